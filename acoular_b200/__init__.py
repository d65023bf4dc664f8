"""B200-native frequency-domain beamforming for Acoular: CSM estimation + steered-response map.

Acoular-compatible classes (same names, attributes and semantics as the reference's):
``MicGeom``, ``RectGrid``, ``RectGrid3D``, ``ImportGrid``, ``LineGrid``, ``MergeGrid``, the sectors
(``RectSector``, ``RectSector3D``, ``CircSector``, ``PolySector``, ``ConvexSector``, ``MultiSector``), ``Environment``, ``TimeSamples``,
``PowerSpectra``, ``PowerSpectraImport``, ``SteeringVector``, ``BeamformerBase``, ``BeamformerEig``,
``BeamformerMusic``, ``BeamformerFunctional``, ``BeamformerOrth``, ``PointSpreadFunction``,
``BeamformerDamas``, ``BeamformerCleansc``, ``L_p``, ``integrate``; the block-wise generators ``RFFT``,
``AutoPowerSpectra``, ``CrossPowerSpectra``; the kernel
entry points ``fastFuncs.calcCSM`` / ``beamformerFreq`` / ``calcPointSpreadFunction`` /
``damasSolverGaussSeidel``; and
the device-level API in :mod:`acoular_b200.device`.  The compute runs in hand-written sm_100a
kernels (``lib/libacoular_b200.so``); there is no CPU fallback.
"""

from .environments import (Environment, GeneralFlowEnvironment, OpenJet, RotatingFlow, SlotJet,
                           UniformFlowEnvironment)
from .fbeamform import (BeamformerBase, BeamformerCleansc, BeamformerDamas, BeamformerEig, BeamformerFunctional,
                        BeamformerMusic, BeamformerOrth, L_p, LazyBfResult, PointSpreadFunction, SteeringVector,
                        integrate)
from .fprocess import RFFT, AutoPowerSpectra, CrossPowerSpectra
from .grids import (CircSector, ConvexSector, ImportGrid, LineGrid, MergeGrid, MultiSector, PolySector, RectGrid,
                    RectGrid3D, RectSector, RectSector3D, Sector, SingleSector)
from .microphones import MicGeom
from .sources import Mixer, PointSource, TimeSamples, WNoiseGenerator
from .spectra import PowerSpectra, PowerSpectraImport

__all__ = [
    'RFFT', 'AutoPowerSpectra', 'CrossPowerSpectra',
    'BeamformerBase', 'BeamformerCleansc', 'BeamformerDamas', 'BeamformerEig', 'BeamformerFunctional',
    'BeamformerOrth', 'BeamformerMusic', 'Environment', 'GeneralFlowEnvironment', 'OpenJet', 'RotatingFlow', 'SlotJet', 'UniformFlowEnvironment', 'ImportGrid', 'L_p', 'LazyBfResult', 'MicGeom', 'Mixer', 'PointSource', 'PointSpreadFunction',
    'PowerSpectra', 'PowerSpectraImport', 'RectGrid', 'RectGrid3D', 'SteeringVector', 'TimeSamples',
    'WNoiseGenerator', 'integrate', 'LineGrid', 'MergeGrid', 'Sector', 'SingleSector', 'RectSector', 'RectSector3D',
    'CircSector', 'PolySector', 'ConvexSector', 'MultiSector',
]
