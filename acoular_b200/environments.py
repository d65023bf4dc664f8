"""Sound propagation environments: distances between grid points and microphones.

Mirrors ``Environment`` (acoular/environments.py:143-238), ``dist_mat`` (65-103) and
``UniformFlowEnvironment`` (254-332).  The hot path
never materialises the distance matrix: the CUDA kernels recompute each mic-grid distance in FP64
from the positions, tile by tile.  :func:`dist_mat` here is the host-side helper behind
``SteeringVector.rm`` / ``r0``, kept for API compatibility.
"""

from __future__ import annotations

import numpy as np


def dist_mat(gpos: np.ndarray, mpos: np.ndarray) -> np.ndarray:
    """``(3, N)`` grid and ``(3, M)`` mic positions -> ``(N, M)`` Euclidean distances."""
    gpos = np.asarray(gpos, dtype=np.float64)
    mpos = np.asarray(mpos, dtype=np.float64)
    d0 = gpos[0][:, None] - mpos[0][None, :]
    d1 = gpos[1][:, None] - mpos[1][None, :]
    d2 = gpos[2][:, None] - mpos[2][None, :]
    return np.sqrt(d0 * d0 + d1 * d1 + d2 * d2)


class Environment:
    """Homogeneous medium with speed of sound ``c`` (default 343 m/s)."""

    def __init__(self, c: float = 343.0):
        self.c = float(c)

    @property
    def digest(self) -> str:
        return f'_env_c{self.c!r}'

    def apparent_r(self, gpos, mpos=0.0):
        """Distances from ``gpos`` (3, N) to ``mpos`` (3, M), or to the origin if ``mpos`` is a scalar."""
        if np.isscalar(mpos):
            mpos = np.array((0, 0, 0), dtype=np.float64)[:, np.newaxis]
        rm = dist_mat(np.ascontiguousarray(gpos), np.ascontiguousarray(mpos))
        if rm.shape[1] == 1:
            rm = rm[:, 0]
        return rm


class UniformFlowEnvironment(Environment):
    """Uniform steady flow of Mach number ``ma`` along ``fdv`` (acoular/environments.py:254-332).

    The apparent distance of a path of length r whose direction makes the angle theta with the flow
    is r / (sqrt(ma^2 cos^2 theta - ma^2 + 1) - ma cos theta).  The map kernels take these distances as
    given (``acb_map_rm_f64``); they cannot be resynthesised from the positions alone.
    """

    def __init__(self, c: float = 343.0, ma: float = 0.0, fdv=(1.0, 0.0, 0.0)):
        super().__init__(c)
        self.ma = float(ma)
        self.fdv = np.asarray(fdv, dtype=np.float64).reshape(3)

    @property
    def digest(self) -> str:
        return f'_uflow_c{self.c!r}_ma{self.ma!r}_{self.fdv.tobytes().hex()}'

    def apparent_r(self, gpos, mpos=0.0):
        if np.isscalar(mpos):
            mpos = np.array((0, 0, 0), dtype=np.float32)[:, np.newaxis]
        gpos = np.asarray(gpos, dtype=np.float64)
        mpos = np.asarray(mpos)
        u = self.fdv / np.sqrt((self.fdv * self.fdv).sum())
        d = gpos[:, :, np.newaxis] - mpos[:, np.newaxis, :]          # (3, N, M)
        r = np.sqrt(np.sum(d * d, 0))
        mc = (self.ma * np.sum(d.reshape((3, -1)) * u[:, np.newaxis], 0) / r.reshape(-1)).reshape(r.shape)
        r = r * (1 / (-mc + np.sqrt(mc * mc - self.ma * self.ma + 1)))
        if r.shape[1] == 1:
            r = r[:, 0]
        return r
