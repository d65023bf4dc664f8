"""Sound propagation environment (no flow): distances between grid points and microphones.

Mirrors ``Environment`` (acoular/environments.py:143-238) and ``dist_mat`` (65-103).  The hot path
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
