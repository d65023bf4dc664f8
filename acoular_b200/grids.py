"""Beamforming grids, mirroring acoular/grids.py.

* :class:`RectGrid`   -- acoular/grids.py:284-472 (``nxsteps`` 332-337, ``pos`` 350-358, ``index`` /
  ``indices`` 385-472 for rectangles and circles)
* :class:`RectGrid3D` -- acoular/grids.py:475-665 (scalar or per-axis increment, ``pos`` 552-560)
* :class:`ImportGrid` -- a grid given by explicit positions (acoular/grids.py:666-833)

Grid positions are ``(3, size)`` float64, x-major as ``np.mgrid`` produces them (flat index
``ix*ny + iy`` in 2D, ``(ix*ny + iy)*nz + iz`` in 3D).  The CUDA map kernels take the grid as
these positions or, for rectangular grids, regenerate them on the device from the same
``linspace`` parameters.
"""

from __future__ import annotations

import hashlib

import numpy as np


class Grid:
    @property
    def pos(self) -> np.ndarray:  # pragma: no cover - interface
        raise NotImplementedError

    @property
    def size(self) -> int:
        return self.pos.shape[-1]

    @property
    def shape(self):
        return (self.size,)

    @property
    def digest(self) -> str:
        p = np.ascontiguousarray(self.pos)
        return '_' + hashlib.blake2b(p.tobytes() + str(self.shape).encode(), digest_size=16).hexdigest()


def _nsteps(lo: float, hi: float, inc: float) -> int:
    i = abs(inc)
    if i != 0:
        return round((abs(hi - lo) + i) / i)
    return 1


class RectGrid(Grid):
    """2D Cartesian grid in the plane ``z``."""

    def __init__(self, x_min=-1.0, x_max=1.0, y_min=-1.0, y_max=1.0, z=1.0, increment=0.1):
        self.x_min, self.x_max = float(x_min), float(x_max)
        self.y_min, self.y_max = float(y_min), float(y_max)
        self.z = float(z)
        self.increment = float(increment)
        self._pos = None

    @property
    def nxsteps(self) -> int:
        return _nsteps(self.x_min, self.x_max, self.increment)

    @property
    def nysteps(self) -> int:
        return _nsteps(self.y_min, self.y_max, self.increment)

    @property
    def size(self) -> int:
        return self.nxsteps * self.nysteps

    @property
    def shape(self):
        return (self.nxsteps, self.nysteps)

    @property
    def extent(self):
        return (self.x_min, self.x_max, self.y_min, self.y_max)

    @property
    def digest(self) -> str:
        """Identifier from the defining parameters (positions follow from them)."""
        return f'_rect|{self.x_min!r}|{self.x_max!r}|{self.y_min!r}|{self.y_max!r}|{self.z!r}|{self.increment!r}'

    @property
    def pos(self) -> np.ndarray:
        key = (self.x_min, self.x_max, self.y_min, self.y_max, self.z, self.increment)
        if self._pos is None or self._pos[0] != key:
            bpos = np.mgrid[self.x_min:self.x_max:self.nxsteps * 1j, self.y_min:self.y_max:self.nysteps * 1j,
                            self.z:self.z + 0.1]
            bpos.resize((3, self.size))
            self._pos = (key, bpos)
        return self._pos[1]

    def index(self, x, y):
        if x < self.x_min or x > self.x_max:
            msg = 'x-value out of range'
            raise ValueError(msg)
        if y < self.y_min or y > self.y_max:
            msg = 'y-value out of range'
            raise ValueError(msg)
        xi = int((x - self.x_min) / self.increment + 0.5)
        yi = int((y - self.y_min) / self.increment + 0.5)
        return xi, yi

    def indices(self, *r):
        """Rectangle ``(x1, y1, x2, y2)`` -> slices; circle ``(x, y, radius)`` -> index arrays."""
        if len(r) == 3:
            xpos = self.pos
            dr2 = (xpos[0, :] - r[0]) ** 2 + (xpos[1, :] - r[1]) ** 2
            inds = dr2 <= r[2] ** 2
            xis, yis = [], []
            for n_p in np.arange(self.size)[inds]:
                xi, yi = self.index(xpos[0, n_p], xpos[1, n_p])
                xis.append(xi)
                yis.append(yi)
            if not (xis and yis):
                return self.index(r[0], r[1])
            return np.array(xis), np.array(yis)
        if len(r) == 4:
            xi1, yi1 = self.index(min(r[0], r[2]), min(r[1], r[3]))
            xi2, yi2 = self.index(max(r[0], r[2]), max(r[1], r[3]))
            return np.s_[xi1:xi2 + 1], np.s_[yi1:yi2 + 1]
        msg = 'polygon sectors are not supported by this grid'
        raise NotImplementedError(msg)

    def linspace_params(self):
        """(x0, dx, nx, y0, dy, ny, z0, dz, nz) such that pos = x0 + i*dx etc. (np.mgrid semantics)."""
        nx, ny = self.nxsteps, self.nysteps
        dx = (self.x_max - self.x_min) / (nx - 1) if nx > 1 else 0.0
        dy = (self.y_max - self.y_min) / (ny - 1) if ny > 1 else 0.0
        return (self.x_min, dx, nx, self.y_min, dy, ny, self.z, 0.0, 1)


class RectGrid3D(RectGrid):
    """3D Cartesian grid ``[x_min, x_max] x [y_min, y_max] x [z_min, z_max]``."""

    def __init__(self, x_min=-1.0, x_max=1.0, y_min=-1.0, y_max=1.0, z_min=-1.0, z_max=1.0, increment=0.1):
        super().__init__(x_min, x_max, y_min, y_max, 0.0, 0.1)
        self.z_min, self.z_max = float(z_min), float(z_max)
        self.increment = increment

    @property
    def digest(self) -> str:
        return (f'_rect3d|{self.x_min!r}|{self.x_max!r}|{self.y_min!r}|{self.y_max!r}|{self.z_min!r}|{self.z_max!r}|'
                f'{self.increment!r}')

    def _inc(self, axis):
        return abs(self.increment) if np.isscalar(self.increment) else abs(self.increment[axis])

    @property
    def nxsteps(self) -> int:
        return _nsteps(self.x_min, self.x_max, self._inc(0))

    @property
    def nysteps(self) -> int:
        return _nsteps(self.y_min, self.y_max, self._inc(1))

    @property
    def nzsteps(self) -> int:
        return _nsteps(self.z_min, self.z_max, self._inc(2))

    @property
    def size(self) -> int:
        return self.nxsteps * self.nysteps * self.nzsteps

    @property
    def shape(self):
        return (self.nxsteps, self.nysteps, self.nzsteps)

    @property
    def pos(self) -> np.ndarray:
        key = (self.x_min, self.x_max, self.y_min, self.y_max, self.z_min, self.z_max, str(self.increment))
        if self._pos is None or self._pos[0] != key:
            bpos = np.mgrid[self.x_min:self.x_max:self.nxsteps * 1j, self.y_min:self.y_max:self.nysteps * 1j,
                            self.z_min:self.z_max:self.nzsteps * 1j]
            bpos.resize((3, self.size))
            self._pos = (key, bpos)
        return self._pos[1]

    def index(self, x, y, z):
        if x < self.x_min or x > self.x_max:
            msg = f'x-value out of range {x:f} ({self.x_min:f}, {self.x_max:f})'
            raise ValueError(msg)
        if y < self.y_min or y > self.y_max:
            msg = f'y-value out of range {y:f} ({self.y_min:f}, {self.y_max:f})'
            raise ValueError(msg)
        if z < self.z_min or z > self.z_max:
            msg = f'z-value out of range {z:f} ({self.z_min:f}, {self.z_max:f})'
            raise ValueError(msg)
        xi = round((x - self.x_min) / self._inc(0))
        yi = round((y - self.y_min) / self._inc(1))
        zi = round((z - self.z_min) / self._inc(2))
        return xi, yi, zi

    def indices(self, x1, y1, z1, x2, y2, z2):
        xi1, yi1, zi1 = self.index(min(x1, x2), min(y1, y2), min(z1, z2))
        xi2, yi2, zi2 = self.index(max(x1, x2), max(y1, y2), max(z1, z2))
        return np.s_[xi1:xi2 + 1], np.s_[yi1:yi2 + 1], np.s_[zi1:zi2 + 1]

    def linspace_params(self):
        nx, ny, nz = self.nxsteps, self.nysteps, self.nzsteps
        dx = (self.x_max - self.x_min) / (nx - 1) if nx > 1 else 0.0
        dy = (self.y_max - self.y_min) / (ny - 1) if ny > 1 else 0.0
        dz = (self.z_max - self.z_min) / (nz - 1) if nz > 1 else 0.0
        return (self.x_min, dx, nx, self.y_min, dy, ny, self.z_min, dz, nz)


class ImportGrid(Grid):
    """Grid given by explicit ``(3, size)`` positions."""

    def __init__(self, pos=None):
        self._p = np.zeros((3, 1)) if pos is None else np.asarray(pos, dtype=np.float64).reshape(3, -1)

    @property
    def pos(self) -> np.ndarray:
        return self._p

    @property
    def size(self) -> int:
        return self._p.shape[-1]

    @property
    def shape(self):
        return (self.size,)
