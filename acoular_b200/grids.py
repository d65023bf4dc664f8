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


class LineGrid(Grid):
    """``num_points`` points spaced ``length / (num_points - 1)`` apart from ``loc`` along ``direction``
    (acoular/grids.py:834-914)."""

    def __init__(self, loc=(0.0, 0.0, 0.0), direction=(1.0, 0.0, 0.0), length=1.0, num_points=1):
        self.loc = tuple(float(v) for v in loc)
        self.direction = tuple(float(v) for v in direction)
        self.length = float(length)
        self.num_points = int(num_points)

    @property
    def pos(self) -> np.ndarray:
        start = np.array(self.loc, dtype=np.float64).reshape(3, 1)
        if self.num_points <= 1:
            return start
        unit = np.array(self.direction, dtype=np.float64) / np.linalg.norm(self.direction)
        steps = np.arange(self.num_points) * (self.length / (self.num_points - 1))
        return start + unit[:, None] * steps[None, :]


class MergeGrid(Grid):
    """The union of the positions of several grids, duplicates removed and sorted as ``np.unique`` along
    the point axis sorts them (acoular/grids.py:917-988)."""

    def __init__(self, grids=()):
        self.grids = list(grids)

    @property
    def pos(self) -> np.ndarray:
        if not self.grids:
            return np.zeros((3, 0))
        return np.unique(np.concatenate([g.pos for g in self.grids], axis=1), axis=1)

    @property
    def subgrids(self) -> np.ndarray:
        """Per point of the concatenated grids, the name and digest of the grid it came from, (1, N)."""
        names = [np.full(g.size, type(g).__name__ + g.digest) for g in self.grids]
        return np.concatenate(names)[None, :] if names else np.zeros((1, 0), dtype=str)


def _subdomain(self, sector):
    """Indices of the grid points in ``sector``: ``np.where`` of its membership mask in the grid's shape
    (acoular/grids.py:187-209)."""
    return np.where(sector.contains(self.pos).reshape(self.shape))


Grid.subdomain = _subdomain


# ------------------------------------------------------------------------------------------------
# Sectors: regions of a grid for integrate() (acoular/grids.py:991-1494).  ``contains(pos)`` maps
# positions (3, N) to a boolean mask (N,).  A single sector may take its border points or not (within
# ``abs_tol``), and, when no point lies in it, the point nearest to its centre (``default_nearest``).
# ------------------------------------------------------------------------------------------------
class Sector:
    """A sector that holds the whole grid."""

    def contains(self, pos):
        return np.ones(np.shape(pos)[1], dtype=bool)


class SingleSector(Sector):
    def __init__(self, include_border=True, abs_tol=1e-12, default_nearest=True):
        self.include_border = bool(include_border)
        self.abs_tol = float(abs_tol)
        self.default_nearest = bool(default_nearest)

    def _or_nearest(self, mask, pos, centre):
        """``mask``, or, if it is empty and ``default_nearest`` is set, only the point of ``pos`` whose
        (x, y) lies nearest to ``centre``."""
        if not mask.any() and self.default_nearest:
            d2 = (pos[0] - centre[0]) ** 2 + (pos[1] - centre[1]) ** 2
            mask[np.argmin(d2)] = True
        return mask

    def _within(self, lo, hi, v):
        """lo <= v <= hi with the border tolerance (inclusive or exclusive)."""
        t = self.abs_tol if self.include_border else -self.abs_tol
        return (v - lo > -t) & (v - hi < t)


class RectSector(SingleSector):
    """Axis-aligned rectangle [x_min, x_max] x [y_min, y_max] in the x-y plane."""

    def __init__(self, x_min=-1.0, x_max=1.0, y_min=-1.0, y_max=1.0, **kw):
        super().__init__(**kw)
        self.x_min, self.x_max, self.y_min, self.y_max = float(x_min), float(x_max), float(y_min), float(y_max)

    def contains(self, pos):
        pos = np.asarray(pos, dtype=np.float64)
        xl, xh = sorted((self.x_min, self.x_max))
        yl, yh = sorted((self.y_min, self.y_max))
        mask = self._within(xl, xh, pos[0]) & self._within(yl, yh, pos[1])
        return self._or_nearest(mask, pos, ((xl + xh) / 2.0, (yl + yh) / 2.0))


class RectSector3D(RectSector):
    """Axis-aligned box: the rectangle and [z_min, z_max]."""

    def __init__(self, x_min=-1.0, x_max=1.0, y_min=-1.0, y_max=1.0, z_min=-1.0, z_max=1.0, **kw):
        super().__init__(x_min, x_max, y_min, y_max, **kw)
        self.z_min, self.z_max = float(z_min), float(z_max)

    def contains(self, pos):
        pos = np.asarray(pos, dtype=np.float64)
        xl, xh = sorted((self.x_min, self.x_max))
        yl, yh = sorted((self.y_min, self.y_max))
        zl, zh = sorted((self.z_min, self.z_max))
        mask = self._within(xl, xh, pos[0]) & self._within(yl, yh, pos[1]) & self._within(zl, zh, pos[2])
        return self._or_nearest(mask, pos, ((xl + xh) / 2.0, (yl + yh) / 2.0))


class CircSector(SingleSector):
    """Disk of radius ``r`` around (x, y) in the x-y plane (the tolerance applies to the squared radius)."""

    def __init__(self, x=0.0, y=0.0, r=1.0, **kw):
        super().__init__(**kw)
        self.x, self.y, self.r = float(x), float(y), float(r)

    def contains(self, pos):
        pos = np.asarray(pos, dtype=np.float64)
        excess = (pos[0] - self.x) ** 2 + (pos[1] - self.y) ** 2 - self.r ** 2
        mask = excess < (self.abs_tol if self.include_border else -self.abs_tol)
        return self._or_nearest(mask, pos, (self.x, self.y))


def _polygon_signed_distance(vx, vy, px, py):
    """Distance of the points (px, py) to the closed polygon (vx, vy): positive inside, negative outside
    (even-odd crossing rule), zero on an edge."""
    ax, ay = np.asarray(vx, dtype=np.float64), np.asarray(vy, dtype=np.float64)
    bx, by = np.roll(ax, -1), np.roll(ay, -1)
    px, py = np.asarray(px, dtype=np.float64)[:, None], np.asarray(py, dtype=np.float64)[:, None]
    ex, ey = bx - ax, by - ay
    len2 = ex * ex + ey * ey
    with np.errstate(divide='ignore', invalid='ignore'):
        t = np.clip(np.where(len2 > 0, ((px - ax) * ex + (py - ay) * ey) / len2, 0.0), 0.0, 1.0)
    dist = np.sqrt(((ax + t * ex - px) ** 2 + (ay + t * ey - py) ** 2).min(axis=1))
    straddle = (ay > py) != (by > py)
    with np.errstate(divide='ignore', invalid='ignore'):
        x_cross = ax + (py - ay) * ex / ey
    inside = (straddle & (px < x_cross)).sum(axis=1) % 2 == 1
    return np.where(inside, dist, -dist)


class PolySector(SingleSector):
    """Polygon with vertices ``edges`` = [x1, y1, x2, y2, ...] (closed implicitly) in the x-y plane.

    When no point lies inside and ``default_nearest`` is set, the point nearest to the vertices' mean is
    taken (the reference's code marks point 0 or 1 there, the index of the smaller centroid coordinate).
    """

    def __init__(self, edges=(), **kw):
        super().__init__(**kw)
        self.edges = [float(e) for e in edges]

    def _vertices(self):
        v = np.asarray(self.edges, dtype=np.float64).reshape(-1, 2)
        if len(v) > 1 and np.array_equal(v[0], v[-1]):
            v = v[:-1]
        return v

    def contains(self, pos):
        pos = np.asarray(pos, dtype=np.float64)
        v = self._vertices()
        d = _polygon_signed_distance(v[:, 0], v[:, 1], pos[0], pos[1])
        mask = d >= -self.abs_tol if self.include_border else d > self.abs_tol
        return self._or_nearest(mask, pos, v.mean(axis=0))


class ConvexSector(PolySector):
    """Convex hull of the points ``edges`` = [x1, y1, x2, y2, ...] in the x-y plane."""

    def contains(self, pos):
        from scipy.spatial import ConvexHull
        pos = np.asarray(pos, dtype=np.float64)
        v = self._vertices()
        hull = v[ConvexHull(v).vertices]
        d = _polygon_signed_distance(hull[:, 0], hull[:, 1], pos[0], pos[1])
        mask = d >= -self.abs_tol if self.include_border else d > self.abs_tol
        return self._or_nearest(mask, pos, v.mean(axis=0))


class MultiSector(Sector):
    """Union of several sectors."""

    def __init__(self, sectors=()):
        self.sectors = list(sectors)

    def contains(self, pos):
        mask = np.zeros(np.shape(pos)[1], dtype=bool)
        for s in self.sectors:
            mask |= s.contains(pos)
        return mask
