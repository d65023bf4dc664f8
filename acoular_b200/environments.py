"""Sound propagation environments: distances between grid points and microphones.

Mirrors ``Environment`` (acoular/environments.py:143-238), ``dist_mat`` (65-103),
``UniformFlowEnvironment`` (254-332), the flow fields ``SlotJet`` / ``OpenJet`` / ``RotatingFlow`` (335-682)
and the ray-traced ``GeneralFlowEnvironment`` (685-980).  The hot path
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


# ------------------------------------------------------------------------------------------------
# Flow fields and the ray-traced environment (acoular/environments.py:335-980).  Host side: they
# produce the apparent distances that the map kernels take as given (SteeringVector.r0 / .rm).
# Every field evaluates many points at once: ``field(x)`` maps positions (3, P) to velocities (3, P)
# and Jacobians (3, 3, P) with J[i, j] = d v_i / d x_j, so that all rays of a microphone advance
# together; ``v(x)`` is the single-point form of the reference's interface.
# ------------------------------------------------------------------------------------------------
class FlowField:
    """A steady flow field."""

    def field(self, x):
        raise NotImplementedError

    def v(self, xx):
        """Velocity (3,) and Jacobian (3, 3) at one position ``xx`` (3,)."""
        vel, jac = self.field(np.asarray(xx, dtype=np.float64).reshape(3, 1))
        return vel[:, 0], jac[:, :, 0]

    @property
    def digest(self) -> str:
        return type(self).__name__ + '|' + '|'.join(f'{k}={np.asarray(v).tobytes().hex()}'
                                                     for k, v in sorted(vars(self).items()))


def _shear_profile(v0, x1, h):
    """Gaussian shear layer of the Albertson et al. (1950) jets, u = v0 exp(-h^2 / (2 x1^2)) for h >= 0
    and the constant core u = v0 for h < 0.  Returns u and its partial derivatives with respect to the
    layer coordinate h and the layer width x1 (both zero in the core)."""
    with np.errstate(divide='ignore', invalid='ignore', over='ignore'):
        w2 = 1.0 / (x1 * x1)
        g = v0 * np.exp(-0.5 * (h * h) * w2)
        d_h = -(h * w2) * g
        d_x1 = (h * h) * w2 * g / x1
    core = h < 0.0
    return np.where(core, v0, g), np.where(core, 0.0, d_h), np.where(core, 0.0, d_x1)


class SlotJet(FlowField):
    """Plane slot jet (Albertson et al. 1950; acoular/environments.py:357-462).

    In the jet frame (x along ``flow``, y normal to the slot plane ``plane``, origin at the slot exit)
    the streamwise velocity u(x, y) has a constant core of half-width B/2 that closes linearly, and a
    Gaussian shear layer whose width grows as x1 = 0.5668 x / l; the layer coordinate is
    h = |y| + (sqrt(pi)/2) x1 - B/2.  Only u is modelled (no entrainment), so the velocity is u along
    ``flow`` and the Jacobian is the outer product of that axis with grad u.
    """

    def __init__(self, v0=0.0, origin=(0.0, 0.0, 0.0), flow=(1.0, 0.0, 0.0), plane=(0.0, 1.0, 0.0), B=0.2, l=5.2):  # noqa: E741
        self.v0 = float(v0)
        self.origin = np.asarray(origin, dtype=np.float64).reshape(3)
        self.flow = np.asarray(flow, dtype=np.float64).reshape(3)
        self.plane = np.asarray(plane, dtype=np.float64).reshape(3)
        self.B = float(B)
        self.l = float(l)

    def _frame(self):
        ax = self.flow / np.linalg.norm(self.flow)
        across = np.cross(self.plane / np.linalg.norm(self.plane), ax)   # normal to the slot plane
        return ax, across

    def field(self, x):
        ax, across = self._frame()
        rel = np.asarray(x, dtype=np.float64) - self.origin[:, None]
        xs, ys = ax @ rel, across @ rel
        rate = 0.5668 / self.l
        x1 = rate * xs
        half_root_pi = 0.5 * np.sqrt(np.pi)
        u, d_h, d_x1 = _shear_profile(self.v0, x1, np.abs(ys) + half_root_pi * x1 - 0.5 * self.B)
        du_dx = rate * (half_root_pi * d_h + d_x1)
        du_dy = np.sign(ys) * d_h
        grad = ax[:, None] * du_dx + across[:, None] * du_dy
        return ax[:, None] * u, ax[:, None, None] * grad[None, :, :]


class OpenJet(FlowField):
    """Round open jet along +x (Albertson et al. 1950; acoular/environments.py:465-573).

    Streamwise velocity with a constant core of diameter D that closes linearly and a Gaussian shear
    layer of width x1 = 0.5022 x / l in the layer coordinate h = r + x1 - D/2, r the distance from the
    jet axis; no entrainment, so only the first row of the Jacobian is non-zero.
    """

    def __init__(self, v0=0.0, origin=(0.0, 0.0, 0.0), D=0.2, l=6.2):  # noqa: E741
        self.v0 = float(v0)
        self.origin = np.asarray(origin, dtype=np.float64).reshape(3)
        self.D = float(D)
        self.l = float(l)

    def field(self, x):
        rel = np.asarray(x, dtype=np.float64) - self.origin[:, None]
        rate = 0.5022 / self.l
        x1 = rate * rel[0]
        radial = np.hypot(rel[1], rel[2])
        u, d_h, d_x1 = _shear_profile(self.v0, x1, radial + x1 - 0.5 * self.D)
        with np.errstate(divide='ignore', invalid='ignore'):
            unit = np.where(radial > 0.0, rel[1:] / radial, 0.0)     # radial unit vector (y, z)
        vel = np.zeros_like(rel)
        vel[0] = u
        jac = np.zeros((3,) + rel.shape)
        jac[0, 0] = rate * (d_h + d_x1)
        jac[0, 1:] = unit * d_h
        return vel, jac


class RotatingFlow(FlowField):
    """Solid-body rotation about the z axis through ``origin`` at ``rps`` revolutions per second with a
    uniform axial velocity ``v0`` (acoular/environments.py:576-682)."""

    def __init__(self, rps=0.0, v0=0.0, origin=(0.0, 0.0, 0.0)):
        self.rps = float(rps)
        self.v0 = float(v0)
        self.origin = np.asarray(origin, dtype=np.float64).reshape(3)

    @property
    def omega(self) -> float:
        return 2 * np.pi * self.rps

    def field(self, x):
        rel = np.asarray(x, dtype=np.float64) - self.origin[:, None]
        om = self.omega
        vel = np.stack((-om * rel[1], om * rel[0], np.full(rel.shape[1], self.v0)))
        spin = np.array(((0.0, -om, 0.0), (om, 0.0, 0.0), (0.0, 0.0, 0.0)))
        return vel, np.repeat(spin[:, :, None], rel.shape[1], axis=2)


def spiral_sphere(N, Om=None, b=None):  # noqa: N803
    """``N`` unit vectors (3, N) spread evenly over the spherical cap of solid angle ``Om`` (default
    2 pi) centred on the direction ``b`` (default +z): the generalised spiral of Saff and Kuijlaars
    (Math. Intelligencer 19, 1997) on the cap around the south pole, reflected onto ``b``.

    The spiral's heights are evenly spaced, h_k = -1 + 2 k / (N 4 pi / Om - 1), and its azimuth advances
    by 3.6 / sqrt(N (4 pi / Om) (1 - h_k^2)) per point; as in acoular/environments.py:685-770 the step
    (not the running angle) is taken modulo 2 pi, which changes no direction.  The reflection is the
    Householder mirror through the plane that bisects the south pole and ``b``.
    """
    Om = 2 * np.pi if Om is None else Om
    axis = np.array((0.0, 0.0, 1.0)) if b is None else np.asarray(b, dtype=np.float64)
    density = N * (4 * np.pi / Om)
    k = np.arange(N)
    height = -1.0 + 2.0 * k / (density - 1.0)
    step = np.zeros(N)
    step[1:] = (3.6 / np.sqrt(density * (1.0 - height[1:] ** 2))) % (2 * np.pi)
    azim = np.cumsum(step)
    ring = np.sqrt(1.0 - height * height)     # sin(arccos h)
    pts = np.stack((ring * np.cos(azim), ring * np.sin(azim), height))
    target = axis / np.linalg.norm(axis)
    mirror = pts[:, 0] - target               # pts[:, 0] is the south pole
    if np.linalg.norm(mirror) < 1e-10:
        return pts
    return pts - np.outer(mirror, mirror @ pts) / (mirror @ pts[:, 0])


class TravelTimeField:
    """Piecewise-linear travel times over a Delaunay tetrahedralisation of ray samples; NaN outside the
    samples' convex hull.  ``field(points (P, 3)) -> (P,)``."""

    def __init__(self, tri, times):
        self.tri = tri
        self.times = np.asarray(times, dtype=np.float64)

    def __call__(self, pts):
        pts = np.atleast_2d(np.asarray(pts, dtype=np.float64))
        cell = self.tri.find_simplex(pts)
        aff = self.tri.transform[cell]                               # (P, 4, 3): barycentric map
        lam = np.einsum('pij,pj->pi', aff[:, :3, :], pts - aff[:, 3, :])
        lam = np.concatenate((lam, 1.0 - lam.sum(axis=1, keepdims=True)), axis=1)
        out = (lam * self.times[self.tri.simplices[cell]]).sum(axis=1)
        out[cell < 0] = np.nan
        return out


# Dormand-Prince 5(4) embedded Runge-Kutta pair (J. R. Dormand, P. J. Prince, J. Comput. Appl. Math. 6,
# 1980): stage nodes, stage weights, 5th-order weights and the 5th - 4th order error weights.
_DP_C = (0.0, 1 / 5, 3 / 10, 4 / 5, 8 / 9, 1.0, 1.0)
_DP_A = ((),
         (1 / 5,),
         (3 / 40, 9 / 40),
         (44 / 45, -56 / 15, 32 / 9),
         (19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729),
         (9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656),
         (35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84))
_DP_B = (35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84, 0.0)
_DP_E = (71 / 57600, 0.0, -71 / 16695, 71 / 1920, -17253 / 339200, 22 / 525, -1 / 40)


def trace_rays(ff, c, x0, dirs, rmax, dt, rtol=1e-9):
    """Trace acoustic rays from ``x0`` backwards in time through the steady flow ``ff``, all rays at once.

    State per ray: position x and wave slowness s, with dx/dt = c s / |s| - v(x) and ds/dt = -J(x) s
    (J the field's Jacobian), started at s = n / (c + v(x0) . n) for the unit directions ``dirs`` (3, R)
    (the ray model of acoular/environments.py:884-980).  Every ray is sampled at t = 0, dt, 2 dt, ... up
    to and including its first sample farther than ``rmax`` from ``x0``.  Between samples each ray
    advances with its own adaptive step (Dormand-Prince 5(4), local error below ``rtol`` relative):
    jet shear layers are thin near the nozzle, and a fixed step smears them.  Returns per ray the
    sample positions (K, 3) and times (K,).
    """
    x0 = np.asarray(x0, dtype=np.float64).reshape(3, 1)
    n = dirs.shape[1]
    vel0, _ = ff.field(x0)
    y = np.concatenate((np.repeat(x0, n, axis=1), dirs / (c + (vel0 * dirs).sum(axis=0))))   # (6, R)
    scale = np.concatenate((np.full(3, rmax), np.full(3, 1.0 / c)))[:, None]                # error floor

    def rate(state):
        vel, jac = ff.field(state[:3])
        sl = state[3:]
        return np.concatenate((c * sl / np.sqrt((sl * sl).sum(axis=0)) - vel, -np.einsum('ijp,jp->ip', jac, sl)))

    paths = [[x0[:, 0].copy()] for _ in range(n)]
    times = [[0.0] for _ in range(n)]
    live = np.arange(n)
    h = np.full(n, 0.25 * dt)
    limit = 64 * int(np.ceil(np.sqrt(n))) + 64     # samples per ray; rays that never leave stop here
    for step in range(1, limit + 1):
        left = np.full(live.size, dt)              # time to the next sample, per live ray
        ys, hs = y[:, live], h[live]
        todo = np.arange(live.size)
        while todo.size:
            yy = ys[:, todo]
            hh = np.minimum(hs[todo], left[todo])
            k = [rate(yy)]
            for i in range(1, 7):
                acc = yy + hh * sum(a * kj for a, kj in zip(_DP_A[i], k) if a != 0.0)
                k.append(rate(acc))
            y5 = yy + hh * sum(b * kj for b, kj in zip(_DP_B, k) if b != 0.0)
            err = hh * sum(e * kj for e, kj in zip(_DP_E, k) if e != 0.0)
            tol = rtol * (np.maximum(np.abs(yy), np.abs(y5)) + scale)
            ratio = np.sqrt(((err / tol) ** 2).mean(axis=0))
            ok = ratio <= 1.0
            grow = np.clip(0.9 * np.where(ratio > 0, ratio, 1e-10) ** -0.2, 0.2, 5.0)
            ys[:, todo[ok]] = y5[:, ok]
            left[todo[ok]] -= hh[ok]
            hs[todo] = np.where(ok & (hh < hs[todo]), hs[todo], hh * grow)
            todo = todo[left[todo] > 1e-12 * dt]
        y[:, live], h[live] = ys, hs
        t = step * dt
        for j, r in enumerate(live):
            paths[r].append(ys[:3, j].copy())
            times[r].append(t)
        live = live[np.sqrt(((ys[:3] - x0) ** 2).sum(axis=0)) <= rmax]
        if live.size == 0:
            break
    return [np.array(p) for p in paths], [np.array(t) for t in times]


class GeneralFlowEnvironment(Environment):
    """Sound propagation through a steady, non-uniform flow field ``ff`` (acoular/environments.py:773-980).

    For each microphone position, ``N`` rays over the solid angle ``Om`` around the direction of the
    region of interest are traced backwards in time (:func:`trace_rays`), sampled every
    range / (c sqrt(N)) seconds until they are one sampling step beyond the farthest region point.
    Rays are taken in spiral order, ``int(sqrt(N))`` at a time, until the region lies inside the hull of
    their samples; a point's travel time is the piecewise-linear interpolant over the Delaunay
    tetrahedralisation of those samples (:class:`TravelTimeField`, NaN outside it), and
    apparent_r = c * time.  The fields are kept per microphone position in ``idict``.

    The reference integrates each ray with VODE (rtol 1e-4); the fourth-order Runge-Kutta steps here
    are finer, and the sampled times agree with the reference's to about 1e-7 relative, the
    interpolated distances to the same order.
    """

    def __init__(self, c: float = 343.0, ff: FlowField | None = None, N: int = 200, Om: float = np.pi, roi=None):  # noqa: N803
        super().__init__(c)
        self.ff = ff
        self.N = int(N)
        self.Om = float(Om)
        self.roi = None if roi is None else np.asarray(roi, dtype=np.float64)
        self.idict = {}

    @property
    def digest(self) -> str:
        return f'_gflow_c{self.c!r}_{self.ff.digest if self.ff else None}_{self.N}_{self.Om!r}'

    def apparent_r(self, gpos, mpos=0.0):
        if np.isscalar(mpos):
            mpos = np.array((0, 0, 0), dtype=np.float32)[:, np.newaxis]
        gpos = np.asarray(gpos)
        mpos = np.asarray(mpos)
        times = np.empty((gpos.shape[-1], mpos.shape[-1]))
        for j in range(mpos.shape[-1]):
            x0 = mpos[:, j]
            key = x0.tobytes()
            if key not in self.idict:
                self.idict[key] = self.get_interpolator(gpos if self.roi is None else self.roi, x0)
            times[:, j] = self.idict[key](gpos.T)
        if times.shape[1] == 1:
            times = times[:, 0]
        return self.c * times

    def get_interpolator(self, roi, x0):
        """Travel-time field (:class:`TravelTimeField`) of the rays from ``x0`` over the region ``roi`` (3, P)."""
        from scipy.spatial import Delaunay

        roi = np.asarray(roi, dtype=np.float64)
        x0 = np.asarray(x0, dtype=np.float64)
        reach = np.sqrt(((roi - x0[:, None]) ** 2).sum(axis=0).max())
        rstep = reach / np.sqrt(self.N)
        dirs = spiral_sphere(self.N, self.Om, b=roi.mean(axis=1) - x0)
        paths, times = trace_rays(self.ff, self.c, x0, dirs, reach + rstep, rstep / self.c)
        group = int(np.sqrt(self.N))
        counts = list(range(group + 1, self.N + 1, group))
        if not counts or counts[-1] != self.N:
            counts.append(self.N)
        for n in counts:          # fewest rays whose samples enclose the region
            tri = Delaunay(np.concatenate(paths[:n]))
            if n == self.N or (tri.find_simplex(roi.T) >= 0).all():
                break
        return TravelTimeField(tri, np.concatenate(times[:n]))
