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
import scipy.linalg as spla


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
# Flow fields and the ray-traced environment (acoular/environments.py:335-980).  Host-side: they
# produce the apparent distances that the map kernels take as given (SteeringVector.r0 / .rm).
# ------------------------------------------------------------------------------------------------
class FlowField:
    """A steady flow field: ``v(x)`` gives the velocity (3,) and its Jacobian (3, 3) at x (3,)."""

    def v(self, xx):
        raise NotImplementedError

    @property
    def digest(self) -> str:
        return type(self).__name__ + '|' + '|'.join(f'{k}={np.asarray(v).tobytes().hex()}'
                                                     for k, v in sorted(vars(self).items()))


class SlotJet(FlowField):
    """Slot jet after Albertson et al. (1950), acoular/environments.py:357-462: constant core, Gaussian
    shear layer of spreading rate 0.5668 / l, in the frame of ``flow`` and the slot plane ``plane``."""

    def __init__(self, v0=0.0, origin=(0.0, 0.0, 0.0), flow=(1.0, 0.0, 0.0), plane=(0.0, 1.0, 0.0), B=0.2, l=5.2):  # noqa: E741
        self.v0 = float(v0)
        self.origin = np.asarray(origin, dtype=np.float64).reshape(3)
        self.flow = np.asarray(flow, dtype=np.float64).reshape(3)
        self.plane = np.asarray(plane, dtype=np.float64).reshape(3)
        self.B = float(B)
        self.l = float(l)

    def v(self, xx):
        ex = self.flow / spla.norm(self.flow)
        pl = self.plane / spla.norm(self.plane)
        ey = -np.cross(ex, pl)
        ez = np.cross(ex, ey)
        rel = xx - self.origin
        x = np.dot(ex, rel)
        y = np.dot(ey, rel)
        x1 = 0.5668 / self.l * x
        h1 = abs(y) + np.sqrt(np.pi) * 0.5 * x1 - 0.5 * self.B
        if h1 < 0.0:            # potential core
            u, dudx, dudy = self.v0, 0, 0
        else:                   # shear layer
            u = self.v0 * np.exp(-h1 * h1 / (2 * x1 * x1))
            dudx = (h1 * h1 / (x * x1 * x1) - np.sqrt(np.pi) * 0.5 * h1 / (x * x1)) * u
            dudy = -np.sign(y) * h1 * u / (x1 * x1)
        jac_local = np.array(((dudx, 0, 0), (dudy, 0, 0), (0, 0, 0))).T
        rot = np.array((ex, ey, ez)).T
        return np.dot(rot, np.array((u, 0, 0))), np.dot(np.dot(rot, jac_local), rot.T)


class OpenJet(FlowField):
    """Round open jet along x after Albertson et al. (1950), acoular/environments.py:465-573: constant
    core, Gaussian shear layer of spreading rate 0.5022 / l."""

    def __init__(self, v0=0.0, origin=(0.0, 0.0, 0.0), D=0.2, l=6.2):  # noqa: E741
        self.v0 = float(v0)
        self.origin = np.asarray(origin, dtype=np.float64).reshape(3)
        self.D = float(D)
        self.l = float(l)

    def v(self, xx):
        x, y, z = xx - self.origin
        r = np.sqrt(y * y + z * z)
        x1 = 0.5022 / self.l * x
        h1 = r + x1 - 0.5 * self.D
        u = self.v0 * np.exp(-h1 * h1 / (2 * x1 * x1))
        if h1 < 0.0:
            dudr = 0.0
            u = self.v0
        else:
            dudr = -h1 * u / (x1 * x1)
        if r > 0.0:
            dudy, dudz = y * dudr / r, z * dudr / r
        else:
            dudy = dudz = 0.0
        dudx = (h1 * h1 / (x * x1 * x1) - h1 / (x * x1)) * u
        if h1 < 0.0:
            dudx = 0
        return np.array((u, 0.0, 0.0)), np.array(((dudx, 0.0, 0.0), (dudy, 0.0, 0.0), (dudz, 0.0, 0.0))).T


class RotatingFlow(FlowField):
    """Rigid rotation about z at ``rps`` revolutions per second plus a constant axial velocity ``v0``
    (acoular/environments.py:576-682)."""

    def __init__(self, rps=0.0, v0=0.0, origin=(0.0, 0.0, 0.0)):
        self.rps = float(rps)
        self.v0 = float(v0)
        self.origin = np.asarray(origin, dtype=np.float64).reshape(3)

    @property
    def omega(self) -> float:
        return 2 * np.pi * self.rps

    def v(self, xx):
        x, y, _ = xx - self.origin
        om = self.omega
        return (np.array((om * -y, om * x, self.v0)),
                np.array(((0.0, om, 0.0), (-om, 0.0, 0.0), (0.0, 0.0, 0.0))).T)


def spiral_sphere(N, Om=None, b=None):  # noqa: N803
    """N unit vectors spread over the solid angle ``Om`` (default 2 pi) around the direction ``b``
    (default +z), as (3, N): a spiral in spherical coordinates, mirrored by a Householder reflection
    onto ``b`` (acoular/environments.py:685-770)."""
    Om = 2 * np.pi if Om is None else Om
    b = np.array((0, 0, 1)) if b is None else np.asarray(b, dtype=np.float64)
    o = 4 * np.pi / Om
    h = -1 + 2 * np.arange(N) / (N * o - 1.0)
    theta = np.arccos(h)
    phi = np.zeros_like(theta)
    for i, hk in enumerate(h[1:]):
        phi[i + 1] = phi[i] + 3.6 / np.sqrt(N * o * (1 - hk * hk)) % (2 * np.pi)
    xyz = np.vstack((np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)))
    first = xyz[:, 0]
    b = b / spla.norm(b)
    d = (first - b)[:, np.newaxis]
    if spla.norm(d) < 1e-10:
        return xyz
    householder = np.identity(3) - np.dot(d, d.T) / np.dot(d.T, first)
    return np.dot(householder, xyz)


class GeneralFlowEnvironment(Environment):
    """Sound propagation through a steady, non-uniform flow field ``ff`` (acoular/environments.py:773-980).

    From each microphone, ``N`` rays over the solid angle ``Om`` (towards the region of interest) are
    traced backwards in time through the flow: x' = c s / |s| - v(x), s' = -J(x)^T s, started with
    s = n / (c + v . n) and integrated by VODE (rtol 1e-4, max step 1e-4 of the range), sampled every
    range / (c sqrt(N)) seconds until they leave the range; ray batches of sqrt(N) are added until the
    convex hull of the samples encloses the region of interest; the travel time of a point is the
    piecewise-linear (Delaunay) interpolant of the sampled times.  apparent_r = c * time.  The steps,
    tolerances and stopping rule are those of the reference, so that the distances agree; the
    interpolators are kept per microphone position.
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
        gt = np.empty((gpos.shape[-1], mpos.shape[-1]))
        for j, x0 in enumerate(np.asarray(mpos).T):
            key = x0.tobytes()
            interp = self.idict.get(key)
            if interp is None:
                interp = self.get_interpolator(gpos if self.roi is None else self.roi, x0)
                self.idict[key] = interp
            gt[:, j] = interp(gpos.T)
        if gt.shape[1] == 1:
            gt = gt[:, 0]
        return self.c * gt

    def get_interpolator(self, roi, x0):
        from scipy.integrate import ode
        from scipy.interpolate import LinearNDInterpolator
        from scipy.spatial import ConvexHull

        c = self.c
        field = self.ff.v

        def rhs(t, y, v):  # noqa: ARG001 - backwards in time: position and wave-normal slowness
            x = y[0:3]
            s = y[3:6]
            vv, dv = v(x)
            sa = np.sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2])
            out = np.empty(6)
            out[0:3] = c * s / sa - vv
            out[3:6] = np.dot(s, -dv.T)
            return out

        def trace(n0, rmax, dt, pts, times):
            s0 = n0 / (c + np.dot(field(x0)[0], n0))
            solver = ode(rhs)
            solver.set_f_params(field)
            solver.set_integrator('vode', rtol=1e-4, max_step=1e-4 * rmax)
            solver.set_initial_value(np.hstack((x0, s0)), 0)
            while solver.successful():
                pts.append(solver.y[0:3])
                times.append(solver.t)
                if spla.norm(solver.y[0:3] - x0) > rmax:
                    break
                solver.integrate(solver.t + dt)

        n_roi = roi.shape[-1]
        batch = int(np.sqrt(self.N))
        centre = roi.mean(1)
        d = x0[:, np.newaxis] - roi
        rmax = np.sqrt((d * d).sum(0).max())
        dirs = spiral_sphere(self.N, self.Om, b=centre - x0)
        rstep = rmax / np.sqrt(self.N)
        rmax += rstep
        tstep = rstep / c
        pts, times = [], []
        done = 0
        hull = None
        for i, n0 in enumerate(dirs.T):
            trace(n0, rmax, tstep, pts, times)
            if i and i % batch == 0:
                if not done:
                    hull = ConvexHull(np.vstack((roi.T, pts)), incremental=True)
                else:
                    hull.add_points(pts[done:], restart=True)
                done = len(pts)
                if hull.simplices.min() >= n_roi:   # no region point on the hull: enclosed
                    break
        return LinearNDInterpolator(np.array(pts), np.array(times))
