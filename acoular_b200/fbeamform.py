"""Frequency-domain beamforming on the B200: ``SteeringVector`` and ``BeamformerBase``.

Mirrors acoular/fbeamform.py:
* :class:`SteeringVector` (105-258): ``grid``, ``mics``, ``steer_type``, ``env``, ``ref``, host-side
  ``r0`` / ``rm`` / ``transfer`` / ``steer_vector``.
* :class:`LazyBfResult` (261-286): per-bin lazy evaluation through ``result[...]``.
* :class:`BeamformerBase` (289-685): ``result``, ``synthetic``, ``integrate``, ``sig_loss_norm``;
  ``_calc`` computes every missing bin of a request in ONE batched device launch instead of the
  reference's per-bin loop (fbeamform.py:475-510), with the same ``_ac`` / ``_fr`` contract.
* :func:`L_p` (2412-2429) and :func:`integrate` (2435-2497).

``BeamformerBase.form`` selects the device form: ``'f64'`` (default) is the plain FP64 form of the
reference method (float32 phase, C-library-faithful cos/sin); ``'tc'`` the tensor-core form.
"""

from __future__ import annotations

import warnings

import numpy as np
import torch

from . import device as D
from .environments import Environment


def _result_array(shape, dtype):
    """Result array in page-locked host memory when a GPU is present (fast, asynchronous copies).

    Left uninitialised: ``LazyBfResult`` returns a bin only after ``_calc`` has written it, so no
    unwritten row is ever read (zero-filling 0.5 GB of host memory would cost tens of ms per result).
    """
    if torch.cuda.is_available():
        t = torch.empty(shape, dtype=getattr(torch, np.dtype(dtype).name), pin_memory=True)
        return t.numpy()
    return np.zeros(shape, dtype=dtype)


class SteeringVector:
    STEER_TYPES = ('true level', 'true location', 'classic', 'inverse')

    def __init__(self, grid=None, mics=None, steer_type: str = 'true level', env: Environment | None = None,
                 ref=None):
        if steer_type not in self.STEER_TYPES:
            msg = f'steer_type must be one of {self.STEER_TYPES}, got {steer_type!r}'
            raise ValueError(msg)
        self.grid = grid
        self.mics = mics
        self.steer_type = steer_type
        self.env = env if env is not None else Environment()
        self._ref = np.array([0.0, 0.0, 0.0])
        if ref is not None:
            self.ref = ref

    @property
    def ref(self):
        return self._ref

    @ref.setter
    def ref(self, ref):
        if np.isscalar(ref):
            self._ref = np.abs(float(ref))
        elif len(ref) == 3:
            self._ref = np.array(ref, dtype=float)
        else:
            msg = 'ref must be a float or a (3,) position'
            raise ValueError(msg)

    @property
    def digest(self) -> str:
        return f'{self.steer_type}|{self.env.digest}|{self.grid.digest}|{self.mics.digest}|{np.asarray(self._ref).tobytes().hex()}'

    @property
    def r0(self):
        if np.isscalar(self.ref):
            if self.ref > 0:
                return np.full((self.grid.size,), self.ref)
            return self.env.apparent_r(self.grid.pos)
        return self.env.apparent_r(self.grid.pos, self.ref[:, np.newaxis])

    @property
    def rm(self):
        return np.atleast_2d(self.env.apparent_r(self.grid.pos, self.mics.pos))

    def transfer(self, f, ind=None):
        """Transfer matrix (G, M) for one frequency (acoular/fastFuncs.py:858-897), host side."""
        r0, rm = self.r0, self.rm
        if ind is not None:
            r0 = r0[ind]
            rm = rm[ind, :] if isinstance(ind, np.ndarray) else rm[ind, :][np.newaxis]
        r0 = np.atleast_1d(r0)
        k = 2 * np.pi * f / self.env.c
        arg = (k * (rm - r0[:, None])).astype(np.float32)
        return (np.cos(arg) - 1j * np.sin(arg)) * r0[:, None] / rm

    def steer_vector(self, f, ind=None):
        x = self.transfer(f, ind)
        if self.steer_type == 'classic':
            return x / np.abs(x) / x.shape[-1]
        if self.steer_type == 'inverse':
            return 1.0 / x.conj() / x.shape[-1]
        if self.steer_type == 'true level':
            return x / np.einsum('ij,ij->i', x, x.conj())[:, np.newaxis]
        return x / np.sqrt(np.einsum('ij,ij->i', x, x.conj()) * x.shape[-1])[:, np.newaxis]


class LazyBfResult:
    def __init__(self, bf):
        self.bf = bf

    def __getitem__(self, key):
        sl = np.index_exp[key][0]
        if isinstance(sl, (int, np.integer)):
            sl = slice(sl, sl + 1)
        missing = np.arange(*sl.indices(self.bf._numfreq))[self.bf._fr[sl] == 0]
        if missing.size:
            self.bf._calc(missing)
        return self.bf._ac.__getitem__(key)


def _upload(a, dev, dtype=None) -> torch.Tensor:
    """A host array as a device tensor, copied from page-locked memory without blocking the host.

    ``torch.as_tensor(a, device=...)`` from ordinary host memory waits for all work queued on the stream;
    inside a chain of launches that wait leaves the GPU idle while the host issues the next launch.  The
    pinned staging block goes back to torch's cache once the copy is done."""
    t = torch.as_tensor(np.ascontiguousarray(a, dtype=dtype))
    return t.pin_memory().to(dev, non_blocking=True)


def _launch_sizes(n: int, cap: int, bin_bytes: int = 0) -> list:
    """Bins per map launch for n bins: the bulk in about 7 equal launches of at most ``cap`` bins, then up to
    three shrinking ones (n / 64, half of it, ...), so that each launch's download overlaps the next launch's
    computation and the download left after the last launch is a few bins' maps.

    A request whose maps total at most 4 MB (``bin_bytes`` per bin) goes in as few launches as ``cap`` allows:
    its download takes well under 100 us, less than what another launch and its copy cost on the host."""
    if n * bin_bytes <= (4 << 20) and bin_bytes > 0:
        return [min(cap, n - i) for i in range(0, n, cap)]
    tail = []
    t, rest = min(max(1, n // 64), cap), n
    while len(tail) < 3 and t >= 1 and rest > 2 * t:
        tail.append(t)
        rest -= t
        t //= 2
    per = max(1, min(cap, -(-rest // 7)))
    return [min(per, rest - i) for i in range(0, rest, per)] + tail


class BeamformerBase:
    """Delay-and-sum beamformer in the frequency domain, computed on the GPU."""

    FORMS = ('f64', 'tc')
    # tensor-core operand forms: split BF16 (~1e-5 of max), TF32 and FP16 (~1e-4; FP16 scales each bin's R')
    TC_PRECISIONS = ('bf16x3', 'tf32', 'fp16')

    def __init__(self, freq_data=None, steer: SteeringVector | None = None, r_diag: bool = True,
                 r_diag_norm: float = 0.0, precision: str = 'float64', cached: bool = False, form: str = 'f64',
                 tc_precision: str = 'bf16x3', glibc_faithful: bool = True, max_bins_per_launch: int | None = None):
        self.freq_data = freq_data
        self.steer = steer if steer is not None else SteeringVector()
        self.r_diag = bool(r_diag)
        self.r_diag_norm = float(r_diag_norm)
        if precision not in ('float64', 'float32'):
            msg = f"precision must be 'float64' or 'float32', got {precision!r}"
            raise ValueError(msg)
        self.precision = precision
        self.cached = cached
        if form not in self.FORMS:
            msg = f'form must be one of {self.FORMS}, got {form!r}'
            raise ValueError(msg)
        self.form = form
        if tc_precision not in self.TC_PRECISIONS:
            msg = f'tc_precision must be one of {self.TC_PRECISIONS}, got {tc_precision!r}'
            raise ValueError(msg)
        self.tc_precision = tc_precision
        self.glibc_faithful = glibc_faithful
        self.max_bins_per_launch = max_bins_per_launch
        self._key = None
        self._ac = None
        self._fr = None
        self._f = None
        self._numfreq = 0

    @property
    def digest(self) -> str:
        return (f'{self.freq_data.digest}|{self.r_diag}|{self.r_diag_norm}|{self.precision}|{self.steer.digest}|'
                f'{self.form}|{self.tc_precision}|{self.glibc_faithful}')

    def _assert_equal_channels(self):
        nc = self.freq_data.num_channels
        if nc != self.steer.mics.num_mics or nc == 0:
            msg = f'{nc:d} channels do not fit {self.steer.mics.num_mics:d} mics'
            raise ValueError(msg)

    @property
    def result(self) -> LazyBfResult:
        key = self.digest
        if key != self._key or self._ac is None:
            self._f = self.freq_data.fftfreq()
            self._numfreq = self._f.shape[0]
            self._assert_equal_channels()
            self._ac = _result_array((self._numfreq, self.steer.grid.size), self.precision)
            self._fr = np.zeros(self._numfreq, dtype='int8')
            self._key = key
        return LazyBfResult(self)

    def sig_loss_norm(self) -> float:
        if not self.r_diag:
            return 1.0
        if self.r_diag_norm == 0.0:
            n = float(self.freq_data.num_channels)
            return n / (n - 1)
        return self.r_diag_norm

    # --- device computation -------------------------------------------------------------------
    def _geometry(self, dev):
        gk = ('geom', self.steer.grid.digest, self.steer.mics.digest, str(dev))
        if getattr(self, '_geom_key', None) != gk:
            self._mpos_d = _upload(self.steer.mics.pos, dev, np.float64)
            self._gpos_d = _upload(self.steer.grid.pos, dev, np.float64)
            self._geom_key = gk
        return self._mpos_d, self._gpos_d

    def _calc(self, ind):
        """Compute bins ``ind`` (array of int) on the device; writes ``_ac[ind]`` and ``_fr[ind] = 1``.

        All requested bins go to the device in a few large launches; contiguous runs of bins are
        passed as views (no copy of the CSM), and each launch's map is copied into ``_ac`` on a side
        stream while the next launch computes.
        """
        ind = np.asarray(ind, dtype=np.int64)
        if ind.size == 0:
            return
        # the reference's _beamformer_params (acoular/fbeamform.py:464-472): the predefined steering
        # vectors of a plain SteeringVector, else the object's own (custom) steering vectors
        if type(self.steer) is not SteeringVector:
            self._calc_custom(ind)
            return
        if type(self.steer.env) is not Environment:
            self._calc_given_distances(ind)
            return
        csm_all = self.freq_data.csm_device
        dev = csm_all.device
        mpos, gpos = self._geometry(dev)
        G = gpos.shape[1]
        M = mpos.shape[1]
        cap = self.max_bins_per_launch or max(1, int((1 << 30) // max(1, G * 8 + M * M * 16)))
        norm = self.sig_loss_norm()
        ref = self.steer.ref
        ac_t = torch.from_numpy(self._ac)
        pinned = ac_t.is_pinned()
        compute = torch.cuda.current_stream(dev)
        copy = D.copy_stream(dev)
        pending = []
        # wave numbers and bin indices of every launch in one upload that does not wait for the stream
        k_all = _upload(2 * np.pi * self._f[ind] / self.steer.env.c, dev, np.float64)
        ind_d = None
        s0 = 0
        for n in _launch_sizes(ind.size, cap, G * self._ac.itemsize):
            sub = ind[s0:s0 + n]
            k = k_all[s0:s0 + n]
            contiguous = bool(np.all(np.diff(sub) == 1))
            if contiguous:
                csm = csm_all[int(sub[0]):int(sub[-1]) + 1]
            else:
                if ind_d is None:
                    ind_d = _upload(ind, dev, np.int64)
                csm = csm_all.index_select(0, ind_d[s0:s0 + n]).contiguous()
            s0 += n
            if self.form == 'f64':
                out = D.map_f64(csm, k, mpos, gpos, self.steer.steer_type, self.r_diag, norm, ref=ref,
                                clip_negative=self.r_diag, glibc_faithful=self.glibc_faithful)
            else:
                out = D.map_tc(csm, k, mpos, gpos, self.steer.steer_type, self.r_diag, norm, ref=ref,
                               clip_negative=self.r_diag, precision=self.tc_precision)
            if self.precision == 'float32':
                out = out.float()
            done = torch.cuda.Event()
            done.record(compute)
            copy.wait_event(done)
            with torch.cuda.stream(copy):
                if contiguous and pinned:
                    ac_t[int(sub[0]):int(sub[-1]) + 1].copy_(out, non_blocking=True)
                    pending.append((None, out))
                else:
                    host = torch.empty(out.shape, dtype=out.dtype, pin_memory=True)
                    host.copy_(out, non_blocking=True)
                    pending.append((sub, host))
            out.record_stream(copy)
        copy.synchronize()
        for sub, host in pending:
            if sub is not None:
                self._ac[sub] = host.numpy()
        self._fr[ind] = 1

    def _store(self, ind, out):
        if self.r_diag:   # set (unphysical) negative output values to 0 (acoular/fbeamform.py:506-508)
            out.clamp_(min=0.0)
        if self.precision == 'float32':
            out = out.float()
        self._ac[ind] = out.cpu().numpy()
        self._fr[ind] = 1

    def _calc_given_distances(self, ind):
        """Environments whose apparent distances are not Euclidean (uniform flow): the map kernel
        takes SteeringVector.r0 / .rm as given (FP64 form, also when ``form == 'tc'``)."""
        csm_all = self.freq_data.csm_device
        dev = csm_all.device
        gk = ('rm', self.steer.digest, str(dev))
        if getattr(self, '_rm_key', None) != gk:
            self._r0_d = torch.as_tensor(np.ascontiguousarray(np.atleast_1d(self.steer.r0), dtype=np.float64),
                                         device=dev)
            self._rm_d = torch.as_tensor(np.ascontiguousarray(self.steer.rm, dtype=np.float64), device=dev)
            self._rm_key = gk
        ind_d = torch.as_tensor(ind, device=dev)
        csm = csm_all.index_select(0, ind_d).contiguous()
        k = torch.as_tensor(2 * np.pi * self._f[ind] / self.steer.env.c, dtype=torch.float64, device=dev)
        out = D.map_rm_f64(csm, k, self._r0_d, self._rm_d, self.steer.steer_type, self.r_diag, self.sig_loss_norm(),
                           clip_negative=False, glibc_faithful=self.glibc_faithful)
        self._store(ind, out)

    def _calc_custom(self, ind):
        """Steering objects other than the plain SteeringVector: their steer_vector(f) (G, M) per bin,
        materialised as the reference does, on the custom-steering kernel."""
        csm_all = self.freq_data.csm_device
        dev = csm_all.device
        norm = self.sig_loss_norm()
        for i in ind:
            h = torch.as_tensor(np.ascontiguousarray(self.steer.steer_vector(self._f[i]), dtype=np.complex128),
                                device=dev)
            out = D.map_custom_f64(csm_all[int(i):int(i) + 1], h[None], self.r_diag, norm)
            self._store(np.array([i]), out)

    # --- band synthesis and integration (acoular/fbeamform.py:512-685) -----------------------
    def synthetic(self, f, num=0):
        res = self.result
        freq = self.freq_data.fftfreq()
        if len(freq) == 0:
            return None
        if num == 0:
            ind = np.searchsorted(freq, f)
            if ind >= len(freq):
                warnings.warn(f'Queried frequency ({f:g} Hz) not in resolved frequency range. Returning zeros.',
                              Warning, stacklevel=2)
                h = np.zeros_like(res[0])
            else:
                if freq[ind] != f:
                    warnings.warn(f'Queried frequency ({f:g} Hz) not in set of discrete FFT sample frequencies. '
                                  f'Using frequency {freq[ind]:g} Hz instead.', Warning, stacklevel=2)
                h = res[ind]
        else:
            if isinstance(num, list):
                f1, f2 = num[0], num[-1]
            else:
                f1 = f * 2.0 ** (-0.5 / num)
                f2 = f * 2.0 ** (+0.5 / num)
            ind1 = np.searchsorted(freq, f1)
            ind2 = np.searchsorted(freq, f2)
            if ind1 == ind2:
                warnings.warn(f'Queried frequency band ({f1:g} to {f2:g} Hz) does not include any discrete FFT '
                              'sample frequencies. Returning zeros.', Warning, stacklevel=2)
                h = np.zeros_like(res[0])
            else:
                h = np.sum(res[ind1:ind2], 0)
        return h.reshape(self.steer.grid.shape)

    def integrate(self, sector, frange=None, num=0):
        grid = self.steer.grid
        ind = _sector_indices(grid, sector)
        gshape = grid.shape
        num_freqs = self.freq_data.fftfreq().shape[0]
        if num == 0 or frange is None:
            if frange is None:
                ind_low = self.freq_data.ind_low
                ind_high = self.freq_data.ind_high
                if ind_low is None:
                    ind_low = 0
                if ind_high is None:
                    ind_high = num_freqs
                irange = (ind_low, ind_high)
                num = 0
            elif len(frange) == 2:
                self.result  # noqa: B018 - sets _f
                irange = (np.searchsorted(self._f, frange[0]), np.searchsorted(self._f, frange[1]))
            else:
                msg = 'Only a tuple of length 2 is allowed for frange if num==0'
                raise TypeError(msg)
            h = np.zeros(num_freqs, dtype=float)
            sl = slice(*irange)
            r = self.result[sl]
            for i in range(num_freqs)[sl]:
                h[i] = r[i - sl.start].reshape(gshape)[ind].sum()
            if frange is None:
                return h
            return self._f[sl], h[sl]
        h = np.zeros(len(frange), dtype=float)
        for i, f in enumerate(frange):
            h[i] = self.synthetic(f, num).reshape(gshape)[ind].sum()
        return h


class BeamformerEig(BeamformerBase):
    """Eigenvalue beamformer (acoular/fbeamform.py:821-888): the map of one eigen-component of the CSM.

    ``n`` selects the component (0 = smallest eigenvalue ... num_mics - 1; negative counts from the
    largest; default -1, the largest); ``na`` is the resolved index.  The eigen-decomposition runs on
    the device (``PowerSpectra.evd_device``; for the largest component alone the selected-eigenpair solver
    ``acb_heevd_select_f64``); the map runs in the plain FP64 form (``acb_map_eig_f64``,
    cost O(G M) per bin and component), with the reference's steering arithmetic.
    """

    def __init__(self, *args, n: int = -1, **kw):
        super().__init__(*args, **kw)
        self.n = int(n)

    @property
    def digest(self) -> str:
        return super().digest + f'|eig{self.n}'

    @property
    def na(self) -> int:
        na = self.n
        nm = self.steer.mics.num_mics
        if na < 0:
            na = max(nm + na, 0)
        return min(nm - 1, na)

    def _eig_select(self, ev, evec, ind):
        na = self.na
        return ev[ind, na:na + 1].contiguous(), evec[ind][:, :, na:na + 1].contiguous(), self.sig_loss_norm()

    def _post(self, out):
        if self.r_diag:
            out.clamp_(min=0.0)
        return out

    def _eig_maps(self, f_rows, lam, vec, norm, r_diag, want_norm=False):
        """Eigenvalue-form maps of B' rows (frequency f_rows[j], components lam (B', E), vec (B', M, E)),
        routed as the reference's _beamformer_params: custom steering objects through their materialised
        steer_vector, non-Euclidean environments through given distances, else the synthesising kernel.
        Returns (maps (B', G), steering norms (B', G) or None)."""
        dev = lam.device
        G = self.steer.grid.size
        out = torch.empty((len(f_rows), G), dtype=torch.float64, device=dev)
        sn = torch.empty_like(out) if want_norm else None
        if type(self.steer) is not SteeringVector:
            # custom steering vectors (acoular/fastFuncs.py:476-559), one row at a time
            for j, f in enumerate(f_rows):
                h = torch.as_tensor(np.ascontiguousarray(self.steer.steer_vector(f), dtype=np.complex128), device=dev)
                D.map_custom_f64(None, h[None], r_diag, norm, out=out[j:j + 1],
                                 steer_norm=None if sn is None else sn[j:j + 1],
                                 eig=(lam[j:j + 1].contiguous(), vec[j:j + 1].contiguous()))
        elif type(self.steer.env) is not Environment:
            # distances of a non-Euclidean environment, given to the kernel as they are
            r0, rm = _steer_distances_device(self.steer, dev, self)
            for j, f in enumerate(f_rows):
                D.map_eig_rm_f64(lam[j:j + 1].contiguous(), vec[j:j + 1].contiguous(),
                                 2 * np.pi * f / self.steer.env.c, r0, rm, self.steer.steer_type, r_diag,
                                 norm, glibc_faithful=self.glibc_faithful, out=out[j],
                                 steer_norm=None if sn is None else sn[j])
        else:
            mpos, gpos = self._geometry(dev)
            k = torch.as_tensor(2 * np.pi * np.asarray(f_rows) / self.steer.env.c, dtype=torch.float64, device=dev)
            D.map_eig_f64(lam.contiguous(), vec.contiguous(), k, mpos, gpos, self.steer.steer_type, r_diag, norm,
                          ref=self.steer.ref, clip_negative=False, glibc_faithful=self.glibc_faithful, out=out,
                          steer_norm=sn)
        return out, sn

    def _components(self, ind):
        """(lam (B', E), vec (B', M, E), norm) of the bins ``ind``.  The largest component alone (n = -1, the
        default) comes from the selected-eigenpair solver (``acb_heevd_select_f64``: no QL sweeps, no other
        eigenvectors) unless the full decomposition is cached already; otherwise ``PowerSpectra.evd_device``."""
        fd = self.freq_data
        M = self.steer.mics.num_mics
        evd = getattr(fd, '_evd_dev', None)
        cached = evd is not None and evd[0] == getattr(fd, '_cache_key', None)
        if (type(self)._eig_select is BeamformerEig._eig_select and self.na == M - 1 and not cached
                and D.heevd_select_supported(M, 1)):
            csm = fd.csm_device
            lam, vec = D.heevd_select_f64(csm[torch.as_tensor(ind, device=csm.device)], [M - 1])
            return lam, vec, self.sig_loss_norm()
        ev, evec = fd.evd_device
        return self._eig_select(ev, evec, torch.as_tensor(ind, device=ev.device))

    def _calc(self, ind):
        ind = np.asarray(ind, dtype=np.int64)
        if ind.size == 0:
            return
        lam, vec, norm = self._components(ind)
        out, _ = self._eig_maps(self._f[ind], lam, vec, norm, self.r_diag)
        out = self._post(out)
        if self.precision == 'float32':
            out = out.float()
        self._ac[ind] = out.cpu().numpy()
        self._fr[ind] = 1


class BeamformerMusic(BeamformerEig):
    """MUSIC (acoular/fbeamform.py:891-944): the noise subspace, the ``num_mics - na`` smallest
    eigen-components, full CSM; each bin's map is returned as 4e-10 * min / map.  ``n`` is the
    assumed number of sources (default 1); ``r_diag`` is False and ``r_diag_norm`` 1.0."""

    def __init__(self, *args, n: int = 1, **kw):
        kw.setdefault('r_diag', False)
        kw.setdefault('r_diag_norm', 1.0)
        super().__init__(*args, n=n, **kw)
        if self.r_diag:
            msg = 'BeamformerMusic is defined for the full CSM only (r_diag=False)'
            raise ValueError(msg)

    @property
    def digest(self) -> str:
        return super().digest + '|music'

    def _eig_select(self, ev, evec, ind):
        M = self.steer.mics.num_mics
        ne = int(M - self.na)
        norm = self.sig_loss_norm() * float(self.freq_data.num_channels) ** 2
        return ev[ind, :ne].contiguous(), evec[ind][:, :, :ne].contiguous(), norm

    def _post(self, out):
        return 4e-10 * out.min(dim=1, keepdim=True).values / out


def _steer_distances_device(steer, dev, holder):
    """SteeringVector.r0 / .rm (any environment) on the device, cached on ``holder`` by steer digest."""
    key = ('r0rm', steer.digest, str(dev))
    if getattr(holder, '_r0rm_key', None) != key:
        holder._r0_dev = torch.as_tensor(np.array(np.broadcast_to(steer.r0, (steer.grid.size,)), dtype=np.float64),
                                         device=dev)
        holder._rm_dev = torch.as_tensor(np.ascontiguousarray(steer.rm, dtype=np.float64), device=dev)
        holder._r0rm_key = key
    return holder._r0_dev, holder._rm_dev


class PointSpreadFunction:
    """Point-spread function of a steering set-up (acoular/fbeamform.py:948-1124), on the GPU.

    ``psf`` is the (G, len(grid_indices)) map of unit sources at ``grid_indices`` (all grid points,
    (G, G), when empty) at frequency ``freq``, rounded to ``precision``.  For a plain
    :class:`SteeringVector` (any environment) the predefined formulation runs on the PSF kernel
    (``acb_psf_f64``, calcPointSpreadFunction); other steering objects take
    |steer_vector^H transfer|^2 as a complex GEMM.  ``calcmode`` ('single', 'block', 'full',
    'readonly') is kept for interface parity; nothing is cached between calls, so every mode
    computes the requested columns (``'full'``: all of them).
    """

    CALCMODES = ('single', 'block', 'full', 'readonly')

    def __init__(self, steer: SteeringVector | None = None, grid_indices=None, calcmode: str = 'single',
                 precision: str = 'float64', freq: float = 1.0, cached: bool = False, glibc_faithful: bool = True):
        if calcmode not in self.CALCMODES:
            msg = f'calcmode must be one of {self.CALCMODES}, got {calcmode!r}'
            raise ValueError(msg)
        if precision not in ('float64', 'float32'):
            msg = f"precision must be 'float64' or 'float32', got {precision!r}"
            raise ValueError(msg)
        self.steer = steer if steer is not None else SteeringVector()
        self.grid_indices = np.array([], dtype=int) if grid_indices is None else np.asarray(grid_indices, dtype=int)
        self.calcmode = calcmode
        self.precision = precision
        self.freq = float(freq)
        self.cached = cached
        self.glibc_faithful = glibc_faithful

    @property
    def digest(self) -> str:
        return f'{self.steer.digest}|{self.precision}'

    def _indices(self):
        gs = self.steer.grid.size
        return self.grid_indices if self.grid_indices.size else np.arange(gs)

    def psf_device(self, ind=None, device=None, out: torch.Tensor | None = None) -> torch.Tensor:
        """The PSF (G, len(ind)) as a float64 device tensor (values rounded to ``precision``);
        written into ``out`` when given."""
        dev = D.require_cuda(device)
        gs = self.steer.grid.size
        ind = self._indices() if ind is None else np.asarray(ind, dtype=int)
        if self.calcmode == 'full':
            cols = np.arange(gs)
        else:
            cols = ind
        if cols.size and (cols.min() < -gs or cols.max() >= gs):
            msg = f'grid indices must lie in [0, {gs})'
            raise IndexError(msg)
        cols = np.where(cols < 0, cols + gs, cols)
        if type(self.steer) is SteeringVector:
            r0, rm = _steer_distances_device(self.steer, dev, self)
            k = 2 * np.pi * self.freq / self.steer.env.c
            direct = out is not None and np.array_equal(ind, cols)
            res = D.psf_f64(r0, rm, k, np.ascontiguousarray(cols, dtype=np.int64), self.steer.steer_type,
                            round_f32=self.precision == 'float32', glibc_faithful=self.glibc_faithful,
                            out=out if direct else None)
            if direct:
                return out
        else:
            # arbitrary steering objects (acoular/fbeamform.py:1119-1124)
            h = torch.as_tensor(np.ascontiguousarray(self.steer.steer_vector(self.freq), dtype=np.complex128),
                                device=dev)
            t = torch.as_tensor(np.ascontiguousarray(np.atleast_2d(self.steer.transfer(self.freq, cols)),
                                                     dtype=np.complex128), device=dev)
            prod = h.conj() @ t.T
            res = (prod * prod.conj()).real.contiguous()
            if self.precision == 'float32':
                res = res.float().double()
        if self.calcmode == 'full' and not np.array_equal(ind, cols):
            res = res[:, torch.as_tensor(ind, device=dev)]
        if out is not None:
            out.copy_(res)
            return out
        return res

    @property
    def psf(self) -> np.ndarray:
        return self.psf_device().cpu().numpy().astype(self.precision)


class BeamformerDamas(BeamformerBase):
    """DAMAS deconvolution (acoular/fbeamform.py:1127-1208), on the GPU.

    Per bin: the conventional map (negative values set to 0 with ``r_diag``), the full PSF of every
    grid point at the bin's frequency (``acb_psf_f64``), and ``n_iter`` Gauss-Seidel sweeps with
    relaxation ``damp`` starting from the map (``acb_damas_gauss_seidel_f64``).  Bins go to the device
    in chunks whose PSFs fit ``psf_budget_bytes``.
    """

    def __init__(self, *args, n_iter: int = 100, damp: float = 1.0, psf_precision: str = 'float64',
                 calcmode: str = 'full', psf_budget_bytes: int = 1 << 30, cta_per_bin: int = 0, **kw):
        super().__init__(*args, **kw)
        if psf_precision not in ('float64', 'float32'):
            msg = f"psf_precision must be 'float64' or 'float32', got {psf_precision!r}"
            raise ValueError(msg)
        if calcmode not in PointSpreadFunction.CALCMODES:
            msg = f'calcmode must be one of {PointSpreadFunction.CALCMODES}, got {calcmode!r}'
            raise ValueError(msg)
        self.n_iter = int(n_iter)
        self.damp = float(damp)
        self.psf_precision = psf_precision
        self.calcmode = calcmode
        self.psf_budget_bytes = int(psf_budget_bytes)
        self.cta_per_bin = int(cta_per_bin)

    @property
    def digest(self) -> str:
        return super().digest + f'|damas{self.n_iter}|{self.damp}|{self.psf_precision}'

    def _dirty_map_device(self, ind, csm_all):
        """Conventional maps (B, G) float64 of bins ``ind`` on the device, the reference's
        beamformerFreq with negative values set to 0 when r_diag is set."""
        dev = csm_all.device
        norm = self.sig_loss_norm()
        ind_d = torch.as_tensor(ind, device=dev)
        if type(self.steer) is not SteeringVector:
            out = torch.empty((ind.size, self.steer.grid.size), dtype=torch.float64, device=dev)
            for j, i in enumerate(ind):
                h = torch.as_tensor(np.ascontiguousarray(self.steer.steer_vector(self._f[i]), dtype=np.complex128),
                                    device=dev)
                D.map_custom_f64(csm_all[int(i):int(i) + 1], h[None], self.r_diag, norm, out=out[j:j + 1])
        else:
            csm = csm_all.index_select(0, ind_d).contiguous()
            k = torch.as_tensor(2 * np.pi * self._f[ind] / self.steer.env.c, dtype=torch.float64, device=dev)
            if type(self.steer.env) is not Environment:
                r0, rm = _steer_distances_device(self.steer, dev, self)
                out = D.map_rm_f64(csm, k, r0, rm, self.steer.steer_type, self.r_diag, norm, clip_negative=False,
                                   glibc_faithful=self.glibc_faithful)
            elif self.form == 'tc':
                mpos, gpos = self._geometry(dev)
                out = D.map_tc(csm, k, mpos, gpos, self.steer.steer_type, self.r_diag, norm, ref=self.steer.ref,
                               clip_negative=False, precision=self.tc_precision)
            else:
                mpos, gpos = self._geometry(dev)
                out = D.map_f64(csm, k, mpos, gpos, self.steer.steer_type, self.r_diag, norm, ref=self.steer.ref,
                                clip_negative=False, glibc_faithful=self.glibc_faithful)
        if self.r_diag:
            out.clamp_(min=0.0)
        return out

    def _calc(self, ind):
        ind = np.asarray(ind, dtype=np.int64)
        if ind.size == 0:
            return
        csm_all = self.freq_data.csm_device
        dev = csm_all.device
        G = self.steer.grid.size
        chunk = max(1, min(ind.size, self.psf_budget_bytes // max(1, G * G * 8)))
        p = PointSpreadFunction(steer=self.steer, calcmode='full', precision=self.psf_precision,
                                glibc_faithful=self.glibc_faithful)
        for s0 in range(0, ind.size, chunk):
            sub = ind[s0:s0 + chunk]
            y = self._dirty_map_device(sub, csm_all)
            psf = torch.empty((sub.size, G, G), dtype=torch.float64, device=dev)
            for j, i in enumerate(sub):
                p.freq = float(self._f[i])
                p.psf_device(device=dev, out=psf[j])
            x = D.damas_gauss_seidel(psf, y, self.n_iter, self.damp, cta_per_bin=self.cta_per_bin)
            del psf
            if self.precision == 'float32':
                x = x.float()
            self._ac[sub] = x.cpu().numpy()
        self._fr[ind] = 1


class BeamformerFunctional(BeamformerEig):
    """Functional beamforming (acoular/fbeamform.py:688-786), full CSM only: the eigenvalues to the power
    1/gamma, the eigenvalue-form map of all components divided by the steering norm, to the power gamma,
    times the norm.  gamma = 1 is the conventional beamformer."""

    def __init__(self, *args, gamma: float = 1.0, **kw):
        kw.setdefault('r_diag', False)
        kw.setdefault('r_diag_norm', 1.0)
        super().__init__(*args, **kw)
        if self.r_diag or self.r_diag_norm != 1.0:
            msg = 'BeamformerFunctional is defined for the full CSM only (r_diag=False, r_diag_norm=1.0)'
            raise ValueError(msg)
        self.gamma = float(gamma)

    @property
    def digest(self) -> str:
        return super().digest + f'|functional{self.gamma}'

    def _calc(self, ind):
        ind = np.asarray(ind, dtype=np.int64)
        if ind.size == 0:
            return
        ev, evec = self.freq_data.evd_device
        ind_d = torch.as_tensor(ind, device=ev.device)
        lam = ev[ind_d].pow(1.0 / self.gamma).contiguous()   # negative round-off eigenvalues give NaN
        out, sn = self._eig_maps(self._f[ind], lam, evec[ind_d].contiguous(), 1.0, False, want_norm=True)
        out = out.div_(sn).pow_(self.gamma).mul_(sn).mul_(self.sig_loss_norm())
        if self.precision == 'float32':
            out = out.float()
        self._ac[ind] = out.cpu().numpy()
        self._fr[ind] = 1


class BeamformerOrth(BeamformerEig):
    """Orthogonal deconvolution (acoular/fbeamform.py:1333-1388): for each eigen-component in
    ``eva_list`` (default the largest, ``[-1]``; ``n`` sets the n largest), its eigenvalue / num_mics
    is placed at the argmax of that component's map.  All components of all bins are mapped in one
    launch; the additions run in the list's order on the host."""

    def __init__(self, *args, eva_list=None, n: int | None = None, **kw):
        super().__init__(*args, **kw)
        self._n = 1
        self._eva_list = np.array([-1])
        if n is not None:
            self.n = n
        if eva_list is not None:
            self.eva_list = eva_list

    @property
    def n(self) -> int:
        return getattr(self, '_n', 1)

    @n.setter
    def n(self, n):
        self._n = int(n)
        self._eva_list = np.arange(-1, -1 - self._n, -1)

    @property
    def eva_list(self) -> np.ndarray:
        return self._eva_list

    @eva_list.setter
    def eva_list(self, v):
        self._eva_list = np.atleast_1d(np.asarray(v, dtype=int))

    @property
    def digest(self) -> str:
        return super().digest + f'|orth{self._eva_list.tobytes().hex()}'

    def _calc(self, ind):
        ind = np.asarray(ind, dtype=np.int64)
        if ind.size == 0:
            return
        ev, evec = self.freq_data.evd_device
        dev = ev.device
        M = evec.shape[-1]
        comps = np.asarray(self._eva_list, dtype=np.int64)
        if comps.size and (comps.min() < -M or comps.max() >= M):
            msg = f'eigenvalue indices must lie in [-{M}, {M})'
            raise IndexError(msg)
        comps = np.where(comps < 0, comps + M, comps)
        L = comps.size
        ind_d = torch.as_tensor(ind, device=dev)
        comp_d = torch.as_tensor(comps, device=dev)
        # rows (bin, component): unit eigenvalue, the component's eigenvector
        vec = evec[ind_d][:, :, comp_d].permute(0, 2, 1).reshape(ind.size * L, M, 1).contiguous()
        lam = torch.ones((ind.size * L, 1), dtype=torch.float64, device=dev)
        f_rows = np.repeat(self._f[ind], L)
        out, _ = self._eig_maps(f_rows, lam, vec, self.sig_loss_norm(), self.r_diag)
        peaks = out.argmax(dim=1).view(ind.size, L).cpu().numpy()
        ev_h = ev[ind_d].cpu().numpy()
        nc = float(self.freq_data.num_channels)
        res = np.zeros((ind.size, self.steer.grid.size))
        for j in range(ind.size):
            for li, c in enumerate(comps):
                res[j, peaks[j, li]] += ev_h[j, c] / nc
        self._ac[ind] = res
        self._fr[ind] = 1


class BeamformerCleansc(BeamformerBase):
    """CLEAN-SC (acoular/fbeamform.py:1391-1490), on the GPU: ``n_iter`` iterations per bin (0 = up
    to 2 num_mics, stopping when the peak exceeds the one ``stopn`` iterations before), damping
    ``damp``.  All bins of a request iterate together on the device (``acb_cleansc_f64``); the
    result rows are float32 values, as the reference's."""

    def __init__(self, *args, n_iter: int = 0, damp: float = 0.6, stopn: int = 3, bin_budget_bytes: int = 1 << 30,
                 **kw):
        super().__init__(*args, **kw)
        if not 0.01 <= float(damp) <= 1.0:
            msg = f'damp must lie in [0.01, 1.0], got {damp!r}'
            raise ValueError(msg)
        self.n_iter = int(n_iter)
        self.damp = float(damp)
        self.stopn = int(stopn)
        self.bin_budget_bytes = int(bin_budget_bytes)

    @property
    def digest(self) -> str:
        return super().digest + f'|cleansc{self.n_iter}|{self.damp}|{self.stopn}'

    def _calc(self, ind):
        ind = np.asarray(ind, dtype=np.int64)
        if ind.size == 0:
            return
        csm_all = self.freq_data.csm_device
        dev = csm_all.device
        G = self.steer.grid.size
        M = csm_all.shape[-1]
        per_bin = 2 * G * 8 + 4 * G + 2 * M * M * 16 + G * M * 16
        chunk = max(1, min(ind.size, self.bin_budget_bytes // per_bin))
        if type(self.steer) is not SteeringVector:
            # a steering object of its own: its steer_vector(f) per bin, materialised as the reference's
            # _beamformer_params does (acoular/fbeamform.py:470-472), on the custom-steering iterations
            for s0 in range(0, ind.size, chunk):
                sub = ind[s0:s0 + chunk]
                csm = csm_all.index_select(0, torch.as_tensor(sub, device=dev))
                steer = torch.as_tensor(np.ascontiguousarray(
                    np.stack([self.steer.steer_vector(self._f[i]) for i in sub]), dtype=np.complex128), device=dev)
                res = D.cleansc_custom_f64(csm, steer, self.r_diag, self.sig_loss_norm(), self.n_iter, self.damp,
                                           self.stopn)
                self._ac[sub] = res.double().cpu().numpy()
            self._fr[ind] = 1
            return
        kw = {}
        if type(self.steer.env) is not Environment:
            kw['r0'], kw['rm'] = _steer_distances_device(self.steer, dev, self)
        else:
            kw['mpos'], kw['gpos'] = self._geometry(dev)
            kw['ref'] = self.steer.ref
        for s0 in range(0, ind.size, chunk):
            sub = ind[s0:s0 + chunk]
            csm = csm_all.index_select(0, torch.as_tensor(sub, device=dev))
            k = torch.as_tensor(2 * np.pi * self._f[sub] / self.steer.env.c, dtype=torch.float64, device=dev)
            res = D.cleansc_f64(csm, k, self.steer.steer_type, self.r_diag, self.sig_loss_norm(), self.n_iter,
                                self.damp, self.stopn, glibc_faithful=self.glibc_faithful, **kw)
            self._ac[sub] = res.double().cpu().numpy()
        self._fr[ind] = 1


def L_p(x):
    """Sound pressure level 10 lg(x / 4e-10), floored at the dtype's eps (acoular/fbeamform.py:2412-2429)."""
    return 10 * np.log10(np.maximum(x / 4e-10, np.finfo(x.dtype).eps))


def _sector_indices(grid, sector):
    """Grid indices of ``sector``: a :class:`~acoular_b200.grids.Sector` through ``grid.subdomain``, or the
    array forms (x1, y1, x2, y2) / (x, y, r) / 3-D box through ``grid.indices`` (acoular/fbeamform.py:2475-2487)."""
    from .grids import Sector
    if isinstance(sector, Sector):
        return grid.subdomain(sector)
    if hasattr(grid, 'indices'):
        return grid.indices(*sector)
    msg = (f'Grid of type {grid.__class__.__name__} does not have an indices method! Please use a sector '
           'derived instance of type Sector instead of type numpy.array.')
    raise NotImplementedError(msg)


def integrate(data, grid, sector):
    """Sum of a map (or of each row of a (F, G) result) over a grid sector (acoular/fbeamform.py:2435-2497)."""
    ind = _sector_indices(grid, sector)
    gshape = grid.shape
    gsize = grid.size
    if np.size(data) == gsize:
        return data.reshape(gshape)[ind].sum()
    if data.ndim == 2 and data.shape[1] == gsize:
        h = np.zeros(data.shape[0])
        for i in range(data.shape[0]):
            h[i] = data[i].reshape(gshape)[ind].sum()
        return h
    return None
