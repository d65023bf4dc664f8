/*
 * acoular_b200 -- C ABI of the B200 (sm_100a) frequency-domain beamforming path.
 *
 * Two stages of Acoular's path are exported:
 *   Stage A  cross-spectral matrix (CSM) estimation       PowerSpectra.calc_csm / calcCSM
 *   Stage B  steered-response map h^H C h per grid point  BeamformerBase._calc / beamformerFreq
 *
 * Conventions
 *   - Every pointer argument is DEVICE memory unless its name ends in _host.
 *   - Complex values are interleaved (re, im): complex128 = 2 doubles, complex64 = 2 floats.
 *   - Matrices are row-major and C-contiguous exactly like the numpy arrays of the reference.
 *   - Every call is asynchronous on `stream` (a cudaStream_t passed as void*; NULL = legacy
 *     default stream) and returns an acb_status code; argument errors are reported before any
 *     work is enqueued.  Kernel-side faults surface at the next synchronising call.
 *   - No call allocates device memory unless its comment says so; scratch space is passed in
 *     by the caller (workspace pointer + size).
 */
#ifndef ACOULAR_B200_H
#define ACOULAR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum acb_status {
    ACB_OK = 0,
    ACB_ERR_SHAPE = 1,        /* a size or shape argument is out of range                */
    ACB_ERR_ARG = 2,          /* an enum / flag / pointer argument is invalid            */
    ACB_ERR_CUDA = 3,         /* a CUDA launch or runtime call failed                    */
    ACB_ERR_UNSUPPORTED = 4,  /* valid request this build does not implement             */
    ACB_ERR_WORKSPACE = 5,    /* workspace pointer missing or too small                  */
    ACB_ERR_TIMEOUT = 6,      /* a bounded device-side wait gave up (error word set)     */
};

enum acb_steer { ACB_STEER_CLASSIC = 1, ACB_STEER_INVERSE = 2, ACB_STEER_TRUE_LEVEL = 3, ACB_STEER_TRUE_LOCATION = 4 };
/* CSM precision: complex128 / complex64 spectra and Welch sums (the reference's `precision`), or the
 * tensor-core form (no counterpart in the reference): FP64 FFT, spectra rounded to TF32 or split
 * into BF16 hi + lo, Gram on tcgen05 with FP32 accumulation, summed into a complex128 csm_upper. */
enum acb_precision { ACB_C128 = 0, ACB_C64 = 1, ACB_CSM_TC_TF32 = 2, ACB_CSM_TC_BF16X3 = 3 };
enum acb_sample_dtype { ACB_F32 = 0, ACB_F64 = 1 };

/* Human-readable text of a status code (static storage). */
const char *acb_status_string(int status);
/* ABI version of this library (bumped on any signature change). */
int acb_abi_version(void);
/* Last CUDA error text seen by the library on this host thread (static storage). */
const char *acb_last_cuda_error(void);

/* ---------------------------------------------------------------------------------------------
 * Stage A: cross-spectral matrix
 * ------------------------------------------------------------------------------------------- */

/* calcCSM drop-in (acoular/fastFuncs.py:19-58): adds one ensemble spectrum to the upper triangle
 * of the CSM, csm[f, r, c] += conj(spec[f, c]) * spec[f, r] for r <= c.
 * csm: complex128 [num_freqs][num_mics][num_mics] (updated in place); spec: complex128 [num_freqs][num_mics]. */
int acb_calc_csm_c128(void *csm, const void *spec, int num_freqs, int num_mics, void *stream);
/* Same for complex64 CSM and spectra. */
int acb_calc_csm_c64(void *csm, const void *spec, int num_freqs, int num_mics, void *stream);

/* Bytes of workspace acb_csm_accumulate needs for `num_windows` windows of `num_bins` bins, for
 * block sizes up to 16384 (the spectra of the chunk). */
size_t acb_csm_workspace_bytes(int num_mics, int num_bins, int64_t num_windows, int precision);
/* The same for any block size: blocks of 32768 and 65536 samples (the largest of the reference's
 * block_size choices, acoular/spectra.py:105-116) add a scratch region for the FFT's sub-spectra,
 * num_windows * num_mics * block_size / 2 complex doubles. */
size_t acb_csm_workspace_bytes_block(int num_mics, int num_bins, int64_t num_windows, int precision, int block_size);

/* Welch accumulation of PowerSpectra.calc_csm (acoular/spectra.py:366-416, windows as yielded by
 * BaseSpectra._get_source_data, acoular/spectra.py:171-184):
 *   for every window w in [first_window, first_window + num_windows):
 *     x   = samples[w*hop : w*hop + block_size, :] * window[:, None]    (FP64)
 *     X   = rfft(x, axis=0)[bin_lo : bin_lo + num_bins]                  (FP64 FFT, then rounded
 *                                                                         to `precision`)
 *     csm_upper[f, r, c] += conj(X[f, c]) * X[f, r]     for r <= c       (in `precision`)
 * samples: [num_samples][num_mics], float32 or float64 (sample_dtype).
 * window: float64 [block_size].  twiddle: complex128 [block_size/2], exp(-2*pi*i*k/block_size).
 * csm_upper: [num_bins][num_mics][num_mics] in `precision` (complex128 for the tensor-core forms,
 * num_mics <= 4032 there); only r <= c is written.
 * block_size: power of two, 16 <= block_size <= 65536.  workspace: >= acb_csm_workspace_bytes_block. */
int acb_csm_accumulate(const void *samples, int sample_dtype, int64_t num_samples, int num_mics,
                       int block_size, int hop, int64_t first_window, int64_t num_windows,
                       const double *window, const void *twiddle, int bin_lo, int num_bins,
                       int precision, void *csm_upper, void *workspace, size_t workspace_bytes,
                       void *stream);

/* Hermitian completion and scaling (acoular/spectra.py:411-416):
 *   csm_out[f, r, c] = scale * (r <= c ? upper[f, r, c] : conj(upper[f, c, r]))
 * upper in `precision`; csm_out always complex128 (as the reference returns). */
int acb_csm_finalize(const void *csm_upper, int num_bins, int num_mics, int precision, double scale,
                     void *csm_out, void *stream);

/* ---------------------------------------------------------------------------------------------
 * Stage B: steered-response map (full CSM, predefined steering vectors)
 * ------------------------------------------------------------------------------------------- */

/* Map parameters shared by the map entry points. */
typedef struct acb_map_params {
    int num_mics;            /* M                                                            */
    int64_t num_grid;        /* G                                                            */
    int num_bins;            /* B: bins computed in this call                                */
    int steer_type;          /* acb_steer                                                    */
    int r_diag;              /* 1: remove the CSM diagonal (fastFuncs.py:277-291)            */
    int clip_negative;       /* 1: set negative map values to 0 (fbeamform.py:506-508)       */
    double norm;             /* signal-loss normalisation (BeamformerBase.sig_loss_norm)     */
    int ref_mode;            /* 0: r0 = |g - ref_point|; 1: r0 = ref_distance (scalar ref)   */
    double ref_point[3];     /* SteeringVector.ref as a position (default origin)            */
    double ref_distance;     /* SteeringVector.ref as a distance (> 0)                       */
    int glibc_faithful;      /* 1: apply the sincos exception table (plain form only)        */
    const uint64_t *sincos_table; /* device hash table from acb_sincos_table_build_host      */
    int64_t sincos_table_slots;   /* power of two                                           */
    /* tensor-core form only (0 = default); no counterpart in the reference:                    */
    int tc_pass_chunks;      /* accumulator width per column pass, in 16-mic chunks: 4, 8 or 16 */
    int tc_splits;           /* CTAs sharing one (bin, 128-point tile): its column passes are   *
                              * split into this many groups whose partial sums are combined in  *
                              * a fixed order (batch entry only; acb_map_tc runs unsplit)       */
} acb_map_params;

/* Plain FP64 form of _freqBeamformer_FullCSM (acoular/fastFuncs.py:217-311), batched over bins:
 *   csm:       complex128 [num_bins][M][M]   (full Hermitian CSM per bin)
 *   wavenumber: float64 [num_bins]           (k = 2*pi*f/c)
 *   mpos:      float64 [3][M];  gpos: float64 [3][G]
 *   out_map:   float64 [num_bins][G];  out_steer_norm: float64 [num_bins][G] or NULL
 * Distances and steering vectors are synthesised on the device from the positions.
 * error_word: int32 on the device or NULL (set nonzero on a device-detected fault). */
int acb_map_f64(const acb_map_params *p, const void *csm, const double *wavenumber, const double *mpos,
                const double *gpos, double *out_map, double *out_steer_norm, int *error_word, void *stream);

/* Eigenvalue form, _freqBeamformer_EigValues (acoular/fastFuncs.py:313-411) batched over bins, as
 * BeamformerEig._calc / BeamformerMusic._calc call it (acoular/fbeamform.py:852-944):
 *   eigval: float64 [num_bins][num_eigs];  eigvec: complex128 [num_bins][M][num_eigs]
 *   map = norm_steer(sum_e eigval[e] (|sum_m conj(eigvec[m][e]) h[m]|^2 - [r_diag] sum_m |..|^2))
 * Plain FP64 form, the same steering synthesis as acb_map_f64.  1 <= num_eigs <= M. */
int acb_map_eig_f64(const acb_map_params *p, int num_eigs, const double *eigval, const void *eigvec,
                    const double *wavenumber, const double *mpos, const double *gpos, double *out_map,
                    double *out_steer_norm, void *stream);

/* The plain FP64 map with the distances given instead of synthesised from positions, batched over
 * bins: r0 float64 [G], rm float64 [G][M] (Environment.apparent_r of any environment, e.g. the
 * uniform-flow one, acoular/environments.py:254-332, as SteeringVector.r0 / .rm pass them,
 * acoular/fbeamform.py:187-197, 464-468).  ref_mode / ref_point are ignored (r0 is given). */
int acb_map_rm_f64(const acb_map_params *p, const void *csm, const double *wavenumber, const double *r0,
                   const double *rm, double *out_map, double *out_steer_norm, void *stream);

/* Custom steering vectors (beamformerFreq('custom', ...), acoular/fastFuncs.py:414-473, as
 * BeamformerBase._calc uses them for steering objects other than the plain SteeringVector,
 * acoular/fbeamform.py:470-472): steer complex128 [num_bins][G][M];
 *   map = norm * (2 Re sum_{a<b} conj(h_a) C_ab h_b + [!r_diag] sum_a C_aa |h_a|^2),
 *   steer_norm = sum_a |h_a|^2.   p->steer_type, ref and glibc_faithful are ignored. */
int acb_map_custom_f64(const acb_map_params *p, const void *csm, const void *steer, double *out_map,
                       double *out_steer_norm, void *stream);

/* Eigenvalue form with custom steering vectors (acoular/fastFuncs.py:476-559). */
int acb_map_eig_custom_f64(const acb_map_params *p, int num_eigs, const double *eigval, const void *eigvec,
                           const void *steer, double *out_map, double *out_steer_norm, void *stream);

/* beamformerFreq with an eigen tuple (eigval[num_eigs], eigvec[M][num_eigs]) for one bin with
 * precomputed distances r0 [G], rm [G][M] (acoular/fastFuncs.py:61-214). */
int acb_beamformer_freq_eig_f64(const acb_map_params *p, int num_eigs, const double *eigval, const void *eigvec,
                                double wavenumber, const double *r0, const double *rm, double *out_map,
                                double *out_steer_norm, void *stream);

/* beamformerFreq drop-in (acoular/fastFuncs.py:61-214) for one bin with precomputed distances:
 *   r0: float64 [G] (distGridToArrayCenter), rm: float64 [G][M] (distGridToAllMics). */
int acb_beamformer_freq_f64(const acb_map_params *p, const void *csm, double wavenumber, const double *r0,
                            const double *rm, double *out_map, double *out_steer_norm, void *stream);

/* Tensor-core operand precisions. */
enum acb_tc_precision {
    ACB_TC_BF16X3 = 0,  /* split-BF16 hi/lo operands, 3 products, FP32 accumulation (~1e-5)      */
    ACB_TC_TF32 = 1,    /* FP32 operands rounded to TF32, 1 product, FP32 accumulation (~1e-4)  */
    ACB_TC_FP16 = 2     /* FP16 operands (R' scaled per bin by a power of two), 1 product, FP32
                           accumulation (~1e-4; steering weights |w| < 65504, i.e. distances
                           below 65 km for 'inverse' and above 15 um for the 1/r types)        */
};

/* Bytes of workspace acb_map_tc needs (the per-bin split-BF16 copy of the real-embedded CSM). */
size_t acb_map_tc_workspace_bytes(int num_mics, int num_bins, int precision);

/* Limit of each bounded device-side wait in the tensor-core kernels (acb_map_tc, acb_map_tc_batch,
 * acb_map_tc_noalloc and the tensor-core CSM forms of acb_csm_accumulate); no counterpart in the
 * reference.  A wait that runs out sets the launch's error word to 1 (where one is given), the CTA
 * lets its own copies and MMAs finish, frees its tensor memory and exits, so the device context stays
 * usable.  Applies to launches enqueued after the call; 0 restores the default of 0.5 s.  Returns
 * the previous limit.  Process-wide (all devices and host threads). */
uint64_t acb_tc_set_wait_limit_ns(uint64_t limit_ns);

/* Tensor-core form of the same map (acoular/fastFuncs.py:217-311 semantics, same arguments and
 * outputs as acb_map_f64): the quadratic form h^H C h is evaluated as the real quadratic form
 * v^T R v of the 2M-dimensional real embedding, R = [[Re C, -Im C], [Im C, Re C]], on tcgen05
 * tensor cores with FP32 accumulation in TMEM; `precision` (acb_tc_precision) picks the operands:
 * split-BF16 (hi*hi + hi*lo + lo*hi), TF32 or FP16.  Steering vectors are synthesised per
 * 128-grid-point tile in shared memory: FP32 distances, the phase k*r with k as a float-float
 * (reduced by a three-term 2*pi for split-BF16), hardware sincos.  The per-point partial sums, the
 * normalisation sums and the final normalisation are FP64.  num_mics <= 2048; above 256 mics the
 * accumulator is computed in column passes of 512 (steering chunks before a pass are synthesised
 * again).  glibc_faithful is ignored.
 * workspace: >= acb_map_tc_workspace_bytes(num_mics, num_bins, precision) bytes.
 * error_word: int32 on the device or NULL; bit 0 is set if a bounded device-side wait gave up,
 * bit 1 (value 2) if an FP16 map value came out non-finite (a steering weight out of FP16 range,
 * or a non-finite CSM entry). */
int acb_map_tc(const acb_map_params *p, int precision, const void *csm, const double *wavenumber,
               const double *mpos, const double *gpos, double *out_map, double *out_steer_norm,
               void *workspace, size_t workspace_bytes, int *error_word, void *stream);

/* Device buffers of one instance of a batched map (sizes given by its acb_map_params). */
typedef struct acb_map_io {
    const void *csm;            /* complex128 [num_bins][M][M]                              */
    const double *wavenumber;   /* float64 [num_bins]                                       */
    const double *mpos;         /* float64 [3][M]                                           */
    const double *gpos;         /* float64 [3][G]                                           */
    double *out_map;            /* float64 [num_bins][G]                                    */
    double *out_steer_norm;     /* float64 [num_bins][G] or NULL                            */
} acb_map_io;

/* Bytes of workspace acb_map_tc_batch needs for these instances. */
size_t acb_map_tc_batch_workspace_bytes(const acb_map_params *params, int num_instances, int precision);

/* Many independent maps of uneven size (mic counts, grids, bin counts) in ONE persistent launch of
 * the tensor-core kernel: the work items (instance, bin, 128-point tile) of all instances share the
 * GPU, so small instances fill the SMs that large ones leave idle.  Each instance's result is the
 * one acb_map_tc gives for it alone.  params/io: host arrays of num_instances (<= 64) entries; all
 * instances use params[0].steer_type.  The instance table travels in the kernel parameters, so the
 * call can be captured in a CUDA graph.  The batched counterpart of BeamformerBase._calc
 * (acoular/fbeamform.py:475-510) over many beamformers. */
int acb_map_tc_batch(const acb_map_params *params, const acb_map_io *io, int num_instances, int precision,
                     void *workspace, size_t workspace_bytes, int *error_word, void *stream);

/* ---------------------------------------------------------------------------------------------
 * Point-spread functions and DAMAS deconvolution
 * ------------------------------------------------------------------------------------------- */

/* calcPointSpreadFunction (acoular/fastFuncs.py:563-801) for one wave number, as
 * PointSpreadFunction._psf_call uses it (acoular/fbeamform.py:1093-1125):
 *   out_psf[g][j] = PSF at grid point g of a unit source at grid point sources[j],
 *   for p->steer_type (1..4), r0 float64 [G], rm float64 [G][M] (SteeringVector.r0 / .rm),
 *   sources int64 [num_sources].  p->num_mics / num_grid / glibc_faithful / sincos_table are used.
 *   round_f32 != 0 rounds each value to float32 (PointSpreadFunction.precision 'float32').
 *   A source index outside [0, G) gives a column of NaN (the kernel reads nothing for it). */
int acb_psf_f64(const acb_map_params *p, int num_sources, const int64_t *sources, double wavenumber,
                const double *r0, const double *rm, int round_f32, double *out_psf, void *stream);

/* damasSolverGaussSeidel (acoular/fastFuncs.py:804-855) for num_bins independent bins, as
 * BeamformerDamas._calc uses it (acoular/fbeamform.py:1167-1208):
 *   psf float64 [num_bins][G][G] (row g = PSF values at g of every source), dirty_map float64
 *   [num_bins][G]; solution float64 [num_bins][G] holds the starting solution and receives the
 *   result after n_iter Gauss-Seidel sweeps with relaxation `relax` (negative values set to 0).
 *   cta_per_bin: 1, 2, 4 or 8 CTAs (one cluster) per bin, 0 = choose from num_bins and the SM count.
 *   ACB_ERR_UNSUPPORTED when a bin's solution (8 G bytes + 38 KB) exceeds a CTA's shared memory
 *   (G above about 24,000). */
int acb_damas_gauss_seidel_f64(const double *psf, int64_t num_grid, int num_bins, const double *dirty_map,
                               double *solution, int n_iter, double relax, int cta_per_bin, void *stream);

/* ---------------------------------------------------------------------------------------------
 * Block-wise spectra generators (acoular/fprocess.py)
 * ------------------------------------------------------------------------------------------- */

/* Workspace (device bytes) of acb_spectra for num_windows windows. */
size_t acb_spectra_workspace_bytes(int num_mics, int block_size, int64_t num_windows);

/* RFFT.result (acoular/fprocess.py:35-181) for windows [first_window, first_window + num_windows) of the
 * samples (the windows of BaseSpectra._get_source_data, acoular/spectra.py:171-184):
 *   out[w][f][m] = rfft(samples[w*hop : w*hop + block_size, m] * window)[f], f = 0 .. block_size/2,
 *   rounded to `precision` (ACB_C128 / ACB_C64); bins 1 .. block_size/2 - 1 doubled when double_inner
 *   (scaling 'energy' / 'amplitude'), then times `scale`, both in the output precision.
 * block_size: power of two, 16 .. 65536 (other even sizes: ACB_ERR_SHAPE / ACB_ERR_UNSUPPORTED). */
int acb_spectra(const void *samples, int sample_dtype, int64_t num_samples, int num_mics, int block_size, int hop,
                int64_t first_window, int64_t num_windows, const double *window, const void *twiddle, int precision,
                double scale, int double_inner, void *out, void *workspace, size_t workspace_bytes, void *stream);

/* AutoPowerSpectra.result (acoular/fprocess.py:286-366): out[i] = (X[i] conj(X[i])).real * scale for
 * num_values spectra values X in `precision`, computed in that precision, stored as float64 or float32. */
int acb_auto_spectra(const void *spectra, int64_t num_values, int precision, int out_float32, double scale, void *out,
                     void *stream);

/* CrossPowerSpectra.result (acoular/fprocess.py:369-467), calc_mode 'full': per window w and bin f,
 *   out[w][f][r][c] = scale * (r <= c ? U[r][c] : conj(U[c][r])),  U[r][c] = conj(X[c]) X[r] (calcCSM),
 * X = spectra[w][f][:] in `precision`; out in `precision`. */
int acb_cross_spectra(const void *spectra, int64_t num_windows, int num_freqs, int num_mics, int precision,
                      double scale, void *out, void *stream);

/* ---------------------------------------------------------------------------------------------
 * CLEAN-SC deconvolution
 * ------------------------------------------------------------------------------------------- */

/* Workspace (device bytes) of acb_heevd_f64. */
size_t acb_heevd_workspace_bytes(int num_mics, int num_bins);

/* Hermitian eigendecomposition of every bin's CSM, PowerSpectra._get__evd (acoular/spectra.py:351-364:
 * numpy.linalg.eigh per bin) on the device: csm complex128 [B][M][M] (read only) -> eigval float64 [B][M]
 * ascending, eigvec complex128 [B][M][M] row-major with the eigenvectors in the columns (numpy's layout;
 * each column may differ from LAPACK's by a unit phase factor).  Householder tridiagonalisation, implicit QL
 * with Wilkinson shifts, back-transformation, all in FP64.  info int [B] (may be NULL): 1 where a QL iteration
 * did not converge in 60 steps.  M <= 4096. */
int acb_heevd_f64(const void *csm, int num_bins, int num_mics, double *eigval, void *eigvec, int *info,
                  void *workspace, size_t workspace_bytes, void *stream);

/* Selected eigenpairs of every bin's CSM: the eigenvalues of ascending ranks sel[0 .. num_sel-1] (the same
 * ranks for every bin, 1 <= num_sel <= 4) and their eigenvectors, as the columns sel of acb_heevd_f64's
 * result (up to a unit phase factor per column): csm complex128 [B][M][M] (read only) -> eigval float64
 * [B][num_sel], eigvec complex128 [B][M][num_sel] row-major.  For consumers of a few components
 * (BeamformerEig n = -1, acoular/fbeamform.py:821-888, uses the largest): Householder tridiagonalisation,
 * the selected eigenvalues by multisection on Sturm counts, their eigenvectors by inverse iteration, the
 * back-transformation; no QL sweeps.  Accurate for eigenvalues separated from the others; inside a cluster
 * of (nearly) equal eigenvalues the vector is some unit vector of the cluster's space, as any solver's is.
 * Workspace: acb_heevd_workspace_bytes(M, B).  M <= 4096 and (3 M + 5 M num_sel) 8 + M num_sel bytes of
 * shared memory <= 200 KB (ACB_ERR_UNSUPPORTED above). */
int acb_heevd_select_f64(const void *csm, int num_bins, int num_mics, int num_sel, const int *sel, double *eigval,
                         void *eigvec, void *workspace, size_t workspace_bytes, void *stream);

/* Workspace (device bytes) of acb_cleansc_f64 for num_bins bins (n_iter 0 = 2 num_mics iterations). */
size_t acb_cleansc_workspace_bytes(int num_mics, int64_t num_grid, int num_bins, int n_iter);

/* BeamformerCleansc._calc (acoular/fbeamform.py:1424-1490) for p->num_bins bins at once:
 *   csm complex128 [B][M][M], the working copy (updated in place: the cleaned CSM on return);
 *   wavenumber [B]; geometry mpos [3][M] / gpos [3][G] with p->ref_*, or given distances r0 [G],
 *   rm [G][M] (then mpos / gpos may be NULL); p->steer_type, r_diag, norm (sig_loss_norm) as for the
 *   map, clip_negative ignored; n_iter 0 = 2 M; damp, stopn as the reference's traits;
 *   result float32 [B][G] (damp * peak at each cleaned peak, as the reference's float32 result).
 * Runs the iterations of all bins with no host synchronisation (2 launches per iteration); the workspace
 * holds, among others, every bin's G x M steering vectors (16 G M bytes per bin). */
int acb_cleansc_f64(const acb_map_params *p, void *csm, const double *wavenumber, const double *mpos,
                    const double *gpos, const double *r0, const double *rm, int n_iter, double damp, int stopn,
                    float *result, void *workspace, size_t workspace_bytes, void *stream);

/* BeamformerCleansc._calc (acoular/fbeamform.py:1424-1490) with a steering object other than the plain
 * SteeringVector (custom steering, as _beamformer_params routes it, acoular/fbeamform.py:470-472):
 * steer complex128 [B][G][M] = the object's steer_vector(f) of each bin; the maps are the custom-steering
 * forms of beamformerFreq (acoular/fastFuncs.py:414-559) and the peak's vector is row xi of steer.
 * csm, n_iter, damp, stopn, result as acb_cleansc_f64 (p->steer_type, ref, glibc_faithful ignored); the
 * workspace may omit the steering region: acb_cleansc_workspace_bytes - 16 G M B bytes suffice. */
int acb_cleansc_custom_f64(const acb_map_params *p, void *csm, const void *steer, int n_iter, double damp, int stopn,
                           float *result, void *workspace, size_t workspace_bytes, void *stream);

/* Size of the fixed device array behind acb_map_tc_noalloc (32 MiB per GPU, held until exit). */
#define ACB_NOALLOC_SCRATCH_BYTES ((size_t)32 << 20)

/* No counterpart in the reference.  Same computation and arguments as acb_map_tc, but it allocates
 * nothing and takes no workspace: the scratch lives in a fixed array of ACB_NOALLOC_SCRATCH_BYTES
 * that the library keeps on every GPU that loads it.  Meant for callers that cannot allocate device
 * memory when they call, such as a real-time acquisition loop that must not risk cudaMalloc's
 * implicit device synchronisation, or a host program with no device allocator of its own.
 * Limit: acb_map_tc_workspace_bytes(num_mics, num_bins, precision) must not exceed
 * ACB_NOALLOC_SCRATCH_BYTES (e.g. 60 bins at 256 mics); larger requests return ACB_ERR_SHAPE before
 * any work is enqueued -- split the bins over several calls.
 * Argument errors return the same status codes as acb_map_tc.
 * The first call on a device looks up the array's device address (once per device, with that
 * device current) and keeps it for the life of the process; make that first call before capturing a
 * stream, and do not call this entry point again on a device after a cudaDeviceReset of it (the
 * reset unloads the array and the kept address goes stale).
 * All calls share the one array: calls whose GPU work overlaps (different streams, or different
 * host threads on one device) race on it; order them on one stream. */
int acb_map_tc_noalloc(const acb_map_params *p, int precision, const void *csm, const double *wavenumber,
                       const double *mpos, const double *gpos, double *out_map, double *out_steer_norm,
                       int *error_word, void *stream);

/* Host-side construction of the sincos exception table used by glibc_faithful=1.
 * The reference evaluates float32 cos/sin of the float32 phase through the C library (numba
 * lowers np.cos/np.sin on float32 to cosf/sinf).  The device computes the correctly rounded
 * float32 value of cos/sin of the same float32 argument; this table lists every float32 argument
 * x in [0, max_arg) where the host C library's cosf/sinf differ from that value, with the
 * difference in units of the last place.  It is built by CALLING the host cosf/sinf on every
 * float32 in the range (no knowledge of their implementation is used).
 * table_host: uint64 [slots] (slots a power of two, >= 2^22 recommended), filled here.
 * Returns the number of exception entries, or a negative acb_status on error. */
int64_t acb_sincos_table_build_host(uint64_t *table_host, int64_t slots, float max_arg, int num_threads);

#ifdef __cplusplus
}
#endif
#endif /* ACOULAR_B200_H */
