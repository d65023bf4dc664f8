// Block-wise spectra generators (acoular/fprocess.py) on the device:
//   acb_spectra        RFFT.result (fprocess.py:35-181): windowed one-sided spectra of consecutive windows,
//                      laid out [window][bin][mic] (the reference's (n, num_freqs * num_channels) blocks),
//                      with its scaling rule (the inner bins doubled for 'energy' / 'amplitude', then the
//                      window factor) applied in the output precision as numpy does;
//   acb_auto_spectra   AutoPowerSpectra.result (fprocess.py:286-366): |X|^2 * scale;
//   acb_cross_spectra  CrossPowerSpectra.result (fprocess.py:369-467), calc_mode 'full': the per-snapshot
//                      CSM, upper triangle by calcCSM's FMA form (fastFuncs.py:19-58), the lower one its
//                      conjugate, times scale.
// The FFT is the CSM path's FP64 kernel (fft_window_kernel); these kernels only pack and combine.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "csm_internal.h"

namespace acb {

// ws [bin][window][mic] complex128 -> out [window][bin][mic]; bins 1 .. F-2 doubled when `twice`, then
// times `scale`, in the output precision (complex64: rounded first, then float32 products).
template <bool C64>
__global__ void spectra_pack_kernel(const double2 *__restrict__ ws, int F, int64_t nw, int M, double scale, int twice,
                                    void *__restrict__ out)
{
    const int64_t n = nw * F * M;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int m = (int)(i % M);
        const int f = (int)((i / M) % F);
        const int64_t w = i / ((int64_t)M * F);
        const double2 x = ws[((int64_t)f * nw + w) * M + m];
        const bool dbl = twice && f > 0 && f < F - 1;
        if (C64) {
            float xr = __double2float_rn(x.x), xi = __double2float_rn(x.y);
            if (dbl) {
                xr *= 2.0f;
                xi *= 2.0f;
            }
            const float s = __double2float_rn(scale);
            reinterpret_cast<float2 *>(out)[i] = make_float2(__fmul_rn(xr, s), __fmul_rn(xi, s));
        } else {
            double xr = x.x, xi = x.y;
            if (dbl) {
                xr *= 2.0;
                xi *= 2.0;
            }
            reinterpret_cast<double2 *>(out)[i] = make_double2(__dmul_rn(xr, scale), __dmul_rn(xi, scale));
        }
    }
}

// (X conj(X)).real * scale in the input's precision, stored as float64 or float32.
template <bool IN64, bool OUT32>
__global__ void auto_spectra_kernel(const void *__restrict__ in, int64_t n, double scale, void *__restrict__ out)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double v;
        if (IN64) {
            const double2 x = reinterpret_cast<const double2 *>(in)[i];
            v = __dmul_rn(__dadd_rn(__dmul_rn(x.x, x.x), __dmul_rn(x.y, x.y)), scale);
        } else {
            const float2 x = reinterpret_cast<const float2 *>(in)[i];
            v = (double)__fmul_rn(__fadd_rn(__fmul_rn(x.x, x.x), __fmul_rn(x.y, x.y)), __double2float_rn(scale));
        }
        if (OUT32) reinterpret_cast<float *>(out)[i] = __double2float_rn(v);
        else reinterpret_cast<double *>(out)[i] = v;
    }
}

// out[w][f][r][c] = scale * (r <= c ? U[r][c] : conj(U[c][r])), U[r][c] = conj(X[c]) X[r] in calcCSM's FMA form.
// One CTA per (window, bin): the M spectra values sit in shared memory, the M x M outputs are written
// in order (coalesced), indices in 32-bit arithmetic.
template <bool C64>
__global__ void __launch_bounds__(256) cross_spectra_kernel(const void *__restrict__ in, int M, double scale,
                                                            void *__restrict__ out)
{
    extern __shared__ double2 xs_d[];
    const int64_t wf = blockIdx.x;   // window * F + f
    const int mm = M * M;
    if (C64) {
        float2 *xs = reinterpret_cast<float2 *>(xs_d);
        const float2 *X = reinterpret_cast<const float2 *>(in) + wf * M;
        for (int m = threadIdx.x; m < M; m += blockDim.x) xs[m] = X[m];
        __syncthreads();
        const float s = __double2float_rn(scale);
        float2 *o = reinterpret_cast<float2 *>(out) + wf * mm;
        for (int e = threadIdx.x; e < mm; e += blockDim.x) {
            const int r = e / M, c = e - r * M;
            const int lo = min(r, c), hi = max(r, c);
            const float2 xr = xs[lo], xc = xs[hi];
            const float tr = xc.x, ti = -xc.y;
            const float ur = __fmaf_rn(-ti, xr.y, __fmaf_rn(tr, xr.x, 0.0f));
            float ui = __fmaf_rn(tr, xr.y, __fmaf_rn(ti, xr.x, 0.0f));
            if (r > c) ui = -ui;
            o[e] = make_float2(__fmul_rn(ur + 0.0f, s), __fmul_rn(ui + 0.0f, s));
        }
    } else {
        double2 *xs = xs_d;
        const double2 *X = reinterpret_cast<const double2 *>(in) + wf * M;
        for (int m = threadIdx.x; m < M; m += blockDim.x) xs[m] = X[m];
        __syncthreads();
        double2 *o = reinterpret_cast<double2 *>(out) + wf * mm;
        for (int e = threadIdx.x; e < mm; e += blockDim.x) {
            const int r = e / M, c = e - r * M;
            const int lo = min(r, c), hi = max(r, c);
            const double2 xr = xs[lo], xc = xs[hi];
            const double tr = xc.x, ti = -xc.y;
            const double ur = __fma_rn(-ti, xr.y, __fma_rn(tr, xr.x, 0.0));
            double ui = __fma_rn(tr, xr.y, __fma_rn(ti, xr.x, 0.0));
            if (r > c) ui = -ui;
            o[e] = make_double2(__dmul_rn(ur + 0.0, scale), __dmul_rn(ui + 0.0, scale));
        }
    }
}

static unsigned grid_for(int64_t n)
{
    const int64_t b = (n + 255) / 256;
    return (unsigned)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

}  // namespace acb

using namespace acb;

extern "C" {

size_t acb_spectra_workspace_bytes(int num_mics, int block_size, int64_t num_windows)
{
    if (num_mics <= 0 || block_size < 2 || num_windows < 0) return 0;
    const size_t spec = (size_t)(block_size / 2 + 1) * (size_t)num_windows * (size_t)num_mics * sizeof(double2);
    const size_t sc = fft_scratch_bytes(num_mics, block_size, num_windows);   // blocks above 16384 samples
    return sc ? (spec + 255) / 256 * 256 + sc : spec;
}

int acb_spectra(const void *samples, int sample_dtype, int64_t num_samples, int num_mics, int block_size, int hop,
                int64_t first_window, int64_t num_windows, const double *window, const void *twiddle, int precision,
                double scale, int double_inner, void *out, void *workspace, size_t workspace_bytes, void *stream)
{
    if (!samples || !window || !twiddle || !out) return ACB_ERR_ARG;
    if (sample_dtype != ACB_F32 && sample_dtype != ACB_F64) return ACB_ERR_ARG;
    if (precision != ACB_C128 && precision != ACB_C64) return ACB_ERR_ARG;
    if (num_mics <= 0 || hop <= 0 || first_window < 0 || num_windows < 0) return ACB_ERR_SHAPE;
    if (block_size < 16 || (block_size & (block_size - 1))) return ACB_ERR_SHAPE;
    if (block_size > 65536) return ACB_ERR_UNSUPPORTED;
    if (num_windows == 0) return ACB_OK;
    if ((first_window + num_windows - 1) * (int64_t)hop + block_size > num_samples) return ACB_ERR_SHAPE;
    if (num_windows > 65535) return ACB_ERR_SHAPE;
    const int F = block_size / 2 + 1;
    if (!workspace || workspace_bytes < acb_spectra_workspace_bytes(num_mics, block_size, num_windows))
        return ACB_ERR_WORKSPACE;
    cudaStream_t s = as_stream(stream);
    void *scratch = nullptr;
    if (fft_scratch_bytes(num_mics, block_size, num_windows))
        scratch = static_cast<uint8_t *>(workspace) +
                  ((size_t)F * (size_t)num_windows * (size_t)num_mics * sizeof(double2) + 255) / 256 * 256;
    int st = fft_launch(samples, sample_dtype, 0, num_mics, block_size, hop, first_window, num_windows, window,
                        reinterpret_cast<const double2 *>(twiddle), 0, F, workspace, 0, 0, 0, scratch, s);
    if (st) return st;
    const int64_t n = num_windows * F * num_mics;
    if (precision == ACB_C64)
        spectra_pack_kernel<true><<<grid_for(n), 256, 0, s>>>(static_cast<const double2 *>(workspace), F, num_windows,
                                                              num_mics, scale, double_inner, out);
    else
        spectra_pack_kernel<false><<<grid_for(n), 256, 0, s>>>(static_cast<const double2 *>(workspace), F,
                                                               num_windows, num_mics, scale, double_inner, out);
    return check_launch();
}

int acb_auto_spectra(const void *spectra, int64_t num_values, int precision, int out_float32, double scale, void *out,
                     void *stream)
{
    if (!spectra || !out) return ACB_ERR_ARG;
    if (precision != ACB_C128 && precision != ACB_C64) return ACB_ERR_ARG;
    if (num_values < 0) return ACB_ERR_SHAPE;
    if (num_values == 0) return ACB_OK;
    cudaStream_t s = as_stream(stream);
    const unsigned g = grid_for(num_values);
    if (precision == ACB_C128) {
        if (out_float32) auto_spectra_kernel<true, true><<<g, 256, 0, s>>>(spectra, num_values, scale, out);
        else auto_spectra_kernel<true, false><<<g, 256, 0, s>>>(spectra, num_values, scale, out);
    } else {
        if (out_float32) auto_spectra_kernel<false, true><<<g, 256, 0, s>>>(spectra, num_values, scale, out);
        else auto_spectra_kernel<false, false><<<g, 256, 0, s>>>(spectra, num_values, scale, out);
    }
    return check_launch();
}

int acb_cross_spectra(const void *spectra, int64_t num_windows, int num_freqs, int num_mics, int precision,
                      double scale, void *out, void *stream)
{
    if (!spectra || !out) return ACB_ERR_ARG;
    if (precision != ACB_C128 && precision != ACB_C64) return ACB_ERR_ARG;
    if (num_windows < 0 || num_freqs <= 0 || num_mics <= 0) return ACB_ERR_SHAPE;
    if (num_windows == 0) return ACB_OK;
    if ((int64_t)num_mics * num_mics > 0x7fffffffLL) return ACB_ERR_SHAPE;
    const int64_t nwf = num_windows * num_freqs;
    if (nwf > 0x7fffffffLL) return ACB_ERR_SHAPE;
    cudaStream_t s = as_stream(stream);
    const size_t smem = (size_t)num_mics * (precision == ACB_C64 ? sizeof(float2) : sizeof(double2));
    if (precision == ACB_C64) {
        cudaFuncSetAttribute(cross_spectra_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cross_spectra_kernel<true><<<(unsigned)nwf, 256, smem, s>>>(spectra, num_mics, scale, out);
    } else {
        cudaFuncSetAttribute(cross_spectra_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cross_spectra_kernel<false><<<(unsigned)nwf, 256, smem, s>>>(spectra, num_mics, scale, out);
    }
    return check_launch();
}

}  // extern "C"
