// Stage A: cross-spectral matrix estimation (PowerSpectra.calc_csm, acoular/spectra.py:366-416).
//
// Data flow per chunk of windows (all on the device, samples resident in HBM):
//   fft_window_kernel : samples [S][M] (f32|f64) -> window (FP64) -> rFFT (FP64, radix-2 in shared
//                       memory) -> spectra [bin][window][mic] rounded to the CSM precision
//   gram_kernel       : csm_upper[bin][r][c] += sum_w conj(X[bin][w][c]) * X[bin][w][r], r <= c,
//                       64x64 upper-triangular tiles, windows streamed through shared memory
//   finalize_kernel   : Hermitian completion and the 2/(N*sum(w^2)*num_blocks) scale
//
// The per-element accumulation runs sequentially over windows with the same two chained FMAs per
// component that the reference's fastmath calcCSM (acoular/fastFuncs.py:53-57) compiles to, so
// given identical spectra the Welch sums are bit-identical to the reference.
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <type_traits>

#include <cuda_bf16.h>

#include "common.cuh"
#include "csm_internal.h"
#include "tc_layout.cuh"

namespace acb {

static thread_local std::string g_last_cuda_error;

void set_cuda_error(cudaError_t e) { g_last_cuda_error = cudaGetErrorString(e); }

// ------------------------------------------------------------------------------------------------
// Windowed real FFT.  One CTA = one window x `mpb` mics; FFT of the N/2-point complex sequence
// z[j] = x[2j] + i x[2j+1], then the split into the N/2+1 real-input bins.
//
// The radix-2 DIT stages run in passes of up to three: a thread loads the 2^s points that s
// consecutive stages combine among themselves, applies the s stages' butterflies in registers
// (same operands, twiddles and operation order as one stage at a time, so the spectra are the
// same bits) and stores them back: one shared-memory round trip and one barrier per pass instead
// of per stage.
// ------------------------------------------------------------------------------------------------
// Shared-memory slot of point j of a mic's sequence: one padding slot after every 8 points, so that
// 8 threads reading 16-byte points 8 apart (the first pass) or 64 apart hit different banks.
__device__ __forceinline__ int zp(int j) { return j + (j >> 3); }
// padded length of one mic's sequence of H points (an odd number of 16-byte slots past the padding)
__host__ __device__ constexpr int fft_stride(int H) { return H + (H >> 3) + 1; }

// s (1..3) consecutive radix-2 DIT stages of lengths L1 = 2^(sg + 1), 2 L1, .., on a bit-reversed
// sequence z of H points (one mic).  Task `task` in [0, H / 2^s) owns points base + t * L1/2,
// t = 0 .. 2^s - 1.  All lengths are powers of two (logN = log2 N): shifts and masks index the
// points and the twiddles W_N^e.
template <int S>
__device__ __forceinline__ void fft_pass(double2 *__restrict__ z, int sg, int task, int logN,
                                         const double2 *__restrict__ tw)
{
    const int half1 = 1 << sg;
    const int base = ((task >> sg) << (sg + S)) + (task & (half1 - 1));   // the pass spans 2^(sg + S) points
    double2 v[1 << S];
#pragma unroll
    for (int t = 0; t < (1 << S); ++t) v[t] = z[zp(base + t * half1)];
#pragma unroll
    for (int q = 0; q < S; ++q) {
        const int hf = half1 << q;                       // half the stage length L = 2^(sg + 1 + q)
        const int shift = logN - (sg + 1 + q);           // W_L^i = W_N^(i N / L)
#pragma unroll
        for (int t = 0; t < (1 << S); ++t) {
            if (t & (1 << q)) continue;
            const int i0 = base + t * half1;
            const double2 w = __ldg(tw + ((i0 & (hf - 1)) << shift));
            const double2 b = v[t + (1 << q)];
            const double br = b.x * w.x - b.y * w.y;
            const double bi = b.x * w.y + b.y * w.x;
            const double2 a = v[t];
            v[t] = make_double2(a.x + br, a.y + bi);
            v[t + (1 << q)] = make_double2(a.x - br, a.y - bi);
        }
    }
#pragma unroll
    for (int t = 0; t < (1 << S); ++t) z[zp(base + t * half1)] = v[t];
}

// Output forms of the spectra (OUT): complex128 or complex64 [bin][window][mic] for the FP64 /
// FP32 Gram; or the tensor-core Gram's operand tiles, TF32 (OUT_TF32) or split BF16 hi + lo
// (OUT_BF16), 32 x 32 tiles [bin][window/32][component/32] with component 2m = Re, 2m + 1 = Im of
// mic m (row) and the window within the chunk (column); `R` row tiles per bin and window block,
// `KC` window blocks; BF16 lo tiles start `lo_elems` elements after the hi tiles.
enum { OUT_C128 = 0, OUT_C64 = 1, OUT_TF32 = 2, OUT_BF16 = 3 };

// Store bin `b` (relative to bin_lo) of window `wi` (within the chunk of nw windows), mic m, in form OUT.
template <int OUT>
__device__ __forceinline__ void put_bin(void *__restrict__ out, int64_t nw, int wi, int M, int m, int b, double xr,
                                        double xi, int R, int KC, int64_t lo_elems)
{
    if (OUT <= OUT_C64) {
        const int64_t o = ((int64_t)b * nw + wi) * M + m;
        if (OUT == OUT_C64)
            reinterpret_cast<float2 *>(out)[o] = make_float2(__double2float_rn(xr), __double2float_rn(xi));
        else reinterpret_cast<double2 *>(out)[o] = make_double2(xr, xi);
    } else {
        const int rowc = 2 * m, col = wi & 31;
        const int64_t tile = ((int64_t)b * KC + (wi >> 5)) * R + (rowc >> 5);
        const float fr = __double2float_rn(xr), fi = __double2float_rn(xi);
        if (OUT == OUT_TF32) {
            uint32_t *t = reinterpret_cast<uint32_t *>(out) + tile * 1024;
            t[tile_off_tf32(rowc & 31, col)] = tf32_bits(fr);
            t[tile_off_tf32((rowc & 31) + 1, col)] = tf32_bits(fi);
        } else {
            __nv_bfloat16 *t = reinterpret_cast<__nv_bfloat16 *>(out) + tile * 1024;
            const __nv_bfloat16 hr = __float2bfloat16_rn(fr), hi = __float2bfloat16_rn(fi);
            const int o0 = tile_off(rowc & 31, col), o1 = tile_off((rowc & 31) + 1, col);
            t[o0] = hr;
            t[o1] = hi;
            t[lo_elems + o0] = __float2bfloat16_rn(fr - __bfloat162float(hr));
            t[lo_elems + o1] = __float2bfloat16_rn(fi - __bfloat162float(hi));
        }
    }
}

template <typename TS, int OUT>
__global__ void __launch_bounds__(256) fft_window_kernel(const TS *__restrict__ samples, int M, int N, int hop,
                                                         int64_t w0, int64_t nw, int mpb,
                                                         const double *__restrict__ window,
                                                         const double2 *__restrict__ tw, int bin_lo, int nbins,
                                                         void *__restrict__ out, int R, int KC, int64_t lo_elems)
{
    extern __shared__ double2 zs[];  // [mpb][fft_stride(H)], point j of mic ml at zs[ml * stride + zp(j)]
    const int H = N >> 1;
    int logH = 0;
    while ((1 << logH) < H) ++logH;
    const int64_t w = w0 + blockIdx.y;
    const int m0 = blockIdx.x * mpb;
    const int nm = min(mpb, M - m0);
    const TS *src = samples + (w * (int64_t)hop) * M;

    // load + window + bit-reversed placement
    for (int idx = threadIdx.x; idx < H * nm; idx += blockDim.x) {
        const int ml = idx % nm;
        const int j = idx / nm;
        const double x0 = (double)src[(int64_t)(2 * j) * M + m0 + ml] * window[2 * j];
        const double x1 = (double)src[(int64_t)(2 * j + 1) * M + m0 + ml] * window[2 * j + 1];
        const int jr = (int)(__brev((unsigned)j) >> (32 - logH));
        zs[ml * fft_stride(H) + zp(logH ? jr : 0)] = make_double2(x0, x1);
    }
    __syncthreads();

    // radix-2 DIT stages, up to three per pass
    for (int st = 0; st < logH;) {
        const int S = logH - st >= 3 ? 3 : logH - st;
        const int logT = logH - S;   // H / 2^S tasks per mic
        for (int idx = threadIdx.x; idx < nm << logT; idx += blockDim.x) {
            const int ml = idx >> logT;
            const int task = idx & ((1 << logT) - 1);
            if (S == 3) fft_pass<3>(zs + ml * fft_stride(H), st, task, logH + 1, tw);
            else if (S == 2) fft_pass<2>(zs + ml * fft_stride(H), st, task, logH + 1, tw);
            else fft_pass<1>(zs + ml * fft_stride(H), st, task, logH + 1, tw);
        }
        __syncthreads();
        st += S;
    }

    // real-input split: X[k] = E + W^k O,  E = (Z[k] + conj(Z[H-k]))/2,  O = -i (Z[k] - conj(Z[H-k]))/2
    for (int idx = threadIdx.x; idx < nbins * nm; idx += blockDim.x) {
        const int ml = idx % nm;
        const int k = bin_lo + idx / nm;
        const double2 *z = zs + ml * fft_stride(H);
        const double2 zk = z[zp(k % H)];
        const double2 zc = z[zp((H - k % H) % H)];
        const double er = 0.5 * (zk.x + zc.x), ei = 0.5 * (zk.y - zc.y);
        const double orr = 0.5 * (zk.y + zc.y), oi = -0.5 * (zk.x - zc.x);
        double2 wk;
        if (k < H) wk = tw[k];
        else wk = make_double2(-1.0, 0.0);
        const double xr = er + (wk.x * orr - wk.y * oi);
        const double xi = ei + (wk.x * oi + wk.y * orr);
        put_bin<OUT>(out, nw, (int)blockIdx.y, M, m0 + ml, k - bin_lo, xr, xi, R, KC, lo_elems);
    }
}

// ------------------------------------------------------------------------------------------------
// Tensor-core operand tiles straight from the samples, four windows per CTA (fft4_tc_kernel).
// The tile layout is K-major: a 16-byte core-matrix row holds 4 consecutive windows (TF32) or 8
// (BF16) of one spectrum component, so a CTA that transforms 4 consecutive windows of `mpb` mics
// stores whole 16-byte rows (TF32) or half rows (BF16) instead of one 4-byte value per window.
// The transform runs in FP32 (the operands are rounded to TF32 or split into BF16 hi + lo right
// after it, so FP64 arithmetic buys nothing): complex points are 8 bytes, half the shared-memory
// traffic of the FP64 transform.  Padded windows (>= the chunk's count, up to 32 KC) and padded
// mics (up to 16 R) are written as zeros, so the operand buffer needs no clearing beforehand.
// ------------------------------------------------------------------------------------------------
// Shared-memory slot of point j: one padding slot per 16 points (8-byte points), so that the passes'
// strided accesses spread over the banks.
__device__ __forceinline__ int zpf(int j) { return j + (j >> 4); }
// Padded length of one sequence: at least H + H/16 slots and congruent to 32 / mpb modulo 16.  In the real
// split a warp reads Z[k] of mpb mics x 32 / mpb consecutive bins; with that stride the mics' slots fall
// on different bank pairs (with the stride 1 modulo 16 of a first version, 4 mics x 8 bins put up to 4
// threads on one bank pair).
__host__ __device__ constexpr int fft_stride_f(int H, int mpb)
{
    return H + (H >> 4) + ((((32 / mpb) & 15) - (H + (H >> 4))) & 15);
}

// s (1..3) consecutive radix-2 DIT stages, the first of length 2^(sg + 1), on a bit-reversed FP32
// sequence (see fft_pass).  The twiddles come from a shared-memory table in stage order: the stage of
// length L = 2 hf reads W_L^i (i < hf) at tws[hf + i], so consecutive threads read consecutive
// entries (the natural-order table read with the stride N / L put up to 16 threads on one bank).  The
// entries are the FP32 roundings of the same W_N^e as the natural-order table.  All lengths are powers
// of two, so the index arithmetic is shifts and masks.
template <int S>
__device__ __forceinline__ void fft_pass_f(float2 *__restrict__ z, int sg, int task, const float2 *__restrict__ tws)
{
    const int half1 = 1 << sg;
    const int base = ((task >> sg) << (sg + S)) + (task & (half1 - 1));
    float2 v[1 << S];
#pragma unroll
    for (int t = 0; t < (1 << S); ++t) v[t] = z[zpf(base + t * half1)];
    // the twiddle of point base + t half1 at stage q is entry (task mod half1) + (t mod 2^q) half1 of the
    // stage's table: 2^q distinct values, each read once
    const int tb = task & (half1 - 1);
#pragma unroll
    for (int q = 0; q < S; ++q) {
        const int hf = half1 << q;                       // half the stage length L = 2^(sg + 1 + q)
        float2 wq[1 << (S - 1)];
#pragma unroll
        for (int u = 0; u < (1 << q); ++u) wq[u] = tws[hf + tb + u * half1];
#pragma unroll
        for (int t = 0; t < (1 << S); ++t) {
            if (t & (1 << q)) continue;
            const float2 w = wq[t & ((1 << q) - 1)];
            const float2 b = v[t + (1 << q)];
            const float br = b.x * w.x - b.y * w.y;
            const float bi = b.x * w.y + b.y * w.x;
            const float2 a = v[t];
            v[t] = make_float2(a.x + br, a.y + bi);
            v[t + (1 << q)] = make_float2(a.x - br, a.y - bi);
        }
    }
#pragma unroll
    for (int t = 0; t < (1 << S); ++t) z[zpf(base + t * half1)] = v[t];
}

constexpr int FFT4_WIN = 4;   // windows per CTA

// V consecutive samples of one row, as float (V = 1, 2 or 4; the address is aligned to the vector)
template <int V>
__device__ __forceinline__ void ld_row(const float *__restrict__ p, float (&x)[V])
{
    if (V == 4) {
        const float4 u = __ldg(reinterpret_cast<const float4 *>(p));
        x[0] = u.x;
        x[1] = u.y;
        x[2] = u.z;
        x[3] = u.w;
    } else if (V == 2) {
        const float2 u = __ldg(reinterpret_cast<const float2 *>(p));
        x[0] = u.x;
        x[1] = u.y;
    } else {
        x[0] = __ldg(p);
    }
}
template <int V>
__device__ __forceinline__ void ld_row(const double *__restrict__ p, float (&x)[V])
{
    if (V == 1) {
        x[0] = (float)__ldg(p);
    } else {
#pragma unroll
        for (int e = 0; e < V; e += 2) {
            const double2 u = __ldg(reinterpret_cast<const double2 *>(p + e));
            x[e] = (float)u.x;
            x[e + 1] = (float)u.y;
        }
    }
}

// Load, window and bit-reversed placement of the CTA's 4 windows x mpb mics: one thread per (window,
// group of V mics, point j), j fastest, so that a warp's stores into the bit-reversed slots of one
// sequence spread over the banks, and each thread loads rows 2j and 2j + 1 as one vector of V mics.
// Windows past the chunk and padding mics are zeros (M % V == 0: a group is all in or all out).
template <typename TS, int V>
__device__ __forceinline__ void fft4_load(const TS *__restrict__ samples, int M, int hop, int64_t w0, int64_t nw,
                                          int wg, int m0, int mpb, int H, int logH, int st,
                                          const float *__restrict__ wf, float2 *__restrict__ zs)
{
    constexpr int logV = V == 4 ? 2 : (V == 2 ? 1 : 0);
    int logG = 0;
    while ((V << logG) < mpb) ++logG;                          // mpb / V groups
    const int total = FFT4_WIN * H << logG;
#pragma unroll 4
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int j = idx & (H - 1);
        const int mg = (idx >> logH) & ((1 << logG) - 1);
        const int wi = idx >> (logH + logG);
        const int64_t w = (int64_t)wg * FFT4_WIN + wi;
        const int m = m0 + (mg << logV);
        float x0[V], x1[V];
        if (w < nw && m < M) {
            const TS *src = samples + ((w0 + w) * (int64_t)hop + 2 * j) * M + m;
            ld_row<V>(src, x0);
            ld_row<V>(src + M, x1);
        } else {
#pragma unroll
            for (int e = 0; e < V; ++e) x0[e] = x1[e] = 0.f;
        }
        const float a0 = wf[2 * j], a1 = wf[2 * j + 1];
        const int jr = logH ? (int)(__brev((unsigned)j) >> (32 - logH)) : 0;
        float2 *z = zs + (wi * mpb + (mg << logV)) * st + zpf(jr);
#pragma unroll
        for (int e = 0; e < V; ++e) z[e * st] = make_float2(x0[e] * a0, x1[e] * a1);
    }
}

template <typename TS, int OUT>
__global__ void __launch_bounds__(256) fft4_tc_kernel(const TS *__restrict__ samples, int M, int N, int hop, int64_t w0,
                                                      int64_t nw, int mpb, int vw, const double *__restrict__ window,
                                                      const double2 *__restrict__ tw, int bin_lo, int nbins,
                                                      void *__restrict__ out, int R, int KC, int64_t lo_elems)
{
    extern __shared__ __align__(16) uint8_t fsm[];
    const int H = N >> 1;
    const int st = fft_stride_f(H, mpb);
    float2 *zs = reinterpret_cast<float2 *>(fsm);                 // [FFT4_WIN][mpb][st]
    float2 *tws = zs + FFT4_WIN * mpb * st;                       // [H] twiddles in stage order (fft_pass_f)
    float *wf = reinterpret_cast<float *>(tws + H);               // [N]
    int logH = 0, logP = 0;
    while ((1 << logH) < H) ++logH;
    while ((1 << logP) < mpb) ++logP;                              // mpb is a power of two
    const int wg = blockIdx.y;                                     // windows 4 wg .. 4 wg + 3 of the chunk
    const int m0 = blockIdx.x * mpb;
    for (int i = threadIdx.x + 1; i < H; i += blockDim.x) {
        // i = hf + r, hf the largest power of two <= i: W_{2 hf}^r = W_N^(r H / hf), N = 2 H
        const int lhf = 31 - __clz(i);
        const double2 u = tw[(i - (1 << lhf)) << (logH - lhf)];
        tws[i] = make_float2((float)u.x, (float)u.y);
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) wf[i] = (float)window[i];
    __syncthreads();

    if (vw == 4) fft4_load<TS, 4>(samples, M, hop, w0, nw, wg, m0, mpb, H, logH, st, wf, zs);
    else if (vw == 2) fft4_load<TS, 2>(samples, M, hop, w0, nw, wg, m0, mpb, H, logH, st, wf, zs);
    else fft4_load<TS, 1>(samples, M, hop, w0, nw, wg, m0, mpb, H, logH, st, wf, zs);
    __syncthreads();

    // radix-2 DIT stages, up to three per pass, over all 4 mpb sequences
    const int nseq = FFT4_WIN * mpb;
    for (int sg = 0; sg < logH;) {
        const int S = logH - sg >= 3 ? 3 : logH - sg;
        const int logT = logH - S;                                 // H / 2^S tasks per sequence
        for (int idx = threadIdx.x; idx < nseq << logT; idx += blockDim.x) {
            const int q = idx >> logT;
            const int task = idx & ((1 << logT) - 1);
            if (S == 3) fft_pass_f<3>(zs + q * st, sg, task, tws);
            else if (S == 2) fft_pass_f<2>(zs + q * st, sg, task, tws);
            else fft_pass_f<1>(zs + q * st, sg, task, tws);
        }
        __syncthreads();
        sg += S;
    }

    // real split of each bin for the 4 windows, then one store per tile row (Re row 2m, Im row 2m+1)
    const int col0 = (wg * FFT4_WIN) & 31;
    const int64_t kc = (wg * FFT4_WIN) >> 5;
    for (int idx = threadIdx.x; idx < nbins * mpb; idx += blockDim.x) {
        const int ml = idx & (mpb - 1);
        const int b = idx >> logP;
        const int k = bin_lo + b;
        const int kh = k & (H - 1), kc2 = (H - kh) & (H - 1);
        float2 wk = make_float2(-1.f, 0.f);
        if (k < H) {
            const double2 t = __ldg(tw + k);
            wk = make_float2((float)t.x, (float)t.y);
        }
        float xr[FFT4_WIN], xi[FFT4_WIN];
#pragma unroll
        for (int wi = 0; wi < FFT4_WIN; ++wi) {
            const float2 *z = zs + (wi * mpb + ml) * st;
            const float2 zk = z[zpf(kh)], zc = z[zpf(kc2)];
            const float er = 0.5f * (zk.x + zc.x), ei = 0.5f * (zk.y - zc.y);
            const float orr = 0.5f * (zk.y + zc.y), oi = -0.5f * (zk.x - zc.x);
            xr[wi] = er + (wk.x * orr - wk.y * oi);
            xi[wi] = ei + (wk.x * oi + wk.y * orr);
        }
        const int m = m0 + ml;                                    // padded mics carry zeros
        const int rowc = 2 * m;
        const int64_t tile = ((int64_t)b * KC + kc) * R + (rowc >> 5);
        const int r0 = rowc & 31;
        if (OUT == OUT_TF32) {
            uint32_t *t = reinterpret_cast<uint32_t *>(out) + tile * 1024;
            *reinterpret_cast<uint4 *>(t + tile_off_tf32(r0, col0)) =
                make_uint4(tf32_bits(xr[0]), tf32_bits(xr[1]), tf32_bits(xr[2]), tf32_bits(xr[3]));
            *reinterpret_cast<uint4 *>(t + tile_off_tf32(r0 + 1, col0)) =
                make_uint4(tf32_bits(xi[0]), tf32_bits(xi[1]), tf32_bits(xi[2]), tf32_bits(xi[3]));
        } else {
            __nv_bfloat16 *t = reinterpret_cast<__nv_bfloat16 *>(out) + tile * 1024;
#pragma unroll
            for (int part = 0; part < 2; ++part) {   // Re row, Im row
                const float *x = part ? xi : xr;
                uint32_t hv[2], lv[2];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const __nv_bfloat162 hi = __floats2bfloat162_rn(x[2 * h], x[2 * h + 1]);
                    const float2 hf = __bfloat1622float2(hi);
                    const __nv_bfloat162 lo = __floats2bfloat162_rn(x[2 * h] - hf.x, x[2 * h + 1] - hf.y);
                    hv[h] = *reinterpret_cast<const uint32_t *>(&hi);
                    lv[h] = *reinterpret_cast<const uint32_t *>(&lo);
                }
                const int o = tile_off(r0 + part, col0);
                *reinterpret_cast<uint2 *>(t + o) = make_uint2(hv[0], hv[1]);
                *reinterpret_cast<uint2 *>(t + lo_elems + o) = make_uint2(lv[0], lv[1]);
            }
        }
    }
}

// Mics per CTA of fft4_tc_kernel: about 72 KB of FP32 sequences (2 to 3 CTAs per SM), power of two
// <= 16 (so that the 16 R padded mics split evenly); 0 if even one mic's 4 windows do not fit.
static int fft4_mics_per_block(int N)
{
    const size_t tables = (size_t)(N / 2) * sizeof(float2) + (size_t)N * sizeof(float);
    if ((size_t)FFT4_WIN * fft_stride_f(N / 2, 1) * sizeof(float2) + tables >= 200 * 1024) return 0;
    int mpb = 16;
    while (mpb > 1 && (size_t)mpb * FFT4_WIN * fft_stride_f(N / 2, mpb) * sizeof(float2) > 72 * 1024) mpb >>= 1;
    return mpb;
}

bool fft_tiles_written_whole(int block_size) { return fft4_mics_per_block(block_size) > 0; }

static size_t fft4_smem_bytes(int N, int mpb)
{
    return (size_t)FFT4_WIN * mpb * fft_stride_f(N / 2, mpb) * sizeof(float2) + (size_t)(N / 2) * sizeof(float2) +
           (size_t)N * sizeof(float);
}

// ------------------------------------------------------------------------------------------------
// Large blocks (N > 16384): one mic's N/2-point sequence no longer fits a CTA's shared memory.  It is
// split by decimation in time into D = N / 16384 interleaved sub-sequences z[d + D i] of 8192 points:
// fft_sub_kernel transforms each one in shared memory with the passes above (sub-spectra Y_d to a
// scratch region [window][mic][d][8192]), and fft_combine_kernel forms, for the requested bins only,
// Z[k] = sum_d W_H^{d k} Y_d[k mod 8192] and Z[H - k] before the same real split.
// ------------------------------------------------------------------------------------------------
constexpr int FFT_MAX_N = 16384;                 // largest block transformed by one CTA
constexpr int FFT_SUB_H = FFT_MAX_N / 2;         // points of each sub-sequence of a larger block

size_t fft_scratch_bytes(int num_mics, int block_size, int64_t num_windows)
{
    if (block_size <= FFT_MAX_N) return 0;
    return (size_t)num_windows * (size_t)num_mics * (size_t)(block_size / 2) * sizeof(double2);
}

template <typename TS>
__global__ void __launch_bounds__(256) fft_sub_kernel(const TS *__restrict__ samples, int M, int N, int hop,
                                                      int64_t w0, const double *__restrict__ window,
                                                      const double2 *__restrict__ tw, double2 *__restrict__ scratch)
{
    extern __shared__ double2 zs[];   // [zp(j)], j < FFT_SUB_H
    const int D = (N >> 1) / FFT_SUB_H;
    int logHs = 0;
    while ((1 << logHs) < FFT_SUB_H) ++logHs;
    const int64_t wi = blockIdx.y;
    const int m = blockIdx.x, d = blockIdx.z;
    const TS *src = samples + ((w0 + wi) * (int64_t)hop) * M + m;
    for (int i = threadIdx.x; i < FFT_SUB_H; i += blockDim.x) {
        const int64_t j = d + (int64_t)D * i;    // complex point j = (x[2j], x[2j+1])
        const double x0 = (double)src[(2 * j) * M] * window[2 * j];
        const double x1 = (double)src[(2 * j + 1) * M] * window[2 * j + 1];
        zs[zp((int)(__brev((unsigned)i) >> (32 - logHs)))] = make_double2(x0, x1);
    }
    __syncthreads();
    int logN = 0;
    while ((1 << logN) < N) ++logN;
    for (int st = 0; st < logHs;) {
        const int S = logHs - st >= 3 ? 3 : logHs - st;
        const int ntask = FFT_SUB_H >> S;
        for (int task = threadIdx.x; task < ntask; task += blockDim.x) {
            if (S == 3) fft_pass<3>(zs, st, task, logN, tw);
            else if (S == 2) fft_pass<2>(zs, st, task, logN, tw);
            else fft_pass<1>(zs, st, task, logN, tw);
        }
        __syncthreads();
        st += S;
    }
    double2 *dst = scratch + ((wi * M + m) * D + d) * (int64_t)FFT_SUB_H;
    for (int k = threadIdx.x; k < FFT_SUB_H; k += blockDim.x) dst[k] = zs[zp(k)];
}

// W_N^e for any integer exponent e (the table holds e < N/2; W_N^{e + N/2} = -W_N^e)
__device__ __forceinline__ double2 twiddle_any(const double2 *__restrict__ tw, int N, int64_t e)
{
    e %= N;
    const int h = N >> 1;
    if (e < h) return tw[e];
    const double2 t = tw[e - h];
    return make_double2(-t.x, -t.y);
}

// Z[k] of one (window, mic) from its D sub-spectra
__device__ __forceinline__ double2 combine_point(const double2 *__restrict__ y, int N, int D, int k,
                                                 const double2 *__restrict__ tw)
{
    const int kk = k % FFT_SUB_H;
    double zr = 0.0, zi = 0.0;
    for (int d = 0; d < D; ++d) {
        const double2 v = y[(int64_t)d * FFT_SUB_H + kk];
        const double2 w = twiddle_any(tw, N, 2 * (int64_t)d * k);   // W_H^{d k} = W_N^{2 d k}
        zr += v.x * w.x - v.y * w.y;
        zi += v.x * w.y + v.y * w.x;
    }
    return make_double2(zr, zi);
}

template <int OUT>
__global__ void __launch_bounds__(256) fft_combine_kernel(const double2 *__restrict__ scratch, int M, int N,
                                                          int64_t nw, int bin_lo, int nbins,
                                                          const double2 *__restrict__ tw, void *__restrict__ out,
                                                          int R, int KC, int64_t lo_elems)
{
    const int H = N >> 1, D = H / FFT_SUB_H;
    const int wi = blockIdx.y;
    const int k = bin_lo + blockIdx.x;
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        const double2 *y = scratch + ((int64_t)wi * M + m) * D * FFT_SUB_H;
        const double2 zk = combine_point(y, N, D, k % H, tw);
        const double2 zc = combine_point(y, N, D, (H - k % H) % H, tw);
        const double er = 0.5 * (zk.x + zc.x), ei = 0.5 * (zk.y - zc.y);
        const double orr = 0.5 * (zk.y + zc.y), oi = -0.5 * (zk.x - zc.x);
        const double2 wk = k < H ? tw[k] : make_double2(-1.0, 0.0);
        const double xr = er + (wk.x * orr - wk.y * oi);
        const double xi = ei + (wk.x * oi + wk.y * orr);
        put_bin<OUT>(out, nw, wi, M, m, k - bin_lo, xr, xi, R, KC, lo_elems);
    }
}

// ------------------------------------------------------------------------------------------------
// Welch Gram accumulation, upper-triangular 64x64 tiles; thread (tx, ty) owns rows ty+16i and
// columns tx+16j of the tile (conflict-free shared-memory reads, coalesced stores).
// ------------------------------------------------------------------------------------------------
template <bool C64>
struct GramT {
    using V = typename std::conditional<C64, float2, double2>::type;
    using S = typename std::conditional<C64, float, double>::type;
};

__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

constexpr int GT = 64;   // tile edge
constexpr int GKC = 16;  // windows per shared-memory stage

template <bool C64>
__global__ void __launch_bounds__(256) gram_kernel(const void *__restrict__ spec_, int M, int64_t nw,
                                                   void *__restrict__ csm_)
{
    using V = typename GramT<C64>::V;
    using S = typename GramT<C64>::S;
    __shared__ V xr_s[GKC][GT];
    __shared__ V xc_s[GKC][GT];
    const V *spec = reinterpret_cast<const V *>(spec_);
    V *csm = reinterpret_cast<V *>(csm_);

    // upper-triangular tile index -> (ti, tj), ti <= tj
    const int T = (M + GT - 1) / GT;
    int t = blockIdx.x, ti = 0;
    while (t >= T - ti) {
        t -= T - ti;
        ++ti;
    }
    const int tj = ti + t;
    const int f = blockIdx.y;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int r0 = ti * GT, c0 = tj * GT;

    S acc_re[4][4], acc_im[4][4];
    V *base = csm + (int64_t)f * M * M;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = r0 + ty + 16 * i, c = c0 + tx + 16 * j;
            V v = {0, 0};
            if (r < M && c < M && r <= c) v = base[(int64_t)r * M + c];
            acc_re[i][j] = v.x;
            acc_im[i][j] = v.y;
        }

    const V *sp = spec + (int64_t)f * nw * M;
    for (int64_t k0 = 0; k0 < nw; k0 += GKC) {
        const int kc = (int)((nw - k0) < GKC ? (nw - k0) : GKC);
        for (int idx = threadIdx.x; idx < GKC * GT; idx += blockDim.x) {
            const int kk = idx / GT, m = idx % GT;
            V a = {0, 0}, b = {0, 0};
            if (kk < kc) {
                if (r0 + m < M) a = sp[(k0 + kk) * M + r0 + m];
                if (c0 + m < M) b = sp[(k0 + kk) * M + c0 + m];
            }
            xr_s[kk][m] = a;
            xc_s[kk][m] = b;
        }
        __syncthreads();
        for (int kk = 0; kk < kc; ++kk) {
            V xr[4], xc[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) xr[i] = xr_s[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) xc[j] = xc_s[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    // temp = conj(X[c]) = (tr, ti); csm += temp * X[r]
                    const S tr = xc[j].x, tim = -xc[j].y;
                    acc_re[i][j] = fma_rn(-tim, xr[i].y, fma_rn(tr, xr[i].x, acc_re[i][j]));
                    acc_im[i][j] = fma_rn(tr, xr[i].y, fma_rn(tim, xr[i].x, acc_im[i][j]));
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = r0 + ty + 16 * i, c = c0 + tx + 16 * j;
            if (r < M && c < M && r <= c) {
                V v;
                v.x = acc_re[i][j];
                v.y = acc_im[i][j];
                base[(int64_t)r * M + c] = v;
            }
        }
}

// ------------------------------------------------------------------------------------------------
// Hermitian completion + scale, 32x32 tiles through shared memory for the transposed half.
// ------------------------------------------------------------------------------------------------
template <bool C64>
__global__ void __launch_bounds__(256) finalize_kernel(const void *__restrict__ up_, int M, double scale,
                                                       double2 *__restrict__ out)
{
    using V = typename GramT<C64>::V;
    __shared__ double2 tile[32][33];
    const V *up = reinterpret_cast<const V *>(up_);
    const int f = blockIdx.z;
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    const V *ub = up + (int64_t)f * M * M;
    double2 *ob = out + (int64_t)f * M * M;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    if (r0 <= c0 + 31) {
        // tile touches the upper triangle: direct read (lower part of a diagonal tile handled below)
        for (int i = ty; i < 32; i += 8) {
            const int r = r0 + i, c = c0 + tx;
            if (r < M && c < M && r <= c) {
                const V v = ub[(int64_t)r * M + c];
                ob[(int64_t)r * M + c] = make_double2((double)v.x * scale, (double)v.y * scale);
            }
        }
    }
    if (c0 <= r0 + 31) {
        // lower elements (r > c) read transposed from upper[c][r]
        for (int i = ty; i < 32; i += 8) {
            const int c = c0 + i, r = r0 + tx;  // coalesced read along r of upper[c][*]
            double2 v = make_double2(0.0, 0.0);
            if (r < M && c < M && c < r) {
                const V u = ub[(int64_t)c * M + r];
                v = make_double2((double)u.x, (double)u.y);
            }
            tile[i][tx] = v;
        }
        __syncthreads();
        for (int i = ty; i < 32; i += 8) {
            const int r = r0 + i, c = c0 + tx;
            if (r < M && c < M && r > c) {
                const double2 u = tile[tx][i];
                ob[(int64_t)r * M + c] = make_double2(u.x * scale, -u.y * scale);
            }
        }
    }
}

// Mics per CTA: at most 32 KB of complex doubles (N/2 per mic), so that several CTAs share an SM
// and hide each other's barrier and FP64 latency; one mic for N > 4096.
static int fft_mics_per_block(int N)
{
    const int cap = 4096 / N;
    return cap >= 16 ? 16 : (cap < 1 ? 1 : cap);
}

// Launch the windowed FFT of `num_windows` windows in output form `out_form`.
int fft_launch(const void *samples, int sample_dtype, int out_form, int num_mics, int block_size, int hop,
               int64_t first_window, int64_t num_windows, const double *window, const double2 *tw, int bin_lo,
               int num_bins, void *out, int R, int KC, int64_t lo_elems, void *scratch, cudaStream_t s)
{
    if (block_size > FFT_MAX_N) {
        if (!scratch) return ACB_ERR_WORKSPACE;
        double2 *sc = reinterpret_cast<double2 *>(scratch);
        const dim3 gs((unsigned)num_mics, (unsigned)num_windows, (unsigned)(block_size / 2 / FFT_SUB_H));
        const size_t smem = (size_t)fft_stride(FFT_SUB_H) * sizeof(double2);
        if (sample_dtype == ACB_F32) {
            cudaFuncSetAttribute(fft_sub_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            fft_sub_kernel<float><<<gs, 256, smem, s>>>(reinterpret_cast<const float *>(samples), num_mics, block_size,
                                                        hop, first_window, window, tw, sc);
        } else {
            cudaFuncSetAttribute(fft_sub_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            fft_sub_kernel<double><<<gs, 256, smem, s>>>(reinterpret_cast<const double *>(samples), num_mics,
                                                         block_size, hop, first_window, window, tw, sc);
        }
        int st = check_launch();
        if (st) return st;
        const dim3 gc((unsigned)num_bins, (unsigned)num_windows);
        const int nt = num_mics < 256 ? (num_mics + 31) / 32 * 32 : 256;
        switch (out_form) {
        case OUT_C128: fft_combine_kernel<OUT_C128><<<gc, nt, 0, s>>>(sc, num_mics, block_size, num_windows, bin_lo,
                                                                      num_bins, tw, out, R, KC, lo_elems); break;
        case OUT_C64: fft_combine_kernel<OUT_C64><<<gc, nt, 0, s>>>(sc, num_mics, block_size, num_windows, bin_lo,
                                                                    num_bins, tw, out, R, KC, lo_elems); break;
        case OUT_TF32: fft_combine_kernel<OUT_TF32><<<gc, nt, 0, s>>>(sc, num_mics, block_size, num_windows, bin_lo,
                                                                      num_bins, tw, out, R, KC, lo_elems); break;
        default: fft_combine_kernel<OUT_BF16><<<gc, nt, 0, s>>>(sc, num_mics, block_size, num_windows, bin_lo,
                                                                num_bins, tw, out, R, KC, lo_elems); break;
        }
        return check_launch();
    }
    if (out_form >= OUT_TF32) {
        const int mpb4 = fft4_mics_per_block(block_size);
        if (mpb4 > 0) {
            // every tile row (16 R padded mics) and column (32 KC padded windows) is written
            const dim3 g4((unsigned)(R * 16 / mpb4), (unsigned)(KC * 32 / FFT4_WIN));
            const size_t smem4 = fft4_smem_bytes(block_size, mpb4);
            // vector width of the sample loads: V mics of a row at once where M and the base allow it
            const size_t es = sample_dtype == ACB_F32 ? 4 : 8;
            int vw = 1;
            for (int v = 4; v >= 2 && vw == 1; v >>= 1)
                if (v <= mpb4 && num_mics % v == 0 && reinterpret_cast<uintptr_t>(samples) % (v * es < 16 ? v * es : 16) == 0)
                    vw = v;
#define ACB_FFT4_LAUNCH(TS, OF)                                                                                     \
    do {                                                                                                            \
        auto kern = fft4_tc_kernel<TS, OF>;                                                                         \
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem4);                        \
        kern<<<g4, 256, smem4, s>>>(reinterpret_cast<const TS *>(samples), num_mics, block_size, hop, first_window,  \
                                    num_windows, mpb4, vw, window, tw, bin_lo, num_bins, out, R, KC, lo_elems);    \
    } while (0)
            if (sample_dtype == ACB_F32) {
                if (out_form == OUT_TF32) ACB_FFT4_LAUNCH(float, OUT_TF32);
                else ACB_FFT4_LAUNCH(float, OUT_BF16);
            } else {
                if (out_form == OUT_TF32) ACB_FFT4_LAUNCH(double, OUT_TF32);
                else ACB_FFT4_LAUNCH(double, OUT_BF16);
            }
#undef ACB_FFT4_LAUNCH
            return check_launch();
        }
    }
    const int mpb = fft_mics_per_block(block_size);
    const dim3 g1((num_mics + mpb - 1) / mpb, (unsigned)num_windows);
    const size_t smem = (size_t)mpb * fft_stride(block_size / 2) * sizeof(double2);
#define ACB_FFT_LAUNCH(TS, OF)                                                                                    \
    do {                                                                                                          \
        auto kern = fft_window_kernel<TS, OF>;                                                                    \
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);                       \
        kern<<<g1, 256, smem, s>>>(reinterpret_cast<const TS *>(samples), num_mics, block_size, hop, first_window, \
                                   num_windows, mpb, window, tw, bin_lo, num_bins, out, R, KC, lo_elems);        \
    } while (0)
#define ACB_FFT_FORMS(TS)                                                \
    switch (out_form) {                                                  \
    case OUT_C128: ACB_FFT_LAUNCH(TS, OUT_C128); break;                  \
    case OUT_C64: ACB_FFT_LAUNCH(TS, OUT_C64); break;                    \
    case OUT_TF32: ACB_FFT_LAUNCH(TS, OUT_TF32); break;                  \
    default: ACB_FFT_LAUNCH(TS, OUT_BF16); break;                        \
    }
    if (sample_dtype == ACB_F32) { ACB_FFT_FORMS(float) }
    else { ACB_FFT_FORMS(double) }
#undef ACB_FFT_FORMS
#undef ACB_FFT_LAUNCH
    return check_launch();
}

}  // namespace acb

using namespace acb;

extern "C" {

const char *acb_status_string(int s)
{
    switch (s) {
    case ACB_OK: return "ok";
    case ACB_ERR_SHAPE: return "size or shape out of range";
    case ACB_ERR_ARG: return "invalid argument";
    case ACB_ERR_CUDA: return "CUDA error";
    case ACB_ERR_UNSUPPORTED: return "unsupported by this build";
    case ACB_ERR_WORKSPACE: return "workspace missing or too small";
    case ACB_ERR_TIMEOUT: return "device-side wait timed out";
    default: return "unknown status";
    }
}

int acb_abi_version(void) { return 2; }   // 2: tensor-core tuning fields, TC CSM forms, eigenvalue maps

const char *acb_last_cuda_error(void) { return g_last_cuda_error.c_str(); }

int acb_calc_csm_c128(void *csm, const void *spec, int num_freqs, int num_mics, void *stream)
{
    if (!csm || !spec) return ACB_ERR_ARG;
    if (num_freqs <= 0 || num_mics <= 0) return ACB_ERR_SHAPE;
    const int T = (num_mics + GT - 1) / GT;
    gram_kernel<false><<<dim3(T * (T + 1) / 2, num_freqs), 256, 0, as_stream(stream)>>>(spec, num_mics, 1, csm);
    return check_launch();
}

int acb_calc_csm_c64(void *csm, const void *spec, int num_freqs, int num_mics, void *stream)
{
    if (!csm || !spec) return ACB_ERR_ARG;
    if (num_freqs <= 0 || num_mics <= 0) return ACB_ERR_SHAPE;
    const int T = (num_mics + GT - 1) / GT;
    gram_kernel<true><<<dim3(T * (T + 1) / 2, num_freqs), 256, 0, as_stream(stream)>>>(spec, num_mics, 1, csm);
    return check_launch();
}

size_t acb_csm_workspace_bytes(int num_mics, int num_bins, int64_t num_windows, int precision)
{
    if (num_mics <= 0 || num_bins <= 0 || num_windows <= 0) return 0;
    if (precision == ACB_CSM_TC_TF32 || precision == ACB_CSM_TC_BF16X3)
        return csm_tc_workspace_bytes(num_mics, num_bins, num_windows);
    const size_t es = precision == ACB_C64 ? 8 : 16;
    return (size_t)num_mics * (size_t)num_bins * (size_t)num_windows * es;
}

size_t acb_csm_workspace_bytes_block(int num_mics, int num_bins, int64_t num_windows, int precision, int block_size)
{
    const size_t base = acb_csm_workspace_bytes(num_mics, num_bins, num_windows, precision);
    if (base == 0) return 0;
    const size_t sc = fft_scratch_bytes(num_mics, block_size, num_windows);
    return sc ? (base + 255) / 256 * 256 + sc : base;
}

int acb_csm_accumulate(const void *samples, int sample_dtype, int64_t num_samples, int num_mics, int block_size,
                       int hop, int64_t first_window, int64_t num_windows, const double *window,
                       const void *twiddle, int bin_lo, int num_bins, int precision, void *csm_upper,
                       void *workspace, size_t workspace_bytes, void *stream)
{
    if (!samples || !window || !twiddle || !csm_upper) return ACB_ERR_ARG;
    if (sample_dtype != ACB_F32 && sample_dtype != ACB_F64) return ACB_ERR_ARG;
    const bool tc = precision == ACB_CSM_TC_TF32 || precision == ACB_CSM_TC_BF16X3;
    if (precision != ACB_C128 && precision != ACB_C64 && !tc) return ACB_ERR_ARG;
    if (num_mics <= 0 || num_windows < 0 || first_window < 0 || hop <= 0) return ACB_ERR_SHAPE;
    if (tc && csm_tc_row_tiles(num_mics) > 252) return ACB_ERR_UNSUPPORTED;
    if (block_size < 16 || (block_size & (block_size - 1))) return ACB_ERR_SHAPE;
    if (block_size > 4 * FFT_MAX_N) return ACB_ERR_UNSUPPORTED;
    if (bin_lo < 0 || num_bins <= 0 || bin_lo + num_bins > block_size / 2 + 1) return ACB_ERR_SHAPE;
    if (num_windows == 0) return ACB_OK;
    if ((first_window + num_windows - 1) * (int64_t)hop + block_size > num_samples) return ACB_ERR_SHAPE;
    if (num_windows > 65535) return ACB_ERR_SHAPE;  // one grid row per window
    const size_t need = acb_csm_workspace_bytes_block(num_mics, num_bins, num_windows, precision, block_size);
    if (!workspace || workspace_bytes < need) return ACB_ERR_WORKSPACE;
    // blocks above 16384 samples: the FFT's sub-spectra go to a scratch region after the spectra
    void *scratch = nullptr;
    if (block_size > FFT_MAX_N)
        scratch = reinterpret_cast<uint8_t *>(workspace) +
                  (acb_csm_workspace_bytes(num_mics, num_bins, num_windows, precision) + 255) / 256 * 256;
    cudaStream_t s = as_stream(stream);
    const double2 *tw = reinterpret_cast<const double2 *>(twiddle);
    if (tc)
        return csm_tc_accumulate(samples, sample_dtype, num_mics, block_size, hop, first_window, num_windows, window,
                                 tw, bin_lo, num_bins, precision == ACB_CSM_TC_TF32, csm_upper, workspace, scratch, s);
    int st = fft_launch(samples, sample_dtype, precision == ACB_C64 ? OUT_C64 : OUT_C128, num_mics, block_size, hop,
                        first_window, num_windows, window, tw, bin_lo, num_bins, workspace, 0, 0, 0, scratch, s);
    if (st) return st;
    const int T = (num_mics + GT - 1) / GT;
    const dim3 g2(T * (T + 1) / 2, num_bins);
    if (precision == ACB_C64) gram_kernel<true><<<g2, 256, 0, s>>>(workspace, num_mics, num_windows, csm_upper);
    else gram_kernel<false><<<g2, 256, 0, s>>>(workspace, num_mics, num_windows, csm_upper);
    return check_launch();
}

int acb_csm_finalize(const void *csm_upper, int num_bins, int num_mics, int precision, double scale, void *csm_out,
                     void *stream)
{
    if (!csm_upper || !csm_out) return ACB_ERR_ARG;
    if (precision != ACB_C128 && precision != ACB_C64) return ACB_ERR_ARG;
    if (num_bins <= 0 || num_mics <= 0 || num_bins > 65535) return ACB_ERR_SHAPE;
    const int T = (num_mics + 31) / 32;
    const dim3 g(T, T, num_bins);
    if (precision == ACB_C64)
        finalize_kernel<true><<<g, 256, 0, as_stream(stream)>>>(csm_upper, num_mics, scale, (double2 *)csm_out);
    else
        finalize_kernel<false><<<g, 256, 0, as_stream(stream)>>>(csm_upper, num_mics, scale, (double2 *)csm_out);
    return check_launch();
}

}  // extern "C"
