// CLEAN-SC (BeamformerCleansc._calc, acoular/fbeamform.py:1424-1490) on the device, all bins of a request
// at once, with no host synchronisation inside the iterations.
//
// Per bin the reference iterates j = 0 .. J-1 on the conventional map h (full-CSM form, no clipping):
//   xi = argmax h (first index), hmax = h[xi], powers[j] = hmax, result[xi] += damp hmax (float32 result);
//   stop when j > stopn and hmax > powers[j - stopn];
//   w = conj(steer_vector(f, xi) sqrt(norm)) (the transfer of calcTransfer, fastFuncs.py:857-897, and the
//   steering formulas of SteeringVector._steer_funcs_freq, fbeamform.py:145-153);
//   D1 = (C^T - diag C) w / hmax; 20 fixed-point steps hh = (D1 + |hh|^2 w) / sqrt(1 + sum |w|^2 |hh|^2);
//   h -= damp * map of the single component (hmax, conj(hh)); C -= damp hmax (hh hh^H)^T.
//
// Device schedule: the steering vectors of every grid point are synthesised once per bin (normalised for
// the steering type, cleansc_steer_kernel); then per iteration cleansc_step_kernel (one CTA per bin: the
// map update h -= damp h1 fused with the argmax, then the peak's steering vector, D1, the fixed point and
// the CSM update) and the eigenvalue-form map of the new component on the cached steering vectors
// (map_eig_custom_launch, E = 1), both over all bins; a bin that has stopped clears its active flag and
// both kernels skip it.  The scalar arithmetic of the steering
// formulas and of the divisions follows numpy's complex arithmetic (x / y for a real y is x * (1 / y));
// sums (einsum, BLAS dot products) are formed in mic order.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "common.cuh"
#include "map_internal.h"

namespace acb {

constexpr int kCscThreads = 512;
constexpr int kCscWarps = kCscThreads / 32;

struct CscArgs {
    int M;
    int64_t G;
    int J;
    int stopn;
    double damp;
    double sqrt_norm;
    int steer_type;
    const double *k;
    const double *r0;   // given distances (non-Euclidean environments), else nullptr
    const double *rm;
    const double *mpos;
    const double *gpos;
    int ref_mode;
    double ref0, ref1, ref2, ref_dist;
    int faithful;
    const uint64_t *table;
    uint64_t mask;
    double2 *csm;      // (B, M, M) working copy, updated
    double *h;         // (B, G) map, updated
    const double *h1;  // (B, G) map of the previous iteration's component
    double *powers;    // (B, J)
    float *result;     // (B, G)
    int *active;       // (B)
    double *lam;       // (B) component eigenvalue (hmax)
    double2 *vec;      // (B, M) component vector conj(hh)
    const double2 *given;   // (B, G, M) a steering object's own vectors (custom steering), else nullptr
};

// numpy's complex division (Smith's method with a reciprocal scale), for a real divisor y = (yr, 0).
__device__ __forceinline__ double2 cdiv_real(double2 x, double yr)
{
    const double rat = __ddiv_rn(0.0, yr);
    const double scl = __ddiv_rn(1.0, __dadd_rn(yr, __dmul_rn(0.0, rat)));
    return make_double2(__dmul_rn(__dadd_rn(x.x, __dmul_rn(x.y, rat)), scl),
                        __dmul_rn(__dsub_rn(x.y, __dmul_rn(x.x, rat)), scl));
}

// numpy's complex division x / y for a general y.
__device__ __forceinline__ double2 cdiv(double2 x, double2 y)
{
    if (fabs(y.x) >= fabs(y.y)) {
        const double rat = __ddiv_rn(y.y, y.x);
        const double scl = __ddiv_rn(1.0, __dadd_rn(y.x, __dmul_rn(y.y, rat)));
        return make_double2(__dmul_rn(__dadd_rn(x.x, __dmul_rn(x.y, rat)), scl),
                            __dmul_rn(__dsub_rn(x.y, __dmul_rn(x.x, rat)), scl));
    }
    const double rat = __ddiv_rn(y.x, y.y);
    const double scl = __ddiv_rn(1.0, __dadd_rn(y.y, __dmul_rn(y.x, rat)));
    return make_double2(__dmul_rn(__dadd_rn(__dmul_rn(x.x, rat), x.y), scl),
                        __dmul_rn(__dsub_rn(__dmul_rn(x.y, rat), x.x), scl));
}

// Steering vectors of every grid point for the component maps, normalised so that the custom-steering
// quadratic form equals the steering type's map: v_m = e^{-i fl32(k r_m)} (times r_m for 'inverse',
// over r_m for 'true level' / 'true location'; the map kernel's synthesis), divided by M (classic),
// M r0 (inverse), r0 S (true level) or sqrt(M S) (true location), S = sum r^2 or sum 1/r^2.
// One warp per grid point, lanes over the mics; out (B, G, M).
__global__ void __launch_bounds__(256) cleansc_steer_kernel(CscArgs a, double2 *__restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const int64_t g = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    const int b = blockIdx.y;
    if (g >= a.G) return;
    const int M = a.M;
    const double k = a.k[b];
    double gx = 0, gy = 0, gz = 0, r0;
    if (a.rm) {
        r0 = a.r0[g];
    } else {
        gx = a.gpos[g];
        gy = a.gpos[a.G + g];
        gz = a.gpos[2 * a.G + g];
        r0 = a.ref_mode == 1 ? a.ref_dist : dist3(gx, gy, gz, a.ref0, a.ref1, a.ref2);
    }
    double2 *o = out + ((int64_t)b * a.G + g) * M;
    double S = 0.0;
    for (int m = lane; m < M; m += 32) {
        const double r = a.rm ? a.rm[g * M + m] : dist3(gx, gy, gz, a.mpos[m], a.mpos[M + m], a.mpos[2 * M + m]);
        const float arg = __double2float_rn(__dmul_rn(k, r));
        float c, sn;
        sincos_f32_arg(arg, a.table, a.mask, a.faithful != 0, c, sn);
        double2 v = make_double2((double)c, -(double)sn);
        if (a.steer_type == 2) {
            v.x = __dmul_rn(v.x, r);
            v.y = __dmul_rn(v.y, r);
            S += r * r;
        } else if (a.steer_type >= 3) {
            v.x = __ddiv_rn(v.x, r);
            v.y = __ddiv_rn(v.y, r);
            S += 1.0 / (r * r);
        }
        o[m] = v;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) S += __shfl_xor_sync(0xffffffffu, S, off);
    const double Md = (double)M;
    const double nf = a.steer_type == 1 ? Md : a.steer_type == 2 ? Md * r0 : a.steer_type == 3 ? r0 * S : sqrt(Md * S);
    const double inv = 1.0 / nf;
    __syncwarp();
    for (int m = lane; m < M; m += 32) {
        const double2 v = o[m];
        o[m] = make_double2(v.x * inv, v.y * inv);
    }
}

__global__ void cleansc_init_kernel(int *active, float *result, int64_t n_result, int B)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < B) active[i] = 1;
    if (i < n_result) result[i] = 0.0f;
}

__global__ void __launch_bounds__(kCscThreads) cleansc_step_kernel(CscArgs a, int j)
{
    extern __shared__ double sm[];
    const int b = blockIdx.x;
    if (!a.active[b]) return;
    const int M = a.M;
    const int64_t G = a.G;
    double2 *w = reinterpret_cast<double2 *>(sm);   // [M] steering of the peak, then its conjugate
    double2 *d1 = w + M;                              // [M]
    double2 *hh = d1 + M;                             // [M]
    double *ww = reinterpret_cast<double *>(hh + M);  // [M] |w|^2
    __shared__ double red_v[kCscWarps];
    __shared__ int64_t red_i[kCscWarps];
    __shared__ double scratch[kCscWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *h = a.h + (int64_t)b * G;
    const double *h1 = a.h1 + (int64_t)b * G;

    // 1. h -= damp h1 (the previous iteration's component), fused with the argmax (first index of the max)
    double best = -INFINITY;
    int64_t bi = G;
    for (int64_t g = threadIdx.x; g < G; g += kCscThreads) {
        double v = h[g];
        if (j > 0) {
            v = __dsub_rn(v, __dmul_rn(a.damp, h1[g]));
            h[g] = v;
        }
        if (v > best || (v == best && g < bi)) {
            best = v;
            bi = g;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int64_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > best || (ov == best && oi < bi)) {
            best = ov;
            bi = oi;
        }
    }
    if (lane == 0) {
        red_v[warp] = best;
        red_i[warp] = bi;
    }
    __syncthreads();
    best = red_v[0];
    bi = red_i[0];
    for (int wv = 1; wv < kCscWarps; ++wv)
        if (red_v[wv] > best || (red_v[wv] == best && red_i[wv] < bi)) {
            best = red_v[wv];
            bi = red_i[wv];
        }
    if (bi >= G) {   // no comparable value (NaN map): stop this bin
        if (threadIdx.x == 0) a.active[b] = 0;
        return;
    }
    const int64_t xi = bi;
    const double hmax = best;
    const bool stop = j > a.stopn && hmax > a.powers[(int64_t)b * a.J + j - a.stopn];
    __syncthreads();   // every thread has read powers before thread 0 writes this iteration's entry
    if (threadIdx.x == 0) {
        a.powers[(int64_t)b * a.J + j] = hmax;
        float *r = a.result + (int64_t)b * G + xi;
        *r = __double2float_rn(__dadd_rn((double)*r, __dmul_rn(a.damp, hmax)));
        if (stop) a.active[b] = 0;
    }
    if (stop) return;

    if (a.given) {
        // 2'. custom steering: the object's own steering vector of the peak, w = conj(v sqrt(norm))
        const double2 *v = a.given + ((int64_t)b * G + xi) * M;
        for (int m = threadIdx.x; m < M; m += kCscThreads) {
            const double2 x = v[m];
            const double2 c = make_double2(__dmul_rn(x.x, a.sqrt_norm), -__dmul_rn(x.y, a.sqrt_norm));
            w[m] = c;
            ww[m] = __dadd_rn(__dmul_rn(c.x, c.x), __dmul_rn(c.y, c.y));
            hh[m] = c;
        }
        __syncthreads();
    } else {
    // 2. steering vector of the peak: transfer x_m = (cos p - i sin p) r0 / rm, p = fl32(k (rm - r0))
    const double k = a.k[b];
    double gx = 0, gy = 0, gz = 0, r0x;
    if (a.rm) {
        r0x = a.r0[xi];
    } else {
        gx = a.gpos[xi];
        gy = a.gpos[G + xi];
        gz = a.gpos[2 * G + xi];
        r0x = a.ref_mode == 1 ? a.ref_dist : dist3(gx, gy, gz, a.ref0, a.ref1, a.ref2);
    }
    for (int m = threadIdx.x; m < M; m += kCscThreads) {
        const double rmm = a.rm ? a.rm[xi * M + m] : dist3(gx, gy, gz, a.mpos[m], a.mpos[M + m], a.mpos[2 * M + m]);
        const float arg = __double2float_rn(__dmul_rn(k, __dsub_rn(rmm, r0x)));
        float c, s;
        sincos_f32_arg(arg, a.table, a.mask, a.faithful != 0, c, s);
        const double xr = __ddiv_rn(__dmul_rn((double)c, r0x), rmm);
        const double xim = __ddiv_rn(__dmul_rn(-(double)s, r0x), rmm);
        w[m] = make_double2(xr, xim);
        ww[m] = __dadd_rn(__dmul_rn(xr, xr), __dmul_rn(xim, xim));   // Re x conj(x)
    }
    __syncthreads();
    double nrm = 0.0;
    if (a.steer_type >= 3) {   // einsum('ij,ij->i', x, x.conj()), in mic order
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int m = 0; m < M; ++m) t = __dadd_rn(t, ww[m]);
            scratch[0] = t;
        }
        __syncthreads();
        nrm = scratch[0];
        if (a.steer_type == 4) nrm = __dsqrt_rn(__dmul_rn(nrm, (double)M));
        __syncthreads();
    }
    for (int m = threadIdx.x; m < M; m += kCscThreads) {
        double2 x = w[m];
        if (a.steer_type == 1) {   // x / |x| / M
            x = cdiv_real(cdiv_real(x, hypot(x.x, x.y)), (double)M);
        } else if (a.steer_type == 2) {   // 1 / conj(x) / M
            x = cdiv_real(cdiv(make_double2(1.0, 0.0), make_double2(x.x, -x.y)), (double)M);
        } else {   // x / sum |x|^2  |  x / sqrt(sum |x|^2 M)
            x = cdiv_real(x, nrm);
        }
        // * sqrt(normfactor), then the conjugate
        const double2 v = make_double2(__dmul_rn(x.x, a.sqrt_norm), -__dmul_rn(x.y, a.sqrt_norm));
        w[m] = v;
        ww[m] = __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));   // conj(w) w
        hh[m] = v;
    }
    __syncthreads();
    }

    // 3. D1 = (C^T - diag C) w / hmax: D1_a = sum_{m != a} C[m][a] w_m, a warp per row a
    const double2 *C = a.csm + (int64_t)b * M * M;
    for (int r = warp; r < M; r += kCscWarps) {
        double sr = 0.0, si = 0.0;
        for (int m = lane; m < M; m += 32) {
            if (m == r) continue;
            const double2 c = C[(int64_t)m * M + r];
            const double2 v = w[m];
            sr = fma(c.x, v.x, fma(-c.y, v.y, sr));
            si = fma(c.x, v.y, fma(c.y, v.x, si));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sr += __shfl_xor_sync(0xffffffffu, sr, o);
            si += __shfl_xor_sync(0xffffffffu, si, o);
        }
        if (lane == 0) d1[r] = cdiv_real(make_double2(sr, si), hmax);
    }
    __syncthreads();

    // 4. 20 fixed-point steps: hh = (D1 + |hh|^2 w) / sqrt(1 + sum_m |w_m|^2 |hh_m|^2), in warp 0 alone
    //    (each lane owns mics lane, lane + 32, ...; the sum is a shuffle reduction, no block barrier)
    if (warp == 0) {
        for (int it = 0; it < 20; ++it) {
            double part = 0.0;
            for (int m = lane; m < M; m += 32) {
                const double2 q = hh[m];
                part = fma(ww[m], __dadd_rn(__dmul_rn(q.x, q.x), __dmul_rn(q.y, q.y)), part);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
            const double den = __dsqrt_rn(__dadd_rn(1.0, part));
            for (int m = lane; m < M; m += 32) {
                const double2 q = hh[m];
                const double H = __dadd_rn(__dmul_rn(q.x, q.x), __dmul_rn(q.y, q.y));
                const double2 v = w[m], d = d1[m];
                hh[m] = cdiv_real(make_double2(__dadd_rn(d.x, __dmul_rn(H, v.x)), __dadd_rn(d.y, __dmul_rn(H, v.y))),
                                  den);
            }
            __syncwarp();
        }
    }
    __syncthreads();

    // 5. C[r][c] -= damp (hmax (hh_c conj(hh_r))); 6. the component for the map: (hmax, conj(hh))
    double2 *Cw = a.csm + (int64_t)b * M * M;
    for (int64_t e = threadIdx.x; e < (int64_t)M * M; e += kCscThreads) {
        const int r = (int)(e / M), c = (int)(e % M);
        const double2 x = hh[c], y = hh[r];
        const double pr = __dsub_rn(__dmul_rn(x.x, y.x), __dmul_rn(x.y, -y.y));
        const double pi = __dadd_rn(__dmul_rn(x.x, -y.y), __dmul_rn(x.y, y.x));
        double2 v = Cw[e];
        v.x = __dsub_rn(v.x, __dmul_rn(a.damp, __dmul_rn(hmax, pr)));
        v.y = __dsub_rn(v.y, __dmul_rn(a.damp, __dmul_rn(hmax, pi)));
        Cw[e] = v;
    }
    for (int m = threadIdx.x; m < M; m += kCscThreads) a.vec[(int64_t)b * M + m] = make_double2(hh[m].x, -hh[m].y);
    if (threadIdx.x == 0) a.lam[b] = hmax;
}

struct CscWorkspace {
    size_t h, h1, powers, lam, vec, active, steer, total;
};

static CscWorkspace csc_layout(int M, int64_t G, int B, int J)
{
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    CscWorkspace w;
    size_t off = 0;
    w.h = off;
    off += up((size_t)B * G * sizeof(double));
    w.h1 = off;
    off += up((size_t)B * G * sizeof(double));
    w.powers = off;
    off += up((size_t)B * J * sizeof(double));
    w.lam = off;
    off += up((size_t)B * sizeof(double));
    w.vec = off;
    off += up((size_t)B * M * sizeof(double2));
    w.active = off;
    off += up((size_t)B * sizeof(int));
    w.steer = off;
    off += up((size_t)B * G * M * sizeof(double2));
    w.total = off;
    return w;
}

}  // namespace acb

using namespace acb;

extern "C" {

size_t acb_cleansc_workspace_bytes(int num_mics, int64_t num_grid, int num_bins, int n_iter)
{
    if (num_mics < 2 || num_grid <= 0 || num_bins <= 0 || n_iter < 0) return 0;
    const int J = n_iter > 0 ? n_iter : 2 * num_mics;
    return csc_layout(num_mics, num_grid, num_bins, J).total;
}

int acb_cleansc_f64(const acb_map_params *p, void *csm, const double *wavenumber, const double *mpos,
                    const double *gpos, const double *r0, const double *rm, int n_iter, double damp, int stopn,
                    float *result, void *workspace, size_t workspace_bytes, void *stream)
{
    if (!p || !csm || !wavenumber || !result || !workspace) return ACB_ERR_ARG;
    if (!rm && (!mpos || !gpos)) return ACB_ERR_ARG;
    if (rm && !r0) return ACB_ERR_ARG;
    if (p->steer_type < 1 || p->steer_type > 4) return ACB_ERR_ARG;
    const int M = p->num_mics, B = p->num_bins;
    const int64_t G = p->num_grid;
    if (M < 2 || M > 2048 || G <= 0 || B <= 0 || B > 65535 || n_iter < 0) return ACB_ERR_SHAPE;
    if (p->glibc_faithful && (!p->sincos_table || p->sincos_table_slots <= 0 ||
                              (p->sincos_table_slots & (p->sincos_table_slots - 1))))
        return ACB_ERR_ARG;
    const int J = n_iter > 0 ? n_iter : 2 * M;
    const CscWorkspace lay = csc_layout(M, G, B, J);
    if (workspace_bytes < lay.total) return ACB_ERR_WORKSPACE;
    cudaStream_t s = as_stream(stream);
    char *ws = static_cast<char *>(workspace);

    acb_map_params q = *p;
    q.clip_negative = 0;   // CLEAN-SC works on the unclipped map
    CscArgs a;
    a.M = M;
    a.G = G;
    a.J = J;
    a.stopn = stopn;
    a.damp = damp;
    a.sqrt_norm = sqrt(p->norm);
    a.steer_type = p->steer_type;
    a.k = wavenumber;
    a.r0 = rm ? r0 : nullptr;
    a.rm = rm;
    a.mpos = mpos;
    a.gpos = gpos;
    a.ref_mode = p->ref_mode;
    a.ref0 = p->ref_point[0];
    a.ref1 = p->ref_point[1];
    a.ref2 = p->ref_point[2];
    a.ref_dist = p->ref_distance;
    a.faithful = p->glibc_faithful;
    a.table = p->sincos_table;
    a.mask = p->glibc_faithful ? (uint64_t)p->sincos_table_slots - 1 : 0;
    a.csm = static_cast<double2 *>(csm);
    a.h = reinterpret_cast<double *>(ws + lay.h);
    a.h1 = reinterpret_cast<const double *>(ws + lay.h1);
    a.powers = reinterpret_cast<double *>(ws + lay.powers);
    a.result = result;
    a.active = reinterpret_cast<int *>(ws + lay.active);
    a.lam = reinterpret_cast<double *>(ws + lay.lam);
    a.vec = reinterpret_cast<double2 *>(ws + lay.vec);
    a.given = nullptr;

    const int64_t n_init = (int64_t)B * G > B ? (int64_t)B * G : B;
    cleansc_init_kernel<<<(unsigned)((n_init + 255) / 256), 256, 0, s>>>(a.active, result, (int64_t)B * G, B);
    int st = check_launch();
    if (st) return st;
    st = map_plain_launch(&q, B, csm, wavenumber, mpos, gpos, r0, rm, a.h, s);
    if (st) return st;
    double2 *steer = reinterpret_cast<double2 *>(ws + lay.steer);
    cleansc_steer_kernel<<<dim3((unsigned)((G + 7) / 8), B), 256, 0, s>>>(a, steer);
    st = check_launch();
    if (st) return st;
    const size_t smem = (size_t)M * (3 * sizeof(double2) + sizeof(double));
    if (cudaFuncSetAttribute(cleansc_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return ACB_ERR_CUDA;
    for (int j = 0; j < J; ++j) {
        cleansc_step_kernel<<<B, kCscThreads, smem, s>>>(a, j);
        st = check_launch();
        if (st) return st;
        if (j + 1 < J) {
            st = map_eig_custom_launch(&q, B, 1, a.lam, a.vec, steer, reinterpret_cast<double *>(ws + lay.h1),
                                       a.active, s);
            if (st) return st;
        }
    }
    return ACB_OK;
}

int acb_cleansc_custom_f64(const acb_map_params *p, void *csm, const void *steer, int n_iter, double damp, int stopn,
                           float *result, void *workspace, size_t workspace_bytes, void *stream)
{
    if (!p || !csm || !steer || !result || !workspace) return ACB_ERR_ARG;
    const int M = p->num_mics, B = p->num_bins;
    const int64_t G = p->num_grid;
    if (M < 2 || M > 2048 || G <= 0 || B <= 0 || B > 65535 || n_iter < 0) return ACB_ERR_SHAPE;
    const int J = n_iter > 0 ? n_iter : 2 * M;
    const CscWorkspace lay = csc_layout(M, G, B, J);
    if (workspace_bytes < lay.steer) return ACB_ERR_WORKSPACE;   // the steering region is not needed
    cudaStream_t s = as_stream(stream);
    char *ws = static_cast<char *>(workspace);

    acb_map_params q = *p;
    q.clip_negative = 0;   // CLEAN-SC works on the unclipped map
    q.glibc_faithful = 0;  // no phase synthesis: the vectors are given
    CscArgs a = {};
    a.M = M;
    a.G = G;
    a.J = J;
    a.stopn = stopn;
    a.damp = damp;
    a.sqrt_norm = sqrt(p->norm);
    a.steer_type = 0;
    a.csm = static_cast<double2 *>(csm);
    a.h = reinterpret_cast<double *>(ws + lay.h);
    a.h1 = reinterpret_cast<const double *>(ws + lay.h1);
    a.powers = reinterpret_cast<double *>(ws + lay.powers);
    a.result = result;
    a.active = reinterpret_cast<int *>(ws + lay.active);
    a.lam = reinterpret_cast<double *>(ws + lay.lam);
    a.vec = reinterpret_cast<double2 *>(ws + lay.vec);
    a.given = static_cast<const double2 *>(steer);

    const int64_t n_init = (int64_t)B * G > B ? (int64_t)B * G : B;
    cleansc_init_kernel<<<(unsigned)((n_init + 255) / 256), 256, 0, s>>>(a.active, result, (int64_t)B * G, B);
    int st = check_launch();
    if (st) return st;
    st = acb_map_custom_f64(&q, csm, steer, a.h, nullptr, stream);
    if (st) return st;
    const size_t smem = (size_t)M * (3 * sizeof(double2) + sizeof(double));
    if (cudaFuncSetAttribute(cleansc_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return ACB_ERR_CUDA;
    for (int j = 0; j < J; ++j) {
        cleansc_step_kernel<<<B, kCscThreads, smem, s>>>(a, j);
        st = check_launch();
        if (st) return st;
        if (j + 1 < J) {
            st = map_eig_custom_launch(&q, B, 1, a.lam, a.vec, steer, reinterpret_cast<double *>(ws + lay.h1),
                                       a.active, s);
            if (st) return st;
        }
    }
    return ACB_OK;
}

}  // extern "C"
