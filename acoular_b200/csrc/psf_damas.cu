// Point-spread functions (calcPointSpreadFunction, acoular/fastFuncs.py:563-801, as
// PointSpreadFunction._psf_call uses it, acoular/fbeamform.py:1093-1125) and the DAMAS Gauss-Seidel
// solver (damasSolverGaussSeidel, acoular/fastFuncs.py:804-855, as BeamformerDamas._calc uses it,
// acoular/fbeamform.py:1167-1208), plain FP64.
//
// PSF: for grid point g and source (grid point) s,
//     P = |sum_m e^{-i fl32(k (rm[g,m] - rm[s,m]))} w_m|^2 * n^2,
// the four steering types weighting w_m and n as the reference does; the phase is rounded to float32
// and its cos/sin are the C library's float32 ones (the exception table of the plain map).
// CTA = 32 grid points (lanes) x 8 sources (warps); the grid points' distance rows are staged in
// shared memory, each source's row is read as a broadcast.
//
// DAMAS: per bin, n_iter sweeps over g = 0 .. G-1 in order, each x[g] = max(0, (1 - relax) x[g] +
// relax (y[g] - sum_{h != g} A[g][h] x[h])) with the latest x.  The sweep is sequential by
// definition; a cluster of 1-8 CTAs per bin keeps x in every CTA's shared memory, splits the bulk of
// each row's dot product over its CTAs' column slices one block of rows ahead, and one warp solves
// each block of 32 rows in order (damas_kernel).
#include <cuda_runtime.h>
#include <stdint.h>

#include <cooperative_groups.h>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace acb {

constexpr int kPsfLanes = 32;
constexpr int kPsfWarps = 8;

template <int ST>
__global__ void __launch_bounds__(256) psf_kernel(int M, int64_t G, int S, const int64_t *__restrict__ src,
                                                  const double *__restrict__ r0, const double *__restrict__ rm,
                                                  double k, const uint64_t *__restrict__ table, uint64_t mask,
                                                  int faithful, int mc, int round_f32, double *__restrict__ out)
{
    extern __shared__ double rg_s[];   // [mc][32]: distance rows of this CTA's grid points, mic-major
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t g = (int64_t)blockIdx.x * kPsfLanes + lane;
    const int sidx = blockIdx.y * kPsfWarps + warp;
    int64_t s = sidx < S ? src[sidx] : 0;
    const bool src_ok = s >= 0 && s < G;   // an index outside the grid yields NaN, never a stray read
    s = src_ok ? s : 0;
    const bool valid = g < G && sidx < S;
    const double *rs = rm + s * M;
    double re = 0.0, im = 0.0, help = 0.0;
    double rs_l = 1.0, irs_l = 1.0;
    for (int m0 = 0; m0 < M; m0 += mc) {
        const int n = min(mc, M - m0);
        __syncthreads();
        for (int i = threadIdx.x; i < n * kPsfLanes; i += blockDim.x) {
            const int mm = i / kPsfLanes, l = i % kPsfLanes;
            const int64_t gg = (int64_t)blockIdx.x * kPsfLanes + l;
            rg_s[i] = gg < G ? rm[gg * M + m0 + mm] : 1.0;
        }
        __syncthreads();
        // every lane runs the loop (the shuffles need the whole warp); invalid lanes write nothing
        for (int mm = 0; mm < n; ++mm) {
            if ((mm & 31) == 0) {   // lane l holds the source distance of mic mm + l and its reciprocal
                rs_l = mm + lane < n ? __ldg(rs + m0 + mm + lane) : 1.0;
                irs_l = 1.0 / rs_l;
            }
            const double rsm = __shfl_sync(0xffffffffu, rs_l, mm & 31);
            const double irs = __shfl_sync(0xffffffffu, irs_l, mm & 31);
            const double rg = rg_s[mm * kPsfLanes + lane];
            const float arg = __double2float_rn(__dmul_rn(k, __dsub_rn(rg, rsm)));
            float c, sn;
            sincos_f32_arg(arg, table, mask, faithful != 0, c, sn);
            // (cos - i sin) / rs  [* rg (inverse) | / rg (true level, true location)]; the divisions as
            // products with reciprocals (within an ulp of the quotients)
            double tr = __dmul_rn((double)c, irs), ti = __dmul_rn(-(double)sn, irs);
            if (ST == 2) {
                tr = __dmul_rn(tr, rg);
                ti = __dmul_rn(ti, rg);
            } else if (ST >= 3) {
                const double ig = 1.0 / rg;
                tr = __dmul_rn(tr, ig);
                ti = __dmul_rn(ti, ig);
                help += ig * ig;
            }
            re += tr;
            im += ti;
        }
    }
    if (!valid) return;
    const double Md = (double)M;
    const double a2 = re * re + im * im;
    double res;
    if (ST == 1) {
        const double nf = r0[s] / Md;
        res = a2 * (nf * nf);
    } else if (ST == 2) {
        const double nf = r0[s] / r0[g] / Md;
        res = a2 * (nf * nf);
    } else if (ST == 3) {
        const double nf = r0[s] / r0[g] / help;
        res = a2 * (nf * nf);
    } else {
        const double nf = r0[s];
        res = a2 * (nf * nf) / Md / help;
    }
    if (!src_ok) res = __longlong_as_double(0x7ff8000000000000ll);
    out[g * S + sidx] = round_f32 ? (double)__double2float_rn(res) : res;
}

constexpr int kDamasThreads = 512;
constexpr int kDamasWarps = kDamasThreads / 32;
constexpr int kDamasRows = 32;        // rows solved per step (one per lane of the solving warp)
constexpr int kDamasMaxCta = 8;       // CTAs per bin (a portable cluster)
constexpr int kDamasPad = kDamasRows + 1;

// Shared memory of one CTA, in doubles: x[G] | partials[2][8][32] | diagonal tile^T[2][32][33] |
// previous-block tile^T[2][32][33] | y[2][32]
__host__ __device__ inline int64_t damas_smem_doubles(int64_t G)
{
    return G + 2 * kDamasMaxCta * kDamasRows + 4 * kDamasRows * kDamasPad + 2 * kDamasRows;
}

// Blocked, pipelined Gauss-Seidel.  Rows are taken in blocks of 32; step t solves block k = t mod nblk.
// Row i of block k needs sum_{h != i} A[i][h] x[h] with the latest x.  It is assembled from
//   (a) the columns outside blocks k and k-1 (final values of this sweep left of k-1, values of the
//       previous sweep right of k): computed one step AHEAD, while block k-1 is being solved, by the
//       warps of the cluster (in the first CTA only those off the solver's SM sub-partition, which
//       would otherwise take its issue slots), each CTA over its own column slice, and summed
//       through distributed shared memory into the first CTA;
//   (b) the columns of block k-1, whose new values are known at the start of step t (tile L);
//   (c) the other columns of block k (tile D), old values for the rows after each row, new ones as
//       they are solved.
// The solving warp (warp 0 of the first CTA) takes (b), (c) and the rows of block k in order, lane i
// owning row i: row j's new value is broadcast with a shuffle and every later lane subtracts its
// contribution.  One cluster barrier per step publishes block k's values to every CTA and the
// partial sums of block k+1 to the solver.  An L2 prefetch of block k+2's rows runs a step ahead
// of their loads.  Sweeps continue across the wrap-around (block 0 follows block nblk-1).
__global__ void __launch_bounds__(kDamasThreads) damas_kernel(const double *__restrict__ A, int64_t G,
                                                             const double *__restrict__ y, double *__restrict__ x,
                                                             int n_iter, double relax)
{
    extern __shared__ double sm[];
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int crank = (int)cluster.block_rank();
    const int64_t bin = blockIdx.x / C;
    double *xs = sm;
    double *red = xs + G;
    double *dT = red + 2 * kDamasMaxCta * kDamasRows;
    double *lT = dT + 2 * kDamasRows * kDamasPad;
    double *ys = lT + 2 * kDamasRows * kDamasPad;
    const double *Ab = A + bin * G * G;
    const double *yg = y + bin * G;
    double *xg = x + bin * G;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nblk = (int)((G + kDamasRows - 1) / kDamasRows);
    const int64_t W = ((G + C - 1) / C + 31) / 32 * 32;
    const int64_t c0 = min((int64_t)crank * W, G), c1 = min(c0 + W, G);
    double *red0 = cluster.map_shared_rank(red, 0);
    double *dT0 = cluster.map_shared_rank(dT, 0);
    double *lT0 = cluster.map_shared_rank(lT, 0);

    for (int64_t i = threadIdx.x; i < G; i += kDamasThreads) xs[i] = xg[i];
    // tiles start zeroed: entries outside a short last block are then finite (0 or an earlier value)
    for (int i = threadIdx.x; i < 4 * kDamasRows * kDamasPad; i += kDamasThreads) dT[i] = 0.0;
    __syncthreads();

    // Partial sums of block k (columns of blocks k and prev excluded) into buffer buf of the first
    // CTA.  The same pass routes the columns of block k (tile D) and of block prev (tile L) to the
    // first CTA's tiles instead of summing them; a warp takes up to three rows at once so that all
    // of its loads of a step are in flight together.
    auto prepare = [&](int k, int prev, int buf, bool spare) {
        if (spare && (warp & 3) == 0) return;
        const int w = spare ? warp - (warp >> 2) - 1 : warp;
        const int nw = spare ? kDamasWarps - kDamasWarps / 4 : kDamasWarps;
        const int64_t g0 = (int64_t)k * kDamasRows, p0 = (int64_t)prev * kDamasRows;
        const int nb = (int)min((int64_t)kDamasRows, G - g0);
        const int np = prev == k ? 0 : (int)min((int64_t)kDamasRows, G - p0);
        if (crank == 0 && w == 0) ys[buf * kDamasRows + lane] = lane < nb ? yg[g0 + lane] : 0.0;
        double *dt0 = dT0 + buf * kDamasRows * kDamasPad;
        double *lt0 = lT0 + buf * kDamasRows * kDamasPad;
        for (int rb = w; rb < nb; rb += 3 * nw) {
            const int r1 = rb + nw, r2 = rb + 2 * nw;
            const bool v1ok = r1 < nb, v2ok = r2 < nb;
            const double *row0 = Ab + (g0 + rb) * G;
            const double *row1 = Ab + (g0 + (v1ok ? r1 : rb)) * G;
            const double *row2 = Ab + (g0 + (v2ok ? r2 : rb)) * G;
            double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
            // chunks of 8 columns per lane: all loads of a chunk are issued before any use
            for (int64_t base = c0 + lane; base < c1; base += 8 * 32) {
                double v0[8], v1[8], v2[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int64_t h = base + u * 32;
                    const bool in = h < c1;
                    v0[u] = in ? __ldg(row0 + h) : 0.0;
                    v1[u] = (in && v1ok) ? __ldg(row1 + h) : 0.0;
                    v2[u] = (in && v2ok) ? __ldg(row2 + h) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int64_t h = base + u * 32;
                    if (h >= c1) break;
                    if (h >= g0 && h < g0 + nb) {
                        double *t = dt0 + (h - g0) * kDamasPad;
                        t[rb] = v0[u];
                        if (v1ok) t[r1] = v1[u];
                        if (v2ok) t[r2] = v2[u];
                    } else if (h >= p0 && h < p0 + np) {
                        double *t = lt0 + (h - p0) * kDamasPad;
                        t[rb] = v0[u];
                        if (v1ok) t[r1] = v1[u];
                        if (v2ok) t[r2] = v2[u];
                    } else {
                        const double xh = xs[h];
                        acc0 = fma(v0[u], xh, acc0);
                        acc1 = fma(v1[u], xh, acc1);
                        acc2 = fma(v2[u], xh, acc2);
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                acc0 += __shfl_xor_sync(0xffffffffu, acc0, o);
                acc1 += __shfl_xor_sync(0xffffffffu, acc1, o);
                acc2 += __shfl_xor_sync(0xffffffffu, acc2, o);
            }
            if (lane == 0) {
                double *rp = red0 + buf * kDamasMaxCta * kDamasRows + crank * kDamasRows;
                rp[rb] = acc0;
                if (v1ok) rp[r1] = acc1;
                if (v2ok) rp[r2] = acc2;
            }
        }
    };

    // Solve the rows of block k in order (warp 0 of the first CTA) and publish them to every CTA.
    // Lane i keeps u_i = c_i - relax (s_i + sum_{l > i} A[i][l] x_l), c_i = (1 - relax) x_i + relax y_i
    // and s_i the sum over the columns outside the block; row j's new value is max(0, u_j), and
    // every lane then subtracts relax A[i][j] times it.  The chain per row is one FMA, one max and
    // one shuffle; the sums feeding it use independent accumulators.
    auto solve = [&](int k, int prev, int buf) {
        const int64_t g0 = (int64_t)k * kDamasRows, p0 = (int64_t)prev * kDamasRows;
        const int nb = (int)min((int64_t)kDamasRows, G - g0);
        const int np = prev == k ? 0 : (int)min((int64_t)kDamasRows, G - p0);
        const int i = lane;
        const double *dt = dT + buf * kDamasRows * kDamasPad;
        const double *lt = lT + buf * kDamasRows * kDamasPad;
        const double *rp = red + buf * kDamasMaxCta * kDamasRows + i;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int c = 0; c < kDamasMaxCta; ++c)
            if (c < C) acc[c & 3] += rp[c * kDamasRows];
#pragma unroll
        for (int j = 0; j < kDamasRows; ++j)
            if (j < np) acc[j & 3] = fma(lt[j * kDamasPad + i], xs[p0 + j], acc[j & 3]);
        double b[kDamasRows];
#pragma unroll
        for (int j = 0; j < kDamasRows; ++j) b[j] = dt[j * kDamasPad + i];
        const double xold = i < nb ? xs[g0 + i] : 0.0;
#pragma unroll
        for (int j = 0; j < kDamasRows; ++j) {
            const double xj = __shfl_sync(0xffffffffu, xold, j);
            if (j > i) acc[j & 3] = fma(b[j], xj, acc[j & 3]);
        }
        const double s = (acc[0] + acc[1]) + (acc[2] + acc[3]);
        double u = (1.0 - relax) * xold + relax * (ys[buf * kDamasRows + i] - s);
#pragma unroll
        for (int j = 0; j < kDamasRows; ++j) b[j] = j < i ? relax * b[j] : 0.0;
        double xv = 0.0;
#pragma unroll
        for (int j = 0; j < kDamasRows; ++j) {
            if (j >= nb) break;
            const double xn = __shfl_sync(0xffffffffu, fmax(u, 0.0), j);
            u = fma(-b[j], xn, u);
            xv = i == j ? xn : xv;
        }
        if (i < nb)
            for (int r = 0; r < C; ++r) cluster.map_shared_rank(xs, r)[g0 + i] = xv;
    };

    // L2 prefetch of this CTA's column slice of the rows of block k (read two steps later).
    auto prefetch = [&](int k, bool spare) {
        if (spare && (warp & 3) == 0) return;
        const int w = spare ? warp - (warp >> 2) - 1 : warp;
        const int64_t g0 = (int64_t)k * kDamasRows;
        const int nb = (int)min((int64_t)kDamasRows, G - g0);
        const int64_t nlines = (c1 - c0 + 15) / 16;     // 128-byte lines of 16 doubles
        const int nthr = (spare ? kDamasWarps - kDamasWarps / 4 : kDamasWarps) * 32;
        for (int64_t e = w * 32 + lane; e < nb * nlines; e += nthr) {
            const double *ptr = Ab + (g0 + e / nlines) * G + c0 + (e % nlines) * 16;
            asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
        }
    };

    prepare(0, nblk - 1, 0, false);
    if (nblk > 1) prefetch(1, false);
    cluster.sync();
    const int64_t steps = (int64_t)n_iter * nblk;
    for (int64_t t = 0; t < steps; ++t) {
        const int k = (int)(t % nblk);
        const int buf = (int)(t & 1);
        const int kn = k + 1 == nblk ? 0 : k + 1;
        if (crank == 0 && warp == 0) solve(k, k == 0 ? nblk - 1 : k - 1, buf);
        if (t + 1 < steps) prepare(kn, k, buf ^ 1, crank == 0);
        if (t + 2 < steps) prefetch(kn + 1 == nblk ? 0 : kn + 1, crank == 0);
        cluster.sync();
    }
    if (crank == 0)
        for (int64_t i = threadIdx.x; i < G; i += kDamasThreads) xg[i] = xs[i];
}

}  // namespace acb

using namespace acb;

extern "C" {

int acb_psf_f64(const acb_map_params *p, int num_sources, const int64_t *sources, double wavenumber, const double *r0,
                const double *rm, int round_f32, double *out_psf, void *stream)
{
    if (!p || !sources || !r0 || !rm || !out_psf) return ACB_ERR_ARG;
    if (p->steer_type < 1 || p->steer_type > 4) return ACB_ERR_ARG;
    if (p->num_mics < 1 || p->num_grid <= 0 || num_sources <= 0) return ACB_ERR_SHAPE;
    if (p->glibc_faithful && (!p->sincos_table || p->sincos_table_slots <= 0 ||
                              (p->sincos_table_slots & (p->sincos_table_slots - 1))))
        return ACB_ERR_ARG;
    const int M = p->num_mics;
    const int64_t G = p->num_grid;
    const int mc = M < 256 ? M : 256;
    const size_t smem = (size_t)mc * kPsfLanes * sizeof(double);
    const dim3 grid((unsigned)((G + kPsfLanes - 1) / kPsfLanes), (unsigned)((num_sources + kPsfWarps - 1) / kPsfWarps));
    if (grid.y > 65535) return ACB_ERR_SHAPE;
    const uint64_t mask = p->glibc_faithful ? (uint64_t)p->sincos_table_slots - 1 : 0;
    cudaStream_t s = as_stream(stream);
#define ACB_PSF(ST)                                                                                          \
    do {                                                                                                     \
        cudaFuncSetAttribute(psf_kernel<ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);        \
        psf_kernel<ST><<<grid, kPsfLanes * kPsfWarps, smem, s>>>(M, G, num_sources, sources, r0, rm, wavenumber, \
                                                                p->sincos_table, mask, p->glibc_faithful, mc, \
                                                                round_f32, out_psf);                         \
    } while (0)
    switch (p->steer_type) {
    case 1: ACB_PSF(1); break;
    case 2: ACB_PSF(2); break;
    case 3: ACB_PSF(3); break;
    default: ACB_PSF(4); break;
    }
#undef ACB_PSF
    return check_launch();
}

int acb_damas_gauss_seidel_f64(const double *psf, int64_t num_grid, int num_bins, const double *dirty_map,
                               double *solution, int n_iter, double relax, int cta_per_bin, void *stream)
{
    if (!psf || !dirty_map || !solution) return ACB_ERR_ARG;
    if (num_grid <= 0 || num_bins <= 0 || n_iter < 0) return ACB_ERR_SHAPE;
    int dev = 0, sms = 0, smem_max = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return ACB_ERR_CUDA;
    const size_t smem = (size_t)damas_smem_doubles(num_grid) * sizeof(double);
    if (smem > (size_t)smem_max) return ACB_ERR_UNSUPPORTED;   // the solution lives in shared memory
    int C = cta_per_bin;
    if (C == 0) {
        C = kDamasMaxCta;
        while (C > 1 && (int64_t)num_bins * C > sms) C >>= 1;
    }
    if (C != 1 && C != 2 && C != 4 && C != 8) return ACB_ERR_ARG;
    if ((int64_t)num_bins * C > 0x7fffffff) return ACB_ERR_SHAPE;
    if (cudaFuncSetAttribute(damas_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return ACB_ERR_CUDA;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(num_bins * C));
    cfg.blockDim = dim3(kDamasThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = as_stream(stream);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, damas_kernel, psf, num_grid, dirty_map, solution, n_iter, relax) != cudaSuccess)
        return ACB_ERR_CUDA;
    return check_launch();
}

}  // extern "C"
