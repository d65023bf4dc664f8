// Stage B, plain FP64 form: h^H C h per (grid point, bin) as in _freqBeamformer_FullCSM
// (acoular/fastFuncs.py:217-311), batched over bins.
//
// CTA = 32 grid points (one per lane) x one bin, 8 warps.
//   1. distances |g - m| in FP64 (same contraction as the reference's dist_mat), phase
//      fl32(k*r), float32 cos/sin (correctly rounded, optionally corrected to the C library's
//      cosf/sinf by the exception table), steering h = cos - i sin, scaled by r (inverse) or 1/r
//      (true level / true location); h lives only in shared memory, chunk by chunk.
//   2. B = 2 Re sum_{a<b} conj(h_a) C_ab h_b (+ sum_a C_aa |h_a|^2 without diagonal removal):
//      warps take 8-row blocks of C (snake order for balance), each lane accumulates
//      y_r = sum_b C_{a_r b} h_b for its grid point with C_ab broadcast from L1/L2 and h_b from
//      shared memory, then conj(h_a) y.
//   3. cross-warp sum, normalisation of the steering type, optional clipping of negatives.
// Mic chunks: M <= 256 is one chunk; larger arrays use 128-mic chunks and loop over chunk pairs.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "map_internal.h"
#include "tc_common.cuh"

namespace acb {

constexpr int kLanes = 32;
constexpr int kWarps = 8;
constexpr int kRowBlock = 8;

struct MapArgs {
    int M;
    int64_t G;
    int steer_type;
    int r_diag;
    int clip;
    double norm;
    int ref_mode;
    double ref0, ref1, ref2, ref_dist;
    int faithful;
    const uint64_t *table;
    uint64_t table_mask;
};

template <bool USE_RM>
__device__ __forceinline__ double grid_mic_dist(const MapArgs &a, const double *__restrict__ rm, int64_t g, int m,
                                                double g0, double g1, double g2, const double *mp)
{
    if (USE_RM) return rm[g * a.M + m];
    return dist3(g0, g1, g2, mp[m], mp[a.M + m], mp[2 * a.M + m]);
}

// Steering value of a grid point and a mic at distance r (acoular/fastFuncs.py:258-273): the phase
// rounded to float32, cos - i sin of it as the C library's float32 functions give them, then the
// weight r (inverse) or 1/r (true level, true location).
__device__ __forceinline__ double2 steer_value(const MapArgs &a, double k, double r)
{
    const float arg = __double2float_rn(__dmul_rn(k, r));
    float c, s;
    sincos_f32_arg(arg, a.table, a.table_mask, a.faithful != 0, c, s);
    double2 h = make_double2((double)c, -(double)s);
    if (a.steer_type == 2) {
        h.x = __dmul_rn(h.x, r);
        h.y = __dmul_rn(h.y, r);
    } else if (a.steer_type >= 3) {
        h.x = __ddiv_rn(h.x, r);
        h.y = __ddiv_rn(h.y, r);
    }
    return h;
}

// Synthesise h for mics [m0, m0+n) of this CTA's 32 grid points into hs[m - m0][lane]; with CUSTOM,
// copy the caller's steering vectors hv[g][m] instead (custom steering, acoular/fastFuncs.py:414-559).
template <bool USE_RM, bool CUSTOM = false, int NW = kWarps>
__device__ __forceinline__ void synth_chunk(const MapArgs &a, const double *__restrict__ rm, double k, int64_t g,
                                           bool gvalid, double g0, double g1, double g2, const double *mp, int m0,
                                           int n, double2 *hs, const double2 *__restrict__ hv = nullptr)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = warp; i < n; i += NW) {
        double2 h = make_double2(0.0, 0.0);
        if (CUSTOM) {
            if (gvalid) h = __ldg(hv + g * a.M + m0 + i);
        } else if (gvalid) {
            h = steer_value(a, k, grid_mic_dist<USE_RM>(a, rm, g, m0 + i, g0, g1, g2, mp));
        }
        hs[i * kLanes + lane] = h;
    }
}

// Quadratic-form contribution of rows [ra0, ra0+na) x cols [cb0, cb0+nb) of C for this lane.
// If `diag_block` the block pair is the same chunk: only b > a counts (plus the diagonal when
// requested).  Returns (off-diagonal sum, diagonal sum).
__device__ __forceinline__ void quad_block(const double2 *__restrict__ C, int M, const double2 *ha, int ra0, int na,
                                           const double2 *hb, int cb0, int nb, bool diag_block, bool with_diag,
                                           double &off, double &dsum)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nrb = (na + kRowBlock - 1) / kRowBlock;
    for (int j = 0; j < nrb; ++j) {
        // snake assignment of row blocks to warps: 0..7, 7..0, 0..7, ...
        const int owner = ((j / kWarps) & 1) ? (kWarps - 1 - (j % kWarps)) : (j % kWarps);
        if (owner != warp) continue;
        const int a0 = j * kRowBlock;  // local row index in chunk A
        double yr[kRowBlock], yi[kRowBlock];
        const double2 *crow[kRowBlock];
#pragma unroll
        for (int r = 0; r < kRowBlock; ++r) {
            yr[r] = 0.0;
            yi[r] = 0.0;
            const int ar = min(a0 + r, na - 1);
            crow[r] = C + (int64_t)(ra0 + ar) * M + cb0;
        }
        const int bstart = diag_block ? a0 + 1 : 0;
        for (int b = bstart; b < nb; ++b) {
            const double2 h = hb[b * kLanes + lane];
#pragma unroll
            for (int r = 0; r < kRowBlock; ++r) {
                const bool use = (a0 + r < na) && (!diag_block || b > a0 + r);
                double2 c = __ldg(crow[r] + b);
                if (!use) c = make_double2(0.0, 0.0);
                yr[r] = fma(c.x, h.x, fma(-c.y, h.y, yr[r]));
                yi[r] = fma(c.x, h.y, fma(c.y, h.x, yi[r]));
            }
        }
#pragma unroll
        for (int r = 0; r < kRowBlock; ++r) {
            if (a0 + r < na) {
                const double2 h = ha[(a0 + r) * kLanes + lane];
                off = fma(h.x, yr[r], fma(h.y, yi[r], off));  // Re(conj(h) y)
                if (with_diag) {
                    const double2 c = __ldg(C + (int64_t)(ra0 + a0 + r) * M + (ra0 + a0 + r));
                    // (C_aa * conj(h)) * h, real part
                    const double pr = c.x * h.x + c.y * h.y;
                    const double pi = -c.x * h.y + c.y * h.x;
                    dsum += pr * h.x - pi * h.y;
                }
            }
        }
    }
}

// Normalisation of the steering type (acoular/fastFuncs.py:293-310) and clipping of negatives.
__device__ __forceinline__ void finish_plain(const MapArgs &a, double scalar, double S, double r0, int bin, int64_t g,
                                             double *out_map, double *out_norm)
{
    const double Md = (double)a.M;
    double res, ns;
    if (a.steer_type == 0) {   // custom steering: no steering normalisation, S = sum |h|^2
        ns = S;
        res = scalar * a.norm;
    } else if (a.steer_type == 1) {
        ns = 1.0 / Md;
        res = scalar / (Md * Md) * a.norm;
    } else if (a.steer_type == 2) {
        const double nf = Md * r0;
        const double nf2 = nf * nf;
        ns = S / nf2;
        res = scalar / nf2 * a.norm;
    } else if (a.steer_type == 3) {
        const double nf = r0 * S;
        ns = 1.0 / (r0 * r0) / S;
        res = scalar / (nf * nf) * a.norm;
    } else {
        const double nf = Md * S;
        ns = 1.0 / Md;
        res = scalar / nf * a.norm;
    }
    if (a.clip && res < 0.0) res = 0.0;
    out_map[(int64_t)bin * a.G + g] = res;
    if (out_norm) out_norm[(int64_t)bin * a.G + g] = ns;
}

template <bool USE_RM, bool CUSTOM = false>
__global__ void __launch_bounds__(256) map_plain_kernel(MapArgs a, const double2 *__restrict__ csm,
                                                        const double *__restrict__ wavenumber, double k_scalar,
                                                        const double *__restrict__ mpos,
                                                        const double *__restrict__ gpos,
                                                        const double *__restrict__ r0_in,
                                                        const double *__restrict__ rm, int mc,
                                                        double *__restrict__ out_map,
                                                        double *__restrict__ out_norm,
                                                        const double2 *__restrict__ steer = nullptr)
{
    extern __shared__ double smem[];
    const int M = a.M;
    double *mp = smem;                                          // [3][M]
    double2 *ha = reinterpret_cast<double2 *>(smem + ((3 * M + 1) & ~1));  // [mc][32]
    double2 *hb = ha + (size_t)mc * kLanes;                      // [mc][32] (only if M > mc)
    __shared__ double red_off[kWarps][kLanes], red_diag[kWarps][kLanes], red_s[kWarps][kLanes];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int bin = blockIdx.y;
    const int64_t g = (int64_t)blockIdx.x * kLanes + lane;
    const bool gvalid = g < a.G;
    const double k = wavenumber ? wavenumber[bin] : k_scalar;
    const double2 *C = csm + (int64_t)bin * M * M;
    const double2 *hv = CUSTOM ? steer + (int64_t)bin * a.G * M : nullptr;

    if (!USE_RM && !CUSTOM)
        for (int i = threadIdx.x; i < 3 * M; i += blockDim.x) mp[i] = mpos[i];
    double g0 = 0, g1 = 0, g2 = 0;
    if (gvalid && !USE_RM && !CUSTOM) {
        g0 = gpos[g];
        g1 = gpos[a.G + g];
        g2 = gpos[2 * a.G + g];
    }
    __syncthreads();

    // steering normalisation sum S (inverse: sum r^2; true level / location: sum 1/r^2; custom: sum |h|^2)
    double s_part = 0.0;
    if (CUSTOM) {
        if (gvalid)
            for (int m = warp; m < M; m += kWarps) {
                const double2 h = __ldg(hv + g * M + m);
                s_part += h.x * h.x + h.y * h.y;
            }
    } else if (gvalid && a.steer_type >= 2) {
        for (int m = warp; m < M; m += kWarps) {
            const double r = grid_mic_dist<USE_RM>(a, rm, g, m, g0, g1, g2, mp);
            s_part += (a.steer_type == 2) ? r * r : 1.0 / (r * r);
        }
    }

    double off = 0.0, dsum = 0.0;
    const int nchunks = (M + mc - 1) / mc;
    for (int ca = 0; ca < nchunks; ++ca) {
        const int ma0 = ca * mc, na = min(mc, M - ma0);
        synth_chunk<USE_RM, CUSTOM>(a, rm, k, g, gvalid, g0, g1, g2, mp, ma0, na, ha, hv);
        __syncthreads();
        quad_block(C, M, ha, ma0, na, ha, ma0, na, true, a.r_diag == 0, off, dsum);
        for (int cb = ca + 1; cb < nchunks; ++cb) {
            const int mb0 = cb * mc, nb = min(mc, M - mb0);
            __syncthreads();
            synth_chunk<USE_RM, CUSTOM>(a, rm, k, g, gvalid, g0, g1, g2, mp, mb0, nb, hb, hv);
            __syncthreads();
            quad_block(C, M, ha, ma0, na, hb, mb0, nb, false, false, off, dsum);
        }
        __syncthreads();
    }

    red_off[warp][lane] = off;
    red_diag[warp][lane] = dsum;
    red_s[warp][lane] = s_part;
    __syncthreads();
    if (warp == 0 && gvalid) {
        double o = 0.0, d = 0.0, S = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            o += red_off[w][lane];
            d += red_diag[w][lane];
            S += red_s[w][lane];
        }
        const double scalar = 2.0 * o + d;
        double r0 = 0.0;
        if (CUSTOM) r0 = 0.0;
        else if (a.ref_mode == 1) r0 = a.ref_dist;
        else if (USE_RM) r0 = r0_in[g];
        else r0 = dist3(g0, g1, g2, a.ref0, a.ref1, a.ref2);
        finish_plain(a, scalar, S, r0, bin, g, out_map, out_norm);
    }
}

// ------------------------------------------------------------------------------------------------
// Staged variant for M <= 256 (one mic chunk): the same steering synthesis and quadratic form, but the
// CSM rows come through shared memory.  Each warp streams the rows of its 8-row blocks in column
// chunks of kCB through a two-stage ring that lane 0 fills with bulk copies (cp.async.bulk into this
// CTA alone; one copy per row, completion on the stage's mbarrier); the next chunk is in flight while
// the warp works on the current one.  Every loaded C value then feeds the 32 grid points of the warp
// from shared memory instead of a broadcast load through L1/L2 per complex FMA, and the masking of the
// triangle is confined to the diagonal 8 x 8 block.  Sixteen warps (four per scheduler, 128 registers
// each) share the CTA's steering block: the FP64 FMA chains of the 8-row blocks need that many warps
// to cover their latency at one CTA per SM (8 warps: 19.7 TFLOP/s on the 256-mic workload, 16: 24.7).
// Waits are bounded; a CTA that gives up raises the error word, writes NaN and returns after its own
// copies have landed.
// ------------------------------------------------------------------------------------------------
constexpr int kSWarps = 16;                              // warps of the staged kernel (4 per scheduler)
constexpr int kCB = 16;                                  // C columns per staged chunk
constexpr int kCStageElems = kRowBlock * kCB;            // double2 per (warp, stage)
constexpr uint64_t kPlainWaitNs = 500ull * 1000 * 1000;  // limit of one wait

struct StagedSmem {
    // byte offsets; M mics
    __host__ __device__ static constexpr size_t mp(int) { return 0; }
    __host__ __device__ static constexpr size_t ha(int M) { return (size_t)((3 * M + 1) & ~1) * 8; }
    __host__ __device__ static constexpr size_t cst(int M) { return ha(M) + (size_t)M * kLanes * 16; }
    __host__ __device__ static constexpr size_t bars(int M) { return cst(M) + (size_t)kSWarps * 2 * kCStageElems * 16; }
    __host__ __device__ static constexpr size_t total(int M) { return bars(M) + kSWarps * 2 * 8 + 16; }
};

// the chunk sequence of one warp: its row blocks in snake order, each block's columns [a0, M) in kCB chunks
struct ChunkCursor {
    int j;    // row block (local index into the warp's list: j-th block of this warp)
    int c0;   // first column of the chunk
};

__device__ __forceinline__ int warp_block(int warp, int t)
{
    // t-th row block of `warp` in the snake assignment 0..7, 7..0, 0..7, ...
    return t * kSWarps + ((t & 1) ? (kSWarps - 1 - warp) : warp);
}

template <bool USE_RM, bool CUSTOM>
__global__ void __launch_bounds__(kLanes * kSWarps, 1)
    map_plain_staged_kernel(MapArgs a, const double2 *__restrict__ csm, const double *__restrict__ wavenumber,
                            double k_scalar, const double *__restrict__ mpos, const double *__restrict__ gpos,
                            const double *__restrict__ r0_in, const double *__restrict__ rm,
                            double *__restrict__ out_map, double *__restrict__ out_norm,
                            const double2 *__restrict__ steer, int *err)
{
    extern __shared__ __align__(16) uint8_t smem_b[];
    const int M = a.M;
    double *mp = reinterpret_cast<double *>(smem_b);
    double2 *ha = reinterpret_cast<double2 *>(smem_b + StagedSmem::ha(M));     // [M][32]
    double2 *cst = reinterpret_cast<double2 *>(smem_b + StagedSmem::cst(M));   // [warp][stage][8][kCB]
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_b + StagedSmem::bars(M));   // [warp][stage]
    volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + kSWarps * 2);
    __shared__ double red_off[kSWarps][kLanes], red_diag[kSWarps][kLanes], red_s[kSWarps][kLanes];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int bin = blockIdx.y;
    const int64_t g = (int64_t)blockIdx.x * kLanes + lane;
    const bool gvalid = g < a.G;
    const double k = wavenumber ? wavenumber[bin] : k_scalar;
    const double2 *C = csm + (int64_t)bin * M * M;
    const double2 *hv = CUSTOM ? steer + (int64_t)bin * a.G * M : nullptr;

    if (threadIdx.x == 0) {
        for (int i = 0; i < kSWarps * 2; ++i) tc::mbar_init(&bars[i], 1);
        *abort_flag = 0;
        tc::fence_mbar_init();
    }
    if (!USE_RM && !CUSTOM)
        for (int i = threadIdx.x; i < 3 * M; i += blockDim.x) mp[i] = mpos[i];
    double g0 = 0, g1 = 0, g2 = 0;
    if (gvalid && !USE_RM && !CUSTOM) {
        g0 = gpos[g];
        g1 = gpos[a.G + g];
        g2 = gpos[2 * a.G + g];
    }
    __syncthreads();

    // this warp's chunk sequence
    const int nblk = (M + kRowBlock - 1) / kRowBlock;
    int nmine = 0;
    while (warp_block(warp, nmine) < nblk) ++nmine;
    double2 *wst = cst + (size_t)warp * 2 * kCStageElems;
    uint64_t *wbar = bars + warp * 2;
    // lane 0: issue the copies of chunk (t, c0) into stage st
    auto issue = [&](int t, int c0, int st) {
        const int a0 = warp_block(warp, t) * kRowBlock;
        const int na = min(kRowBlock, M - a0), nc = min(kCB, M - c0);
        tc::mbar_arrive_expect_tx(&wbar[st], (uint32_t)(na * nc * 16));
        for (int r = 0; r < na; ++r)
            tc::bulk_g2s(wst + (size_t)st * kCStageElems + r * kCB, C + (int64_t)(a0 + r) * M + c0, (uint32_t)(nc * 16),
                         &wbar[st]);
    };
    auto next = [&](int &t, int &c0) {
        c0 += kCB;
        if (c0 >= M) {
            ++t;
            if (t < nmine) c0 = warp_block(warp, t) * kRowBlock;
        }
    };
    // the first two chunks go out before the steering synthesis, so their latency hides under it
    int it_t = 0, it_c = nmine > 0 ? warp_block(warp, 0) * kRowBlock : 0;   // issue cursor
    int issued = 0;
    if (lane == 0)
        for (int q = 0; q < 2 && it_t < nmine; ++q, ++issued) {
            issue(it_t, it_c, q);
            next(it_t, it_c);
        }
    issued = __shfl_sync(0xffffffffu, issued, 0);
    it_t = __shfl_sync(0xffffffffu, it_t, 0);
    it_c = __shfl_sync(0xffffffffu, it_c, 0);

    // steering normalisation sum S (inverse: sum r^2; true level / location: sum 1/r^2; custom: sum |h|^2)
    double s_part = 0.0;
    if (CUSTOM) {
        if (gvalid)
            for (int m = warp; m < M; m += kSWarps) {
                const double2 h = __ldg(hv + g * M + m);
                s_part += h.x * h.x + h.y * h.y;
            }
    } else if (gvalid && a.steer_type >= 2) {
        for (int m = warp; m < M; m += kSWarps) {
            const double r = grid_mic_dist<USE_RM>(a, rm, g, m, g0, g1, g2, mp);
            s_part += (a.steer_type == 2) ? r * r : 1.0 / (r * r);
        }
    }
    synth_chunk<USE_RM, CUSTOM, kSWarps>(a, rm, k, g, gvalid, g0, g1, g2, mp, 0, M, ha, hv);
    __syncthreads();

    double off = 0.0, dsum = 0.0;
    const bool with_diag = a.r_diag == 0;
    int q = 0;   // chunk counter: stage q & 1, phase (q >> 1) & 1
    bool ok = true;
    for (int t = 0; t < nmine && ok; ++t) {
        const int a0 = warp_block(warp, t) * kRowBlock;
        const int na = min(kRowBlock, M - a0);
        double yr[kRowBlock], yi[kRowBlock];
#pragma unroll
        for (int r = 0; r < kRowBlock; ++r) yr[r] = yi[r] = 0.0;
        for (int c0 = a0; c0 < M; c0 += kCB, ++q) {
            const int st = q & 1;
            ok = __all_sync(0xffffffffu, tc::mbar_wait(&wbar[st], (uint32_t)((q >> 1) & 1), abort_flag, kPlainWaitNs));
            if (!ok) break;
            const double2 *cs = wst + (size_t)st * kCStageElems;
            const int nc = min(kCB, M - c0);
            int bb = 0;
            if (c0 == a0) {
                // the diagonal 8 x 8 block: row r takes columns b > a0 + r (and its diagonal term)
#pragma unroll
                for (int d = 0; d < kRowBlock; ++d) {
                    if (d >= nc) break;
                    const double2 h = ha[(c0 + d) * kLanes + lane];
#pragma unroll
                    for (int r = 0; r < kRowBlock; ++r) {
                        if (r >= na) continue;
                        const double2 c = cs[r * kCB + d];
                        if (d > r) {
                            yr[r] = fma(c.x, h.x, fma(-c.y, h.y, yr[r]));
                            yi[r] = fma(c.x, h.y, fma(c.y, h.x, yi[r]));
                        } else if (d == r && with_diag) {
                            // (C_aa * conj(h)) * h, real part
                            const double pr = c.x * h.x + c.y * h.y;
                            const double pi = -c.x * h.y + c.y * h.x;
                            dsum += pr * h.x - pi * h.y;
                        }
                    }
                }
                bb = kRowBlock;
            }
            if (na == kRowBlock) {
#pragma unroll 4
                for (; bb < nc; ++bb) {
                    const double2 h = ha[(c0 + bb) * kLanes + lane];
#pragma unroll
                    for (int r = 0; r < kRowBlock; ++r) {
                        const double2 c = cs[r * kCB + bb];
                        yr[r] = fma(c.x, h.x, fma(-c.y, h.y, yr[r]));
                        yi[r] = fma(c.x, h.y, fma(c.y, h.x, yi[r]));
                    }
                }
            } else {
                for (; bb < nc; ++bb) {
                    const double2 h = ha[(c0 + bb) * kLanes + lane];
#pragma unroll
                    for (int r = 0; r < kRowBlock; ++r) {
                        if (r >= na) continue;
                        const double2 c = cs[r * kCB + bb];
                        yr[r] = fma(c.x, h.x, fma(-c.y, h.y, yr[r]));
                        yi[r] = fma(c.x, h.y, fma(c.y, h.x, yi[r]));
                    }
                }
            }
            // the stage is consumed: lane 0 refills it with the chunk two ahead
            __syncwarp();
            if (it_t < nmine) {
                if (lane == 0) {
                    tc::fence_proxy_async_smem();
                    issue(it_t, it_c, st);
                }
                next(it_t, it_c);
                ++issued;
            }
        }
        if (!ok) break;
#pragma unroll
        for (int r = 0; r < kRowBlock; ++r) {
            if (r < na) {
                const double2 h = ha[(a0 + r) * kLanes + lane];
                off = fma(h.x, yr[r], fma(h.y, yi[r], off));   // Re(conj(h) y)
            }
        }
    }
    if (!ok && lane == 0) {
        // let this warp's copies still in flight (chunks q .. issued - 1) land before the CTA exits
        for (int qq = q; qq < issued; ++qq)
            tc::mbar_drain(&wbar[qq & 1], (uint32_t)((qq >> 1) & 1), tc::drain_limit_ns(kPlainWaitNs));
    }

    red_off[warp][lane] = off;
    red_diag[warp][lane] = dsum;
    red_s[warp][lane] = s_part;
    __syncthreads();
    if (warp == 0 && gvalid) {
        double o = 0.0, d = 0.0, S = 0.0;
#pragma unroll
        for (int w = 0; w < kSWarps; ++w) {
            o += red_off[w][lane];
            d += red_diag[w][lane];
            S += red_s[w][lane];
        }
        double r0 = 0.0;
        if (CUSTOM) r0 = 0.0;
        else if (a.ref_mode == 1) r0 = a.ref_dist;
        else if (USE_RM) r0 = r0_in[g];
        else r0 = dist3(g0, g1, g2, a.ref0, a.ref1, a.ref2);
        if (*abort_flag) {
            out_map[(int64_t)bin * a.G + g] = __longlong_as_double(0x7ff8000000000000ll);
            if (out_norm) out_norm[(int64_t)bin * a.G + g] = __longlong_as_double(0x7ff8000000000000ll);
        } else {
            finish_plain(a, 2.0 * o + d, S, r0, bin, g, out_map, out_norm);
        }
    }
    if (threadIdx.x == 0 && *abort_flag && err) atomicOr(err, 1);
}

// ------------------------------------------------------------------------------------------------
// Eigenvalue form of _freqBeamformer_EigValues (acoular/fastFuncs.py:313-411): with eigenvalues
// lambda_e and eigenvectors V[:, e] of the CSM (E of them),
//     scalar = sum_e lambda_e (|sum_m conj(V[m][e]) h[m]|^2 - [r_diag] sum_m |conj(V[m][e]) h[m]|^2),
// then the steering-type normalisation of the full-CSM form.  Same steering synthesis (float32
// phase, libm-faithful cos/sin) as map_plain_kernel; the warps take the eigenvectors in groups of
// 32 (four per warp, partial sums in registers across mic chunks), each eigenvector's mic sum in
// the reference's order.  Cost O(G M E) per bin.
// ------------------------------------------------------------------------------------------------
constexpr int kEigPerWarp = 4;

template <bool USE_RM, bool CUSTOM = false>
__global__ void __launch_bounds__(256) map_eig_kernel(MapArgs a, int E, const double *__restrict__ eigval,
                                                      const double2 *__restrict__ eigvec,
                                                      const double *__restrict__ wavenumber, double k_scalar,
                                                      const double *__restrict__ mpos, const double *__restrict__ gpos,
                                                      const double *__restrict__ r0_in, const double *__restrict__ rm,
                                                      int mc, double *__restrict__ out_map,
                                                      double *__restrict__ out_norm,
                                                      const double2 *__restrict__ steer = nullptr,
                                                      const int *__restrict__ active = nullptr)
{
    extern __shared__ double smem[];
    if (active && !active[blockIdx.y]) return;   // a bin whose iteration has stopped (CLEAN-SC)
    const int M = a.M;
    double *mp = smem;                                                     // [3][M]
    double2 *hs = reinterpret_cast<double2 *>(smem + ((3 * M + 1) & ~1));  // [mc][32]
    __shared__ double red_sc[kWarps][kLanes], red_s[kWarps][kLanes];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int bin = blockIdx.y;
    const int64_t g = (int64_t)blockIdx.x * kLanes + lane;
    const bool gvalid = g < a.G;
    const double k = wavenumber ? wavenumber[bin] : k_scalar;
    const double *lam = eigval + (int64_t)bin * E;
    const double2 *V = eigvec + (int64_t)bin * M * E;
    const double2 *hv = CUSTOM ? steer + (int64_t)bin * a.G * M : nullptr;

    if (!USE_RM && !CUSTOM)
        for (int i = threadIdx.x; i < 3 * M; i += blockDim.x) mp[i] = mpos[i];
    double g0 = 0, g1 = 0, g2 = 0;
    if (gvalid && !USE_RM && !CUSTOM) {
        g0 = gpos[g];
        g1 = gpos[a.G + g];
        g2 = gpos[2 * a.G + g];
    }
    __syncthreads();

    double s_part = 0.0;
    if (CUSTOM) {
        if (gvalid)
            for (int m = warp; m < M; m += kWarps) {
                const double2 h = __ldg(hv + g * M + m);
                s_part += h.x * h.x + h.y * h.y;
            }
    } else if (gvalid && a.steer_type >= 2) {
        for (int m = warp; m < M; m += kWarps) {
            const double r = grid_mic_dist<USE_RM>(a, rm, g, m, g0, g1, g2, mp);
            s_part += (a.steer_type == 2) ? r * r : 1.0 / (r * r);
        }
    }

    double scal = 0.0;
    const int nchunks = (M + mc - 1) / mc;
    for (int eg = 0; eg < E; eg += kWarps * kEigPerWarp) {
        double fr[kEigPerWarp], fi[kEigPerWarp], dg[kEigPerWarp];
#pragma unroll
        for (int j = 0; j < kEigPerWarp; ++j) fr[j] = fi[j] = dg[j] = 0.0;
        const int e0 = eg + warp * kEigPerWarp;
        for (int ca = 0; ca < nchunks; ++ca) {
            const int m0 = ca * mc, n = min(mc, M - m0);
            synth_chunk<USE_RM, CUSTOM>(a, rm, k, g, gvalid, g0, g1, g2, mp, m0, n, hs, hv);
            __syncthreads();
            for (int mm = 0; mm < n; ++mm) {
                const double2 h = hs[mm * kLanes + lane];
                const double2 *vrow = V + (int64_t)(m0 + mm) * E;
#pragma unroll
                for (int j = 0; j < kEigPerWarp; ++j) {
                    if (e0 + j >= E) break;
                    const double2 v = __ldg(vrow + e0 + j);
                    // temp1 = conj(V[m][e]) * h[m]
                    const double tr = v.x * h.x + v.y * h.y, ti = v.x * h.y - v.y * h.x;
                    fr[j] += tr;
                    fi[j] += ti;
                    if (a.r_diag) dg[j] += tr * tr + ti * ti;
                }
            }
            __syncthreads();   // hs is rewritten by the next chunk
        }
#pragma unroll
        for (int j = 0; j < kEigPerWarp; ++j) {
            if (e0 + j >= E) break;
            const double full = fr[j] * fr[j] + fi[j] * fi[j];
            scal += (a.r_diag ? full - dg[j] : full) * lam[e0 + j];
        }
    }

    red_sc[warp][lane] = scal;
    red_s[warp][lane] = s_part;
    __syncthreads();
    if (warp == 0 && gvalid) {
        double sc = 0.0, S = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            sc += red_sc[w][lane];
            S += red_s[w][lane];
        }
        double r0 = 0.0;
        if (CUSTOM) r0 = 0.0;
        else if (a.ref_mode == 1) r0 = a.ref_dist;
        else if (USE_RM) r0 = r0_in[g];
        else r0 = dist3(g0, g1, g2, a.ref0, a.ref1, a.ref2);
        finish_plain(a, sc, S, r0, bin, g, out_map, out_norm);
    }
}

// Eigenvalue form for a few components (E <= kEigSmall, e.g. BeamformerEig's default n = -1 and each
// CLEAN-SC iteration's single component): one thread per grid point walks the mics in order,
// synthesises each steering value once and accumulates the E projections and the normalisation sum in
// registers.  Without shared memory a CTA of 4 warps holds no resources but registers, so many warps
// per SM hide the latency of the FP64 synthesis and of the exception-table probes; the shared-memory
// form above (one CTA of 8 warps per SM) serves larger E, where the projections outnumber the
// registers.  Each component's mic sum runs in the reference's order.
constexpr int kEigSmall = 4;
constexpr int kEigSmallThreads = 128;

template <bool USE_RM, bool CUSTOM, int EMAX>
__global__ void __launch_bounds__(kEigSmallThreads)
    map_eig_small_kernel(MapArgs a, int E, const double *__restrict__ eigval, const double2 *__restrict__ eigvec,
                         const double *__restrict__ wavenumber, double k_scalar, const double *__restrict__ mpos,
                         const double *__restrict__ gpos, const double *__restrict__ r0_in,
                         const double *__restrict__ rm, double *__restrict__ out_map, double *__restrict__ out_norm,
                         const double2 *__restrict__ steer, const int *__restrict__ active)
{
    const int bin = blockIdx.y;
    if (active && !active[bin]) return;   // a bin whose iteration has stopped (CLEAN-SC)
    const int64_t g = (int64_t)blockIdx.x * kEigSmallThreads + threadIdx.x;
    if (g >= a.G) return;
    const int M = a.M;
    const double k = wavenumber ? wavenumber[bin] : k_scalar;
    const double *lam = eigval + (int64_t)bin * E;
    const double2 *V = eigvec + (int64_t)bin * M * E;
    const double2 *hv = CUSTOM ? steer + ((int64_t)bin * a.G + g) * M : nullptr;
    double g0 = 0, g1 = 0, g2 = 0;
    if (!USE_RM && !CUSTOM) {
        g0 = gpos[g];
        g1 = gpos[a.G + g];
        g2 = gpos[2 * a.G + g];
    }
    double fr[EMAX], fi[EMAX], dg[EMAX];
#pragma unroll
    for (int j = 0; j < EMAX; ++j) fr[j] = fi[j] = dg[j] = 0.0;
    double S = 0.0;
    for (int m = 0; m < M; ++m) {
        double2 h;
        if (CUSTOM) {
            h = __ldg(hv + m);
            S += h.x * h.x + h.y * h.y;
        } else {
            const double r = USE_RM ? __ldg(rm + g * M + m)
                                    : dist3(g0, g1, g2, __ldg(mpos + m), __ldg(mpos + M + m), __ldg(mpos + 2 * M + m));
            h = steer_value(a, k, r);
            if (a.steer_type >= 2) S += (a.steer_type == 2) ? r * r : 1.0 / (r * r);
        }
        const double2 *vrow = V + (int64_t)m * E;
#pragma unroll
        for (int j = 0; j < EMAX; ++j) {
            if (j >= E) break;
            const double2 v = __ldg(vrow + j);
            // temp1 = conj(V[m][e]) * h[m]
            const double tr = v.x * h.x + v.y * h.y, ti = v.x * h.y - v.y * h.x;
            fr[j] += tr;
            fi[j] += ti;
            if (a.r_diag) dg[j] += tr * tr + ti * ti;
        }
    }
    double scal = 0.0;
#pragma unroll
    for (int j = 0; j < EMAX; ++j) {
        if (j >= E) break;
        const double full = fr[j] * fr[j] + fi[j] * fi[j];
        scal += (a.r_diag ? full - dg[j] : full) * lam[j];
    }
    double r0 = 0.0;
    if (CUSTOM) r0 = 0.0;
    else if (a.ref_mode == 1) r0 = a.ref_dist;
    else if (USE_RM) r0 = r0_in[g];
    else r0 = dist3(g0, g1, g2, a.ref0, a.ref1, a.ref2);
    finish_plain(a, scal, S, r0, bin, g, out_map, out_norm);
}

static int make_args(const acb_map_params *p, MapArgs &a)
{
    if (!p) return ACB_ERR_ARG;
    if (p->num_mics < 2 || p->num_mics > 2048 || p->num_grid <= 0 || p->num_bins <= 0 || p->num_bins > 65535)
        return ACB_ERR_SHAPE;
    if (p->steer_type < 1 || p->steer_type > 4) return ACB_ERR_ARG;
    if (p->glibc_faithful && (!p->sincos_table || p->sincos_table_slots <= 0 ||
                              (p->sincos_table_slots & (p->sincos_table_slots - 1))))
        return ACB_ERR_ARG;
    a.M = p->num_mics;
    a.G = p->num_grid;
    a.steer_type = p->steer_type;
    a.r_diag = p->r_diag;
    a.clip = p->clip_negative;
    a.norm = p->norm;
    a.ref_mode = p->ref_mode;
    a.ref0 = p->ref_point[0];
    a.ref1 = p->ref_point[1];
    a.ref2 = p->ref_point[2];
    a.ref_dist = p->ref_distance;
    a.faithful = p->glibc_faithful;
    a.table = p->sincos_table;
    a.table_mask = p->glibc_faithful ? (uint64_t)p->sincos_table_slots - 1 : 0;
    return ACB_OK;
}

template <bool USE_RM, bool CUSTOM = false>
static int launch_plain(const MapArgs &a, int nbins, const void *csm, const double *k, double k_scalar,
                        const double *mpos,
                        const double *gpos, const double *r0, const double *rm, double *out_map, double *out_norm,
                        cudaStream_t s, const void *steer = nullptr, int *err = nullptr)
{
    if (a.M <= 256) {   // one mic chunk: the staged kernel
        const size_t smem = StagedSmem::total(a.M);
        auto kern = map_plain_staged_kernel<USE_RM, CUSTOM>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        const dim3 grid((unsigned)((a.G + kLanes - 1) / kLanes), nbins);
        kern<<<grid, kLanes * kSWarps, smem, s>>>(a, reinterpret_cast<const double2 *>(csm), k, k_scalar, mpos, gpos,
                                                 r0, rm, out_map, out_norm, reinterpret_cast<const double2 *>(steer),
                                                 err);
        return check_launch();
    }
    const int mc = a.M <= 256 ? a.M : 128;
    const int nbuf = a.M <= mc ? 1 : 2;
    const size_t smem = (size_t)(((3 * a.M + 1) & ~1) * sizeof(double)) + (size_t)nbuf * mc * kLanes * sizeof(double2);
    auto kern = map_plain_kernel<USE_RM, CUSTOM>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const dim3 grid((unsigned)((a.G + kLanes - 1) / kLanes), nbins);
    kern<<<grid, kLanes * kWarps, smem, s>>>(a, reinterpret_cast<const double2 *>(csm), k, k_scalar, mpos, gpos, r0,
                                            rm, mc, out_map, out_norm, reinterpret_cast<const double2 *>(steer));
    return check_launch();
}

template <bool USE_RM, bool CUSTOM = false>
static int launch_eig(const MapArgs &a, int nbins, int E, const double *eigval, const void *eigvec, const double *k,
                      double k_scalar, const double *mpos, const double *gpos, const double *r0, const double *rm,
                      double *out_map, double *out_norm, cudaStream_t s, const void *steer = nullptr,
                      const int *active = nullptr)
{
    if (E <= kEigSmall) {
        const dim3 grid((unsigned)((a.G + kEigSmallThreads - 1) / kEigSmallThreads), nbins);
        auto kern = E == 1 ? map_eig_small_kernel<USE_RM, CUSTOM, 1> : map_eig_small_kernel<USE_RM, CUSTOM, kEigSmall>;
        kern<<<grid, kEigSmallThreads, 0, s>>>(a, E, eigval, reinterpret_cast<const double2 *>(eigvec), k, k_scalar,
                                               mpos, gpos, r0, rm, out_map, out_norm,
                                               reinterpret_cast<const double2 *>(steer), active);
        return check_launch();
    }
    const int mc = a.M <= 256 ? a.M : 128;
    const size_t smem = (size_t)(((3 * a.M + 1) & ~1) * sizeof(double)) + (size_t)mc * kLanes * sizeof(double2);
    auto kern = map_eig_kernel<USE_RM, CUSTOM>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const dim3 grid((unsigned)((a.G + kLanes - 1) / kLanes), nbins);
    kern<<<grid, kLanes * kWarps, smem, s>>>(a, E, eigval, reinterpret_cast<const double2 *>(eigvec), k, k_scalar, mpos,
                                            gpos, r0, rm, mc, out_map, out_norm,
                                            reinterpret_cast<const double2 *>(steer), active);
    return check_launch();
}

// Launchers for other translation units (map_internal.h).
int map_plain_launch(const acb_map_params *p, int nbins, const void *csm, const double *k, const double *mpos,
                     const double *gpos, const double *r0, const double *rm, double *out_map, cudaStream_t s)
{
    MapArgs a;
    const int rc = make_args(p, a);
    if (rc != ACB_OK) return rc;
    if (rm) {
        a.ref_mode = 0;   // r0 is given
        return launch_plain<true>(a, nbins, csm, k, 0.0, nullptr, nullptr, r0, rm, out_map, nullptr, s);
    }
    return launch_plain<false>(a, nbins, csm, k, 0.0, mpos, gpos, nullptr, nullptr, out_map, nullptr, s);
}

int map_eig_launch(const acb_map_params *p, int nbins, int E, const double *eigval, const void *eigvec,
                   const double *k, const double *mpos, const double *gpos, const double *r0, const double *rm,
                   double *out_map, const int *active, cudaStream_t s)
{
    MapArgs a;
    const int rc = make_args(p, a);
    if (rc != ACB_OK) return rc;
    if (rm) {
        a.ref_mode = 0;
        return launch_eig<true>(a, nbins, E, eigval, eigvec, k, 0.0, nullptr, nullptr, r0, rm, out_map, nullptr, s,
                                nullptr, active);
    }
    return launch_eig<false>(a, nbins, E, eigval, eigvec, k, 0.0, mpos, gpos, nullptr, nullptr, out_map, nullptr, s,
                             nullptr, active);
}

int map_eig_custom_launch(const acb_map_params *p, int nbins, int E, const double *eigval, const void *eigvec,
                          const void *steer, double *out_map, const int *active, cudaStream_t s);

}  // namespace acb

using namespace acb;

extern "C" {

int acb_map_f64(const acb_map_params *p, const void *csm, const double *wavenumber, const double *mpos,
                const double *gpos, double *out_map, double *out_steer_norm, int *error_word, void *stream)
{
    MapArgs a;
    int st = make_args(p, a);
    if (st) return st;
    if (!csm || !wavenumber || !mpos || !gpos || !out_map) return ACB_ERR_ARG;
    if ((a.G + kLanes - 1) / kLanes > 0x7fffffffLL) return ACB_ERR_SHAPE;
    return launch_plain<false>(a, p->num_bins, csm, wavenumber, 0.0, mpos, gpos, nullptr, nullptr, out_map,
                               out_steer_norm, as_stream(stream), nullptr, error_word);
}

int acb_map_eig_f64(const acb_map_params *p, int num_eigs, const double *eigval, const void *eigvec,
                    const double *wavenumber, const double *mpos, const double *gpos, double *out_map,
                    double *out_steer_norm, void *stream)
{
    MapArgs a;
    int st = make_args(p, a);
    if (st) return st;
    if (!eigval || !eigvec || !wavenumber || !mpos || !gpos || !out_map) return ACB_ERR_ARG;
    if (num_eigs < 1 || num_eigs > p->num_mics) return ACB_ERR_SHAPE;
    if ((a.G + kLanes - 1) / kLanes > 0x7fffffffLL) return ACB_ERR_SHAPE;
    return launch_eig<false>(a, p->num_bins, num_eigs, eigval, eigvec, wavenumber, 0.0, mpos, gpos, nullptr, nullptr,
                             out_map, out_steer_norm, as_stream(stream));
}

int acb_beamformer_freq_eig_f64(const acb_map_params *p, int num_eigs, const double *eigval, const void *eigvec,
                                double wavenumber, const double *r0, const double *rm, double *out_map,
                                double *out_steer_norm, void *stream)
{
    MapArgs a;
    int st = make_args(p, a);
    if (st) return st;
    if (p->num_bins != 1) return ACB_ERR_SHAPE;
    if (!eigval || !eigvec || !r0 || !rm || !out_map) return ACB_ERR_ARG;
    if (num_eigs < 1 || num_eigs > p->num_mics) return ACB_ERR_SHAPE;
    a.ref_mode = 0;
    return launch_eig<true>(a, 1, num_eigs, eigval, eigvec, nullptr, wavenumber, nullptr, nullptr, r0, rm, out_map,
                            out_steer_norm, as_stream(stream));
}

int acb_map_rm_f64(const acb_map_params *p, const void *csm, const double *wavenumber, const double *r0,
                   const double *rm, double *out_map, double *out_steer_norm, void *stream)
{
    MapArgs a;
    int st = make_args(p, a);
    if (st) return st;
    if (!csm || !wavenumber || !r0 || !rm || !out_map) return ACB_ERR_ARG;
    if ((a.G + kLanes - 1) / kLanes > 0x7fffffffLL) return ACB_ERR_SHAPE;
    a.ref_mode = 0;
    return launch_plain<true>(a, p->num_bins, csm, wavenumber, 0.0, nullptr, nullptr, r0, rm, out_map, out_steer_norm,
                              as_stream(stream));
}

// Custom steering: p->steer_type is ignored; steer: complex128 [num_bins][G][M].
static int custom_args(const acb_map_params *p, MapArgs &a)
{
    if (!p) return ACB_ERR_ARG;
    acb_map_params q = *p;
    q.steer_type = 1;            // any valid type for the shared checks; replaced below
    q.glibc_faithful = 0;        // the steering is given: no phase synthesis
    int st = make_args(&q, a);
    if (st) return st;
    a.steer_type = 0;
    return ACB_OK;
}

int acb_map_custom_f64(const acb_map_params *p, const void *csm, const void *steer, double *out_map,
                       double *out_steer_norm, void *stream)
{
    MapArgs a;
    int st = custom_args(p, a);
    if (st) return st;
    if (!csm || !steer || !out_map) return ACB_ERR_ARG;
    if ((a.G + kLanes - 1) / kLanes > 0x7fffffffLL) return ACB_ERR_SHAPE;
    return launch_plain<false, true>(a, p->num_bins, csm, nullptr, 0.0, nullptr, nullptr, nullptr, nullptr, out_map,
                                     out_steer_norm, as_stream(stream), steer);
}

int acb_map_eig_custom_f64(const acb_map_params *p, int num_eigs, const double *eigval, const void *eigvec,
                           const void *steer, double *out_map, double *out_steer_norm, void *stream)
{
    MapArgs a;
    int st = custom_args(p, a);
    if (st) return st;
    if (!eigval || !eigvec || !steer || !out_map) return ACB_ERR_ARG;
    if (num_eigs < 1 || num_eigs > p->num_mics) return ACB_ERR_SHAPE;
    if ((a.G + kLanes - 1) / kLanes > 0x7fffffffLL) return ACB_ERR_SHAPE;
    return launch_eig<false, true>(a, p->num_bins, num_eigs, eigval, eigvec, nullptr, 0.0, nullptr, nullptr, nullptr,
                                   nullptr, out_map, out_steer_norm, as_stream(stream), steer);
}

int acb_beamformer_freq_f64(const acb_map_params *p, const void *csm, double wavenumber, const double *r0,
                            const double *rm, double *out_map, double *out_steer_norm, void *stream)
{
    MapArgs a;
    int st = make_args(p, a);
    if (st) return st;
    if (p->num_bins != 1) return ACB_ERR_SHAPE;
    if (!csm || !r0 || !rm || !out_map) return ACB_ERR_ARG;
    a.ref_mode = 0;
    st = launch_plain<true>(a, 1, csm, nullptr, wavenumber, nullptr, nullptr, r0, rm, out_map, out_steer_norm,
                            as_stream(stream));
    return st;
}

}  // extern "C"

namespace acb {

int map_eig_custom_launch(const acb_map_params *p, int nbins, int E, const double *eigval, const void *eigvec,
                          const void *steer, double *out_map, const int *active, cudaStream_t s)
{
    MapArgs a;
    const int rc = custom_args(p, a);
    if (rc != ACB_OK) return rc;
    return launch_eig<false, true>(a, nbins, E, eigval, eigvec, nullptr, 0.0, nullptr, nullptr, nullptr, nullptr,
                                   out_map, nullptr, s, steer, active);
}

}  // namespace acb
