// Stage B, tensor-core form: the steered-response map as a real GEMM on tcgen05 with split-BF16
// operands (hi + lo, three products, FP32 accumulation in TMEM).
//
// Formulation.  With h_g = (cos phi - i sin phi) * w(r) the steering vector of grid point g and
// v_g = (Re h_0, Im h_0, Re h_1, Im h_1, ...) in R^{2M}, the map value is
//     B_g = Re(h_g^H C h_g) = v_g^T R v_g,   R[2a+p][2b+q] = [[Re C, -Im C], [Im C, Re C]]_ab,
// with R real symmetric.  Split the 2M components into chunks of 32 (16 mics).  Because R is
// symmetric,  B = sum_j D'_j . v_j  with  D'_j = sum_{i<=j} v_i^T R'_ij,  R'_ij = 2 R_ij (i < j),
// R'_jj = R_jj.  The kernel runs the K loop over chunks i and for each i issues the MMAs into the
// accumulator columns of every chunk j >= i; after chunk i the columns of chunk i are final, so
// the epilogue dots them with v_i while v_i is still in the synthesising thread's registers.
// Steering vectors are never re-synthesised and about half of the dense GEMM is skipped.
//
// Per CTA: 128 grid points (UMMA M = 128, one TMEM lane each) x one frequency bin.
//   warp 0      : bulk copies of the R' tiles of chunk i (pre-laid in HBM in the shared-memory
//                 core-matrix order by tc_prep_kernel) into a 2-stage ring
//   warp 1      : TMEM allocation; one thread issues tcgen05.mma (A = steering chunk, B = R'
//                 tiles; products hi*hi + hi*lo + lo*hi) and commits to the stage's mbarrier
//   warps 2..17 : steering synthesis of chunk i (four threads per grid point, 4 mics each):
//                 FP32 distance (Newton rsqrt), the phase k*r as an exact float-float product,
//                 Cody-Waite reduction by a three-term 2*pi, hardware sincos, bf16 hi/lo split
//                 into the A stage; then the epilogue of chunk i-1 from TMEM.  No FP64<->FP32
//                 conversion sits in the per-element path (the conversion pipe is the scarce one).
// Every mbarrier wait is bounded (globaltimer); on timeout the CTA raises an error word and exits
// its loops without further work.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "tc_common.cuh"

namespace acb {

constexpr int TC_ROWS = 128;
constexpr int TC_CHUNK = 32;               // real components per chunk
constexpr int TC_MPC = TC_CHUNK / 2;       // mics per chunk
constexpr int TC_MAX_CHUNKS = 16;          // 2M <= 512 TMEM columns in one pass
constexpr int TC_TILE_ELEMS = TC_CHUNK * TC_CHUNK;
constexpr int TC_TILE_BYTES = TC_TILE_ELEMS * 2;          // bf16
constexpr int TC_A_BYTES = TC_ROWS * TC_CHUNK * 2;        // 8 KB per (stage, hi|lo)
constexpr int TC_ASTAGES = 3;              // steering (A) ring: synthesis runs up to 2 chunks ahead
constexpr int TC_BSTAGES = 2;              // R' tile (B) ring
constexpr int TC_PARTS = 4;                 // synthesis threads per grid point (one per 4 mics of a chunk)
constexpr int TC_SYNTH_WARPS = 4 * TC_PARTS;  // TC_PARTS warps per TMEM lane quarter
constexpr int TC_SYNTH_THREADS = 32 * TC_SYNTH_WARPS;
constexpr int TC_THREADS = 64 + TC_SYNTH_THREADS;

// 2*pi = P2A + P2B + P2C (Cody-Waite split; P2A has 8 significant bits so n*P2A is exact)
__device__ constexpr float TC_P2A = 0x1.92p+2f;
__device__ constexpr float TC_P2B = 0x1.fb5444p-10f;
__device__ constexpr float TC_P2C = 0x1.68c234p-37f;
__device__ constexpr float TC_INV2PI = 0.15915493667125702f;

struct TcArgs {
    int M, Mp, C;
    int64_t G;
    int steer_type;
    int clip;
    double norm;
    int ref_mode;
    double ref0, ref1, ref2, ref_dist;
    uint64_t wait_limit_ns;
    int64_t bin_stride_elems;  // R' elements per bin (hi and lo separately)
};

__host__ __device__ constexpr int tri_tiles(int C) { return C * (C + 1) / 2; }
// index of tile (i, j >= i) in the row-major upper-triangular tile order
__host__ __device__ constexpr int tile_index(int C, int i, int j) { return i * C - i * (i - 1) / 2 + (j - i); }

// Element offset inside a 32x32 tile (row = n, col = k), K-major no-swizzle core-matrix order.
__device__ __forceinline__ int tile_off(int row, int col)
{
    return (((row >> 3) * 4 + (col >> 3)) << 6) + ((row & 7) << 3) + (col & 7);
}

// ------------------------------------------------------------------------------------------------
// R' in split-BF16, per bin: tiles (i, j >= i) of 32 x 32, stored row = n (column of D), col = k.
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) tc_prep_kernel(const double2 *__restrict__ csm, int M, int C, int r_diag,
                                                      int64_t bin_stride, __nv_bfloat16 *__restrict__ rh,
                                                      __nv_bfloat16 *__restrict__ rl)
{
    int t = blockIdx.x, i = 0;
    while (t >= C - i) {
        t -= C - i;
        ++i;
    }
    const int j = i + t;
    const int bin = blockIdx.y;
    const double2 *Cb = csm + (int64_t)bin * M * M;
    __nv_bfloat16 *th = rh + (int64_t)bin * bin_stride + (int64_t)tile_index(C, i, j) * TC_TILE_ELEMS;
    __nv_bfloat16 *tl = rl + (int64_t)bin * bin_stride + (int64_t)tile_index(C, i, j) * TC_TILE_ELEMS;
    const double factor = (j > i) ? 2.0 : 1.0;
    for (int e = threadIdx.x; e < TC_TILE_ELEMS; e += blockDim.x) {
        const int rr = e >> 5, kk = e & 31;
        const int n = TC_CHUNK * j + rr, k = TC_CHUNK * i + kk;
        const int a = k >> 1, pa = k & 1, b = n >> 1, pb = n & 1;
        double val = 0.0;
        if (a < M && b < M && !(r_diag && a == b)) {
            const double2 c = Cb[(int64_t)a * M + b];
            val = (pa == pb) ? c.x : (pa == 0 ? -c.y : c.y);
            val *= factor;
        }
        const float vf = (float)val;
        const __nv_bfloat16 h = __float2bfloat16_rn(vf);
        const __nv_bfloat16 l = __float2bfloat16_rn(vf - __bfloat162float(h));
        const int o = tile_off(rr, kk);
        th[o] = h;
        tl[o] = l;
    }
}

struct TcSmem {
    // offsets in bytes from the 1024-aligned dynamic shared-memory base
    __host__ __device__ static constexpr int a_off(int stage, int lo) { return (stage * 2 + lo) * TC_A_BYTES; }
    __host__ __device__ static constexpr int b_base() { return TC_ASTAGES * 2 * TC_A_BYTES; }
    __host__ __device__ static constexpr int b_off(int C, int stage, int lo)
    {
        return b_base() + (stage * 2 + lo) * C * TC_TILE_BYTES;
    }
    __host__ __device__ static constexpr int mic_off(int C) { return b_base() + TC_BSTAGES * 2 * C * TC_TILE_BYTES; }
    __host__ __device__ static constexpr int red_off(int C, int Mp) { return mic_off(C) + Mp * 16; }
    __host__ __device__ static constexpr int bar_off(int C, int Mp) { return red_off(C, Mp) + 2 * TC_PARTS * TC_ROWS * 8; }
    __host__ __device__ static constexpr int total(int C, int Mp) { return bar_off(C, Mp) + 128; }
};

template <int ST>
__global__ void __launch_bounds__(TC_THREADS, 1) map_tc_kernel(TcArgs a, const double *__restrict__ wavenumber,
                                                               const double *__restrict__ mpos,
                                                               const double *__restrict__ gpos,
                                                               const __nv_bfloat16 *__restrict__ rh,
                                                               const __nv_bfloat16 *__restrict__ rl,
                                                               double *__restrict__ out_map,
                                                               double *__restrict__ out_norm, int *err)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // operand tiles start on a 1 KB boundary (the launch reserves 1 KB of slack for this)
    uint8_t *smem = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
    const int C = a.C, Mp = a.Mp;
    float4 *mp4 = reinterpret_cast<float4 *>(smem + TcSmem::mic_off(C));        // [Mp] (x, y, z, 0)
    double *red = reinterpret_cast<double *>(smem + TcSmem::red_off(C, Mp));     // [2][parts][128]
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + TcSmem::bar_off(C, Mp));
    uint64_t *full_a = bars;        // [3] steering chunk t in A stage t % 3
    uint64_t *full_b = bars + 3;    // [2] R' tiles of chunk t in B stage t % 2
    uint64_t *done = bars + 5;      // [3] MMAs of chunk t complete (committed to done[t % 3])
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 8);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + 9);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bin = blockIdx.y;
    const int64_t tile0 = (int64_t)blockIdx.x * TC_ROWS;
    const uint32_t ncols = (uint32_t)(C <= 1 ? 32 : (C <= 2 ? 64 : (C <= 4 ? 128 : (C <= 8 ? 256 : 512))));

    for (int m = threadIdx.x; m < Mp; m += blockDim.x) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (m < a.M) v = make_float4((float)mpos[m], (float)mpos[a.M + m], (float)mpos[2 * a.M + m], 0.f);
        mp4[m] = v;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_ASTAGES; ++s) {
            tc::mbar_init(&full_a[s], TC_SYNTH_THREADS);
            tc::mbar_init(&done[s], 1);
        }
        for (int s = 0; s < TC_BSTAGES; ++s) tc::mbar_init(&full_b[s], 1);
        *abort_flag = 0;
        tc::fence_mbar_init();
    }
    if (warp == 1) tc::tmem_alloc(tmem_slot, ncols);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t taddr = *tmem_slot;
    const int64_t bin_off = (int64_t)bin * a.bin_stride_elems;

    if (warp == 0) {
        // ---------------- producer: R' tiles of chunk t ----------------
        if (lane == 0) {
            int last = -1;
            for (int t = 0; t < C && !*abort_flag; ++t) {
                const int s = t & 1;
                // B stage t % 2 was last read by the MMAs of chunk t - 2
                if (t >= TC_BSTAGES &&
                    !tc::mbar_wait(&done[(t - 2) % 3], ((t - 2) / 3) & 1, abort_flag, a.wait_limit_ns))
                    break;
                const uint32_t bytes = (uint32_t)(C - t) * TC_TILE_BYTES;
                tc::mbar_arrive_expect_tx(&full_b[s], 2 * bytes);
                const int64_t src = bin_off + (int64_t)tile_index(C, t, t) * TC_TILE_ELEMS;
                tc::bulk_g2s(smem + TcSmem::b_off(C, s, 0), rh + src, bytes, &full_b[s]);
                tc::bulk_g2s(smem + TcSmem::b_off(C, s, 1), rl + src, bytes, &full_b[s]);
                last = t;
            }
            // on an abort, let the last copies land before the CTA releases its shared memory
            if (*abort_flag && last >= 0)
                tc::mbar_wait(&full_b[last & 1], (last >> 1) & 1, abort_flag, 4 * a.wait_limit_ns);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int last = -1;
            for (int t = 0; t < C && !*abort_flag; ++t) {
                const int sa = t % 3, sb = t & 1;
                if (!tc::mbar_wait(&full_a[sa], (t / 3) & 1, abort_flag, a.wait_limit_ns)) break;
                if (!tc::mbar_wait(&full_b[sb], (t >> 1) & 1, abort_flag, a.wait_limit_ns)) break;
                tc::tc_fence_after();
                const int ntot = TC_CHUNK * (C - t);
                const uint32_t c0 = (uint32_t)(TC_CHUNK * t);
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) {
#pragma unroll
                    for (int prod = 0; prod < 3; ++prod) {
                        const uint32_t a_addr = tc::smem_u32(smem + TcSmem::a_off(sa, prod == 2)) + ks * 256;
                        const uint32_t b_addr = tc::smem_u32(smem + TcSmem::b_off(C, sb, prod == 1)) + ks * 256;
                        const uint64_t ad = tc::sdesc_noswizzle(a_addr, 128, 512);
                        for (int n0 = 0; n0 < ntot; n0 += 256) {
                            const int np = min(256, ntot - n0);
                            const uint64_t bd = tc::sdesc_noswizzle(b_addr + (n0 / TC_CHUNK) * TC_TILE_BYTES, 128, 512);
                            const uint32_t accum = (t == 0 && ks == 0 && prod == 0) ? 0u : 1u;
                            tc::mma_bf16(taddr + c0 + (uint32_t)n0, ad, bd, tc::idesc_m128(1, (uint32_t)np), accum);
                        }
                    }
                }
                tc::mma_commit(&done[sa]);
                last = t;
            }
            if (last >= 0) tc::mbar_wait(&done[last % 3], (last / 3) & 1, abort_flag, 4 * a.wait_limit_ns);
        }
    } else {
        // ---------------- steering synthesis + epilogue (warps 2..17) ----------------
        // Warp w serves TMEM lane quarter q = w % 4 (grid points 32q..32q+31 of the tile) and
        // part p of every chunk: mics 4p..4p+3 of the chunk's 16, components 8p..8p+7, which is
        // exactly one 16-byte core-matrix column of the A tile.
        const int q = warp & 3;
        const int p = (warp - 2) >> 2;
        const int row = q * 32 + lane;     // A row == TMEM lane == grid point in the tile
        const int64_t g = tile0 + row;
        const bool gvalid = g < a.G;
        double gx = 0, gy = 0, gz = 0;
        if (gvalid) {
            gx = gpos[g];
            gy = gpos[a.G + g];
            gz = gpos[2 * a.G + g];
        }
        const float gxf = (float)gx, gyf = (float)gy, gzf = (float)gz;
        const double k = wavenumber[bin];
        const float khi = (float)k, klo = (float)(k - (double)khi);
        const uint32_t lane_addr = taddr + ((uint32_t)(q * 32) << 16);
        constexpr int PC = TC_CHUNK / TC_PARTS;   // components per part
        double S = 0.0, acc = 0.0;
        float va[PC], vb[PC];
        const int a_off_row = (((row >> 3) * 4 + p) << 7) + ((row & 7) << 4);

        auto synth = [&](int t, float (&v)[PC]) {
            const int s = t % 3;
            float s_part = 0.f;
            uint32_t hw[4], lw[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int m = t * TC_MPC + p * 4 + e;
                const bool valid = gvalid && m < a.M;
                const float4 mv = mp4[m];
                const float dx = gxf - mv.x, dy = gyf - mv.y, dz = gzf - mv.z;
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                const float y = tc::rsqrt_approx(r2);           // 1/r, ~2^-22 relative
                float r = r2 * y;
                r = fmaf(fmaf(-r, r, r2), 0.5f * y, r);         // r to ~0.5 ulp
                // phase k*r as an exact float-float product, reduced by the 3-term 2*pi
                const float ph = khi * r;
                const float pl = fmaf(klo, r, fmaf(khi, r, -ph));
                const float nq = __fsub_rn(__fmaf_rn(ph, TC_INV2PI, 12582912.f), 12582912.f);
                float x = fmaf(-nq, TC_P2A, ph);
                x = fmaf(-nq, TC_P2B, x);
                x = fmaf(-nq, TC_P2C, x);
                x += pl;
                float sn, cs;
                tc::sincos_approx(x, sn, cs);
                float w = 1.f;
                if (ST == 2) {
                    w = r;
                    s_part += valid ? r2 : 0.f;
                } else if (ST >= 3) {
                    w = y;
                    s_part += valid ? y * y : 0.f;
                }
                const float vr = valid ? cs * w : 0.f;
                const float vi = valid ? -sn * w : 0.f;
                v[2 * e] = vr;
                v[2 * e + 1] = vi;
                // split-BF16 by integer rounding (half away from zero) of the upper 16 bits:
                // hi = round16(x), lo = round16(x - hi); byte permutes pack (re, im) pairs
                const uint32_t rr = __float_as_uint(vr) + 0x8000u, ri = __float_as_uint(vi) + 0x8000u;
                hw[e] = __byte_perm(rr, ri, 0x7632);
                const float lr = vr - __uint_as_float(rr & 0xFFFF0000u);
                const float li = vi - __uint_as_float(ri & 0xFFFF0000u);
                lw[e] = __byte_perm(__float_as_uint(lr) + 0x8000u, __float_as_uint(li) + 0x8000u, 0x7632);
            }
            *reinterpret_cast<uint4 *>(smem + TcSmem::a_off(s, 0) + a_off_row) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
            *reinterpret_cast<uint4 *>(smem + TcSmem::a_off(s, 1) + a_off_row) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
            S += (double)s_part;
            tc::fence_proxy_async_smem();
            tc::mbar_arrive(&full_a[s]);
        };
        // warp-uniform waits: tcgen05.ld is .sync.aligned, all 32 lanes must take the same path
        auto warp_wait = [&](uint64_t *bar, uint32_t parity) -> bool {
            const bool ok = tc::mbar_wait(bar, parity, abort_flag, a.wait_limit_ns);
            return __all_sync(0xffffffffu, ok);
        };
        auto warp_abort = [&]() -> bool { return __any_sync(0xffffffffu, *abort_flag != 0); };
        auto epilogue = [&](int t, const float (&v)[PC]) {
            if (!warp_wait(&done[t % 3], (t / 3) & 1)) return;
            tc::tc_fence_after();
            float d[PC];
            tc::tmem_ld_x8(lane_addr + (uint32_t)(TC_CHUNK * t + PC * p), d);
            float part = 0.f;
#pragma unroll
            for (int e = 0; e < PC; ++e) part = fmaf(d[e], v[e], part);
            acc += (double)part;
        };
        // Synthesis runs two chunks ahead of the epilogue: chunk t is written to A stage t % 3 while
        // the MMAs of chunks t-1 and t-2 may still run; the columns of chunk t-2 are read after.
        // Stage t % 3 was last used by chunk t-3, whose epilogue (and hence MMA completion) was
        // awaited one iteration earlier.
        float vc[PC];
        auto step = [&](int t, float (&cur)[PC], const float (&old)[PC]) {
            synth(t, cur);
            if (t >= 2) epilogue(t - 2, old);
        };
        int t = 0;
        for (; t + 3 <= C && !warp_abort(); t += 3) {
            step(t, va, vb);       // va: chunk t % 3 == 0; vb: chunk (t - 2) % 3 == 1
            step(t + 1, vb, vc);   // vb: 1; vc: (t - 1) % 3 == 2
            step(t + 2, vc, va);   // vc: 2; va: t % 3 == 0
        }
        if (t < C && !warp_abort()) step(t, va, vb);
        if (t + 1 < C && !warp_abort()) step(t + 1, vb, vc);
        // drain: the last two chunks (slots follow chunk % 3: 0 -> va, 1 -> vb, 2 -> vc)
        for (int tt = (C >= 2 ? C - 2 : 0); tt < C && !warp_abort(); ++tt) {
            if (tt % 3 == 0) epilogue(tt, va);
            else if (tt % 3 == 1) epilogue(tt, vb);
            else epilogue(tt, vc);
        }
        tc::tc_fence_before();
        // combine the per-part partial sums of each grid point (named barrier over the synth warps)
        if (p > 0) {
            red[p * TC_ROWS + row] = acc;
            red[(TC_PARTS + p) * TC_ROWS + row] = S;
        }
        asm volatile("bar.sync 1, %0;" ::"r"(TC_SYNTH_THREADS) : "memory");
        if (p == 0 && gvalid && !*abort_flag) {
            double scalar = acc;
#pragma unroll
            for (int pp = 1; pp < TC_PARTS; ++pp) {
                scalar += red[pp * TC_ROWS + row];
                S += red[(TC_PARTS + pp) * TC_ROWS + row];
            }
            double r0;
            if (a.ref_mode == 1) r0 = a.ref_dist;
            else r0 = dist3(gx, gy, gz, a.ref0, a.ref1, a.ref2);
            const double Md = (double)a.M;
            double res, ns;
            if (ST == 1) {
                ns = 1.0 / Md;
                res = scalar / (Md * Md) * a.norm;
            } else if (ST == 2) {
                const double nf = Md * r0;
                const double nf2 = nf * nf;
                ns = S / nf2;
                res = scalar / nf2 * a.norm;
            } else if (ST == 3) {
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
    }
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc::tc_fence_after();
        tc::tmem_dealloc(taddr, ncols);
    }
    if (threadIdx.x == 0 && *abort_flag && err) atomicOr(err, 1);
}

}  // namespace acb

using namespace acb;

extern "C" {

size_t acb_map_tc_workspace_bytes(int num_mics, int num_bins, int precision)
{
    (void)precision;
    if (num_mics < 2 || num_bins <= 0) return 0;
    const int Mp = (num_mics + TC_MPC - 1) / TC_MPC * TC_MPC;
    const int C = Mp / TC_MPC;
    return (size_t)2 * (size_t)num_bins * (size_t)tri_tiles(C) * TC_TILE_BYTES;
}

int acb_map_tc(const acb_map_params *p, int precision, const void *csm, const double *wavenumber, const double *mpos,
               const double *gpos, double *out_map, double *out_steer_norm, void *workspace, size_t workspace_bytes,
               int *error_word, void *stream)
{
    if (!p || !csm || !wavenumber || !mpos || !gpos || !out_map) return ACB_ERR_ARG;
    if (precision != ACB_TC_BF16X3) return ACB_ERR_UNSUPPORTED;
    if (p->steer_type < 1 || p->steer_type > 4) return ACB_ERR_ARG;
    if (p->num_mics < 2 || p->num_grid <= 0 || p->num_bins <= 0 || p->num_bins > 65535) return ACB_ERR_SHAPE;
    const int M = p->num_mics;
    const int Mp = (M + TC_MPC - 1) / TC_MPC * TC_MPC;
    const int C = Mp / TC_MPC;
    if (C > TC_MAX_CHUNKS) return ACB_ERR_UNSUPPORTED;
    const size_t need = acb_map_tc_workspace_bytes(M, p->num_bins, precision);
    if (!workspace || workspace_bytes < need) return ACB_ERR_WORKSPACE;
    if ((p->num_grid + TC_ROWS - 1) / TC_ROWS > 0x7fffffffLL) return ACB_ERR_SHAPE;
    cudaStream_t s = as_stream(stream);
    TcArgs a;
    a.M = M;
    a.Mp = Mp;
    a.C = C;
    a.G = p->num_grid;
    a.steer_type = p->steer_type;
    a.clip = p->clip_negative;
    a.norm = p->norm;
    a.ref_mode = p->ref_mode;
    a.ref0 = p->ref_point[0];
    a.ref1 = p->ref_point[1];
    a.ref2 = p->ref_point[2];
    a.ref_dist = p->ref_distance;
    a.wait_limit_ns = 500ull * 1000 * 1000;
    a.bin_stride_elems = (int64_t)tri_tiles(C) * TC_TILE_ELEMS;
    __nv_bfloat16 *rh = reinterpret_cast<__nv_bfloat16 *>(workspace);
    __nv_bfloat16 *rl = rh + (size_t)p->num_bins * a.bin_stride_elems;
    tc_prep_kernel<<<dim3(tri_tiles(C), p->num_bins), 256, 0, s>>>(reinterpret_cast<const double2 *>(csm), M, C,
                                                                   p->r_diag, a.bin_stride_elems, rh, rl);
    int st = check_launch();
    if (st) return st;
    int smem = TcSmem::total(C, Mp) + 1024;
    // a CTA that takes all 512 TMEM columns must be alone on its SM: size the shared memory so
    // that no second CTA fits (a second one would stall in tcgen05.alloc until the first exits)
    if (C > 8 && smem < 116 * 1024) smem = 116 * 1024;
    const dim3 grid((unsigned)((p->num_grid + TC_ROWS - 1) / TC_ROWS), p->num_bins);
    auto kern = p->steer_type == 1 ? map_tc_kernel<1>
                : p->steer_type == 2 ? map_tc_kernel<2>
                : p->steer_type == 3 ? map_tc_kernel<3>
                                     : map_tc_kernel<4>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    kern<<<grid, TC_THREADS, smem, s>>>(a, wavenumber, mpos, gpos, rh, rl, out_map, out_steer_norm, error_word);
    return check_launch();
}

}  // extern "C"
