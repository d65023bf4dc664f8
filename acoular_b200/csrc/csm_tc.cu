// Stage A, tensor-core form: the Welch Gram sum_w conj(X_w[c]) X_w[r] of PowerSpectra.calc_csm
// (acoular/spectra.py:407-410, the calcCSM contraction acoular/fastFuncs.py:19-58) as a real
// symmetric rank-K update on tcgen05.
//
// Formulation.  With Y[w][2m] = Re X_w[m], Y[w][2m+1] = Im X_w[m] (K windows x 2M components),
//     D = Y^T Y,   C[r][c] = sum_w conj(X_w[c]) X_w[r]:
//     Re C[r][c] = D[2r][2c] + D[2r+1][2c+1],   Im C[r][c] = D[2r+1][2c] - D[2r][2c+1].
// D is symmetric, so only its upper block triangle is computed: 2 M^2 K multiply-adds per bin
// (the 3M complex product would take 3 M^2 K).  The operand Y^T is written by the FFT directly as
// TF32 or split-BF16 (hi + lo; three products hi*hi + hi*lo + lo*hi) 32 x 32 K-major tiles
// [bin][window/32][component/32]; FP32 accumulation in TMEM over the window chunk, then an FP64
// add into the complex128 upper triangle that the FP64 path also fills.
//
// Work item: one bin x one block of 128 rows (4 row tiles) x 4 column tiles (128 columns) at or
// right of the block's diagonal.  Persistent CTAs (one per SM) walk the items in bin order; per item
// the K loop streams 32-window stages of the A (4 tiles) and B (4 tiles) operands through a 6-stage
// ring of bulk copies into this CTA alone.  Two TMEM accumulators alternate between items so that the
// epilogue of one item overlaps the MMAs of the next.  All items cost the same, so the CTAs stay in
// step and the items of a bin run at about the same time, reading the bin's tiles from L2: with
// items of 4 and 8 column tiles mixed, the CTAs drifted apart by several waves and read the
// operands 2.3 times from DRAM (measured: the Gram 0.19 ms faster on the 256-mic workload).
//   warp 0     : bulk-copy producer (one thread)
//   warp 1     : TMEM allocation; one thread issues the MMAs and commits
//   warps 2..5 : epilogue: a thread owns one accumulator row (component); even/odd neighbours
//                exchange their rows with a shuffle and each forms half of the complex entries
// Every mbarrier wait is bounded (globaltimer); on timeout the CTA raises an error word and exits.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "csm_internal.h"
#include "tc_common.cuh"
#include "tc_layout.cuh"

namespace acb {

constexpr int GTC_TILE_BYTES = 4096;        // a TF32 tile, or a BF16 hi + lo tile pair
constexpr int GTC_ROWT = 4;                 // row tiles per item (128 rows)
constexpr int GTC_MAXC = 4;                 // column tiles per item (N <= 128)
constexpr int GTC_STAGE_BYTES = (GTC_ROWT + GTC_MAXC) * GTC_TILE_BYTES;   // 32 KB
constexpr int GTC_STAGES = 6;
constexpr int GTC_THREADS = 192;
constexpr int GTC_MAX_ITEMS = 1024;         // items per bin (row block, first column tile)

struct GtcItem {
    uint8_t rb, c0, nc, pad;
};

struct GtcArgs {
    const uint8_t *ops;        // operand tiles (TF32, or BF16 hi tiles followed by lo tiles)
    int64_t lo_bytes;          // BF16: byte offset of the lo tiles from the hi tiles
    int R, KC, M, nbins, nper;
    int64_t nitems;
    double2 *csm;              // complex128 [nbins][M][M], upper triangle accumulated
    uint64_t wait_limit_ns;
    GtcItem it[GTC_MAX_ITEMS];
};

__host__ __device__ constexpr int gtc_smem_bytes() { return GTC_STAGES * GTC_STAGE_BYTES + 1024 + 256; }

template <bool TF32>
__global__ void __launch_bounds__(GTC_THREADS, 1) gram_tc_kernel(const __grid_constant__ GtcArgs a, int *err)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + GTC_STAGES * GTC_STAGE_BYTES);
    uint64_t *full = bars;                         // [GTC_STAGES] stage landed
    uint64_t *empty = bars + GTC_STAGES;           // [GTC_STAGES] MMAs reading the stage are complete
    uint64_t *accf = bars + 2 * GTC_STAGES;        // [2] accumulator buffer complete
    uint64_t *acce = accf + 2;                     // [2] epilogue has read the accumulator buffer
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(acce + 2);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(acce + 3);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t nmine = a.nitems > blockIdx.x ? (a.nitems - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const int64_t tiles_bin = (int64_t)a.KC * a.R;

    if (threadIdx.x == 0) {
        for (int s = 0; s < GTC_STAGES; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&accf[b], 1);
            tc::mbar_init(&acce[b], 128);
        }
        *abort_flag = 0;
        tc::fence_mbar_init();
    }
    if (warp == 1) tc::tmem_alloc(tmem_slot, 512);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t taddr = *tmem_slot;

    if (warp == 0) {
        // ---------------- producer: A (4 row tiles) and B (nc column tiles) per 32-window stage
        if (lane == 0) {
            int s = 0, u = 0, lastS = -1, lastU = 0;
            int64_t n = 0;   // stages issued
            bool ok = true;
            for (int64_t li = 0; li < nmine && ok; ++li) {
                const int64_t item = blockIdx.x + li * gridDim.x;
                const int64_t bin = item / a.nper;
                const GtcItem g = a.it[item - bin * a.nper];
                for (int kc = 0; kc < a.KC && ok; ++kc, ++n) {
                    if (n >= GTC_STAGES) ok = tc::mbar_wait(&empty[s], (uint32_t)(u ^ 1), abort_flag, a.wait_limit_ns);
                    if (!ok) break;
                    const int64_t t0 = bin * tiles_bin + (int64_t)kc * a.R;
                    const uint32_t abytes = GTC_ROWT * GTC_TILE_BYTES, bbytes = (uint32_t)g.nc * GTC_TILE_BYTES;
                    tc::mbar_arrive_expect_tx(&full[s], abytes + bbytes);
                    uint8_t *st = smem + s * GTC_STAGE_BYTES;
                    if (TF32) {
                        tc::bulk_g2s(st, a.ops + (t0 + GTC_ROWT * g.rb) * GTC_TILE_BYTES, abytes, &full[s]);
                        tc::bulk_g2s(st + abytes, a.ops + (t0 + g.c0) * GTC_TILE_BYTES, bbytes, &full[s]);
                    } else {
                        // stage: A hi | A lo | B hi | B lo, 2 KB tiles
                        const uint32_t ah = abytes / 2, bh = bbytes / 2;
                        const uint8_t *hi = a.ops, *lo = a.ops + a.lo_bytes;
                        tc::bulk_g2s(st, hi + (t0 + GTC_ROWT * g.rb) * (GTC_TILE_BYTES / 2), ah, &full[s]);
                        tc::bulk_g2s(st + ah, lo + (t0 + GTC_ROWT * g.rb) * (GTC_TILE_BYTES / 2), ah, &full[s]);
                        tc::bulk_g2s(st + abytes, hi + (t0 + g.c0) * (GTC_TILE_BYTES / 2), bh, &full[s]);
                        tc::bulk_g2s(st + abytes + bh, lo + (t0 + g.c0) * (GTC_TILE_BYTES / 2), bh, &full[s]);
                    }
                    lastS = s;
                    lastU = u;
                    if (++s == GTC_STAGES) { s = 0; u ^= 1; }
                }
            }
            // on an abort, let every copy still in flight land before the CTA releases its shared
            // memory: the last GTC_STAGES issued stages (n of them at most)
            if (*abort_flag)
                for (int j = 0; j < GTC_STAGES && j < n; ++j) {
                    const int st = (lastS - j + GTC_STAGES) % GTC_STAGES;
                    tc::mbar_drain(&full[st], (uint32_t)(lastS - j >= 0 ? lastU : lastU ^ 1),
                                   tc::drain_limit_ns(a.wait_limit_ns));
                }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer
        if (lane == 0) {
            constexpr uint32_t SBO = TF32 ? 1024 : 512;
            const uint64_t sbase = tc::sdesc_noswizzle(tc::smem_u32(smem), 128, SBO);
            const uint32_t idesc0 = tc::idesc_m128(TF32 ? 2 : 1, 0);
            int s = 0, u = 0;
            uint64_t *lastBar = nullptr;   // barrier of the last commit (commits complete in order)
            uint32_t lastPar = 0;
            bool ok = true;
            for (int64_t li = 0; li < nmine && ok; ++li) {
                const int64_t item = blockIdx.x + li * gridDim.x;
                const int64_t bin = item / a.nper;
                const GtcItem g = a.it[item - bin * a.nper];
                const int buf = (int)(li & 1);
                if (li >= 2) ok = tc::mbar_wait(&acce[buf], (uint32_t)(((li >> 1) - 1) & 1), abort_flag, a.wait_limit_ns);
                if (!ok) break;
                tc::tc_fence_after();
                const uint32_t dcol = taddr + (uint32_t)(buf * 256);
                const uint32_t idesc = idesc0 | ((uint32_t)(g.nc * 4) << 17);   // N = 32 nc
                const uint32_t abytes = GTC_ROWT * GTC_TILE_BYTES;
                for (int kc = 0; kc < a.KC && ok; ++kc) {
                    ok = tc::mbar_wait(&full[s], (uint32_t)u, abort_flag, a.wait_limit_ns);
                    if (!ok) break;
                    tc::tc_fence_after();
                    const uint64_t sd = sbase + (uint64_t)((s * GTC_STAGE_BYTES) >> 4);
                    if (TF32) {
                        const uint64_t ad = sd, bd = sd + (abytes >> 4);
#pragma unroll
                        for (int ks = 0; ks < 4; ++ks)
                            tc::mma_tf32(dcol, ad + ks * 16, bd + ks * 16, idesc, (kc | ks) ? 1u : 0u);
                    } else {
                        const uint32_t ah = abytes / 2, bh = (uint32_t)g.nc * GTC_TILE_BYTES / 2;
                        const uint64_t ahi = sd, alo = sd + (ah >> 4), bhi = sd + (abytes >> 4),
                                       blo = sd + ((abytes + bh) >> 4);
#pragma unroll
                        for (int ks = 0; ks < 2; ++ks) {
                            tc::mma_bf16(dcol, ahi + ks * 16, bhi + ks * 16, idesc, (kc | ks) ? 1u : 0u);
                            tc::mma_bf16(dcol, ahi + ks * 16, blo + ks * 16, idesc, 1u);
                            tc::mma_bf16(dcol, alo + ks * 16, bhi + ks * 16, idesc, 1u);
                        }
                    }
                    tc::mma_commit(&empty[s]);
                    lastBar = &empty[s];
                    lastPar = (uint32_t)u;
                    if (++s == GTC_STAGES) { s = 0; u ^= 1; }
                }
                if (!ok) break;
                tc::mma_commit(&accf[buf]);
                lastBar = &accf[buf];
                lastPar = (uint32_t)((li >> 1) & 1);
            }
            // before TMEM is released: every MMA issued has completed
            if (lastBar) tc::mbar_drain(lastBar, lastPar, tc::drain_limit_ns(a.wait_limit_ns));
        }
    } else {
        // ---------------- epilogue (warps 2..5: TMEM lane quarters 2, 3, 0, 1)
        const int q = warp & 3;
        const int rho = q * 32 + lane;              // accumulator row = component in the row block
        const int p = lane & 1;                     // 0: Re row 2r, 1: Im row 2r+1
        bool ok = true;
        for (int64_t li = 0; li < nmine && ok; ++li) {
            const int64_t item = blockIdx.x + li * gridDim.x;
            const int64_t bin = item / a.nper;
            const GtcItem g = a.it[item - bin * a.nper];
            const int buf = (int)(li & 1);
            ok = __all_sync(0xffffffffu,
                            tc::mbar_wait(&accf[buf], (uint32_t)((li >> 1) & 1), abort_flag, a.wait_limit_ns));
            if (!ok) break;
            tc::tc_fence_after();
            const int r = (GTC_ROWT * 32 * g.rb + rho) >> 1;   // mic of this row
            double2 *crow = a.csm + ((int64_t)bin * a.M + r) * a.M;
            for (int j = 0; j < g.nc; ++j) {
                float v[32], w[32];
                tc::tmem_ld_x32(taddr + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 256 + 32 * j), v);
#pragma unroll
                for (int t = 0; t < 32; ++t) w[t] = __shfl_xor_sync(0xffffffffu, v[t], 1);
                // even lane: columns (mics) 0..7 of the tile, odd lane: 8..15; re = row 2r, im = row 2r+1
                const int cb = 16 * (g.c0 + j) + 8 * p;
#pragma unroll
                for (int t2 = 0; t2 < 8; ++t2) {
                    const float dre_re = p ? w[2 * (t2 + 8)] : v[2 * t2];              // D[2r][2c]
                    const float dre_im = p ? w[2 * (t2 + 8) + 1] : v[2 * t2 + 1];      // D[2r][2c+1]
                    const float dim_re = p ? v[2 * (t2 + 8)] : w[2 * t2];              // D[2r+1][2c]
                    const float dim_im = p ? v[2 * (t2 + 8) + 1] : w[2 * t2 + 1];      // D[2r+1][2c+1]
                    const int c = cb + t2;
                    if (r < a.M && c < a.M && c >= r) {
                        double2 cur = crow[c];
                        cur.x += (double)dre_re + (double)dim_im;
                        // the diagonal sum_w |X_w[r]|^2 is real; its two mirrored accumulator
                        // entries differ by FP32 rounding only
                        if (c != r) cur.y += (double)dim_re - (double)dre_im;
                        crow[c] = cur;
                    }
                }
            }
            tc::tc_fence_before();
            tc::mbar_arrive(&acce[buf]);
        }
    }
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc::tc_fence_after();
        tc::tmem_dealloc(taddr, 512);
    }
    if (threadIdx.x == 0 && *abort_flag && err) atomicOr(err, 1);
}

// Rows of the operand: mics padded to a multiple of 64 (whole 128-row blocks), 2 components each.
int csm_tc_row_tiles(int num_mics) { return (num_mics + 63) / 64 * 4; }

size_t csm_tc_workspace_bytes(int num_mics, int num_bins, int64_t num_windows)
{
    const int64_t KC = (num_windows + 31) / 32;
    return (size_t)num_bins * (size_t)KC * (size_t)csm_tc_row_tiles(num_mics) * GTC_TILE_BYTES;
}

int csm_tc_accumulate(const void *samples, int sample_dtype, int num_mics, int block_size, int hop,
                      int64_t first_window, int64_t num_windows, const double *window, const double2 *tw,
                      int bin_lo, int num_bins, bool tf32, void *csm_upper, void *workspace, void *fft_scratch,
                      cudaStream_t s)
{
    const int R = csm_tc_row_tiles(num_mics);
    const int KC = (int)((num_windows + 31) / 32);
    const size_t ops_bytes = csm_tc_workspace_bytes(num_mics, num_bins, num_windows);
    // padded windows and padded mics must read as zero (the four-window transform writes them itself)
    if (!fft_tiles_written_whole(block_size)) {
        const cudaError_t e = cudaMemsetAsync(workspace, 0, ops_bytes, s);
        if (e != cudaSuccess) {
            set_cuda_error(e);
            return ACB_ERR_CUDA;
        }
    }
    const int64_t lo_elems = (int64_t)num_bins * KC * R * 1024;   // BF16: lo tiles after the hi tiles
    int st = fft_launch(samples, sample_dtype, tf32 ? 2 : 3, num_mics, block_size, hop, first_window, num_windows,
                        window, tw, bin_lo, num_bins, workspace, R, KC, lo_elems, fft_scratch, s);
    if (st) return st;

    GtcArgs a;
    a.ops = reinterpret_cast<const uint8_t *>(workspace);
    a.lo_bytes = lo_elems * 2;
    a.R = R;
    a.KC = KC;
    a.M = num_mics;
    a.nbins = num_bins;
    int n = 0;
    for (int rb = 0; rb < R / GTC_ROWT; ++rb)
        for (int c0 = GTC_ROWT * rb; c0 < R; c0 += GTC_MAXC) {
            if (n >= GTC_MAX_ITEMS) return ACB_ERR_UNSUPPORTED;
            a.it[n].rb = (uint8_t)rb;
            a.it[n].c0 = (uint8_t)c0;
            a.it[n].nc = (uint8_t)(R - c0 < GTC_MAXC ? R - c0 : GTC_MAXC);
            a.it[n].pad = 0;
            ++n;
        }
    a.nper = n;
    a.nitems = (int64_t)n * num_bins;
    a.csm = reinterpret_cast<double2 *>(csm_upper);
    a.wait_limit_ns = tc_wait_limit_ns();
    int dev = 0, nsm = kNumSMs;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = (unsigned)(a.nitems < nsm ? a.nitems : nsm);
    const int smem = gtc_smem_bytes();
    auto kern = tf32 ? gram_tc_kernel<true> : gram_tc_kernel<false>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    kern<<<grid, GTC_THREADS, smem, s>>>(a, nullptr);
    return check_launch();
}

}  // namespace acb
