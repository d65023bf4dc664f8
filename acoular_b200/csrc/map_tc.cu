// Stage B, tensor-core form: the steered-response map as a real GEMM on tcgen05 with FP32
// accumulation in TMEM, in one of three operand forms: split BF16 (hi + lo, three products), FP32
// rounded to TF32, or FP16 with each bin's R' scaled by a power of two.
//
// Formulation.  With h_g = (cos phi - i sin phi) * w(r) the steering vector of grid point g and
// v_g = (Re h_0, Im h_0, Re h_1, Im h_1, ...) in R^{2M}, the map value is
//     B_g = Re(h_g^H C h_g) = v_g^T R v_g,   R[2a+p][2b+q] = [[Re C, -Im C], [Im C, Re C]]_ab,
// with R real symmetric.  Split the 2M components into chunks of 32 (16 mics).  Because R is
// symmetric,  B = sum_j D'_j . v_j  with  D'_j = sum_{i<=j} v_i^T R'_ij,  R'_ij = 2 R_ij (i < j),
// R'_jj = R_jj.  The kernel runs the K loop over chunks i and for each i issues the MMAs into the
// accumulator columns of every chunk j >= i; after chunk i the columns of chunk i are final, so
// the epilogue dots them with v_i while v_i is still in the A stage.  Steering vectors are never
// re-synthesised and about half of the dense GEMM is skipped.
//
// Work item: 128 grid points (UMMA M = 128, one TMEM lane each) x one frequency bin x one group of
// column passes.  The accumulator columns of an item are covered in passes of `pw` chunks (a
// runtime tile width: 4, 8 or 16 chunks = 128, 256 or 512 TMEM columns); with `splits` > 1 the
// passes of one (bin, tile) are shared among several items whose partial sums (B and the
// normalisation sum S are both additive over chunks) are combined by the last item to finish, in
// split order, before the steering-type normalisation.
//
// Pipeline step: one A stage (16 KB), i.e. one chunk (split BF16, TF32) or two (FP16, 8 KB each).
// Every role works per step: one steering arrival, one R' tile barrier, one MMA commit, one
// epilogue wait and release.
//   warp 5      : bulk copies of the step's R' tiles (pre-laid in HBM in the shared-memory
//                 core-matrix order by tc_prep_kernel) into a 128 KB tile ring, running ahead
//   warp 1      : TMEM allocation; one thread issues tcgen05.mma (A = steering chunk, B = R'
//                 tiles) and commits to the step's mbarrier
//   warps 0,9,2,3: epilogue (TMEM lane quarters 0..3): after the step's MMAs, read the final
//                 accumulator columns from TMEM and dot them with the steering chunks read back
//                 from the A stage
//   16 warps    : steering synthesis (four threads per grid point, 4 mics of each chunk), packed
//                 FP32: distance by rsqrt, the phase (k as a float-float; reduced by a three-term
//                 2*pi for split BF16), hardware sincos, the operand conversion into the A stage.
//                 No FP64 arithmetic and no TMEM access sits in the per-element path.
// Every mbarrier wait is bounded (globaltimer); on timeout the CTA raises an error word and exits
// its loops without further work.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "common.cuh"
#include "tc_common.cuh"
#include "tc_layout.cuh"

namespace acb {

constexpr uint64_t TC_DEFAULT_WAIT_LIMIT_NS = 500ull * 1000 * 1000;
static std::atomic<uint64_t> g_tc_wait_limit_ns{TC_DEFAULT_WAIT_LIMIT_NS};

uint64_t tc_wait_limit_ns() { return g_tc_wait_limit_ns.load(std::memory_order_relaxed); }

constexpr int TC_ROWS = 128;
constexpr int TC_CHUNK = 32;               // real components per chunk
constexpr int TC_MPC = TC_CHUNK / 2;       // mics per chunk
constexpr int TC_PASS_CHUNKS = 16;         // widest column pass (512 TMEM columns), the default
constexpr int TC_MAX_SPLIT = 8;            // pass groups per (bin, tile)
constexpr int TC_MAX_MICS = 2048;          // mic positions live in shared memory
constexpr int TC_TILE_ELEMS = TC_CHUNK * TC_CHUNK;
constexpr int TC_TILE_BYTES = TC_TILE_ELEMS * 2;          // bf16
constexpr int TC_A_BYTES = TC_ROWS * TC_CHUNK * 2;        // 8 KB per (stage, hi|lo)
// steering (A) ring: 3 to 5 stages, the most that fit in shared memory beside the batch's mic table
// (synthesis runs up to stages - 1 chunks ahead of the MMAs)
constexpr int TC_ASTAGES_MIN = 3;
constexpr int TC_ASTAGES_MAX = 5;
constexpr int TC_RING = 32;                // R' tile (B) ring: 32 tiles of hi + lo (128 KB)
constexpr int TC_PARTS = 4;                 // synthesis threads per grid point (one per 4 mics of a chunk)
constexpr int TC_SYNTH_WARPS = 4 * TC_PARTS;  // TC_PARTS warps per TMEM lane quarter
constexpr int TC_SYNTH_THREADS = 32 * TC_SYNTH_WARPS;
constexpr int TC_EPI_WARPS = 4;             // one per TMEM lane quarter
constexpr int TC_EPI_THREADS = 32 * TC_EPI_WARPS;
// Warp layout.  A warp's scheduler (SM sub-partition) is warp % 4.  The single-thread MMA issuer must
// not share its scheduler with many compute-bound synthesis warps: a scheduler that always has a
// ready FMA warp leaves the issuer's scalar instructions waiting for issue slots, and the tensor pipe
// idles (measured on B200: a tcgen05.mma stream 50x slower next to FMA-bound warps on the same
// scheduler, unchanged when they sit on the other three).  Scheduler 1 holds the MMA issuer (warp 1),
// the bulk-copy producer (warp 5), the epilogue warp of TMEM lane quarter 1 (warp 9; a warp reads the
// TMEM lanes of quarter warp % 4) and one synthesis warp (13); warps 17 and 21 idle.  Schedulers 0, 2
// and 3 hold one epilogue warp and five synthesis warps each.  Six warps per scheduler leave 80
// registers per thread (registers are allocated per scheduler, 16,384 each).
constexpr int TC_WARPS = 24;
constexpr int TC_THREADS = 32 * TC_WARPS;
constexpr int TC_WARP_MMA = 1;
constexpr int TC_WARP_PRODUCER = 5;
__host__ __device__ constexpr bool tc_is_epi(int w) { return w == 0 || w == 2 || w == 3 || w == 9; }
// index 0..15 of a synthesis warp, -1 for other warps
__host__ __device__ constexpr int tc_synth_index(int w)
{
    return (w < 4 || w >= TC_WARPS || w == 5 || w == 9 || w == 17 || w == 21)
               ? -1
               : (w - 4) - (w > 5) - (w > 9) - (w > 17) - (w > 21);
}
static_assert(tc_synth_index(4) == 0 && tc_synth_index(13) == 7 && tc_synth_index(23) == TC_SYNTH_WARPS - 1,
              "synthesis warp indices");

// 2*pi = P2A + P2B + P2C (Cody-Waite split; P2A has 8 significant bits so n*P2A is exact)
__device__ constexpr float TC_P2A = 0x1.92p+2f;
__device__ constexpr float TC_P2B = 0x1.fb5444p-10f;
__device__ constexpr float TC_P2C = 0x1.68c234p-37f;
__device__ constexpr float TC_INV2PI = 0.15915493667125702f;

// One beamforming instance of a batch: its geometry, CSM operand and outputs.  The batch's
// instances travel in the kernel parameters (grid constant), so a launch needs no device-side
// descriptor upload and can be captured in a CUDA graph as it is.
struct TcInst {
    int64_t item_off;          // first global work item of this instance
    int64_t ntiles;            // 128-point grid tiles
    int64_t G;
    int M, Mp, C, nbins;
    int clip, ref_mode;
    double norm, ref0, ref1, ref2, ref_dist;
    const double *k;           // [nbins] wave numbers
    const double *mpos;        // [3][M]
    const double *gpos;        // [3][G]
    double *out;               // [nbins][G]
    double *out_norm;          // [nbins][G] or null
    const __nv_bfloat16 *rh, *rl;   // split-BF16 R' tiles, bin_stride elements per bin
    int64_t bin_stride;
    int pw, P, splits;         // pass width (chunks), passes per (bin, tile), pass groups
    uint8_t sp0[TC_MAX_SPLIT + 1];  // pass group s covers passes [sp0[s], sp0[s+1])
    double2 *part;             // [nbins * ntiles][splits][128] partial (B, S) when splits > 1
    int *cnt;                  // [nbins * ntiles][4] finished groups per epilogue warp (zeroed per launch)
    int small;                 // every item number of the batch < 2^31: item decoding in 32-bit arithmetic
};

// Position of a work item inside its instance: items run (bin, tile, group) with the group fastest.
struct TcItem {
    int64_t base;              // bin * ntiles + tile
    int bin, split, pa, pz;    // passes [pa, pz)
    int64_t tile;
};

__device__ __forceinline__ TcItem decode_item(const TcInst &in, int64_t item)
{
    TcItem t;
    if (in.small) {
        // 32-bit division: the decode sits on the single-thread MMA issuer's path once per item
        const uint32_t local = (uint32_t)(item - in.item_off), sp = (uint32_t)in.splits, nt = (uint32_t)in.ntiles;
        const uint32_t base = local / sp;
        t.split = (int)(local - base * sp);
        t.base = base;
        t.bin = (int)(base / nt);
        t.tile = base - (uint32_t)t.bin * nt;
    } else {
        const int64_t local = item - in.item_off;
        t.split = (int)(local % in.splits);
        t.base = local / in.splits;
        t.bin = (int)(t.base / in.ntiles);
        t.tile = t.base % in.ntiles;
    }
    t.pa = in.sp0[t.split];
    t.pz = in.sp0[t.split + 1];
    return t;
}

constexpr int TC_MAX_INST = 64;

struct TcBatch {
    int n_inst;
    int mp_max;                // largest padded mic count (shared-memory mic table size)
    int nstages;               // A stages (TC_ASTAGES_MIN .. TC_ASTAGES_MAX)
    int64_t nitems;
    uint64_t wait_limit_ns;
    TcInst inst[TC_MAX_INST];
};

__device__ __forceinline__ int find_inst(const TcBatch &b, int64_t item)
{
    int lo = 0, hi = b.n_inst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (b.inst[mid].item_off <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

constexpr int TC_NB = 8;       // chunk barrier ring (full_b / done); the producer runs <= 7 chunks ahead
// The epilogue waits on every step's `done` barrier in turn; the MMAs of step T + TC_NB complete the
// same barrier slot again.  They need the A stage of step T + TC_NB, which the epilogue frees at step
// T + TC_NB - stages, so with at most TC_NB A stages the epilogue has always seen step T first (more
// stages would let a slot run two phases ahead of its waiter and the parity wait would never pass).
static_assert(TC_ASTAGES_MAX <= TC_NB, "A ring deeper than the step barrier ring");

__host__ __device__ constexpr int tri_tiles(int C) { return C * (C + 1) / 2; }
// index of tile (i, j >= i) in the row-major upper-triangular tile order
__host__ __device__ constexpr int tile_index(int C, int i, int j) { return i * C - i * (i - 1) / 2 + (j - i); }

// ------------------------------------------------------------------------------------------------
// R' in split-BF16, per bin: tiles (i, j >= i) of 32 x 32, stored row = n (column of D), col = k.
// ------------------------------------------------------------------------------------------------
// Position of padding mics and of grid rows past the end of the grid: far away, so that 1/r and
// its square vanish (1e-18, 1e-37) while r, r^2 and the phase stay finite.  Padding mics have zero
// R' rows and columns, and the rows past the grid are never written, so neither needs masking.
constexpr float TC_FAR = 1e18f;

// Operand precisions of the tensor-core form (the values of acb_tc_precision).
constexpr int TC_SPLIT = 0;   // split-BF16 hi/lo, three products
constexpr int TC_TF = 1;      // FP32 rounded to TF32
constexpr int TC_HALF = 2;    // FP16, R' scaled per bin by a power of two

// FP16 operands: the R' tiles of a bin are scaled by 2^e with e = 15 - ceil-exponent of the bin's
// largest |R'| entry, so that every entry lies below 2^15 (FP16 holds up to 65504) and the bin keeps
// FP16's full 11-bit precision down to 2^-14 of that scale; the map sums are scaled back by 2^-e.
// The largest entry of each bin is found first (tc_binmax_kernel) and kept as FP64 bits in the
// workspace half that the FP16 tiles leave unused.
__device__ __forceinline__ int tc_half_shift(const unsigned long long *bmax, int bin)
{
    const double mx = __longlong_as_double((long long)bmax[bin]);
    int ex = 0;
    if (mx > 0.0) frexp(mx, &ex);   // mx < 2^ex
    return mx > 0.0 ? 15 - ex : 0;
}

// Tile (i, j >= i) of the CTA's blockIdx.x in the upper-triangular tile order of C chunks.
__device__ __forceinline__ void tc_tile_of_block(int C, int &i, int &j)
{
    int t = blockIdx.x;
    i = 0;
    while (t >= C - i) {
        t -= C - i;
        ++i;
    }
    j = i + t;
}

// Entry (rr, kk) of R' tile (i, j): row n = 32 j + rr of D (column of R), column k = 32 i + kk.
__device__ __forceinline__ double tc_rprime(const double2 *Cb, int M, int r_diag, int i, int j, int rr, int kk)
{
    const int n = TC_CHUNK * j + rr, k = TC_CHUNK * i + kk;
    const int a = k >> 1, pa = k & 1, b = n >> 1, pb = n & 1;
    if (a >= M || b >= M || (r_diag && a == b)) return 0.0;
    const double2 c = Cb[(int64_t)a * M + b];
    const double val = (pa == pb) ? c.x : (pa == 0 ? -c.y : c.y);
    return (j > i) ? 2.0 * val : val;
}

// Largest |R'| entry of every bin: one CTA per (tile, bin), an atomic max on the FP64 bit pattern
// (non-negative doubles order like their bits); bmax is zeroed before the launch.
__global__ void __launch_bounds__(256) tc_binmax_kernel(const double2 *__restrict__ csm, int M, int C, int r_diag,
                                                        unsigned long long *__restrict__ bmax)
{
    int i, j;
    tc_tile_of_block(C, i, j);
    const int bin = blockIdx.y;
    const double2 *Cb = csm + (int64_t)bin * M * M;
    double m = 0.0;
    for (int e = threadIdx.x; e < TC_TILE_ELEMS; e += blockDim.x)
        m = fmax(m, fabs(tc_rprime(Cb, M, r_diag, i, j, e >> 5, e & 31)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ double wm[8];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, wm[w]);
        if (m > 0.0) atomicMax(&bmax[bin], (unsigned long long)__double_as_longlong(m));
    }
}

template <int PREC>
__global__ void __launch_bounds__(256) tc_prep_kernel(const double2 *__restrict__ csm, int M, int C, int r_diag,
                                                      int64_t bin_stride, __nv_bfloat16 *__restrict__ rh,
                                                      __nv_bfloat16 *__restrict__ rl)
{
    int i, j;
    tc_tile_of_block(C, i, j);
    const int bin = blockIdx.y;
    const double2 *Cb = csm + (int64_t)bin * M * M;
    __nv_bfloat16 *th = rh + (int64_t)bin * bin_stride + (int64_t)tile_index(C, i, j) * TC_TILE_ELEMS;
    __nv_bfloat16 *tl = rl + (int64_t)bin * bin_stride + (int64_t)tile_index(C, i, j) * TC_TILE_ELEMS;
    const int shift = PREC == TC_HALF ? tc_half_shift(reinterpret_cast<const unsigned long long *>(rl), bin) : 0;
    for (int e = threadIdx.x; e < TC_TILE_ELEMS; e += blockDim.x) {
        const int rr = e >> 5, kk = e & 31;
        const double val = tc_rprime(Cb, M, r_diag, i, j, rr, kk);
        if (PREC == TC_HALF) {
            reinterpret_cast<__half *>(th)[tile_off(rr, kk)] = __double2half(ldexp(val, shift));
            continue;
        }
        const float vf = (float)val;
        if (PREC == TC_TF) {
            // FP32 tiles of 4 KB: the whole workspace (hi and lo halves) holds them, 2 x bin_stride
            // bf16 elements per bin
            uint32_t *t32 = reinterpret_cast<uint32_t *>(rh + 2 * (int64_t)bin * bin_stride) +
                            (int64_t)tile_index(C, i, j) * TC_TILE_ELEMS;
            t32[tile_off_tf32(rr, kk)] = tf32_bits(vf);
        } else {
            const __nv_bfloat16 h = __float2bfloat16_rn(vf);
            const __nv_bfloat16 l = __float2bfloat16_rn(vf - __bfloat162float(h));
            const int o = tile_off(rr, kk);
            th[o] = h;
            tl[o] = l;
        }
    }
}

struct TcSmem {
    // offsets in bytes from the 1024-aligned dynamic shared-memory base; ns = number of A stages
    __host__ __device__ static constexpr int a_off(int stage, int lo) { return (stage * 2 + lo) * TC_A_BYTES; }
    __host__ __device__ static constexpr int b_base(int ns) { return ns * 2 * TC_A_BYTES; }
    // ring slot of R' tile pair: hi at b_off(slot, 0), lo at b_off(slot, 1)
    __host__ __device__ static constexpr int b_off(int ns, int slot, int lo)
    {
        return b_base(ns) + (lo * TC_RING + slot) * TC_TILE_BYTES;
    }
    __host__ __device__ static constexpr int mic_off(int ns) { return b_base(ns) + 2 * TC_RING * TC_TILE_BYTES; }
    __host__ __device__ static constexpr int red_off(int ns, int Mp) { return mic_off(ns) + Mp * 16; }
    // per-item normalisation partial sums, double-buffered by item parity: [2][parts][128]
    __host__ __device__ static constexpr int bar_off(int ns, int Mp) { return red_off(ns, Mp) + 2 * TC_PARTS * TC_ROWS * 8; }
    __host__ __device__ static constexpr int nbars() { return 2 * TC_ASTAGES_MAX + 3 * TC_NB + 4 + 2; }
    __host__ __device__ static constexpr int total(int ns, int Mp) { return bar_off(ns, Mp) + nbars() * 8 + 16; }
};

// Reference distance of grid point g (loaded at an item's start, so the epilogue does not wait for
// the grid positions after the item's last step).
__device__ __forceinline__ double ref_distance(const TcInst &a, int64_t g)
{
    if (a.ref_mode == 1 || g >= a.G) return a.ref_dist;
    return dist3(a.gpos[g], a.gpos[a.G + g], a.gpos[2 * a.G + g], a.ref0, a.ref1, a.ref2);
}

// Normalisation of the steering type (acoular/fastFuncs.py:293-310) and clipping.
template <int ST>
__device__ __forceinline__ void finish_point(const TcInst &a, double scalar, double S, double r0, int bin, int64_t g,
                                             double *out_map, double *out_norm)
{
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

// Persistent kernel: one CTA per SM walks the batch's work items (instance, bin, 128-point tile)
// blockIdx.x, +gridDim.x, ...; the step pipeline runs on across item and instance boundaries.
template <int ST, int PREC>
__global__ void __launch_bounds__(TC_THREADS, 1) map_tc_kernel(const __grid_constant__ TcBatch b, int *err)
{
    constexpr bool TF32 = PREC == TC_TF, HALF = PREC == TC_HALF, SPLIT = PREC == TC_SPLIT;
    // R' tile ring: 32 split-BF16 pairs (hi and lo halves of the ring region), 32 FP32 tiles, or
    // 64 FP16 tiles in the same 128 KB; FP16 ring slot s sits at b_base + s * 2 KB
    constexpr int RING = HALF ? 2 * TC_RING : TC_RING;
    // chunks per step: an FP16 chunk fills half an A stage (8 KB), so a stage carries two, and a step
    // (one A stage, one R' tile barrier, one MMA commit) covers a chunk pair: the steering -> MMA ->
    // epilogue hand-offs run once per pair (a pass's chunks pair up from its first; an odd last chunk
    // is a step alone)
    constexpr int CPS = HALF ? 2 : 1;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // operand tiles start on a 1 KB boundary (the launch reserves 1 KB of slack for this)
    uint8_t *smem = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
    const int MPX = b.mp_max;
    const int NST = b.nstages;
    float4 *mp4 = reinterpret_cast<float4 *>(smem + TcSmem::mic_off(NST));        // [MPX] (x, y, z, w)
    double *red = reinterpret_cast<double *>(smem + TcSmem::red_off(NST, MPX));   // [2][parts][128] sums S
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + TcSmem::bar_off(NST, MPX));
    uint64_t *full_a = bars;                          // [NST] step T written to A stage T % NST
    uint64_t *afree = bars + TC_ASTAGES_MAX;          // [NST] epilogue of step T has released A stage T % NST
    uint64_t *full_b = bars + 2 * TC_ASTAGES_MAX;     // [8]  R' tiles of step T landed
    uint64_t *done = full_b + TC_NB;                  // [8]  MMAs of step T complete
    uint64_t *tfree = done + TC_NB;                   // [8]  epilogue has read all columns of window W
    uint64_t *s_ready = tfree + TC_NB;                // [2]  synthesis sums S of item parity written
    // [2] epilogue has read the sums S of item parity: an item can have fewer steps than the A ring
    // has stages, so the synthesis warps may finish item li + 2 before the epilogue reaches item li
    uint64_t *s_free = s_ready + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(s_free + 2);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(s_free + 3);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t nmine = b.nitems > blockIdx.x ? (b.nitems - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const uint32_t ncols = 512;   // the whole TMEM: accumulator windows rotate through it

    if (threadIdx.x == 0) {
        for (int s = 0; s < NST; ++s) {
            tc::mbar_init(&full_a[s], TC_SYNTH_THREADS);
            tc::mbar_init(&afree[s], TC_EPI_THREADS);
        }
        for (int s = 0; s < TC_NB; ++s) {
            tc::mbar_init(&full_b[s], 1);
            tc::mbar_init(&done[s], 1);
        }
        for (int s = 0; s < TC_NB; ++s) tc::mbar_init(&tfree[s], TC_EPI_THREADS);
        tc::mbar_init(&s_ready[0], TC_SYNTH_THREADS);
        tc::mbar_init(&s_ready[1], TC_SYNTH_THREADS);
        tc::mbar_init(&s_free[0], TC_EPI_THREADS);
        tc::mbar_init(&s_free[1], TC_EPI_THREADS);
        *abort_flag = 0;
        tc::fence_mbar_init();
    }
    if (warp == 1) tc::tmem_alloc(tmem_slot, ncols);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t taddr = *tmem_slot;

    // Step sequence of one item: column passes p = 0 .. P-1, each covering accumulator chunks
    // [16p, je) with je = min(C, 16p + 16); in pass p the K chunks i = 0 .. je-1 run, chunk i feeding
    // the columns of chunks j in [max(i, 16p), je).  Chunk i's columns are final after step (p, i)
    // when i >= 16p; those steps also carry chunk i's dot product and normalisation sum.
    if (warp == TC_WARP_PRODUCER) {
        // ---------------- producer: R' tiles of every step into the tile ring ----------------
        // Step T (the CPS chunks of one A stage) takes n consecutive ring tiles starting at the running
        // tile counter U; tile U reuses slot U % RING, free once the step that held tile U - RING is
        // complete.
        if (lane == 0) {
            uint32_t ustart[TC_NB];   // first ring tile of the last TC_NB steps
            uint32_t U = 0;
            int T = 0, freed = -1, lastT = -1;
            bool ok = true;
            for (int64_t li = 0; li < nmine && ok; ++li) {
                const int64_t item = blockIdx.x + li * gridDim.x;
                const TcInst &in = b.inst[find_inst(b, item)];
                const TcItem it = decode_item(in, item);
                const int C = in.C, pw = in.pw;
                const int64_t bin = it.bin;
                const __nv_bfloat16 *bh = in.rh + (TF32 ? 2 : 1) * bin * in.bin_stride;   // FP16: halves
                const __nv_bfloat16 *bl = in.rl + bin * in.bin_stride;
                for (int pp = it.pa; pp < it.pz && ok; ++pp) {
                    const int jb = pp * pw, je = min(C, jb + pw);
                    for (int i0 = 0; i0 < je && ok; i0 += CPS, ++T) {
                        const int i1 = min(je, i0 + CPS);
                        int n = 0;   // the step's tiles: chunk i feeds columns j >= max(i, jb)
                        for (int i = i0; i < i1; ++i) n += je - max(i, jb);
                        // step barriers form a ring of TC_NB: step T - TC_NB must be complete; ring
                        // slots: every step holding a tile <= U + n - 1 - RING must be complete
                        while (ok && (freed < T - TC_NB ||
                                      (freed + 1 < T &&
                                       (int)(ustart[(freed + 1) & (TC_NB - 1)] - (U + n - 1 - RING)) <= 0))) {
                            ok = tc::mbar_wait(&done[(freed + 1) & (TC_NB - 1)], (uint32_t)(((freed + 1) / TC_NB) & 1),
                                               abort_flag, b.wait_limit_ns);
                            if (ok) ++freed;
                        }
                        if (!ok) break;
                        ustart[T & (TC_NB - 1)] = U;
                        uint64_t *fb = &full_b[T & (TC_NB - 1)];
                        tc::mbar_arrive_expect_tx(fb, (HALF ? 1u : 2u) * n * TC_TILE_BYTES);   // hi + lo, FP32, FP16
                        for (int i = i0; i < i1; ++i) {
                            const int j0 = max(i, jb), nc = je - j0;
                            const int64_t src = (int64_t)tile_index(C, i, j0) * TC_TILE_ELEMS;
                            int j = 0;
                            while (j < nc) {   // contiguous runs of ring slots
                                const int slot = (int)((U + j) & (RING - 1));
                                const int run = min(nc - j, RING - slot);
                                const uint32_t bytes = (uint32_t)run * TC_TILE_BYTES;
                                if (HALF) {
                                    tc::bulk_g2s(smem + TcSmem::b_base(NST) + slot * TC_TILE_BYTES,
                                                 bh + src + (int64_t)j * TC_TILE_ELEMS, bytes, fb);
                                } else if (TF32) {   // FP32 tiles of 4 KB, ring slot s at b_base + s * 4 KB
                                    tc::bulk_g2s(smem + TcSmem::b_base(NST) + slot * 2 * TC_TILE_BYTES,
                                                 reinterpret_cast<const uint32_t *>(bh) + src +
                                                     (int64_t)j * TC_TILE_ELEMS,
                                                 2 * bytes, fb);
                                } else {
                                    tc::bulk_g2s(smem + TcSmem::b_off(NST, slot, 0),
                                                 bh + src + (int64_t)j * TC_TILE_ELEMS, bytes, fb);
                                    tc::bulk_g2s(smem + TcSmem::b_off(NST, slot, 1),
                                                 bl + src + (int64_t)j * TC_TILE_ELEMS, bytes, fb);
                                }
                                j += run;
                            }
                            U += (uint32_t)nc;
                        }
                        lastT = T;
                    }
                }
            }
            // on an abort, let every copy still in flight land before the CTA releases its shared
            // memory: the last TC_NB steps (the producer runs at most TC_NB - 1 steps ahead) each own
            // one barrier slot
            if (*abort_flag)
                for (int t = max(0, lastT - (TC_NB - 1)); t <= lastT; ++t)
                    tc::mbar_drain(&full_b[t & (TC_NB - 1)], (uint32_t)((t / TC_NB) & 1),
                                   tc::drain_limit_ns(b.wait_limit_ns));
        }
    } else if (warp == TC_WARP_MMA) {
        // ---------------- MMA issuer ----------------
        // Kept lean: it sits on every step's critical path.  Descriptors are built once and
        // advanced by adding byte offsets >> 4 to their 14-bit start-address field; ring and
        // stage indices are 32-bit counters advanced incrementally.
        if (lane == 0) {
            // BF16: 8-row x 8-element core matrices, 4 per 32-component row group (SBO 512);
            // TF32: 8-row x 4-element core matrices, 8 per row group (SBO 1024)
            constexpr uint32_t SBO = TF32 ? 1024 : 512;
            const uint64_t a_base = tc::sdesc_noswizzle(tc::smem_u32(smem + TcSmem::a_off(0, 0)), 128, SBO);
            const uint64_t b_base = tc::sdesc_noswizzle(tc::smem_u32(smem + TcSmem::b_off(NST, 0, 0)), 128, SBO);
            constexpr uint32_t A_STEP = TC_A_BYTES >> 4;          // next (stage, hi|lo) block
            constexpr uint32_t T_STEP = (TF32 ? 2 : 1) * (TC_TILE_BYTES >> 4);   // next ring tile
            constexpr uint32_t LO_B = (TC_RING * TC_TILE_BYTES) >> 4;
            // operand format: 0 = FP16, 1 = BF16 (kind::f16), 2 = TF32 (kind::tf32)
            const uint32_t idesc0 = tc::idesc_m128(TF32 ? 2 : (HALF ? 0 : 1), 0);
            int sa = 0, ua = 0;     // A stage and its phase parity
            int sb = 0, ub = 0;     // step barrier slot and parity
            uint32_t slot0 = 0;     // ring slot of the step's first tile
            int lastb = -1, lastu = 0;
            // accumulator windows (one per column pass) rotate through TMEM in slots of the
            // instance's width; a slot is reused once the epilogue has released the window that
            // last held it.  An instance change drains all windows and restarts the rotation.
            int W = 0, w_start = 0, wpt = 1, width = 512, cur_inst = -1;
            bool ok = true;
            for (int64_t li = 0; li < nmine && ok; ++li) {
                const int64_t item = blockIdx.x + li * gridDim.x;
                const int ii = find_inst(b, item);
                const TcItem it = decode_item(b.inst[ii], item);
                const int C = b.inst[ii].C, pw = b.inst[ii].pw;
                if (ii != cur_inst) {
                    if (W > 0)
                        ok = tc::mbar_wait(&tfree[(W - 1) & (TC_NB - 1)], (uint32_t)(((W - 1) / TC_NB) & 1), abort_flag,
                                           b.wait_limit_ns);
                    width = TC_CHUNK * min(C, pw);
                    wpt = min(TC_NB, 512 / width);
                    w_start = W;
                    cur_inst = ii;
                }
                for (int pp = it.pa; pp < it.pz && ok; ++pp, ++W) {
                    const int jb = pp * pw, je = min(C, jb + pw);
                    if (W - w_start >= wpt)
                        ok = tc::mbar_wait(&tfree[(W - wpt) & (TC_NB - 1)], (uint32_t)(((W - wpt) / TC_NB) & 1),
                                           abort_flag, b.wait_limit_ns);
                    const uint32_t wcol = taddr + (uint32_t)(((W - w_start) % wpt) * width);
                    for (int i0 = 0; i0 < je && ok; i0 += CPS) {
                        ok = tc::mbar_wait(&full_a[sa], (uint32_t)ua, abort_flag, b.wait_limit_ns) &&
                             tc::mbar_wait(&full_b[sb], (uint32_t)ub, abort_flag, b.wait_limit_ns);
                        if (!ok) break;
                        tc::tc_fence_after();
                        for (int i = i0; i < min(je, i0 + CPS); ++i) {
                            const int j0 = max(i, jb), n = je - j0;
                            const uint32_t dcol = wcol + (uint32_t)(TC_CHUNK * (j0 - jb));
                            // split the step's n tiles into runs of <= 8 (N <= 256) that do not wrap
                            const int run0 = min(min(n, 8), (int)(RING - slot0));
                            const uint32_t slot1 = (slot0 + run0) & (RING - 1);
                            const int rest = n - run0;
                            const int run1 = min(min(rest, 8), (int)(RING - slot1));
                            const uint32_t slot2 = (slot1 + run1) & (RING - 1);
                            const int run2 = rest - run1;   // at most one more run (n <= 16)
                            // BF16: K steps of 16 (2) x products hi*hi, hi*lo, lo*hi; TF32: K steps of 8 (4) x 1;
                            // FP16: K steps of 16 (2) x 1
                            constexpr int KS = TF32 ? 4 : 2, NPROD = SPLIT ? 3 : 1;
#pragma unroll
                            for (int ks = 0; ks < KS; ++ks) {
#pragma unroll
                                for (int prod = 0; prod < NPROD; ++prod) {
                                    // A: split-BF16 hi (lo for the third product), FP32, or FP16 chunk
                                    // i - i0 of the stage
                                    const int ablk = sa * 2 + (HALF ? (i - i0) : (prod == 2));
                                    const uint64_t ad = a_base + (uint64_t)(ablk * A_STEP + ks * 16);
                                    const uint64_t bd = b_base + (uint64_t)((prod == 1 ? LO_B : 0u) + ks * 16);
                                    const uint32_t accum = (i == 0 && ks == 0 && prod == 0) ? 0u : 1u;
                                    const uint32_t n0 = idesc0 | ((uint32_t)(run0 * 4) << 17);
                                    const uint32_t n1 = idesc0 | ((uint32_t)(run1 * 4) << 17);
                                    const uint32_t n2 = idesc0 | ((uint32_t)(run2 * 4) << 17);
                                    if (TF32) {
                                        tc::mma_tf32(dcol, ad, bd + slot0 * T_STEP, n0, accum);
                                        if (run1 > 0)
                                            tc::mma_tf32(dcol + (uint32_t)(run0 * TC_CHUNK), ad, bd + slot1 * T_STEP, n1,
                                                        accum);
                                        if (run2 > 0)
                                            tc::mma_tf32(dcol + (uint32_t)((run0 + run1) * TC_CHUNK), ad,
                                                        bd + slot2 * T_STEP, n2, accum);
                                    } else {
                                        tc::mma_bf16(dcol, ad, bd + slot0 * T_STEP, n0, accum);
                                        if (run1 > 0)
                                            tc::mma_bf16(dcol + (uint32_t)(run0 * TC_CHUNK), ad, bd + slot1 * T_STEP, n1,
                                                        accum);
                                        if (run2 > 0)
                                            tc::mma_bf16(dcol + (uint32_t)((run0 + run1) * TC_CHUNK), ad,
                                                        bd + slot2 * T_STEP, n2, accum);
                                    }
                                }
                            }
                            slot0 = (slot0 + (uint32_t)n) & (RING - 1);
                        }
                        tc::mma_commit(&done[sb]);
                        lastb = sb;
                        lastu = ub;
                        if (++sa == NST) { sa = 0; ua ^= 1; }
                        if (++sb == TC_NB) { sb = 0; ub ^= 1; }
                    }
                }
            }
            // MMAs complete in issue order: the last commit covers all of them
            if (lastb >= 0) tc::mbar_drain(&done[lastb], (uint32_t)lastu, tc::drain_limit_ns(b.wait_limit_ns));
        }
    } else if (tc_is_epi(warp)) {
        // ---------------- epilogue (warps 0, 9, 2, 3 for lane quarters 0..3): one thread per grid point
        // After step (p, i) with i >= 16p the accumulator columns of chunk i are final; dot them
        // with the steering chunk as the MMA saw it (hi + lo from the A stage).  Every step then
        // releases its A stage.
        const int q = warp & 3;
        const int row = q * 32 + lane;
        const uint32_t lane_addr = taddr + ((uint32_t)(q * 32) << 16);
        const int a_row = ((row >> 3) << 9) + ((row & 7) << 4);   // byte offset of the row's first chunk
        int T = 0, sa = 0;
        int W = 0, w_start = 0, wpt = 1, width = 512, cur_inst = -1;   // same window rotation as the MMAs
        bool ok = true;
        for (int64_t li = 0; li < nmine && ok; ++li) {
            const int64_t item = blockIdx.x + li * gridDim.x;
            const int ii = find_inst(b, item);
            const TcInst &in = b.inst[ii];
            const TcItem it = decode_item(in, item);
            const int C = in.C, pw = in.pw;
            if (ii != cur_inst) {
                width = TC_CHUNK * min(C, pw);
                wpt = min(TC_NB, 512 / width);
                w_start = W;
                cur_inst = ii;
            }
            const int bin = it.bin;
            const int64_t g = it.tile * TC_ROWS + row;
            // (split BF16 has no registers to spare across the steps: it loads them after the last one)
            const double r0 = SPLIT ? 0.0 : ref_distance(in, g);
            double acc = 0.0;
            for (int pp = it.pa; pp < it.pz && ok; ++pp, ++W) {
                const int jb = pp * pw, je = min(C, jb + pw);
                const uint32_t wcol = lane_addr + (uint32_t)(((W - w_start) % wpt) * width);
                for (int i0 = 0; i0 < je; i0 += CPS, ++T) {
                    ok = __all_sync(0xffffffffu, tc::mbar_wait(&done[T & (TC_NB - 1)], (uint32_t)((T / TC_NB) & 1),
                                                               abort_flag, b.wait_limit_ns));
                    if (!ok) break;
                    for (int i = i0; i < min(je, i0 + CPS); ++i) {
                        if (i >= jb) {
                            tc::tc_fence_after();
                            float d[TC_CHUNK];
                            tc::tmem_ld_x32(wcol + (uint32_t)(TC_CHUNK * (i - jb)), d);
                            const uint8_t *ahi = smem + TcSmem::a_off(sa, HALF ? (i - i0) : 0) + a_row;
                            const uint8_t *alo = smem + TcSmem::a_off(sa, 1) + a_row;   // split BF16 only
                            float part = 0.f;
                            // the 11-bit forms dot in packed FP32: (re, im) component pairs, two accumulators
                            uint64_t pacc[2] = {0, 0};
                            if (TF32) {
                                // FP32 row: 8 core-matrix columns of 4 values, 128 bytes apart
                                const uint8_t *a32 =
                                    smem + TcSmem::a_off(sa, 0) + ((row >> 3) << 10) + ((row & 7) << 4);
#pragma unroll
                                for (int c4 = 0; c4 < 8; ++c4) {
                                    const float4 v = *reinterpret_cast<const float4 *>(a32 + c4 * 128);
                                    const float *dc = d + c4 * 4;
                                    pacc[0] = tc::f2_fma(tc::f2(dc[0], dc[1]), tc::f2(v.x, v.y), pacc[0]);
                                    pacc[1] = tc::f2_fma(tc::f2(dc[2], dc[3]), tc::f2(v.z, v.w), pacc[1]);
                                }
                            }
                            if (HALF) {
                                // FP16 row: 4 core-matrix columns of 4 (re, im) pairs, 128 bytes apart
#pragma unroll
                                for (int grp = 0; grp < 4; ++grp) {
                                    const uint4 hw = *reinterpret_cast<const uint4 *>(ahi + grp * 128);
                                    const uint32_t hv[4] = {hw.x, hw.y, hw.z, hw.w};
#pragma unroll
                                    for (int e = 0; e < 4; ++e) {
                                        const float2 v = __half22float2(*reinterpret_cast<const __half2 *>(&hv[e]));
                                        pacc[0] = tc::f2_fma(tc::f2(d[grp * 8 + 2 * e], d[grp * 8 + 2 * e + 1]),
                                                             tc::f2(v.x, v.y), pacc[0]);
                                    }
                                }
                            }
                            if (!SPLIT) {
                                float p0, p1, p2, p3;
                                tc::f2_split(pacc[0], p0, p1);
                                tc::f2_split(pacc[1], p2, p3);
                                part = (p0 + p1) + (p2 + p3);
                            }
#pragma unroll
                            for (int grp = 0; grp < (SPLIT ? 4 : 0); ++grp) {
                                const uint4 hw = *reinterpret_cast<const uint4 *>(ahi + grp * 128);
                                const uint4 lw = *reinterpret_cast<const uint4 *>(alo + grp * 128);
                                const uint32_t hv[4] = {hw.x, hw.y, hw.z, hw.w}, lv[4] = {lw.x, lw.y, lw.z, lw.w};
#pragma unroll
                                for (int e = 0; e < 4; ++e) {
                                    const float vr = __uint_as_float(hv[e] << 16) + __uint_as_float(lv[e] << 16);
                                    const float vi =
                                        __uint_as_float(hv[e] & 0xFFFF0000u) + __uint_as_float(lv[e] & 0xFFFF0000u);
                                    part = fmaf(d[grp * 8 + 2 * e], vr, part);
                                    part = fmaf(d[grp * 8 + 2 * e + 1], vi, part);
                                }
                            }
                            acc += (double)part;
                            tc::tc_fence_before();
                        }
                    }
                    tc::mbar_arrive(&afree[sa]);
                    if (++sa == NST) sa = 0;
                }
                if (!ok) break;
                tc::mbar_arrive(&tfree[W & (TC_NB - 1)]);
            }
            if (!ok) break;
            if (HALF) {
                // undo the bin's R' scale; an FP16 steering value out of range (|w| >= 65520) shows as a
                // non-finite sum and raises bit 2 of the error word
                acc = ldexp(acc, -tc_half_shift(reinterpret_cast<const unsigned long long *>(in.rl), bin));
                if (g < in.G && !isfinite(acc) && err) atomicOr(err, 2);
            }
            // normalisation sums of this item from the synthesis warps
            ok = __all_sync(0xffffffffu, tc::mbar_wait(&s_ready[li & 1], (uint32_t)((li >> 1) & 1), abort_flag,
                                                       b.wait_limit_ns));
            if (!ok) break;
            const double *rs = red + (li & 1) * TC_PARTS * TC_ROWS;
            double S = 0.0;
#pragma unroll
            for (int pp = 0; pp < TC_PARTS; ++pp) S += rs[pp * TC_ROWS + row];
            tc::mbar_arrive(&s_free[li & 1]);
            if (in.splits > 1) {
                // publish this group's partial sums; the last group of the (bin, tile) to finish
                // adds all groups' partials in group order and writes the map
                // (per warp: a warp's 32 rows are counted on their own, so no barrier spans warps)
                double2 *pb = in.part + it.base * in.splits * TC_ROWS;
                pb[it.split * TC_ROWS + row] = make_double2(acc, S);
                __threadfence();
                __syncwarp();
                int last = 0;
                if (lane == 0) last = atomicAdd(&in.cnt[it.base * 4 + q], 1) == in.splits - 1;
                last = __shfl_sync(0xffffffffu, last, 0);
                if (!last) continue;
                __threadfence();
                acc = 0.0;
                S = 0.0;
                for (int s = 0; s < in.splits; ++s) {
                    const double2 v = __ldcg(pb + s * TC_ROWS + row);
                    acc += v.x;
                    S += v.y;
                }
            }
            if (g < in.G) finish_point<ST>(in, acc, S, SPLIT ? ref_distance(in, g) : r0, bin, g, in.out, in.out_norm);
        }
    } else if (tc_synth_index(warp) >= 0) {
        // ---------------- steering synthesis (16 warps off scheduler 1) ----------------
        // Synthesis warp s serves grid points 32q..32q+31 (q = s % 4) and part p = s / 4 of every
        // chunk: mics 4p..4p+3 of the chunk's 16, i.e. one 16-byte core-matrix column of the A tile.
        // The arithmetic runs on mic pairs in packed FP32 (.f32x2): one instruction per pair.
        const int sidx = tc_synth_index(warp);
        const int q = sidx & 3;
        const int p = sidx >> 2;
        const int row = q * 32 + lane;
        const int a_off_row = (((row >> 3) * 4 + p) << 7) + ((row & 7) << 4);
        const int sid = sidx * 32 + lane;   // 0 .. TC_SYNTH_THREADS-1
        const uint64_t NHALF = tc::f2_splat(-0.5f), THALF = tc::f2_splat(1.5f);
        int T = 0, sa = 0, ua = 0, cur_inst = -1;
        bool ok = true;
        // the grid point and wave number of an item are loaded one item ahead, so that their global-memory
        // latency overlaps the previous item's steps (at the item's start for split BF16, whose
        // synthesis has no registers to spare)
        float nx = -TC_FAR, ny = -TC_FAR, nz = -TC_FAR;
        double nk = 0.0;
        auto fetch = [&](int64_t lj) {
            const int64_t itm = blockIdx.x + lj * gridDim.x;
            const TcInst &ij = b.inst[find_inst(b, itm)];
            const TcItem tj = decode_item(ij, itm);
            const int64_t gj = tj.tile * TC_ROWS + row;
            nx = ny = nz = -TC_FAR;
            if (gj < ij.G) {
                nx = (float)ij.gpos[gj];
                ny = (float)ij.gpos[ij.G + gj];
                nz = (float)ij.gpos[2 * ij.G + gj];
            }
            nk = ij.k[tj.bin];
        };
        if (!SPLIT && nmine > 0) fetch(0);
        for (int64_t li = 0; li < nmine && ok; ++li) {
            const int64_t item = blockIdx.x + li * gridDim.x;
            const int ii = find_inst(b, item);
            const TcInst &in = b.inst[ii];
            if (SPLIT) fetch(li);
            const float gxf = nx, gyf = ny, gzf = nz;
            const double k = nk;
            if (!SPLIT && li + 1 < nmine) fetch(li + 1);
            if (ii != cur_inst) {
                // new instance: every synthesis thread is past the previous item, reload the mics
                asm volatile("bar.sync 2, %0;" ::"r"(TC_SYNTH_THREADS) : "memory");
                // pair layout: mics 2j, 2j+1 as (x, x', y, y') (z, z', w, w') in float4s 2j, 2j+1;
                // padding mics beyond M sit far away with weight 0 (the weight is needed only by the
                // inverse steering's sum of r^2)
                float *mpf = reinterpret_cast<float *>(mp4);
                for (int m = sid; m < in.Mp; m += TC_SYNTH_THREADS) {
                    float4 v = make_float4(TC_FAR, TC_FAR, TC_FAR, 0.f);
                    if (m < in.M)
                        v = make_float4((float)in.mpos[m], (float)in.mpos[in.M + m], (float)in.mpos[2 * in.M + m], 1.f);
                    float *d = mpf + (m >> 1) * 8 + (m & 1);
                    d[0] = v.x;
                    d[2] = v.y;
                    d[4] = v.z;
                    d[6] = v.w;
                }
                asm volatile("bar.sync 2, %0;" ::"r"(TC_SYNTH_THREADS) : "memory");
                cur_inst = ii;
            }
            const TcItem it = decode_item(in, item);
            const int C = in.C, pw = in.pw;
            const uint64_t GX = tc::f2_splat(gxf), GY = tc::f2_splat(gyf), GZ = tc::f2_splat(gzf);
            const float khi = (float)k, klo = (float)(k - (double)khi);
            const uint64_t KH = tc::f2_splat(khi), KL = tc::f2_splat(klo);
            const uint64_t NKH = tc::f2_splat(-khi), NKL = tc::f2_splat(-klo);
            double S = 0.0;
            for (int pp = it.pa; pp < it.pz && ok; ++pp) {
                const int jb = pp * pw, je = min(C, jb + pw);
                // packed FP32 running sums of the normalisation terms of 4 consecutive chunks (8 per lane),
                // added to the FP64 sum per group: passes start at multiples of 4 chunks, so the groups, and
                // with them the sum's bits, do not depend on the pass width
                uint64_t s2run = 0;
                // T counts A stages: each holds CPS chunks t0 .. t0 + CPS - 1 of the pass
                for (int t0 = 0; t0 < je; t0 += CPS, ++T) {
                    if (T >= NST) {
                        // the A stage is free once the epilogue has released stage T - NST
                        ok = __all_sync(0xffffffffu, tc::mbar_wait(&afree[sa], (uint32_t)(ua ^ 1), abort_flag,
                                                                   b.wait_limit_ns));
                        if (!ok) break;
                    }
#pragma unroll
                    for (int c = 0; c < CPS; ++c) {
                        // a pass's odd last chunk: the second slot repeats the first chunk's arithmetic (so both
                        // slots' instructions interleave) and stores nothing
                        const bool live = c == 0 || t0 + c < je;
                        const int t = live ? t0 + c : t0;
                        uint64_t s2 = 0;   // packed normalisation partial sums (0.0f, 0.0f)
                        uint32_t hw[4], lw[4];
#pragma unroll
                        for (int e2 = 0; e2 < 2; ++e2) {
                            const int j = t * (TC_MPC / 2) + p * 2 + e2;   // mics 2j, 2j+1
                            const float4 pa = mp4[2 * j], pb = mp4[2 * j + 1];
                            const uint64_t dx = tc::f2_sub(GX, tc::f2(pa.x, pa.y));
                            const uint64_t dy = tc::f2_sub(GY, tc::f2(pa.z, pa.w));
                            const uint64_t dz = tc::f2_sub(GZ, tc::f2(pb.x, pb.y));
                            const uint64_t r2 = tc::f2_fma(dz, dz, tc::f2_fma(dy, dy, tc::f2_mul(dx, dx)));
                            float r2a, r2b;
                            tc::f2_split(r2, r2a, r2b);
                            // 1/r: hardware rsqrt (~2^-22 relative); split BF16 (16 significant bits) adds one
                            // Newton step y *= 1.5 - 0.5 r^2 y^2, the 11-bit forms do not need it
                            uint64_t y = tc::f2(tc::rsqrt_approx(r2a), tc::rsqrt_approx(r2b));
                            if (SPLIT) y = tc::f2_mul(y, tc::f2_fma(tc::f2_mul(tc::f2_mul(r2, y), y), NHALF, THALF));
                            const uint64_t r = tc::f2_mul(r2, y);
                            // xn = -(k r) reduced: cos(xn) = Re h / w and sin(xn) = Im h / w
                            float xa, xb;
                            if (!SPLIT) {
                                // TF32 and FP16 keep 11 significant bits: -k r in FP32 (k as a float-float) feeds
                                // the hardware sincos directly, which reduces the argument by whole turns
                                tc::f2_split(tc::f2_fma(NKL, r, tc::f2_mul(NKH, r)), xa, xb);
                            } else {
                                // k r as an exact float-float product, reduced by the 3-term 2*pi
                                const uint64_t ph = tc::f2_mul(KH, r);
                                const uint64_t pl = tc::f2_fma(KL, r, tc::f2_fma(KH, r, tc::f2_mul(NKH, r)));
                                const uint64_t MAG = tc::f2_splat(12582912.f);
                                const uint64_t nnq = tc::f2_sub(MAG, tc::f2_fma(ph, tc::f2_splat(TC_INV2PI), MAG));
                                uint64_t x = tc::f2_fma(nnq, tc::f2_splat(TC_P2A), ph);
                                x = tc::f2_fma(nnq, tc::f2_splat(TC_P2B), x);
                                x = tc::f2_fma(nnq, tc::f2_splat(TC_P2C), x);
                                tc::f2_split(tc::f2_add(x, pl), xa, xb);
                                xa = -xa;
                                xb = -xb;
                            }
                            float sa_, ca_, sb_, cb_;
                            tc::sincos_approx(xa, sa_, ca_);
                            tc::sincos_approx(xb, sb_, cb_);
                            uint64_t vre = tc::f2(ca_, cb_), vim = tc::f2(sa_, sb_);
                            // steering weight: 1, r (inverse, times the mics' table weights: 0 for padding)
                            // or 1/r (true level / location)
                            if (ST == 2) {
                                const uint64_t wt = tc::f2(pb.z, pb.w);
                                const uint64_t w = tc::f2_mul(r, wt);
                                s2 = tc::f2_fma(r2, wt, s2);
                                vre = tc::f2_mul(vre, w);
                                vim = tc::f2_mul(vim, w);
                            } else if (ST >= 3) {
                                s2 = tc::f2_fma(y, y, s2);
                                vre = tc::f2_mul(vre, y);
                                vim = tc::f2_mul(vim, y);
                            }
                            float vr[2], vi[2];
                            tc::f2_split(vre, vr[0], vr[1]);
                            tc::f2_split(vim, vi[0], vi[1]);
#pragma unroll
                            for (int h = 0; h < 2; ++h) {
                                const int e = 2 * e2 + h;
                                if (TF32) {   // FP32 operand rounded to TF32: (re, im) of mic e in hw[e], lw[e]
                                    hw[e] = tf32_bits(vr[h]);
                                    lw[e] = tf32_bits(vi[h]);
                                    continue;
                                }
                                if (HALF) {   // FP16 pair (re, im), one packed conversion
                                    const __half2 f2h = __floats2half2_rn(vr[h], vi[h]);
                                    hw[e] = *reinterpret_cast<const uint32_t *>(&f2h);
                                    continue;
                                }
                                // split-BF16: hi = bf16(x) (packed pair conversion), lo = bf16(x - hi)
                                const __nv_bfloat162 h2 = __floats2bfloat162_rn(vr[h], vi[h]);
                                hw[e] = *reinterpret_cast<const uint32_t *>(&h2);
                                const float lr = vr[h] - __uint_as_float(hw[e] << 16);
                                const float li_ = vi[h] - __uint_as_float(hw[e] & 0xFFFF0000u);
                                const __nv_bfloat162 l2 = __floats2bfloat162_rn(lr, li_);
                                lw[e] = *reinterpret_cast<const uint32_t *>(&l2);
                            }
                        }
                        if (TF32) {
                            // components 8p..8p+7 = core-matrix columns 2p, 2p+1 of the FP32 row
                            uint8_t *a32 = smem + TcSmem::a_off(sa, 0) + ((row >> 3) << 10) + ((row & 7) << 4) + p * 256;
                            *reinterpret_cast<uint4 *>(a32) = make_uint4(hw[0], lw[0], hw[1], lw[1]);
                            *reinterpret_cast<uint4 *>(a32 + 128) = make_uint4(hw[2], lw[2], hw[3], lw[3]);
                        } else if (live) {
                            // FP16: chunk c of the stage in slot c; split BF16: hi and lo halves
                            *reinterpret_cast<uint4 *>(smem + TcSmem::a_off(sa, HALF ? c : 0) + a_off_row) =
                                make_uint4(hw[0], hw[1], hw[2], hw[3]);
                            if (SPLIT)
                                *reinterpret_cast<uint4 *>(smem + TcSmem::a_off(sa, 1) + a_off_row) =
                                    make_uint4(lw[0], lw[1], lw[2], lw[3]);
                        }
                        // each mic's normalisation term once, in its own pass
                        if (ST >= 2 && live && t >= jb) {
                            s2run = tc::f2_add(s2run, s2);
                            if ((t & 3) == 3 || t == je - 1) {
                                float sa2, sb2;
                                tc::f2_split(s2run, sa2, sb2);
                                S += (double)sa2 + (double)sb2;
                                s2run = 0;
                            }
                        }
                    }
                    tc::fence_proxy_async_smem();
                    tc::mbar_arrive(&full_a[sa]);
                    if (++sa == NST) { sa = 0; ua ^= 1; }
                }
            }
            if (!ok) break;
            // the slot of item li - 2 must have been read (one phase of s_free per item of that parity)
            if (li >= 2) {
                ok = __all_sync(0xffffffffu, tc::mbar_wait(&s_free[li & 1], (uint32_t)(((li >> 1) - 1) & 1),
                                                           abort_flag, b.wait_limit_ns));
                if (!ok) break;
            }
            red[((li & 1) * TC_PARTS + p) * TC_ROWS + row] = S;
            tc::mbar_arrive(&s_ready[li & 1]);
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

// Host side: validate and lay out one instance; the R' region of the instance starts at `ws`.
static int tc_fill_inst(const acb_map_params *p, const void *csm, const double *wavenumber, const double *mpos,
                        const double *gpos, double *out_map, double *out_steer_norm, __nv_bfloat16 *ws,
                        int64_t item_off, TcInst &in)
{
    if (!p || !csm || !wavenumber || !mpos || !gpos || !out_map) return ACB_ERR_ARG;
    if (p->steer_type < 1 || p->steer_type > 4) return ACB_ERR_ARG;
    if (p->num_mics < 2 || p->num_grid <= 0 || p->num_bins <= 0 || p->num_bins > 65535) return ACB_ERR_SHAPE;
    if (p->num_mics > TC_MAX_MICS) return ACB_ERR_UNSUPPORTED;
    const int M = p->num_mics;
    in.M = M;
    in.Mp = (M + TC_MPC - 1) / TC_MPC * TC_MPC;
    in.C = in.Mp / TC_MPC;
    in.G = p->num_grid;
    in.nbins = p->num_bins;
    in.ntiles = (p->num_grid + TC_ROWS - 1) / TC_ROWS;
    in.item_off = item_off;
    in.clip = p->clip_negative;
    in.norm = p->norm;
    in.ref_mode = p->ref_mode;
    in.ref0 = p->ref_point[0];
    in.ref1 = p->ref_point[1];
    in.ref2 = p->ref_point[2];
    in.ref_dist = p->ref_distance;
    in.k = wavenumber;
    in.mpos = mpos;
    in.gpos = gpos;
    in.out = out_map;
    in.out_norm = out_steer_norm;
    in.bin_stride = (int64_t)tri_tiles(in.C) * TC_TILE_ELEMS;
    in.rh = ws;
    in.rl = ws + (size_t)p->num_bins * in.bin_stride;
    const int pw = p->tc_pass_chunks;
    if (pw != 0 && pw != 4 && pw != 8 && pw != 16) return ACB_ERR_ARG;
    if (p->tc_splits < 0) return ACB_ERR_ARG;
    in.pw = pw ? pw : TC_PASS_CHUNKS;
    in.P = (in.C + in.pw - 1) / in.pw;
    in.splits = 1;
    in.sp0[0] = 0;
    in.sp0[1] = (uint8_t)in.P;
    in.part = nullptr;
    in.cnt = nullptr;
    in.small = 0;   // set once the batch's item count is known
    return ACB_OK;
}

// Split the passes [0, P) of an instance into `splits` contiguous groups of balanced cost.  Cost of
// pass p in units of one R' tile step: its MMA tiles sum_{j in pass} (j + 1) plus its steering
// synthesis (chunks 0 .. je-1), weighted 2 tiles per chunk.
static void tc_split_passes(TcInst &in, int splits)
{
    const int P = in.P;
    if (splits > P) splits = P;
    if (splits > TC_MAX_SPLIT) splits = TC_MAX_SPLIT;
    if (splits < 1) splits = 1;
    double cost[TC_MAX_MICS / TC_MPC + 1];
    for (int pp = 0; pp < P; ++pp) {
        const int jb = pp * in.pw, je = in.C < jb + in.pw ? in.C : jb + in.pw;
        double c = 2.0 * je;
        for (int j = jb; j < je; ++j) c += j + 1;
        cost[pp] = c;
    }
    // minimise the largest group cost: dp[s][e] = best max over the first e passes in s groups
    static thread_local double dp[TC_MAX_SPLIT + 1][TC_MAX_MICS / TC_MPC + 1];
    static thread_local int cut[TC_MAX_SPLIT + 1][TC_MAX_MICS / TC_MPC + 1];
    double pre[TC_MAX_MICS / TC_MPC + 2];
    pre[0] = 0.0;
    for (int pp = 0; pp < P; ++pp) pre[pp + 1] = pre[pp] + cost[pp];
    for (int e = 0; e <= P; ++e) dp[1][e] = pre[e];
    for (int sgrp = 2; sgrp <= splits; ++sgrp)
        for (int e = sgrp; e <= P; ++e) {
            dp[sgrp][e] = 1e300;
            for (int c = sgrp - 1; c < e; ++c) {
                const double v = dp[sgrp - 1][c] > pre[e] - pre[c] ? dp[sgrp - 1][c] : pre[e] - pre[c];
                if (v < dp[sgrp][e]) {
                    dp[sgrp][e] = v;
                    cut[sgrp][e] = c;
                }
            }
        }
    in.splits = splits;
    int e = P;
    in.sp0[splits] = (uint8_t)P;
    for (int sgrp = splits; sgrp >= 2; --sgrp) {
        e = cut[sgrp][e];
        in.sp0[sgrp - 1] = (uint8_t)e;
    }
    in.sp0[0] = 0;
}

static inline size_t round256(size_t x) { return (x + 255) / 256 * 256; }

// Workspace of one batch instance: R' tiles, then (when split) the partial sums and group counters.
static size_t tc_inst_ws_bytes(const acb_map_params &p, int precision)
{
    const size_t r = acb_map_tc_workspace_bytes(p.num_mics, p.num_bins, precision);
    if (r == 0) return 0;
    size_t tot = round256(r);
    if (p.tc_splits > 1) {
        const int64_t nbase = (int64_t)p.num_bins * ((p.num_grid + TC_ROWS - 1) / TC_ROWS);
        tot += round256((size_t)nbase * TC_MAX_SPLIT * TC_ROWS * sizeof(double2));
        tot += round256((size_t)nbase * 4 * sizeof(int));
    }
    return tot;
}

// Launch the R' preparation of every instance and the persistent map kernel over the batch.
static int tc_launch(TcBatch &bt, const acb_map_params *const *params, const void *const *csms, int steer_type,
                     int precision, int *error_word, cudaStream_t s)
{
    int mp_max = 16;
    for (int i = 0; i < bt.n_inst; ++i) {
        const TcInst &in = bt.inst[i];
        if (in.splits > 1) {
            const cudaError_t e = cudaMemsetAsync(in.cnt, 0, (size_t)in.nbins * in.ntiles * 4 * sizeof(int), s);
            if (e != cudaSuccess) {
                set_cuda_error(e);
                return ACB_ERR_CUDA;
            }
        }
        if (precision == ACB_TC_FP16) {
            // the bins' largest |R'| entries, for the FP16 scale, in the workspace half the tiles leave free
            unsigned long long *bmax = reinterpret_cast<unsigned long long *>(const_cast<__nv_bfloat16 *>(in.rl));
            const cudaError_t e = cudaMemsetAsync(bmax, 0, (size_t)in.nbins * sizeof(unsigned long long), s);
            if (e != cudaSuccess) {
                set_cuda_error(e);
                return ACB_ERR_CUDA;
            }
            tc_binmax_kernel<<<dim3(tri_tiles(in.C), in.nbins), 256, 0, s>>>(
                reinterpret_cast<const double2 *>(csms[i]), in.M, in.C, params[i]->r_diag, bmax);
            const int st = check_launch();
            if (st) return st;
        }
        auto prep = precision == ACB_TC_TF32   ? tc_prep_kernel<TC_TF>
                    : precision == ACB_TC_FP16 ? tc_prep_kernel<TC_HALF>
                                               : tc_prep_kernel<TC_SPLIT>;
        prep<<<dim3(tri_tiles(in.C), in.nbins), 256, 0, s>>>(reinterpret_cast<const double2 *>(csms[i]), in.M, in.C,
                                                            params[i]->r_diag, in.bin_stride,
                                                            const_cast<__nv_bfloat16 *>(in.rh),
                                                            const_cast<__nv_bfloat16 *>(in.rl));
        const int st = check_launch();
        if (st) return st;
        mp_max = max(mp_max, in.Mp);
    }
    bt.mp_max = mp_max;
    bt.wait_limit_ns = tc_wait_limit_ns();
    int dev = 0, nsm = kNumSMs, smem_max = 232448;
    if (cudaGetDevice(&dev) == cudaSuccess) {
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    }
    // the deepest A ring that fits beside this batch's mic table (+1 KB of alignment slack)
    int ns = TC_ASTAGES_MAX;
    while (ns > TC_ASTAGES_MIN && TcSmem::total(ns, mp_max) + 1024 > smem_max) --ns;
    bt.nstages = ns;
    int smem = TcSmem::total(ns, mp_max) + 1024;
    // each CTA takes all 512 TMEM columns and must be alone on its SM: size the shared memory so
    // that no second CTA fits (a second one would stall in tcgen05.alloc until the first exits)
    if (smem < 116 * 1024) smem = 116 * 1024;
    const dim3 grid((unsigned)(bt.nitems < nsm ? bt.nitems : nsm));
    using KernT = void (*)(const TcBatch, int *);
    static const KernT kernels[4][3] = {
        {map_tc_kernel<1, TC_SPLIT>, map_tc_kernel<1, TC_TF>, map_tc_kernel<1, TC_HALF>},
        {map_tc_kernel<2, TC_SPLIT>, map_tc_kernel<2, TC_TF>, map_tc_kernel<2, TC_HALF>},
        {map_tc_kernel<3, TC_SPLIT>, map_tc_kernel<3, TC_TF>, map_tc_kernel<3, TC_HALF>},
        {map_tc_kernel<4, TC_SPLIT>, map_tc_kernel<4, TC_TF>, map_tc_kernel<4, TC_HALF>}};
    const KernT kern = kernels[steer_type - 1][precision];
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    kern<<<grid, TC_THREADS, smem, s>>>(bt, error_word);
    return check_launch();
}

}  // namespace acb

using namespace acb;

extern "C" {

uint64_t acb_tc_set_wait_limit_ns(uint64_t limit_ns)
{
    return g_tc_wait_limit_ns.exchange(limit_ns ? limit_ns : TC_DEFAULT_WAIT_LIMIT_NS);
}

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
    if (!p) return ACB_ERR_ARG;
    if (precision != ACB_TC_BF16X3 && precision != ACB_TC_TF32 && precision != ACB_TC_FP16) return ACB_ERR_UNSUPPORTED;
    TcBatch bt;
    bt.n_inst = 1;
    int st = tc_fill_inst(p, csm, wavenumber, mpos, gpos, out_map, out_steer_norm,
                          reinterpret_cast<__nv_bfloat16 *>(workspace), 0, bt.inst[0]);
    if (st) return st;
    const size_t need = acb_map_tc_workspace_bytes(p->num_mics, p->num_bins, precision);
    if (!workspace || workspace_bytes < need) return ACB_ERR_WORKSPACE;
    bt.nitems = bt.inst[0].ntiles * bt.inst[0].nbins;
    bt.inst[0].small = bt.nitems < (int64_t(1) << 31);
    const acb_map_params *pp[1] = {p};
    const void *cc[1] = {csm};
    return tc_launch(bt, pp, cc, p->steer_type, precision, error_word, as_stream(stream));
}

size_t acb_map_tc_batch_workspace_bytes(const acb_map_params *params, int num_instances, int precision)
{
    if (!params || num_instances <= 0) return 0;
    size_t tot = 0;
    for (int i = 0; i < num_instances; ++i) {
        const size_t b = tc_inst_ws_bytes(params[i], precision);
        if (b == 0) return 0;
        tot += b;
    }
    return tot;
}

int acb_map_tc_batch(const acb_map_params *params, const acb_map_io *io, int num_instances, int precision,
                     void *workspace, size_t workspace_bytes, int *error_word, void *stream)
{
    if (!params || !io) return ACB_ERR_ARG;
    if (num_instances <= 0 || num_instances > TC_MAX_INST) return ACB_ERR_SHAPE;
    if (precision != ACB_TC_BF16X3 && precision != ACB_TC_TF32 && precision != ACB_TC_FP16) return ACB_ERR_UNSUPPORTED;
    const size_t need = acb_map_tc_batch_workspace_bytes(params, num_instances, precision);
    if (need == 0) return ACB_ERR_SHAPE;
    if (!workspace || workspace_bytes < need) return ACB_ERR_WORKSPACE;
    const int steer = params[0].steer_type;
    TcBatch bt;
    bt.n_inst = num_instances;
    int64_t items = 0;
    uint8_t *w = reinterpret_cast<uint8_t *>(workspace);
    const acb_map_params *pp[TC_MAX_INST];
    const void *cc[TC_MAX_INST];
    for (int i = 0; i < num_instances; ++i) {
        if (params[i].steer_type != steer) return ACB_ERR_ARG;   // one steering type per launch
        TcInst &in = bt.inst[i];
        const int st = tc_fill_inst(&params[i], io[i].csm, io[i].wavenumber, io[i].mpos, io[i].gpos, io[i].out_map,
                                    io[i].out_steer_norm, reinterpret_cast<__nv_bfloat16 *>(w), items, in);
        if (st) return st;
        if (params[i].tc_splits > 1) {
            tc_split_passes(in, params[i].tc_splits);
            const size_t r = round256(acb_map_tc_workspace_bytes(params[i].num_mics, params[i].num_bins, precision));
            const int64_t nbase = (int64_t)in.nbins * in.ntiles;
            in.part = reinterpret_cast<double2 *>(w + r);
            in.cnt = reinterpret_cast<int *>(w + r + round256((size_t)nbase * TC_MAX_SPLIT * TC_ROWS * sizeof(double2)));
        }
        items += in.ntiles * in.nbins * in.splits;
        w += tc_inst_ws_bytes(params[i], precision);
        pp[i] = &params[i];
        cc[i] = io[i].csm;
    }
    bt.nitems = items;
    for (int i = 0; i < num_instances; ++i) bt.inst[i].small = items < (int64_t(1) << 31);
    return tc_launch(bt, pp, cc, steer, precision, error_word, as_stream(stream));
}

}  // extern "C"
