// Batched Hermitian eigendecomposition of CSMs (PowerSpectra._get__evd, acoular/spectra.py:351-364: numpy's
// eigh per bin, eigenvalues ascending, eigenvectors in the columns), hand-written for the device.
//
// Three kernels, one matrix per CTA (or per column slab), every bin of a request in one launch each:
//   heevd_tridiag_kernel : Householder reduction to a real symmetric tridiagonal matrix, A = Q T Q^H.
//                          Step i reflects column i below the diagonal, x -> beta e1 with H = I - tau v v^H
//                          (beta real, tau complex, v_0 = 1), then updates the trailing matrix
//                          A22 <- H^H A22 H = A22 - v w^H - w v^H, p = tau A22 v, w = p - (tau/2)(p^H v) v,
//                          on A22's lower triangle only (half the memory traffic of the full update).
//   heevd_tql_kernel     : eigenvalues and eigenvectors of T by implicit QL sweeps with Wilkinson shifts
//                          (the EISPACK tql2 scheme), eigenvectors accumulated in Z.  One thread forms a
//                          sweep's plane rotations from d and e; all threads then apply them to their rows of
//                          Z (no barrier per rotation).  Then the ascending order of the eigenvalues.
//   heevd_back_kernel    : eigenvectors of A, V = Q Z = H_0 H_1 ... H_{M-2} Z, for a slab of columns held in
//                          shared memory, reflectors applied from the last; each warp owns columns of the
//                          slab, so the reflectors need no barrier; columns written in ascending eigenvalue
//                          order.
// All arithmetic is FP64.  The eigenvectors differ from LAPACK's by a phase per column (any unit factor is an
// eigenvector); the eigenvalue beamformers use them only through |v^H h|.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "common.cuh"

namespace acb {

constexpr int kEvThreads = 256;
constexpr int kEvWarps = kEvThreads / 32;
// the QL kernel's CTA: 128 threads, so that every matrix of a 513-bin request has its CTA resident at once
// (the sweeps are one thread's serial recurrence, so a matrix takes the same time in any wave)
constexpr int kQlThreads = 128;
constexpr int kQlMaxIter = 60;   // QL iterations per eigenvalue before giving up (info = 1)

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b)   // conj(a) * b
{
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// Block sum of a double (all threads receive it); `red` holds kEvWarps doubles.
__device__ __forceinline__ double block_sum(double v, double *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kEvWarps; ++w) t += red[w];
    return t;
}

// A (B, M, M) complex128 row-major, overwritten; d, e (B, M); tau (B, M) complex; vh (B, M - 1, M): reflector i
// in entries i + 1 .. M - 1 of row i.
__global__ void __launch_bounds__(kEvThreads) heevd_tridiag_kernel(double2 *__restrict__ Aall, int M,
                                                                   double *__restrict__ dall, double *__restrict__ eall,
                                                                   double2 *__restrict__ tauall,
                                                                   double2 *__restrict__ vhall)
{
    extern __shared__ double2 ev_sm[];
    double2 *v = ev_sm;        // [M]
    double2 *p = ev_sm + M;    // [M]
    __shared__ double red[kEvWarps];
    __shared__ double2 s_tau, s_scale;
    __shared__ double s_beta;
    const int b = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double2 *A = Aall + (int64_t)b * M * M;
    double *d = dall + (int64_t)b * M;
    double *e = eall + (int64_t)b * M;
    double2 *tau = tauall + (int64_t)b * M;
    double2 *vh = vhall + (int64_t)b * (M > 1 ? M - 1 : 1) * M;

    for (int i = 0; i < M - 1; ++i) {
        for (int r = i + 1 + tid; r < M; r += kEvThreads) v[r] = A[(int64_t)r * M + i];
        __syncthreads();
        double part = 0.0;
        for (int r = i + 2 + tid; r < M; r += kEvThreads) part += v[r].x * v[r].x + v[r].y * v[r].y;
        const double xn2 = block_sum(part, red);
        if (tid == 0) {
            const double2 al = v[i + 1];
            d[i] = A[(int64_t)i * M + i].x;
            if (xn2 == 0.0 && al.y == 0.0) {   // already real and reduced: H = I
                s_beta = al.x;
                s_tau = make_double2(0.0, 0.0);
                s_scale = make_double2(0.0, 0.0);
            } else {
                const double beta = -copysign(sqrt(al.x * al.x + al.y * al.y + xn2), al.x);
                s_beta = beta;
                s_tau = make_double2((beta - al.x) / beta, -al.y / beta);
                // 1 / (alpha - beta)
                const double2 den = make_double2(al.x - beta, al.y);
                const double dd = den.x * den.x + den.y * den.y;
                s_scale = make_double2(den.x / dd, -den.y / dd);
            }
            e[i] = s_beta;
            tau[i] = s_tau;
        }
        __syncthreads();
        const double2 tu = s_tau;
        if (tu.x == 0.0 && tu.y == 0.0) {
            for (int r = i + 1 + tid; r < M; r += kEvThreads)
                vh[(int64_t)i * M + r] = make_double2(r == i + 1 ? 1.0 : 0.0, 0.0);
            __syncthreads();
            continue;
        }
        const double2 sc = s_scale;
        for (int r = i + 1 + tid; r < M; r += kEvThreads) {
            const double2 vr = r == i + 1 ? make_double2(1.0, 0.0) : cmul(v[r], sc);
            v[r] = vr;
            vh[(int64_t)i * M + r] = vr;
        }
        __syncthreads();
        // p = tau A22 v: a warp per row, lanes along the row.  Only the lower triangle of A22 is kept up to
        // date (A is Hermitian): row r's entries right of the diagonal are conj(A[c][r]), read down column r
        for (int r = i + 1 + warp; r < M; r += kEvWarps) {
            const double2 *row = A + (int64_t)r * M;
            double ar = 0.0, ai = 0.0;
            for (int c = i + 1 + lane; c < M; c += 32) {
                double2 a;
                if (c <= r) {
                    a = row[c];
                } else {
                    a = A[(int64_t)c * M + r];
                    a.y = -a.y;
                }
                const double2 x = v[c];
                ar = fma(a.x, x.x, fma(-a.y, x.y, ar));
                ai = fma(a.x, x.y, fma(a.y, x.x, ai));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                ar += __shfl_xor_sync(0xffffffffu, ar, o);
                ai += __shfl_xor_sync(0xffffffffu, ai, o);
            }
            if (lane == 0) p[r] = cmul(tu, make_double2(ar, ai));
        }
        __syncthreads();
        // alpha2 = -(tau / 2) (p^H v);  w = p + alpha2 v  (into p)
        double pr = 0.0, pi = 0.0;
        for (int r = i + 1 + tid; r < M; r += kEvThreads) {
            const double2 t = cmulc(p[r], v[r]);
            pr += t.x;
            pi += t.y;
        }
        const double sr = block_sum(pr, red);
        const double si = block_sum(pi, red);
        const double2 al2 = cmul(make_double2(-0.5 * tu.x, -0.5 * tu.y), make_double2(sr, si));
        for (int r = i + 1 + tid; r < M; r += kEvThreads) {
            const double2 t = cmul(al2, v[r]);
            p[r] = make_double2(p[r].x + t.x, p[r].y + t.y);
        }
        __syncthreads();
        // A22 -= v w^H + w v^H on the lower triangle (c <= r): a warp per row, lanes along the row
        for (int r = i + 1 + warp; r < M; r += kEvWarps) {
            for (int c = i + 1 + lane; c <= r; c += 32) {
                const double2 vr = v[r], wr = p[r], vc = v[c], wc = p[c];
                const double2 t1 = cmulc(wc, vr);   // v_r conj(w_c)
                const double2 t2 = cmulc(vc, wr);   // w_r conj(v_c)
                double2 a = A[(int64_t)r * M + c];
                a.x -= t1.x + t2.x;
                a.y -= t1.y + t2.y;
                A[(int64_t)r * M + c] = a;
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        d[M - 1] = A[(int64_t)(M - 1) * M + (M - 1)].x;
        e[M - 1] = 0.0;
        tau[M - 1] = make_double2(0.0, 0.0);
    }
}

// d, e (B, M) -> eigenvalues w (B, M) ascending, Z (B, M, M) column-major (column j = eigenvector of the
// unsorted eigenvalue j), perm (B, M): sorted position q holds unsorted index perm[q]; info[b] = 1 if a QL
// iteration did not converge.
__global__ void __launch_bounds__(kQlThreads) heevd_tql_kernel(const double *__restrict__ dall,
                                                               const double *__restrict__ eall, int M,
                                                               double *__restrict__ wall, double *__restrict__ Zall,
                                                               int *__restrict__ permall, int *__restrict__ info)
{
    extern __shared__ double ql_sm[];
    double *d = ql_sm;          // [M]
    double *e = ql_sm + M;      // [M]
    double *cs = ql_sm + 2 * M; // [M] cosine of the rotation of (i, i + 1)
    double *sn = ql_sm + 3 * M; // [M] sine
    __shared__ int s_m, s_stop, s_done, s_fail;
    const int b = blockIdx.x;
    const int tid = threadIdx.x;
    double *Z = Zall + (int64_t)b * M * M;
    for (int k = tid; k < M; k += kQlThreads) {
        d[k] = dall[(int64_t)b * M + k];
        e[k] = eall[(int64_t)b * M + k];
    }
    for (int64_t idx = tid; idx < (int64_t)M * M; idx += kQlThreads) Z[idx] = (idx / M == idx % M) ? 1.0 : 0.0;
    if (tid == 0) s_fail = 0;
    __syncthreads();
    const double eps = 2.220446049250313e-16;
    for (int l = 0; l < M; ++l) {
        int iter = 0;
        while (true) {
            if (tid == 0) {
                int m = l;
                while (m < M - 1) {
                    const double dd = fabs(d[m]) + fabs(d[m + 1]);
                    if (fabs(e[m]) <= eps * dd) break;
                    ++m;
                }
                s_done = (m == l) || (iter >= kQlMaxIter);
                if (m != l && iter >= kQlMaxIter) s_fail = 1;
                if (!s_done) {
                    double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                    double r = hypot(g, 1.0);
                    g = d[m] - d[l] + e[l] / (g + copysign(r, g));
                    double s = 1.0, c = 1.0, p = 0.0;
                    int i = m - 1;
                    bool restart = false;
                    for (; i >= l; --i) {
                        const double f = s * e[i], bb = c * e[i];
                        r = hypot(f, g);
                        e[i + 1] = r;
                        if (r == 0.0) {   // split: deflate and restart from the same l
                            d[i + 1] -= p;
                            e[m] = 0.0;
                            restart = true;
                            break;
                        }
                        const double rinv = 1.0 / r;   // one division for both ratios
                        s = f * rinv;
                        c = g * rinv;
                        g = d[i + 1] - p;
                        r = (d[i] - g) * s + 2.0 * c * bb;
                        p = s * r;
                        d[i + 1] = g + p;
                        g = c * r - bb;
                        cs[i] = c;
                        sn[i] = s;
                    }
                    if (!restart) {
                        d[l] -= p;
                        e[l] = g;
                        e[m] = 0.0;
                    }
                    s_m = m;
                    s_stop = restart ? i + 1 : l;   // rotations i = m - 1 .. s_stop were formed
                }
            }
            __syncthreads();
            const int done = s_done, m = s_m, stop = s_stop;
            __syncthreads();   // every thread has read the control words before thread 0 writes them again
            if (done) break;
            ++iter;
            // apply the rotations in the order they were formed to every row k of Z.  Rotation i reads entry i
            // and writes entry i + 1 of the row, so every entry is read before it is written: the reads of 8
            // rotations are issued together, ahead of their writes, and their latency is paid once per 8
            // (one read at a time waited for the previous write, about one L2 round trip per rotation)
            for (int k = tid; k < M; k += kQlThreads) {
                double *zk = Z + k;   // entry i of row k at zk[i * M]
                double carry = zk[(int64_t)m * M];
                int i = m - 1;
                for (; i - 7 >= stop; i -= 8) {
                    double zv[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) zv[j] = zk[(int64_t)(i - j) * M];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int ii = i - j;
                        zk[(int64_t)(ii + 1) * M] = sn[ii] * zv[j] + cs[ii] * carry;
                        carry = cs[ii] * zv[j] - sn[ii] * carry;
                    }
                }
                for (; i >= stop; --i) {
                    const double zi = zk[(int64_t)i * M];
                    zk[(int64_t)(i + 1) * M] = sn[i] * zi + cs[i] * carry;
                    carry = cs[i] * zi - sn[i] * carry;
                }
                zk[(int64_t)stop * M] = carry;
            }
            __syncthreads();
        }
    }
    // ascending order, ties by index (as a stable sort)
    for (int k = tid; k < M; k += kQlThreads) {
        const double dk = d[k];
        int rank = 0;
        for (int j = 0; j < M; ++j) rank += (d[j] < dk) || (d[j] == dk && j < k);
        wall[(int64_t)b * M + rank] = dk;
        permall[(int64_t)b * M + rank] = k;
    }
    if (tid == 0 && info) info[b] = s_fail;
}

// V = Q Z for the output columns [c0, c0 + W) of one matrix, reflectors applied from the last.  The slab
// sits in shared memory column by column (stride M + 1), and warp w owns the slab's columns w, w + 8, ..:
// for each reflector a warp forms tau v^H S[:, j] over its own columns (lanes along the rows, a shuffle
// reduction) and updates them, so no barrier separates the reflectors.  The reflector's entries are read
// by all warps from L1.  V (B, M, M) complex128 row-major, columns = eigenvectors in ascending order.
template <int CPW>
__global__ void __launch_bounds__(kEvThreads) heevd_back_kernel(const double2 *__restrict__ vhall,
                                                                const double2 *__restrict__ tauall,
                                                                const double *__restrict__ Zall,
                                                                const int *__restrict__ permall, int M, int W,
                                                                int ldv, double2 *__restrict__ Vall)
{
    extern __shared__ double2 bk_sm[];
    const int Mp = M + 1;
    double2 *S = bk_sm;                    // [W][Mp]: entry r of slab column j at S[j * Mp + r]
    const int b = blockIdx.x;
    const int c0 = blockIdx.y * W;
    const int nw = min(W, M - c0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double2 *vh = vhall + (int64_t)b * (M > 1 ? M - 1 : 1) * M;
    const double2 *tau = tauall + (int64_t)b * M;
    const double *Z = Zall + (int64_t)b * M * M;
    const int *perm = permall + (int64_t)b * M;
    for (int j = warp; j < nw; j += kEvWarps) {
        const double *zc = Z + (int64_t)perm[c0 + j] * M;   // column-major Z: eigenvector of T
        for (int r = lane; r < M; r += 32) S[j * Mp + r] = make_double2(zc[r], 0.0);
    }
    // this warp's columns (j < nw)
    int nq = 0;
    while (nq < CPW && warp + kEvWarps * nq < nw) ++nq;
    for (int i = M - 2; i >= 0 && nq > 0; --i) {
        const double2 t = __ldg(tau + i);
        if (t.x == 0.0 && t.y == 0.0) continue;
        const double2 *v = vh + (int64_t)i * M;
        double ar[CPW], ai[CPW];
#pragma unroll
        for (int q = 0; q < CPW; ++q) ar[q] = ai[q] = 0.0;
        for (int r = i + 1 + lane; r < M; r += 32) {
            const double2 vr = __ldg(v + r);
#pragma unroll
            for (int q = 0; q < CPW; ++q) {
                if (q >= nq) break;
                const double2 x = cmulc(vr, S[(warp + kEvWarps * q) * Mp + r]);
                ar[q] += x.x;
                ai[q] += x.y;
            }
        }
        double2 sc[CPW];
#pragma unroll
        for (int q = 0; q < CPW; ++q) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                ar[q] += __shfl_xor_sync(0xffffffffu, ar[q], o);
                ai[q] += __shfl_xor_sync(0xffffffffu, ai[q], o);
            }
            sc[q] = cmul(t, make_double2(ar[q], ai[q]));
        }
        for (int r = i + 1 + lane; r < M; r += 32) {
            const double2 vr = __ldg(v + r);
#pragma unroll
            for (int q = 0; q < CPW; ++q) {
                if (q >= nq) break;
                double2 *sp = S + (warp + kEvWarps * q) * Mp + r;
                const double2 u = cmul(vr, sc[q]);
                *sp = make_double2(sp->x - u.x, sp->y - u.y);
            }
        }
    }
    __syncthreads();
    double2 *V = Vall + (int64_t)b * M * ldv;   // row stride ldv (M, or the number of selected columns)
    for (int idx = tid; idx < M * W; idx += kEvThreads) {
        const int r = idx / W, j = idx % W;
        if (j < nw) V[(int64_t)r * ldv + c0 + j] = S[j * Mp + r];
    }
}

// ------------------------------------------------------------------------------------------------
// Selected eigenpairs (acb_heevd_select_f64): the eigenvalues of chosen ranks and their eigenvectors
// only, for consumers that use a few components (BeamformerEig's default n = -1 takes the largest).
// After the same tridiagonalisation, one warp per selected rank k:
//   - the k-th smallest eigenvalue of T by multisection: each round the 32 lanes evaluate the Sturm
//     count (the number of negative pivots of the LDL^T factorisation of T - x I, i.e. of eigenvalues
//     below x) at 32 points spread over the current interval, which then narrows to the gap between two
//     neighbouring points (about 33x per round, from the Gershgorin interval down to 2 eps |lambda|, or
//     eps ||T|| for eigenvalues near zero, the accuracy of the QL iteration);
//   - its eigenvector by inverse iteration: T - lambda I factored once by Gaussian elimination with
//     partial pivoting (a tridiagonal factor gains one superdiagonal of fill-in), then three solves from
//     a fixed start vector, each rescaled by its largest entry; zero pivots are replaced by eps ||T||;
//   - the back-transformation by the reflectors (heevd_back_kernel on the selected columns).
// The QL sweeps and their accumulation of all M eigenvectors are skipped.
// ------------------------------------------------------------------------------------------------
constexpr int kSelMax = 4;

struct EvSel {
    int n;
    int idx[kSelMax];
};

// Number of eigenvalues of T (diagonal d, squared off-diagonal e2) below x.
__device__ __forceinline__ int ev_sturm(const double *d, const double *e2, int M, double x, double pivmin)
{
    double q = d[0] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    int cnt = q < 0.0;
    for (int i = 1; i < M; ++i) {
        q = (d[i] - x) - e2[i - 1] / q;
        if (fabs(q) < pivmin) q = -pivmin;
        cnt += q < 0.0;
    }
    return cnt;
}

__host__ __device__ constexpr size_t ev_select_smem(int M, int E)
{
    return ((size_t)3 * M + (size_t)5 * M * E) * sizeof(double) + (size_t)M * E;
}

__global__ void __launch_bounds__(32 * kSelMax) heevd_select_kernel(const double *__restrict__ dall,
                                                                    const double *__restrict__ eall, int M,
                                                                    EvSel sel, double *__restrict__ wsel,
                                                                    double *__restrict__ Zall,
                                                                    int *__restrict__ permall)
{
    extern __shared__ double sl_sm[];
    double *d = sl_sm;           // [M]
    double *e = sl_sm + M;       // [M] off-diagonal (e[M - 1] = 0)
    double *e2 = sl_sm + 2 * M;  // [M] its squares
    const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    double *u0 = sl_sm + 3 * M + (size_t)w * 5 * M;   // pivots (as reciprocals after the factorisation)
    double *u1 = u0 + M;                              // first superdiagonal of U
    double *u2 = u1 + M;                              // second superdiagonal (fill-in)
    double *mu = u2 + M;                              // multipliers
    double *y = mu + M;                               // iterate
    unsigned char *pv = reinterpret_cast<unsigned char *>(sl_sm + 3 * M + (size_t)sel.n * 5 * M) + (size_t)w * M;
    for (int i = tid; i < M; i += blockDim.x) {
        d[i] = dall[(int64_t)b * M + i];
        const double ei = i < M - 1 ? eall[(int64_t)b * M + i] : 0.0;
        e[i] = ei;
        e2[i] = ei * ei;
    }
    __syncthreads();
    if (w >= sel.n) return;
    const double eps = 2.220446049250313e-16;
    // Gershgorin interval, the norm of T and the pivot floor
    double lo = INFINITY, hi = -INFINITY, emax2 = 0.0;
    for (int i = lane; i < M; i += 32) {
        const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + fabs(e[i]);
        lo = fmin(lo, d[i] - r);
        hi = fmax(hi, d[i] + r);
        emax2 = fmax(emax2, e2[i]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        emax2 = fmax(emax2, __shfl_xor_sync(0xffffffffu, emax2, o));
    }
    const double pivmin = 2.2250738585072014e-308 * fmax(1.0, emax2);
    const double tnorm = fmax(fabs(lo), fabs(hi));
    const double fudge = 2.0 * eps * tnorm + 2.0 * pivmin;
    lo -= fudge;
    hi += fudge;
    const int k = sel.idx[w];
    for (int it = 0; it < 64; ++it) {
        const double width = hi - lo;
        if (width <= fmax(2.0 * eps * fmax(fabs(lo), fabs(hi)), eps * tnorm) || width <= 4.0 * pivmin) break;
        const double x = lo + width * (double)(lane + 1) / 33.0;
        const int c = ev_sturm(d, e2, M, x, pivmin);
        const unsigned bal = __ballot_sync(0xffffffffu, c > k);   // points above the k-th eigenvalue
        const double x31 = __shfl_sync(0xffffffffu, x, 31);
        if (bal == 0) {
            lo = x31;
        } else {
            const int j0 = __ffs(bal) - 1;
            const double xh = __shfl_sync(0xffffffffu, x, j0);
            const double xl = __shfl_sync(0xffffffffu, x, j0 > 0 ? j0 - 1 : 0);
            if (j0 > 0) lo = xl;
            hi = xh;
        }
    }
    const double lam = 0.5 * (lo + hi);
    if (lane == 0) {
        wsel[(int64_t)b * sel.n + w] = lam;
        const double tiny = tnorm > 0.0 ? eps * tnorm : 2.2250738585072014e-308;
        // T - lam I = P L U
        double a = d[0] - lam, bs = M > 1 ? e[0] : 0.0;
        for (int i = 0; i < M - 1; ++i) {
            const double l = e[i], m = d[i + 1] - lam, n = i + 2 < M ? e[i + 1] : 0.0;
            if (fabs(a) >= fabs(l)) {
                if (fabs(a) < tiny) a = a < 0.0 ? -tiny : tiny;
                const double f = l / a;
                pv[i] = 0;
                u0[i] = a;
                u1[i] = bs;
                u2[i] = 0.0;
                mu[i] = f;
                a = m - f * bs;
                bs = n;
            } else {
                const double f = a / l;
                pv[i] = 1;
                u0[i] = l;
                u1[i] = m;
                u2[i] = n;
                mu[i] = f;
                a = bs - f * m;
                bs = -f * n;
            }
        }
        if (fabs(a) < tiny) a = a < 0.0 ? -tiny : tiny;
        u0[M - 1] = a;
        for (int i = 0; i < M; ++i) u0[i] = 1.0 / u0[i];
        for (int i = 0; i < M; ++i) y[i] = 1.0 + 0.25 * (double)((i * 2654435761u) % 1009u) / 1009.0;
        for (int it = 0; it < 3; ++it) {
            double cur = y[0];
            for (int i = 0; i < M - 1; ++i) {
                const double nx = y[i + 1];
                if (pv[i]) {
                    y[i] = nx;
                    cur -= mu[i] * nx;
                } else {
                    y[i] = cur;
                    cur = nx - mu[i] * cur;
                }
            }
            y[M - 1] = cur * u0[M - 1];
            if (M > 1) y[M - 2] = (y[M - 2] - u1[M - 2] * y[M - 1]) * u0[M - 2];
            for (int i = M - 3; i >= 0; --i) y[i] = (y[i] - u1[i] * y[i + 1] - u2[i] * y[i + 2]) * u0[i];
            double mx = 0.0;
            for (int i = 0; i < M; ++i) mx = fmax(mx, fabs(y[i]));
            const double sc = mx > 0.0 ? 1.0 / mx : 1.0;
            for (int i = 0; i < M; ++i) y[i] *= sc;
        }
    }
    __syncwarp();
    double ss = 0.0;
    for (int i = lane; i < M; i += 32) ss += y[i] * y[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    const double inv = ss > 0.0 ? 1.0 / sqrt(ss) : 0.0;
    double *zc = Zall + (int64_t)b * M * M + (int64_t)w * M;   // column w of Z
    for (int i = lane; i < M; i += 32) zc[i] = y[i] * inv;
    if (lane == 0) permall[(int64_t)b * M + w] = w;
}

struct EvWorkspace {
    size_t A, d, e, tau, vh, Z, perm, total;
};

static EvWorkspace ev_layout(int M, int B)
{
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    EvWorkspace w;
    size_t off = 0;
    w.A = off;
    off += up((size_t)B * M * M * sizeof(double2));
    w.d = off;
    off += up((size_t)B * M * sizeof(double));
    w.e = off;
    off += up((size_t)B * M * sizeof(double));
    w.tau = off;
    off += up((size_t)B * M * sizeof(double2));
    w.vh = off;
    off += up((size_t)B * (M > 1 ? M - 1 : 1) * M * sizeof(double2));
    w.Z = off;
    off += up((size_t)B * M * M * sizeof(double));
    w.perm = off;
    off += up((size_t)B * M * sizeof(int));
    w.total = off;
    return w;
}

// Columns per back-transformation slab: as many as fit beside the reflector in the shared memory (<= 32).
static int ev_slab(int M)
{
    int W = 32;
    while (W > 1 && (size_t)(M + 1) * W * sizeof(double2) > 200 * 1024) W >>= 1;
    return W;
}

}  // namespace acb

using namespace acb;

extern "C" {

size_t acb_heevd_workspace_bytes(int num_mics, int num_bins)
{
    if (num_mics < 1 || num_bins < 1) return 0;
    return ev_layout(num_mics, num_bins).total;
}

int acb_heevd_f64(const void *csm, int num_bins, int num_mics, double *eigval, void *eigvec, int *info,
                  void *workspace, size_t workspace_bytes, void *stream)
{
    if (!csm || !eigval || !eigvec || !workspace) return ACB_ERR_ARG;
    const int M = num_mics, B = num_bins;
    if (M < 1 || B < 1 || M > 4096 || B > 65535) return ACB_ERR_SHAPE;
    const EvWorkspace lay = ev_layout(M, B);
    if (workspace_bytes < lay.total) return ACB_ERR_WORKSPACE;
    const int W = ev_slab(M);
    if ((size_t)(M + 1) * W * sizeof(double2) > 200 * 1024) return ACB_ERR_UNSUPPORTED;
    cudaStream_t s = as_stream(stream);
    char *ws = static_cast<char *>(workspace);
    double2 *A = reinterpret_cast<double2 *>(ws + lay.A);
    double *d = reinterpret_cast<double *>(ws + lay.d);
    double *e = reinterpret_cast<double *>(ws + lay.e);
    double2 *tau = reinterpret_cast<double2 *>(ws + lay.tau);
    double2 *vh = reinterpret_cast<double2 *>(ws + lay.vh);
    double *Z = reinterpret_cast<double *>(ws + lay.Z);
    int *perm = reinterpret_cast<int *>(ws + lay.perm);
    cudaError_t err = cudaMemcpyAsync(A, csm, (size_t)B * M * M * sizeof(double2), cudaMemcpyDeviceToDevice, s);
    if (err != cudaSuccess) {
        set_cuda_error(err);
        return ACB_ERR_CUDA;
    }
    const size_t sm1 = 2 * (size_t)M * sizeof(double2), sm2 = 4 * (size_t)M * sizeof(double);
    if (cudaFuncSetAttribute(heevd_tridiag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1) !=
            cudaSuccess ||
        cudaFuncSetAttribute(heevd_tql_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2) != cudaSuccess)
        return ACB_ERR_CUDA;
    heevd_tridiag_kernel<<<B, kEvThreads, sm1, s>>>(A, M, d, e, tau, vh);
    int st = check_launch();
    if (st) return st;
    heevd_tql_kernel<<<B, kQlThreads, sm2, s>>>(d, e, M, eigval, Z, perm, info);
    st = check_launch();
    if (st) return st;
    const size_t smem = (size_t)(M + 1) * W * sizeof(double2);
    // columns per warp: the slab's W columns over the 8 warps
    auto back = W >= 32 ? heevd_back_kernel<4> : (W >= 16 ? heevd_back_kernel<2> : heevd_back_kernel<1>);
    if (cudaFuncSetAttribute(back, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return ACB_ERR_CUDA;
    back<<<dim3(B, (M + W - 1) / W), kEvThreads, smem, s>>>(vh, tau, Z, perm, M, W, M,
                                                           static_cast<double2 *>(eigvec));
    return check_launch();
}

int acb_heevd_select_f64(const void *csm, int num_bins, int num_mics, int num_sel, const int *sel, double *eigval,
                         void *eigvec, void *workspace, size_t workspace_bytes, void *stream)
{
    if (!csm || !sel || !eigval || !eigvec || !workspace) return ACB_ERR_ARG;
    const int M = num_mics, B = num_bins, E = num_sel;
    if (M < 1 || B < 1 || M > 4096 || B > 65535 || E < 1 || E > kSelMax || E > M) return ACB_ERR_SHAPE;
    EvSel es;
    es.n = E;
    for (int j = 0; j < kSelMax; ++j) es.idx[j] = 0;
    for (int j = 0; j < E; ++j) {
        if (sel[j] < 0 || sel[j] >= M) return ACB_ERR_ARG;
        es.idx[j] = sel[j];
    }
    const size_t sm3 = ev_select_smem(M, E);
    if (sm3 > 200 * 1024) return ACB_ERR_UNSUPPORTED;
    const EvWorkspace lay = ev_layout(M, B);
    if (workspace_bytes < lay.total) return ACB_ERR_WORKSPACE;
    cudaStream_t s = as_stream(stream);
    char *ws = static_cast<char *>(workspace);
    double2 *A = reinterpret_cast<double2 *>(ws + lay.A);
    double *d = reinterpret_cast<double *>(ws + lay.d);
    double *e = reinterpret_cast<double *>(ws + lay.e);
    double2 *tau = reinterpret_cast<double2 *>(ws + lay.tau);
    double2 *vh = reinterpret_cast<double2 *>(ws + lay.vh);
    double *Z = reinterpret_cast<double *>(ws + lay.Z);
    int *perm = reinterpret_cast<int *>(ws + lay.perm);
    cudaError_t err = cudaMemcpyAsync(A, csm, (size_t)B * M * M * sizeof(double2), cudaMemcpyDeviceToDevice, s);
    if (err != cudaSuccess) {
        set_cuda_error(err);
        return ACB_ERR_CUDA;
    }
    const size_t sm1 = 2 * (size_t)M * sizeof(double2);
    if (cudaFuncSetAttribute(heevd_tridiag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1) !=
            cudaSuccess ||
        cudaFuncSetAttribute(heevd_select_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm3) !=
            cudaSuccess)
        return ACB_ERR_CUDA;
    heevd_tridiag_kernel<<<B, kEvThreads, sm1, s>>>(A, M, d, e, tau, vh);
    int st = check_launch();
    if (st) return st;
    heevd_select_kernel<<<B, 32 * E, sm3, s>>>(d, e, M, es, eigval, Z, perm);
    st = check_launch();
    if (st) return st;
    // the E eigenvectors of T sit in columns 0 .. E-1 of each matrix's Z, perm[j] = j: one slab of E columns
    const size_t smem = (size_t)(M + 1) * E * sizeof(double2);
    if (cudaFuncSetAttribute(heevd_back_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return ACB_ERR_CUDA;
    heevd_back_kernel<1><<<dim3(B, 1), kEvThreads, smem, s>>>(vh, tau, Z, perm, M, E, E,
                                                              static_cast<double2 *>(eigvec));
    return check_launch();
}

}  // extern "C"
