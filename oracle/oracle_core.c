/*
 * CPU oracle for the Acoular frequency-domain beamforming path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the numba kernels that the
 * reference (Acoular 26.08) runs on this path.  It is the checker for the CUDA kernels and the
 * timed CPU baseline ("port") in the benchmark; no product code path may call it.
 *
 * Every function follows the reference's arithmetic order so that its results reproduce the
 * reference's own numba results to rounding:
 *   orc_calc_csm_c128 / _c64   acoular/fastFuncs.py:19-58     (calcCSM)
 *   orc_dist_mat               acoular/environments.py:65-103 (dist_mat)
 *   orc_beamformer_fullcsm     acoular/fastFuncs.py:217-311   (_freqBeamformer_FullCSM)
 *   orc_beamformer_eig         acoular/fastFuncs.py:313-411   (_freqBeamformer_EigValues)
 *   orc_beamformer_custom      acoular/fastFuncs.py:414-559   (_freqBeamformer_SpecificSteerVec_*)
 *   orc_psf                    acoular/fastFuncs.py:563-801   (calcPointSpreadFunction)
 *   orc_damas_gauss_seidel     acoular/fastFuncs.py:804-855   (damasSolverGaussSeidel)
 *   orc_transfer               acoular/fastFuncs.py:857-897   (calcTransfer)
 * Parity of this restatement is pinned against golden vectors produced by running the reference's
 * own code (tests/golden/make_golden.py) and against the reference's committed regression arrays
 * for Environment.apparent_r.
 *
 * Float32 phase semantics: the reference rounds k*r to float32 and evaluates np.cos / np.sin in
 * float32, which numba lowers to the C library's cosf / sinf.  This file calls the same cosf / sinf.
 *
 * Build: oracle/build_oracle.sh (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* calcCSM, complex128 signature (fastFuncs.py:19-58).
 * csm: [F][M][M] interleaved (re, im) doubles, updated in place (upper triangle r <= c).
 * spec: [F][M] interleaved.  csm[f,r,c] += conj(spec[f,c]) * spec[f,r]. */
void orc_calc_csm_c128(double *csm, const double *spec, int64_t F, int64_t M)
{
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F; ++f) {
        const double *s = spec + 2 * f * M;
        double *c = csm + 2 * f * M * M;
        for (int64_t col = 0; col < M; ++col) {
            const double tr = s[2 * col], ti = -s[2 * col + 1]; /* temp = conj(spec[col]) */
            for (int64_t row = 0; row <= col; ++row) {
                const double xr = s[2 * row], xi = s[2 * row + 1];
                /* csm += temp * spec[row]; the reference compiles this with fastmath, which LLVM
                 * contracts into two chained FMAs per component in this order (verified bit-exact
                 * against the reference's numba build). */
                double *dst = c + 2 * (row * M + col);
                dst[0] = fma(-ti, xi, fma(tr, xr, dst[0]));
                dst[1] = fma(tr, xi, fma(ti, xr, dst[1]));
            }
        }
    }
}

/* calcCSM, complex64 signature: same arithmetic in float32. */
void orc_calc_csm_c64(float *csm, const float *spec, int64_t F, int64_t M)
{
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F; ++f) {
        const float *s = spec + 2 * f * M;
        float *c = csm + 2 * f * M * M;
        for (int64_t col = 0; col < M; ++col) {
            const float tr = s[2 * col], ti = -s[2 * col + 1];
            for (int64_t row = 0; row <= col; ++row) {
                const float xr = s[2 * row], xi = s[2 * row + 1];
                float *dst = c + 2 * (row * M + col);
                dst[0] = fmaf(-ti, xi, fmaf(tr, xr, dst[0]));
                dst[1] = fmaf(tr, xi, fmaf(ti, xr, dst[1]));
            }
        }
    }
}

/* Welch accumulation over K blocks of spectra [K][F][M] (one calcCSM call per block, the loop
 * of PowerSpectra.calc_csm, spectra.py:407-410).  Used by the CPU baseline timing. */
void orc_calc_csm_blocks_c128(double *csm, const double *spec, int64_t K, int64_t F, int64_t M)
{
    for (int64_t b = 0; b < K; ++b)
        orc_calc_csm_c128(csm, spec + 2 * b * F * M, F, M);
}

void orc_calc_csm_blocks_c64(float *csm, const float *spec, int64_t K, int64_t F, int64_t M)
{
    for (int64_t b = 0; b < K; ++b)
        orc_calc_csm_c64(csm, spec + 2 * b * F * M, F, M);
}

/* dist_mat (environments.py:65-103): rm[n, m] = |g_n - m_m|.  gpos [3][N], mpos [3][M]. */
void orc_dist_mat(const double *gpos, const double *mpos, int64_t N, int64_t M, double *rm)
{
#pragma omp parallel for schedule(static)
    for (int64_t n = 0; n < N; ++n) {
        const double g0 = gpos[n], g1 = gpos[N + n], g2 = gpos[2 * N + n];
        for (int64_t m = 0; m < M; ++m) {
            const double d0 = g0 - mpos[m], d1 = g1 - mpos[M + m], d2 = g2 - mpos[2 * M + m];
            /* fastmath contraction of d0^2 + d1^2 + d2^2 as numba emits it (bit-exact) */
            rm[n * M + m] = sqrt(fma(d2, d2, fma(d1, d1, d0 * d0)));
        }
    }
}

/* _freqBeamformer_FullCSM (fastFuncs.py:217-311) for one frequency bin.
 * csm: [M][M] interleaved complex128; r0: [G]; rm: [G][M]; k: wave number.
 * steer_type: 1 classic, 2 inverse, 3 true level, 4 true location.
 * Writes result[G] and normsteer[G]. */
void orc_beamformer_fullcsm(const double *csm, const double *r0, const double *rm, double k, double norm,
                            int r_diag, int steer_type, int64_t G, int64_t M, double *result, double *normsteer)
{
    const int st2 = steer_type == 2;
    const int st34 = steer_type == 3 || steer_type == 4;
#pragma omp parallel
    {
        double *vr = (double *)__builtin_alloca(sizeof(double) * M);
        double *vi = (double *)__builtin_alloca(sizeof(double) * M);
#pragma omp for schedule(static)
        for (int64_t gi = 0; gi < G; ++gi) {
            const double *r = rm + gi * M;
            double help = 0.0;
            for (int64_t m = 0; m < M; ++m) {
                const float arg = (float)(k * r[m]);  /* np.float32(waveNumber * dist) */
                vr[m] = (double)cosf(arg);            /* cos(arg) - 1j*sin(arg), float32 libm */
                vi[m] = -(double)sinf(arg);
            }
            if (st2) {
                help = 0.0;
                for (int64_t m = 0; m < M; ++m) {
                    help += r[m] * r[m];
                    vr[m] *= r[m];
                    vi[m] *= r[m];
                }
            }
            if (st34) {
                help = 0.0;
                for (int64_t m = 0; m < M; ++m) {
                    help += 1.0 / (r[m] * r[m]);
                    vr[m] /= r[m];
                    vi[m] /= r[m];
                }
            }
            double scalar = 0.0;
            for (int64_t b = 0; b < M; ++b) {
                double lr = 0.0, li = 0.0;
                for (int64_t a = 0; a < b; ++a) {
                    /* csm[a, b] * conj(v[a]) */
                    const double cr = csm[2 * (a * M + b)], ci = csm[2 * (a * M + b) + 1];
                    const double hr = vr[a], hi = -vi[a];
                    lr += cr * hr - ci * hi;
                    li += cr * hi + ci * hr;
                }
                /* 2 * (left * v[b]).real */
                scalar += 2.0 * (lr * vr[b] - li * vi[b]);
            }
            if (!r_diag) {
                for (int64_t m = 0; m < M; ++m) {
                    const double cr = csm[2 * (m * M + m)], ci = csm[2 * (m * M + m) + 1];
                    const double hr = vr[m], hi = -vi[m];
                    const double pr = cr * hr - ci * hi, pi = cr * hi + ci * hr;
                    scalar += pr * vr[m] - pi * vi[m];
                }
            }
            if (steer_type == 1) {
                const double nf = (double)M;
                normsteer[gi] = 1.0 / (double)M;
                result[gi] = scalar / (nf * nf) * norm;
            } else if (steer_type == 2) {
                const double nf = (double)M * r0[gi];
                const double nf2 = nf * nf;
                normsteer[gi] = help / nf2;
                result[gi] = scalar / nf2 * norm;
            } else if (steer_type == 3) {
                const double nf = r0[gi] * help;
                normsteer[gi] = 1.0 / (r0[gi] * r0[gi]) / help;
                result[gi] = scalar / (nf * nf) * norm;
            } else {
                const double nf = (double)M * help;
                normsteer[gi] = 1.0 / (double)M;
                result[gi] = scalar / nf * norm;
            }
        }
    }
}

/* _freqBeamformer_EigValues (fastFuncs.py:313-411) for one frequency bin.
 * eigval: [E]; eigvec: [M][E] interleaved complex128; r0: [G]; rm: [G][M]; k: wave number.
 * Per grid point: steering as in the full-CSM kernel, then
 *   scalar = sum_e eigval[e] * (|sum_m conj(V[m][e]) v[m]|^2 - [r_diag] sum_m |conj(V[m][e]) v[m]|^2).
 * Writes result[G] and normsteer[G]. */
void orc_beamformer_eig(const double *eigval, const double *eigvec, const double *r0, const double *rm, double k,
                        double norm, int r_diag, int steer_type, int64_t G, int64_t M, int64_t E, double *result,
                        double *normsteer)
{
    const int st2 = steer_type == 2;
    const int st34 = steer_type == 3 || steer_type == 4;
#pragma omp parallel
    {
        double *vr = (double *)__builtin_alloca(sizeof(double) * M);
        double *vi = (double *)__builtin_alloca(sizeof(double) * M);
#pragma omp for schedule(static)
        for (int64_t gi = 0; gi < G; ++gi) {
            const double *r = rm + gi * M;
            double help = 0.0;
            for (int64_t m = 0; m < M; ++m) {
                const float arg = (float)(k * r[m]);
                vr[m] = (double)cosf(arg);
                vi[m] = -(double)sinf(arg);
            }
            if (st2) {
                help = 0.0;
                for (int64_t m = 0; m < M; ++m) {
                    help += r[m] * r[m];
                    vr[m] *= r[m];
                    vi[m] *= r[m];
                }
            }
            if (st34) {
                help = 0.0;
                for (int64_t m = 0; m < M; ++m) {
                    help += 1.0 / (r[m] * r[m]);
                    vr[m] /= r[m];
                    vi[m] /= r[m];
                }
            }
            double scalar = 0.0;
            for (int64_t e = 0; e < E; ++e) {
                double fr = 0.0, fi = 0.0, dg = 0.0;
                for (int64_t m = 0; m < M; ++m) {
                    /* temp1 = conj(V[m][e]) * v[m] */
                    const double er = eigvec[2 * (m * E + e)], ei = -eigvec[2 * (m * E + e) + 1];
                    const double tr = er * vr[m] - ei * vi[m], ti = er * vi[m] + ei * vr[m];
                    fr += tr;
                    fi += ti;
                    if (r_diag) dg += tr * tr + ti * ti;
                }
                const double full = fr * fr + fi * fi;
                scalar += (r_diag ? full - dg : full) * eigval[e];
            }
            if (steer_type == 1) {
                const double nf = (double)M;
                normsteer[gi] = 1.0 / (double)M;
                result[gi] = scalar / (nf * nf) * norm;
            } else if (steer_type == 2) {
                const double nf = (double)M * r0[gi];
                const double nf2 = nf * nf;
                normsteer[gi] = help / nf2;
                result[gi] = scalar / nf2 * norm;
            } else if (steer_type == 3) {
                const double nf = r0[gi] * help;
                normsteer[gi] = 1.0 / (r0[gi] * r0[gi]) / help;
                result[gi] = scalar / (nf * nf) * norm;
            } else {
                const double nf = (double)M * help;
                normsteer[gi] = 1.0 / (double)M;
                result[gi] = scalar / nf * norm;
            }
        }
    }
}

/* _freqBeamformer_SpecificSteerVec_FullCSM / _CsmRemovedDiag (fastFuncs.py:414-473) and the
 * eigenvalue variants (fastFuncs.py:476-559): custom steering vectors h [G][M] (interleaved complex).
 * eig != 0: eigval [E], eigvec [M][E] instead of csm.  result = scalar * norm, normsteer = sum |h|^2. */
void orc_beamformer_custom(const double *csm, const double *eigval, const double *eigvec, int64_t E, const double *h,
                           double norm, int r_diag, int64_t G, int64_t M, double *result, double *normsteer)
{
#pragma omp parallel for schedule(static)
    for (int64_t gi = 0; gi < G; ++gi) {
        const double *v = h + 2 * gi * M;
        double help = 0.0, scalar = 0.0;
        for (int64_t m = 0; m < M; ++m) help += v[2 * m] * v[2 * m] + v[2 * m + 1] * v[2 * m + 1];
        if (!eigval) {
            for (int64_t m = 0; m < M; ++m) {
                double lr = 0.0, li = 0.0;
                for (int64_t a = 0; a < m; ++a) {   /* csm[a, m] * conj(h[a]) */
                    const double cr = csm[2 * (a * M + m)], ci = csm[2 * (a * M + m) + 1];
                    const double hr = v[2 * a], hi = -v[2 * a + 1];
                    lr += cr * hr - ci * hi;
                    li += cr * hi + ci * hr;
                }
                scalar += 2.0 * (lr * v[2 * m] - li * v[2 * m + 1]);
                if (!r_diag) {
                    const double cr = csm[2 * (m * M + m)], ci = csm[2 * (m * M + m) + 1];
                    const double hr = v[2 * m], hi = -v[2 * m + 1];
                    const double pr = cr * hr - ci * hi, pi = cr * hi + ci * hr;
                    scalar += pr * v[2 * m] - pi * v[2 * m + 1];
                }
            }
        } else {
            for (int64_t e = 0; e < E; ++e) {
                double fr = 0.0, fi = 0.0, dg = 0.0;
                for (int64_t m = 0; m < M; ++m) {
                    const double er = eigvec[2 * (m * E + e)], ei = -eigvec[2 * (m * E + e) + 1];
                    const double tr = er * v[2 * m] - ei * v[2 * m + 1], ti = er * v[2 * m + 1] + ei * v[2 * m];
                    fr += tr;
                    fi += ti;
                    dg += tr * tr + ti * ti;
                }
                const double full = fr * fr + fi * fi;
                scalar += (r_diag ? full - dg : full) * eigval[e];
            }
        }
        normsteer[gi] = help;
        result[gi] = scalar * norm;
    }
}

/* Number of OpenMP threads the library will use (reported as the baseline's core count). */
int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* calcPointSpreadFunction (fastFuncs.py:563-801) for one wave number: the four
 * _psf_Formulation* kernels.  r0: [G]; rm: [G][M]; src: [S] grid indices of the unit sources.
 * out: [G][S], out[g][s] = |sum_m e^{-i fl32(k (rm[g][m] - rm[src][m]))} w_m|^2 * n^2 with the weights
 * and normalisation of steering type steer_type (1..4), in the reference's order of operations. */
void orc_psf(const double *r0, const double *rm, double k, const int64_t *src, int64_t S, int steer_type, int64_t G,
             int64_t M, double *out)
{
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < G; ++g) {
        const double *rg = rm + g * M;
        for (int64_t j = 0; j < S; ++j) {
            const double *rs = rm + src[j] * M;
            double pr = 0.0, pi = 0.0, help = 0.0;
            for (int64_t m = 0; m < M; ++m) {
                const float arg = (float)(k * (rg[m] - rs[m]));
                double tr = (double)cosf(arg) / rs[m], ti = -(double)sinf(arg) / rs[m];
                if (steer_type == 2) {
                    tr *= rg[m];
                    ti *= rg[m];
                } else if (steer_type >= 3) {
                    tr /= rg[m];
                    ti /= rg[m];
                    help += 1.0 / (rg[m] * rg[m]);
                }
                pr += tr;
                pi += ti;
            }
            const double a2 = pr * pr + pi * pi;
            double nf;
            if (steer_type == 1) {
                nf = r0[src[j]] / (double)M;
                out[g * S + j] = a2 * (nf * nf);
            } else if (steer_type == 2) {
                nf = r0[src[j]] / r0[g] / (double)M;
                out[g * S + j] = a2 * (nf * nf);
            } else if (steer_type == 3) {
                nf = r0[src[j]] / r0[g] / help;
                out[g * S + j] = a2 * (nf * nf);
            } else {
                nf = r0[src[j]];
                out[g * S + j] = a2 * (nf * nf) / (double)M / help;
            }
        }
    }
}

/* damasSolverGaussSeidel (fastFuncs.py:804-855) for one bin: n_iter sweeps over g = 0..G-1, in order,
 * x[g] = max(0, (1 - relax) x[g] + relax (y[g] - (sum_h A[g][h] x[h] - A[g][g] x[g]))) with the latest x.
 * A: [G][G]; y: [G]; x: [G] starting solution, overwritten. */
void orc_damas_gauss_seidel(const double *A, const double *y, int64_t G, int64_t n_iter, double relax, double *x)
{
    for (int64_t it = 0; it < n_iter; ++it) {
        for (int64_t g = 0; g < G; ++g) {
            const double *row = A + g * G;
            double s = 0.0;
            for (int64_t h = 0; h < G; ++h) s += row[h] * x[h];
            s -= row[g] * x[g];
            s = (1.0 - relax) * x[g] + relax * (y[g] - s);
            x[g] = s > 0.0 ? s : 0.0;
        }
    }
}

/* damasSolverGaussSeidel over F independent bins (the guvectorize loop over the leading axis). */
void orc_damas_gauss_seidel_bins(const double *A, const double *y, int64_t F, int64_t G, int64_t n_iter, double relax,
                                 double *x)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t f = 0; f < F; ++f) orc_damas_gauss_seidel(A + f * G * G, y + f * G, G, n_iter, relax, x + f * G);
}

/* calcTransfer / _transferCoreFunc (fastFuncs.py:857-897): out[g][m] = (cos a - i sin a) r0[g] / rm[g][m],
 * a = fl32(k (rm[g][m] - r0[g])), cos/sin the C library's float32 ones.  out interleaved complex128. */
void orc_transfer(const double *r0, const double *rm, double k, int64_t G, int64_t M, double *out)
{
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < G; ++g) {
        for (int64_t m = 0; m < M; ++m) {
            const float arg = (float)(k * (rm[g * M + m] - r0[g]));
            const double tr = (double)cosf(arg) * r0[g], ti = -(double)sinf(arg) * r0[g];
            out[2 * (g * M + m)] = tr / rm[g * M + m];
            out[2 * (g * M + m) + 1] = ti / rm[g * M + m];
        }
    }
}
