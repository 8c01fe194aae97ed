/*
 * CPU restatement of the Legendre stage of cuHPX's CPU transforms -- TEST
 * INFRASTRUCTURE AND CPU BASELINE ONLY (never linked into the product).
 *
 * cuHPX's CPU SHT.forward / iSHT.forward (cuhpx/hpx_sht.py:214-236, 268-283)
 * contract the ring spectra with a dense [M][L][rings] table of orthonormal
 * Pbar_l^m(cos theta_t) (quadrature weights folded in for the analysis),
 * real and imaginary parts separately:
 *     a[l][m]  = sum_t w_t Pbar_l^m(x_t) F[t][m]                 (analysis)
 *     F[t][m]  = sum_l Pbar_l^m(x_t) a[l][m]                     (synthesis)
 * The table is built once at construction (cuhpx/sht_tools.py:192-229,
 * legpoly); at nside 1024, L = M = 2047 it is 68.6 GB in FP32 and 137 GB in
 * FP64.  Here the same values are regenerated per order by the same
 * recurrence (seed 1/sqrt(4 pi), diagonal sqrt((2l+1)(1+x)(1-x)/2/l),
 * sub-diagonal sqrt(2l+1) x, three-term coefficients of sht_tools.py:215-218)
 * so that no table is held; the rows l < m, which are zero in the table,
 * are skipped.  Orders run in parallel (OpenMP), each on its own buffers.
 *
 * Layouts (row-major, complex interleaved re, im):
 *   ftm [R][M] complex, alm [L][M] complex, w and x [R].
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* diag[m][t] = Pbar_m^m(x_t), m < M (cuhpx/sht_tools.py:207-209) */
static double* diagonal(const double* x, int R, int M) {
    double* d = (double*)malloc(sizeof(double) * (size_t)M * R);
    if (!d) return NULL;
    const double c0 = 1.0 / sqrt(4.0 * M_PI);
#pragma omp parallel for schedule(static)
    for (int t = 0; t < R; ++t) {
        double v = c0;
        d[t] = v;
        for (int l = 1; l < M; ++l) {
            v = sqrt((2.0 * l + 1.0) * (1.0 + x[t]) * (1.0 - x[t]) / 2.0 / l) * v;
            d[(size_t)l * R + t] = v;
        }
    }
    return d;
}

/* the three-term coefficients of cuhpx/sht_tools.py:215-218 */
static inline void rec_coeffs(int l, int m, double* f1, double* f2) {
    *f1 = sqrt((2.0 * l - 1.0) / (l - m) * (2.0 * l + 1.0) / (l + m));
    *f2 = sqrt((l + m - 1.0) / (l - m) * (2.0 * l + 1.0) / (2.0 * l - 3.0) * (l - m - 1.0) / (l + m));
}

int hpx_ref_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void hpx_ref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* a[l][m] = sum_t w_t Pbar_l^m(x_t) ftm[t][m]; alm is overwritten (zeros for l < m). */
int hpx_ref_sht_contract(const double* ftm, const double* w, const double* x, int R, int L, int M, double* alm) {
    double* dg = diagonal(x, R, M);
    if (!dg) return 1;
    memset(alm, 0, sizeof(double) * 2 * (size_t)L * M);
    int fail = 0;
#pragma omp parallel
    {
        double* buf = (double*)malloc(sizeof(double) * 4 * (size_t)R);
        if (!buf) {
#pragma omp atomic write
            fail = 1;
        }
#pragma omp for schedule(dynamic, 1)
        for (int m = 0; m < M; ++m) {
            if (!buf || m >= L) continue;
            double *fr = buf, *fi = buf + R, *p2 = buf + 2 * R, *p1 = buf + 3 * R;
            for (int t = 0; t < R; ++t) {
                fr[t] = w[t] * ftm[2 * ((size_t)t * M + m)];
                fi[t] = w[t] * ftm[2 * ((size_t)t * M + m) + 1];
            }
            const double* dm = dg + (size_t)m * R;
            const double s1 = sqrt(2.0 * (m + 1) + 1.0);
            double ar = 0.0, ai = 0.0, br = 0.0, bi = 0.0;
#pragma omp simd reduction(+ : ar, ai, br, bi)
            for (int t = 0; t < R; ++t) {
                const double q0 = dm[t], q1 = s1 * x[t] * dm[t];
                p2[t] = q0;
                p1[t] = q1;
                ar += q0 * fr[t];
                ai += q0 * fi[t];
                br += q1 * fr[t];
                bi += q1 * fi[t];
            }
            alm[2 * ((size_t)m * M + m)] = ar;
            alm[2 * ((size_t)m * M + m) + 1] = ai;
            if (m + 1 < L) {
                alm[2 * ((size_t)(m + 1) * M + m)] = br;
                alm[2 * ((size_t)(m + 1) * M + m) + 1] = bi;
            }
            for (int l = m + 2; l < L; ++l) {
                double f1, f2;
                rec_coeffs(l, m, &f1, &f2);
                double sr = 0.0, si = 0.0;
#pragma omp simd reduction(+ : sr, si)
                for (int t = 0; t < R; ++t) {
                    const double v = x[t] * f1 * p1[t] - f2 * p2[t];
                    p2[t] = p1[t];
                    p1[t] = v;
                    sr += v * fr[t];
                    si += v * fi[t];
                }
                alm[2 * ((size_t)l * M + m)] = sr;
                alm[2 * ((size_t)l * M + m) + 1] = si;
            }
        }
        free(buf);
    }
    free(dg);
    return fail;
}

/* ftm[t][m] = sum_l Pbar_l^m(x_t) alm[l][m]; ftm is overwritten. */
int hpx_ref_isht_contract(const double* alm, const double* x, int R, int L, int M, double* ftm) {
    double* dg = diagonal(x, R, M);
    if (!dg) return 1;
    int fail = 0;
#pragma omp parallel
    {
        double* buf = (double*)malloc(sizeof(double) * 4 * (size_t)R);
        if (!buf) {
#pragma omp atomic write
            fail = 1;
        }
#pragma omp for schedule(dynamic, 1)
        for (int m = 0; m < M; ++m) {
            if (!buf) continue;
            double *gr = buf, *gi = buf + R, *p2 = buf + 2 * R, *p1 = buf + 3 * R;
            if (m >= L) {
                for (int t = 0; t < R; ++t) {
                    ftm[2 * ((size_t)t * M + m)] = 0.0;
                    ftm[2 * ((size_t)t * M + m) + 1] = 0.0;
                }
                continue;
            }
            const double* dm = dg + (size_t)m * R;
            const double s1 = sqrt(2.0 * (m + 1) + 1.0);
            const double a0r = alm[2 * ((size_t)m * M + m)], a0i = alm[2 * ((size_t)m * M + m) + 1];
            const double a1r = m + 1 < L ? alm[2 * ((size_t)(m + 1) * M + m)] : 0.0;
            const double a1i = m + 1 < L ? alm[2 * ((size_t)(m + 1) * M + m) + 1] : 0.0;
#pragma omp simd
            for (int t = 0; t < R; ++t) {
                const double q0 = dm[t], q1 = s1 * x[t] * dm[t];
                p2[t] = q0;
                p1[t] = q1;
                gr[t] = q0 * a0r + q1 * a1r;
                gi[t] = q0 * a0i + q1 * a1i;
            }
            for (int l = m + 2; l < L; ++l) {
                double f1, f2;
                rec_coeffs(l, m, &f1, &f2);
                const double ar = alm[2 * ((size_t)l * M + m)], ai = alm[2 * ((size_t)l * M + m) + 1];
#pragma omp simd
                for (int t = 0; t < R; ++t) {
                    const double v = x[t] * f1 * p1[t] - f2 * p2[t];
                    p2[t] = p1[t];
                    p1[t] = v;
                    gr[t] += v * ar;
                    gi[t] += v * ai;
                }
            }
            for (int t = 0; t < R; ++t) {
                ftm[2 * ((size_t)t * M + m)] = gr[t];
                ftm[2 * ((size_t)t * M + m) + 1] = gi[t];
            }
        }
        free(buf);
    }
    free(dg);
    return fail;
}

/*
 * The same analysis contraction with the Legendre recurrence carried in
 * 80-bit extended precision (long double, exponent range to 1e-4951) at the
 * nodes x_t with sin^2(theta_t) = s2_t given by the caller: the reference's
 * FP64 diagonal Pbar_m^m ~ sin^m(theta) goes subnormal for high orders near
 * the poles, and the recurrence carries the lost bits up to degrees where the
 * values matter.  This is the accurate transform the CUDA FP64 path is checked
 * against at large nside.  Products with the spectra are summed in long double.
 */
int hpx_ref_sht_contract_ext(const double* ftm, const double* w, const double* x, const double* s2, int R, int L,
                             int M, double* alm) {
    memset(alm, 0, sizeof(double) * 2 * (size_t)L * M);
    int fail = 0;
#pragma omp parallel
    {
        long double* buf = (long double*)malloc(sizeof(long double) * 5 * (size_t)R);
        if (!buf) {
#pragma omp atomic write
            fail = 1;
        }
#pragma omp for schedule(dynamic, 1)
        for (int m = 0; m < M; ++m) {
            if (!buf || m >= L) continue;
            long double *fr = buf, *fi = buf + R, *p2 = buf + 2 * R, *p1 = buf + 3 * R, *xl = buf + 4 * R;
            for (int t = 0; t < R; ++t) {
                fr[t] = (long double)w[t] * ftm[2 * ((size_t)t * M + m)];
                fi[t] = (long double)w[t] * ftm[2 * ((size_t)t * M + m) + 1];
                xl[t] = x[t];
                long double d = 1.0L / sqrtl(4.0L * 3.14159265358979323846264338327950288L);
                for (int l = 1; l <= m; ++l) d = sqrtl((2.0L * l + 1.0L) * (long double)s2[t] / (2.0L * l)) * d;
                p2[t] = d;
                p1[t] = sqrtl(2.0L * (m + 1) + 1.0L) * xl[t] * d;
            }
            long double ar = 0, ai = 0, br = 0, bi = 0;
            for (int t = 0; t < R; ++t) {
                ar += p2[t] * fr[t];
                ai += p2[t] * fi[t];
                br += p1[t] * fr[t];
                bi += p1[t] * fi[t];
            }
            alm[2 * ((size_t)m * M + m)] = (double)ar;
            alm[2 * ((size_t)m * M + m) + 1] = (double)ai;
            if (m + 1 < L) {
                alm[2 * ((size_t)(m + 1) * M + m)] = (double)br;
                alm[2 * ((size_t)(m + 1) * M + m) + 1] = (double)bi;
            }
            for (int l = m + 2; l < L; ++l) {
                const long double f1 = sqrtl((2.0L * l - 1.0L) / (l - m) * (2.0L * l + 1.0L) / (l + m));
                const long double f2 = sqrtl((l + m - 1.0L) / (l - m) * (2.0L * l + 1.0L) / (2.0L * l - 3.0L) *
                                             (l - m - 1.0L) / (l + m));
                long double sr = 0, si = 0;
                for (int t = 0; t < R; ++t) {
                    const long double v = xl[t] * f1 * p1[t] - f2 * p2[t];
                    p2[t] = p1[t];
                    p1[t] = v;
                    sr += v * fr[t];
                    si += v * fi[t];
                }
                alm[2 * ((size_t)l * M + m)] = (double)sr;
                alm[2 * ((size_t)l * M + m) + 1] = (double)si;
            }
        }
        free(buf);
    }
    return fail;
}

/* The synthesis contraction in extended precision (as hpx_ref_sht_contract_ext). */
int hpx_ref_isht_contract_ext(const double* alm, const double* x, const double* s2, int R, int L, int M,
                              double* ftm) {
    int fail = 0;
#pragma omp parallel
    {
        long double* buf = (long double*)malloc(sizeof(long double) * 5 * (size_t)R);
        if (!buf) {
#pragma omp atomic write
            fail = 1;
        }
#pragma omp for schedule(dynamic, 1)
        for (int m = 0; m < M; ++m) {
            if (!buf) continue;
            long double *gr = buf, *gi = buf + R, *p2 = buf + 2 * R, *p1 = buf + 3 * R, *xl = buf + 4 * R;
            if (m >= L) {
                for (int t = 0; t < R; ++t) {
                    ftm[2 * ((size_t)t * M + m)] = 0.0;
                    ftm[2 * ((size_t)t * M + m) + 1] = 0.0;
                }
                continue;
            }
            const long double a0r = alm[2 * ((size_t)m * M + m)], a0i = alm[2 * ((size_t)m * M + m) + 1];
            const long double a1r = m + 1 < L ? alm[2 * ((size_t)(m + 1) * M + m)] : 0.0;
            const long double a1i = m + 1 < L ? alm[2 * ((size_t)(m + 1) * M + m) + 1] : 0.0;
            for (int t = 0; t < R; ++t) {
                xl[t] = x[t];
                long double d = 1.0L / sqrtl(4.0L * 3.14159265358979323846264338327950288L);
                for (int l = 1; l <= m; ++l) d = sqrtl((2.0L * l + 1.0L) * (long double)s2[t] / (2.0L * l)) * d;
                p2[t] = d;
                p1[t] = sqrtl(2.0L * (m + 1) + 1.0L) * xl[t] * d;
                gr[t] = p2[t] * a0r + (m + 1 < L ? p1[t] * a1r : 0.0L);
                gi[t] = p2[t] * a0i + (m + 1 < L ? p1[t] * a1i : 0.0L);
            }
            for (int l = m + 2; l < L; ++l) {
                const long double f1 = sqrtl((2.0L * l - 1.0L) / (l - m) * (2.0L * l + 1.0L) / (l + m));
                const long double f2 = sqrtl((l + m - 1.0L) / (l - m) * (2.0L * l + 1.0L) / (2.0L * l - 3.0L) *
                                             (l - m - 1.0L) / (l + m));
                const long double ar = alm[2 * ((size_t)l * M + m)], ai = alm[2 * ((size_t)l * M + m) + 1];
                for (int t = 0; t < R; ++t) {
                    const long double v = xl[t] * f1 * p1[t] - f2 * p2[t];
                    p2[t] = p1[t];
                    p1[t] = v;
                    gr[t] += v * ar;
                    gi[t] += v * ai;
                }
            }
            for (int t = 0; t < R; ++t) {
                ftm[2 * ((size_t)t * M + m)] = (double)gr[t];
                ftm[2 * ((size_t)t * M + m) + 1] = (double)gi[t];
            }
        }
        free(buf);
    }
    return fail;
}
