/*
 * tce_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the toroidal
 * ERI path of ALRAKIK/William_CI.  See tce_oracle.h for the rules of use and
 * the parity status.  Each routine names the reference file:line it restates
 * (paths relative to the reference project root).
 *
 * The pair-vector memo (clifford_tools.f90:467-549) is compiled only into the
 * timing build (ORC_PAIR_MEMO); the parity build recomputes the vectors, which
 * gives the same values.  Not restated: the point-group "symmetry" keyword and
 * the timers.
 */
#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include "tce_oracle.h"
#include "debye_coeffs.h"
#ifdef _OPENMP
#include <omp.h>
#endif

#define NMC 16                /* NMAX_CLIFF, clifford_tools.f90:82 */
#define MAXP 64               /* primitives per shell supported by the oracle */
#define PI_D 3.14159265358979323846

/* =====================================================================
 * log I_v(x) scaled by e^-x : bessel_iv_log.f90:43-318 (CUSF port).
 * ===================================================================== */
static double debye_poly(int k, double t2)
{   /* P_k(t^2) by Horner, u_k(t) = t^k P_k(t^2) */
    double s = 0.0;
    for (int j = k; j >= 0; --j) s = s * t2 + DEBYE_P[k][j];
    return s;
}

static double iv_uniform(double v, double x, int order)
{   /* bessel_iv_log.f90:141-171 (and the identical blocks for 6, 9, 13) */
    double u = v / x, v_eta, x_prime, x_prime_2;
    if (u < 0.5) {
        double asinh_u = asinh(u);
        double t1 = u / (sqrt(1.0 + u * u) + 1.0);
        v_eta = v * (t1 - asinh_u);
        x_prime = 1.0 / u;
        x_prime_2 = 1.0 / (u * u);
    } else {
        x_prime = 1.0 / u;
        x_prime_2 = x_prime * x_prime;
        double s = sqrt(1.0 + x_prime_2);
        v_eta = v * (s - x_prime + log(x_prime / (1.0 + s)));
    }
    double sq = sqrt(1.0 + x_prime_2);
    double t = 1.0 / sq, t2 = t * t;
    double sum = 1.0, vp = 1.0, tp = 1.0;
    for (int k = 1; k <= order; ++k) {
        vp *= v; tp *= t;
        sum += tp * debye_poly(k, t2) / vp;
    }
    return -0.91893853320467267 - 0.5 * log(v) + v_eta - 0.25 * log(1.0 + x_prime_2) + log(fabs(sum));
}

double orc_iv_log(double v_in, double x)
{
    const double LOG_INV_SQRT_2PI = -0.91893853320467267;
    const double LOG_2 = 0.69314718055994529;
    if (x < 0.0 || (v_in < 0.0 && v_in != floor(v_in))) return NAN;
    if (x == 0.0) return (v_in == 0.0) ? 0.0 : -DBL_MAX;
    double v = v_in < 0.0 ? -v_in : v_in;
    double log_x = log(x), log_v = log(v);
    if (v == 0.0) log_v = -1000.0;

    /* Method 1: mu-series order 3 (:95-114) */
    if ((x > 1.4e3 && v < 3.05) ||
        (((0.6229 * log_x - 3.2318) > log_v) && v > 3.1 && (pow(v, 8) / (384.0 * pow(x, 4)) < 1e-16))) {
        double mu = 4.0 * v * v, cur = 1.0, sum = 1.0;
        for (int k = 1, c = 1; k <= 5; k += 2, ++c) {
            cur = cur * (-(mu - (double)(k * k)) / ((double)c * 8.0 * x));
            sum += cur;
        }
        return LOG_INV_SQRT_2PI - 0.5 * log_x + log(fabs(sum));
    }
    /* Method 2: mu-series order 20 (:118-135) */
    if ((x > 30.0 && v < 15.3919) ||
        ((0.5113 * log_x + 0.7939 > log_v) && x > 59.6925 && v < sqrt(3.0 * x))) {
        double mu = 4.0 * v * v, cur = 1.0, sum = 1.0;
        for (int k = 1, c = 1; k <= 39; k += 2, ++c) {
            cur = cur * (-(mu - (double)(k * k)) / ((double)c * 8.0 * x));
            sum += cur;
        }
        return LOG_INV_SQRT_2PI - 0.5 * log_x + log(fabs(sum));
    }
    /* Methods 3-6: uniform (Debye) expansions of order 4, 6, 9, 13 (:138-288) */
    if ((x > 274.2377 && v > 0.3) || v > 163.6993) return iv_uniform(v, x, 4);
    if ((x > 84.4153 && v > 0.46) || v > 56.9971) return iv_uniform(v, x, 6);
    if ((x > 35.9074 && v > 0.6) || v > 20.1534) return iv_uniform(v, x, 9);
    if ((x > 19.6931 && v > 0.7) || v > 12.6964) return iv_uniform(v, x, 13);

    /* Method 7: power series in log form, 41 terms (:292-314) */
    {
        enum { N_TERMS = 41 };
        double terms[N_TERMS];
        double x2o4 = x * x / 4.0, inv = 1.0 / x2o4, vinv = v * inv;
        terms[0] = -lgamma(v + 1.0);
        for (int k = 1; k < N_TERMS; ++k)
            terms[k] = terms[k - 1] - log((double)k * ((double)k * inv + vinv));
        int peak = (int)floor((-v + sqrt(v * v + x * x)) / 2.0);
        if (peak < 0) peak = 0;
        if (peak > N_TERMS - 1) peak = N_TERMS - 1; /* outside the region this branch serves */
        double s = 0.0;
        for (int k = 0; k < N_TERMS; ++k) s += exp(terms[k] - terms[peak]);
        return v * (log_x - LOG_2) + terms[peak] + log(s) - x;
    }
}

double orc_iv_scaled(int n, double x) { return exp(orc_iv_log((double)n, x)); } /* :320-328 */

/* =====================================================================
 * clifford_tools.f90
 * ===================================================================== */

/* bessel_scaled_vector :386-421 (Miller, start N+30+sqrt(80A)) */
void orc_bessel_scaled_vector(int N, double A, double *Iv)
{
    if (A < 1e-12) { for (int k = 0; k <= N; ++k) Iv[k] = 0.0; Iv[0] = 1.0; return; }
    int n0 = N + 30 + (int)sqrt(80.0 * A);
    double *w = (double *)malloc(sizeof(double) * (size_t)(n0 + 1));
    double ip1 = 0.0, ik = 1e-300, im1;
    w[n0] = ik;
    for (int k = n0; k >= 1; --k) {
        im1 = ip1 + (2.0 * (double)k / A) * ik;
        ip1 = ik; ik = im1;
        w[k - 1] = ik;
        if (fabs(ik) > 1e250) {
            for (int m = k - 1; m <= n0; ++m) w[m] *= 1e-250;
            ip1 *= 1e-250; ik *= 1e-250;
        }
    }
    double norm = orc_iv_scaled(0, A) / w[0];
    for (int k = 0; k <= N; ++k) Iv[k] = w[k] * norm;
    free(w);
}

/* bessel_scaled_vector_fast :429-461 (Miller started at N itself) */
void orc_bessel_scaled_vector_fast(int N, double A, double *Iv)
{
    if (A < 1e-10) { for (int k = 0; k <= N; ++k) Iv[k] = 0.0; Iv[0] = 1.0; return; }
    if (N < 2) { for (int k = 0; k <= N; ++k) Iv[k] = orc_iv_scaled(k, A); return; }
    double inv_A2 = 2.0 / A;
    Iv[N] = 1e-280;
    Iv[N - 1] = Iv[N] * (double)N * inv_A2;
    for (int k = N - 1; k >= 1; --k) {
        Iv[k - 1] = Iv[k + 1] + (double)k * inv_A2 * Iv[k];
        if (Iv[k - 1] > 1e250) for (int m = k - 1; m <= N; ++m) Iv[m] *= 1e-250;
    }
    double s = orc_iv_scaled(0, A) / Iv[0];
    for (int k = 0; k <= N; ++k) Iv[k] *= s;
}

/* bessel_nmax_estimate :566-572 */
int orc_bessel_nmax_estimate(double A) { return 20 + (int)ceil(9.0 * sqrt(A > 0.0 ? A : 0.0)); }

/* fourier_sin_product :578-607 ; d has 2(i+l)+1 entries, d[k + (i+l)] */
void orc_fourier_sin_product(int i, int l, double phA, double phB, double *dre, double *dim)
{
    int M = i + l, deg = 0;
    double tre[2 * NMC + 8], tim[2 * NMC + 8];
    for (int k = 0; k <= 2 * M; ++k) { dre[k] = 0.0; dim[k] = 0.0; }
    dre[M] = 1.0;
    for (int m = 1; m <= M; ++m) {
        double ph = (m <= i) ? phA : phB;
        /* cp = e^{i ph}/(2i) = (sin ph - i cos ph)/2 ; cm = -e^{-i ph}/(2i) = (sin ph + i cos ph)/2 */
        double s = sin(ph), c = cos(ph);
        double cpr = 0.5 * s, cpi = -0.5 * c;
        double cmr = 0.5 * s, cmi = 0.5 * c;
        for (int k = 0; k <= 2 * M + 2; ++k) { tre[k] = 0.0; tim[k] = 0.0; }
        for (int k = -deg; k <= deg; ++k) {
            double ar = dre[k + M], ai = dim[k + M];
            /* tmp index shifted by +1 so that k-1 >= -M-1 maps to >= 0 */
            tre[k + 1 + M + 1] += cpr * ar - cpi * ai;
            tim[k + 1 + M + 1] += cpr * ai + cpi * ar;
            tre[k - 1 + M + 1] += cmr * ar - cmi * ai;
            tim[k - 1 + M + 1] += cmr * ai + cmi * ar;
        }
        deg += 1;
        for (int k = -deg; k <= deg; ++k) { dre[k + M] = tre[k + M + 1]; dim[k + M] = tim[k + M + 1]; }
    }
}

/* pair Fourier vector (the value pair_vector_cached :467-549 returns) */
void orc_pair_vector(int N, double A, int i, int l, double phA, double phB, int sgn,
                     double *vre, double *vim)
{
    int M = i + l;
    double *Iv = (double *)malloc(sizeof(double) * (size_t)(N + M + 1));
    orc_bessel_scaled_vector_fast(N + M, A, Iv);
    if (M == 0) {
        for (int m = 0; m <= N; ++m) { vre[m] = Iv[m]; vim[m] = 0.0; }
    } else {
        double dre[2 * NMC + 1], dim[2 * NMC + 1];
        orc_fourier_sin_product(i, l, phA, phB, dre, dim);
        for (int m = 0; m <= N; ++m) {
            double ar = 0.0, ai = 0.0;
            for (int kk = -M; kk <= M; ++kk) {
                double b = Iv[abs(m - sgn * kk)];
                ar += dre[kk + M] * b; ai += dim[kk + M] * b;
            }
            vre[m] = ar; vim[m] = ai;
        }
    }
    free(Iv);
}

/* Memo of the pair Fourier vectors, as pair_vector_cached keeps them
 * (clifford_tools.f90:467-549): one table shared by the OpenMP threads, keyed
 * by the bits of (A, phA, phB) and (N, i, l, sgn), open addressing with up to
 * 64 probes, lock-free lookups (the slot's offset is published last), inserts
 * one at a time, a pool of at most 16e6 complex numbers (256 MB); a vector that
 * does not fit is returned uncached.  Compiled only into the timing build
 * (ORC_PAIR_MEMO, Makefile target `fast`): the parity build recomputes every
 * vector, which gives the same values. */
#ifdef ORC_PAIR_MEMO
#define PV_SLOTS (1u << 18)
#define PV_POOL_MAX 16000000LL
static int64_t *pv_key;            /* [4 * PV_SLOTS] */
static int64_t *pv_off;            /* [PV_SLOTS], -1 = empty; offset in complex numbers */
static double *pv_pool;            /* [2 * PV_POOL_MAX], re/im interleaved */
static int64_t pv_used;
static int pv_ready;

static void pv_init(void)
{
    if (__atomic_load_n(&pv_ready, __ATOMIC_ACQUIRE)) return;
    #pragma omp critical(orc_pv_cache)
    {
        if (!pv_ready) {
            pv_key = (int64_t *)malloc(sizeof(int64_t) * 4 * (size_t)PV_SLOTS);
            pv_off = (int64_t *)malloc(sizeof(int64_t) * (size_t)PV_SLOTS);
            pv_pool = (double *)malloc(sizeof(double) * 2 * (size_t)PV_POOL_MAX);
            for (size_t h = 0; h < PV_SLOTS; ++h) pv_off[h] = -1;
            pv_used = 0;
            __atomic_store_n(&pv_ready, 1, __ATOMIC_RELEASE);
        }
    }
}

void orc_pair_cache_free(void)
{
    free(pv_key); free(pv_off); free(pv_pool);
    pv_key = pv_off = NULL; pv_pool = NULL;
    pv_used = 0;
    pv_ready = 0;
}

static void pair_vector_memo(int N, double A, int i, int l, double phA, double phB, int sgn, double *vre, double *vim)
{
    pv_init();
    int64_t k[4];
    memcpy(&k[0], &A, 8); memcpy(&k[1], &phA, 8); memcpy(&k[2], &phB, 8);
    k[3] = (int64_t)N + 1000000LL * ((int64_t)i + 64LL * ((int64_t)l + 64LL * (int64_t)(sgn + 1)));
    uint64_t hh = (uint64_t)k[0] * 31u + (uint64_t)k[1];
    hh = hh * 31u + (uint64_t)k[2];
    hh = hh * 31u + (uint64_t)k[3];
    hh ^= hh >> 31;
    const unsigned h0 = (unsigned)(hh & (PV_SLOTS - 1));
    unsigned h = h0;
    for (int probe = 0; probe < 64; ++probe) {
        int64_t o = __atomic_load_n(&pv_off[h], __ATOMIC_ACQUIRE);
        if (o < 0) break;
        const int64_t *key = pv_key + 4 * (size_t)h;
        if (key[0] == k[0] && key[1] == k[1] && key[2] == k[2] && key[3] == k[3]) {
            const double *v = pv_pool + 2 * o;
            for (int m = 0; m <= N; ++m) { vre[m] = v[2 * m]; vim[m] = v[2 * m + 1]; }
            return;
        }
        h = (h + 1) & (PV_SLOTS - 1);
    }
    orc_pair_vector(N, A, i, l, phA, phB, sgn, vre, vim);
    #pragma omp critical(orc_pv_cache)
    {
        unsigned g = h0;
        int free_slot = 0;
        for (int probe = 0; probe < 64; ++probe) {
            if (pv_off[g] < 0) { free_slot = 1; break; }
            const int64_t *key = pv_key + 4 * (size_t)g;
            if (key[0] == k[0] && key[1] == k[1] && key[2] == k[2] && key[3] == k[3]) break;
            g = (g + 1) & (PV_SLOTS - 1);
        }
        if (free_slot && pv_used + N + 1 <= PV_POOL_MAX) {
            const int64_t o = pv_used;
            double *v = pv_pool + 2 * o;
            for (int m = 0; m <= N; ++m) { v[2 * m] = vre[m]; v[2 * m + 1] = vim[m]; }
            pv_used += N + 1;
            memcpy(pv_key + 4 * (size_t)g, k, sizeof k);
            __atomic_store_n(&pv_off[g], o, __ATOMIC_RELEASE);
        }
    }
}
#define PAIR_VECTOR pair_vector_memo
#else
void orc_pair_cache_free(void) {}
#define PAIR_VECTOR orc_pair_vector
#endif

/* fast_quad_points precompute_t.f90:906-942 : GL on [0,1], t = 0.6u/(1-u) */
void orc_fast_quad_points(int n, double *t, double *w)
{
    const double s = 0.6;
    for (int i = 1; i <= n; ++i) {
        double x = cos(PI_D * ((double)i - 0.25) / ((double)n + 0.5));
        double p0, p1, p2, dp, dx;
        for (int it = 0; it < 100; ++it) {
            p0 = 1.0; p1 = x;
            for (int j = 2; j <= n; ++j) { p2 = ((2.0 * j - 1.0) * x * p1 - (j - 1.0) * p0) / (double)j; p0 = p1; p1 = p2; }
            dp = (double)n * (x * p1 - p0) / (x * x - 1.0);
            dx = p1 / dp;
            x = x - dx;
            if (fabs(dx) < 1e-15) break;
        }
        p0 = 1.0; p1 = x;
        for (int j = 2; j <= n; ++j) { p2 = ((2.0 * j - 1.0) * x * p1 - (j - 1.0) * p0) / (double)j; p0 = p1; p1 = p2; }
        dp = (double)n * (x * p1 - p0) / (x * x - 1.0);
        double u = 0.5 * (1.0 - x);
        double wu = 1.0 / ((1.0 - x * x) * dp * dp);
        t[i - 1] = s * u / (1.0 - u);
        w[i - 1] = wu * s / ((1.0 - u) * (1.0 - u));
    }
}

/* tools.f90:1-264 (bary_center_toroidal_*, bary_exponent_*) via bary_dir :715-733 */
void orc_bary(double e1, double e2, double x1, double x2, double L, double a, double *pe, double *cen)
{
    const double eps = 1e-6;
    double x = x1 - x2, p;
    if (fabs(x) > 0.5 * L - eps && fabs(x) < 0.5 * L + eps)
        p = (fabs(e1 - e2) < 1e-8) ? 0.0 : fabs(e1 - e2);
    else {
        p = e1 * e1 + e2 * e2 + 2.0 * e1 * e2 * cos(a * x);
        p = sqrt(fabs(p));
    }
    if (p > e1 + e2) p = e1 + e2;
    if (e1 + e2 - p < 1e-14) p = e1 + e2;
    *pe = p;

    double r1 = x1, r2 = x2, rp;
    double d = fabs(r1 - r2);
    if (d < 0.5 * L + eps && d > 0.5 * L - eps) {
        if (fabs(e1 - e2) < 1e-10) rp = 0.5 * (r1 + r2);
        else if (e1 > e2) rp = r1;
        else if (e2 > e1) rp = r2;
        else rp = 0.5 * (r1 + r2);
    } else if (fabs(e1 - e2) < 1e-10) {
        rp = (d > 0.5 * L + eps) ? 0.5 * (r1 + r2) - 0.5 * L : 0.5 * (r1 + r2);
    } else {
        double val = e1 * cos(a * r1) + e2 * cos(a * r2);
        double H = (-val >= 0.0) ? 1.0 : 0.0; /* HeavisideModule */
        rp = atan((e1 * sin(a * r1) + e2 * sin(a * r2)) / val) / a + 0.5 * L * H;
    }
    *cen = rp;
}

/* hermite_E_1D :757-785 ; E has NMC+1 entries */
void orc_hermite_E_1D(int i, int j, double p, double PA, double PB, double *E)
{
    double Eold[NMC + 4], Enew[NMC + 4]; /* Eold index t+1 (t = -1 .. NMC+1) */
    double inv2p = 0.5 / p;
    for (int t = 0; t < NMC + 4; ++t) { Eold[t] = 0.0; Enew[t] = 0.0; }
    Eold[1] = 1.0;
    int deg = 0;
    for (int m = 1; m <= i + j; ++m) {
        double X = (m <= i) ? PA : PB;
        for (int t = 0; t <= deg + 1; ++t)
            Enew[t] = inv2p * Eold[t] + X * Eold[t + 1] + (double)(t + 1) * Eold[t + 2];
        deg += 1;
        for (int t = 0; t <= deg; ++t) Eold[t + 1] = Enew[t];
        Eold[deg + 2] = 0.0;
    }
    for (int t = 0; t <= NMC; ++t) E[t] = 0.0;
    for (int t = 0; t <= deg; ++t) E[t] = Eold[t + 1];
}

/* =====================================================================
 * one-electron overlap (normalisation input): clifford_tools.f90:120-380,
 * 1D_Overlap_toroidal.f90:83-157, 2D/3D analogues.
 * ===================================================================== */
static double Ttab[NMC + 1][NMC + 1][NMC / 2 + 1][NMC + 1];   /* filled once by init_clifford, outside parallel regions */
static double binom_t[NMC + 1][NMC + 1];
static double dfact_t[2 * NMC + 2]; /* dfact(n) at [n+1] */
static int clifford_ready = 0;

static void init_clifford(void) /* :120-165 */
{
    if (clifford_ready) return;
    memset(binom_t, 0, sizeof binom_t);
    binom_t[0][0] = 1.0;
    for (int n = 1; n <= NMC; ++n) {
        binom_t[n][0] = 1.0;
        for (int k = 1; k <= n; ++k) binom_t[n][k] = binom_t[n - 1][k - 1] + (k <= n - 1 ? binom_t[n - 1][k] : 0.0);
    }
    dfact_t[0] = 1.0; dfact_t[1] = 1.0;
    for (int n = 1; n <= 2 * NMC; ++n) { int m = n - 2 < -1 ? -1 : n - 2; dfact_t[n + 1] = (double)n * dfact_t[m + 1]; }
    memset(Ttab, 0, sizeof Ttab);
    static double Tcur[NMC + 1][NMC + 1], Tnew[NMC + 1][NMC + 1];
    for (int s = 0; s <= NMC / 2; ++s) {
        memset(Tcur, 0, sizeof Tcur);
        Tcur[s][s] = 1.0;
        for (int e = 0; e <= NMC; ++e) for (int nu = 0; nu <= NMC; ++nu) Ttab[e][nu][s][0] = Tcur[e][nu];
        for (int m = 1; m <= NMC - 2 * s; ++m) {
            memset(Tnew, 0, sizeof Tnew);
            for (int e = 0; e <= NMC; ++e)
                for (int nu = e; nu <= NMC - 1; ++nu) {
                    if (Tcur[e][nu] == 0.0) continue;
                    Tnew[e][nu + 1] += Tcur[e][nu];
                    if (nu > e) Tnew[e + 1][nu] += (double)(nu - e) * Tcur[e][nu];
                }
            memcpy(Tcur, Tnew, sizeof Tcur);
            for (int e = 0; e <= NMC; ++e) for (int nu = 0; nu <= NMC; ++nu) Ttab[e][nu][s][m] = Tcur[e][nu];
        }
    }
    clifford_ready = 1;
}

static void clifford_bessel_ratios(int nmax, double A, double R[NMC + 1][NMC + 1]) /* :171-220 */
{
    memset(R, 0, sizeof(double) * (NMC + 1) * (NMC + 1));
    if (A < 1.0) {
        double eA = exp(-A), q = 0.25 * A * A;
        for (int nu = 0; nu <= nmax; ++nu) {
            double term = 1.0;
            for (int k = 1; k <= nu; ++k) term = term / (2.0 * (double)k);
            double ser = term;
            for (int k = 1; k <= 14; ++k) { term = term * q / ((double)k * (double)(k + nu)); ser += term; }
            for (int e = 0; e <= nu; ++e) R[e][nu] = (nu == e) ? eA * ser : eA * ser * pow(A, nu - e);
        }
    } else {
        double ive[NMC + 1];
        for (int nu = 0; nu <= nmax; ++nu) ive[nu] = orc_iv_scaled(nu, A);
        for (int e = 0; e <= nmax; ++e) {
            double Ae = pow(A, e);
            for (int nu = e; nu <= nmax; ++nu) R[e][nu] = ive[nu] / Ae;
        }
    }
}

static double Icliff_from_R(int n, int m, double R[NMC + 1][NMC + 1], double L) /* :227-246 */
{
    if (n % 2 != 0) return 0.0;
    int s = n / 2;
    double acc = 0.0;
    for (int e = s; e <= s + m; ++e)
        for (int nu = e; nu <= s + m; ++nu)
            if (Ttab[e][nu][s][m] != 0.0) acc += Ttab[e][nu][s][m] * R[e][nu];
    return L * dfact_t[n - 1 + 1] * acc;
}

static double overlap_1D_clifford_ext(int i, int l, int ds, int dc, double spa, double cpa, double spb,
                                      double cpb, double inv_ax, double R[NMC + 1][NMC + 1], double L)
{   /* :268-293 */
    if (i < 0 || l < 0) return 0.0;
    double acc = 0.0;
    for (int k = 0; k <= i; ++k) {
        double fa = binom_t[i][k] * pow(cpa, k) * pow(spa, i - k);
        if (fa == 0.0) continue;
        for (int q = 0; q <= l; ++q) {
            int ns = k + q + ds;
            if (ns % 2 != 0) continue;
            int nc = (i - k) + (l - q) + dc;
            double fb = binom_t[l][q] * pow(cpb, q) * pow(spb, l - q);
            acc += fa * fb * Icliff_from_R(ns, nc, R, L);
        }
    }
    return acc * pow(inv_ax, i + l);
}

static double overlap_1D_real(int j, int m, double p, double pa, double pb) /* :336-361 */
{
    double base = sqrt(PI_D / p), mom[NMC + 1];
    for (int n = 0; n <= j + m; ++n)
        mom[n] = (n % 2 == 0) ? dfact_t[n - 1 + 1] / pow(2.0 * p, n / 2) * base : 0.0;
    double acc = 0.0;
    for (int k = 0; k <= j; ++k)
        for (int q = 0; q <= m; ++q) {
            if ((k + q) % 2 != 0) continue;
            acc += binom_t[j][k] * binom_t[m][q] * pow(pa, j - k) * pow(pb, m - q) * mom[k + q];
        }
    return acc;
}

double orc_overlap_pair(int ndp, const double L[3], const int32_t l1[3], const int32_t l2[3],
                        const double r1[3], const double r2[3], int n1, const double *e1,
                        const double *c1, int n2, const double *e2, const double *c2)
{
    init_clifford();
    double S = 0.0, R[NMC + 1][NMC + 1];
    for (int i = 0; i < n1; ++i)
        for (int j = 0; j < n2; ++j) {
            double al = e1[i], be = e2[j], prod = 1.0;
            for (int d = 0; d < 3; ++d) {
                if (d < ndp) {
                    double a = 2.0 * PI_D / L[d], pe, cen;
                    orc_bary(al, be, r1[d], r2[d], L[d], a, &pe, &cen);
                    double A = 2.0 * pe / (a * a);
                    double kd = exp(-2.0 * (al + be - pe) / (a * a));
                    int nmax = l1[d] + l2[d] < NMC ? l1[d] + l2[d] : NMC;
                    clifford_bessel_ratios(nmax, A, R);
                    prod *= kd * overlap_1D_clifford_ext(l1[d], l2[d], 0, 0, sin(a * (cen - r1[d])), cos(a * (cen - r1[d])),
                                                         sin(a * (cen - r2[d])), cos(a * (cen - r2[d])), 1.0 / a, R, L[d]);
                } else {
                    double es = al + be, mu = al * be / es;
                    double P = (al * r1[d] + be * r2[d]) / es;
                    prod *= exp(-mu * (r1[d] - r2[d]) * (r1[d] - r2[d])) * overlap_1D_real(l1[d], l2[d], es, P - r1[d], P - r2[d]);
                }
            }
            S += c1[i] * c2[j] * prod;
        }
    return S;
}

/* normalize_1D.f90:17-79 (2D, 3D identical with their overlap) */
double orc_normalize(int ndp, const double L[3], int nbas, const double *ctr, const int32_t *lxyz,
                     const int32_t *prim_off, const double *exps, double *coefs)
{
    double dev = 0.0;
    for (int f = 0; f < nbas; ++f) {
        int o = prim_off[f], np = prim_off[f + 1] - prim_off[f];
        const double *r = ctr + 3 * f;
        const int32_t *l = lxyz + 3 * f;
        for (int i = 0; i < np; ++i) {
            double one = 1.0;
            double S = orc_overlap_pair(ndp, L, l, l, r, r, 1, exps + o + i, &one, 1, exps + o + i, &one);
            coefs[o + i] /= sqrt(S);
        }
        double S = orc_overlap_pair(ndp, L, l, l, r, r, np, exps + o, coefs + o, np, exps + o, coefs + o);
        for (int i = 0; i < np; ++i) coefs[o + i] /= sqrt(S);
        S = orc_overlap_pair(ndp, L, l, l, r, r, np, exps + o, coefs + o, np, exps + o, coefs + o);
        if (fabs(S - 1.0) > dev) dev = fabs(S - 1.0);
    }
    return dev;
}

/* =====================================================================
 * The engine context: t-tables + shells + cells + Schwarz + prim table
 * (ERI_toroidal.f90:93-337, eri_direct.f90:76-225)
 * ===================================================================== */
typedef struct {
    int n;                 /* components */
    double r[3];
    int pw[15][3];
    int np;
    double e[MAXP];
    double c[15][MAXP];
} shellv;

struct orc_ctx {
    orc_system s;
    int nbas, nfuc, ndp, nq, ncap;
    double L[3], a[3];
    /* copies of AO data */
    double *ctr, *exps, *coefs;
    int32_t *lxyz, *poff;
    /* t tables (clifford_tools.f90:58-67) */
    double *t_node, *t_weight, *t_bessel, *t_bt;
    int *t_nmax, *t_kfirst, t_nmaxall[3], t_nsplit[3];
    /* shells */
    int nsh, nshuc, *sh_first, *sh_n;
    int sym_ok, ncl[3], ncell;
    int *scell, *sloc, *fcell, *floc, *relc;
    double *Q, *Qsh, Qmax;
    int mp;
    double *ps_qp;
};

#define TB(c, n, k, d) ((c)->t_bessel[(size_t)(n) + (size_t)((c)->ncap + 1) * ((size_t)(k) + (size_t)(c)->nq * (size_t)(d))])
#define TBT(c, k, n, d) ((c)->t_bt[(size_t)(k) + (size_t)(c)->nq * ((size_t)(n) + (size_t)((c)->ncap + 1) * (size_t)(d))])

/* setup_t_tables :620-709 */
static void setup_t_tables(orc_ctx *c)
{
    int nq = c->nq, ncap = c->ncap, ndp = c->ndp;
    c->t_bessel = (double *)calloc((size_t)(ncap + 1) * nq * ndp, sizeof(double));
    c->t_nmax = (int *)calloc((size_t)nq * ndp, sizeof(int));
    for (int d = 0; d < ndp; ++d)
        for (int k = 0; k < nq; ++k)
            orc_bessel_scaled_vector(ncap, 2.0 * c->t_node[k] * c->t_node[k] / (c->a[d] * c->a[d]), &TB(c, 0, k, d));
    for (int d = 0; d < ndp; ++d)
        for (int k = 0; k < nq; ++k) {
            int nm = ncap;
            for (int n = 0; n <= ncap; ++n)
                if (TB(c, n, k, d) < 1e-16 * TB(c, 0, k, d)) { nm = (n + 5 < ncap) ? n + 5 : ncap; break; }
            c->t_nmax[k + nq * d] = nm;
        }
    c->t_bt = (double *)calloc((size_t)nq * (ncap + 1) * ndp, sizeof(double));
    for (int d = 0; d < ndp; ++d) {
        int mx = 0;
        for (int k = 0; k < nq; ++k) {
            int nm = c->t_nmax[k + nq * d];
            if (nm > mx) mx = nm;
            TBT(c, k, 0, d) = TB(c, 0, k, d);
            for (int n = 1; n <= nm; ++n) TBT(c, k, n, d) = 2.0 * TB(c, n, k, d);
        }
        c->t_nmaxall[d] = mx;
    }
    c->t_kfirst = (int *)calloc((size_t)(ncap + 1) * ndp, sizeof(int));
    for (int d = 0; d < ndp; ++d)
        for (int n = 0; n <= ncap; ++n) {
            int kf = nq; /* 0-based "nq+1" */
            for (int k = 0; k < nq && kf == nq; ++k)
                for (int kk = k; kk < nq; ++kk)
                    if (TBT(c, kk, n, d) != 0.0) { kf = k; break; }
            c->t_kfirst[n + (ncap + 1) * d] = kf;
        }
    for (int d = 0; d < ndp; ++d) {
        int ns = 0, need = nq < 8 ? nq : 8;
        for (int n = 0; n <= ncap; ++n) {
            int cnt = 0;
            for (int k = 0; k < nq; ++k) if (c->t_nmax[k + nq * d] >= n) ++cnt;
            if (cnt >= need) ns = n;
        }
        c->t_nsplit[d] = ns;
    }
}

static void make_shell(const orc_ctx *c, int first, int n, shellv *s)
{
    s->n = n;
    for (int d = 0; d < 3; ++d) s->r[d] = c->ctr[3 * first + d];
    s->np = c->poff[first + 1] - c->poff[first];
    for (int i = 0; i < s->np; ++i) s->e[i] = c->exps[c->poff[first] + i];
    for (int a = 0; a < n; ++a) {
        for (int d = 0; d < 3; ++d) s->pw[a][d] = c->lxyz[3 * (first + a) + d];
        for (int i = 0; i < s->np; ++i) s->c[a][i] = c->coefs[c->poff[first + a] + i];
    }
}

static void single_prim(const shellv *src, int p, shellv *dst)
{
    *dst = *src;
    dst->np = 1;
    dst->e[0] = src->e[p];
    for (int a = 0; a < src->n; ++a) dst->c[a][0] = src->c[a][p];
}

/* =====================================================================
 * ERI_shell_block_toroidal : ERI_shell_block_toroidal.f90:28-390
 *   ps_noscreen: no prefactor screens; ps_bra/ps_ket (mp x mp): prim screen
 * ===================================================================== */
static void shell_block(const orc_ctx *c, const shellv *SA, const shellv *SB, const shellv *SC,
                        const shellv *SD, int ps_noscreen, const double *ps_bra, const double *ps_ket,
                        int mp, double *blk)
{
    const double screen_tol = 2.22e-16;
    const int ndp = c->ndp, nq = c->nq;
    int nA = SA->n, nB = SB->n, nC = SC->n, nD = SD->n;
    for (int x = 0; x < nA * nB * nC * nD; ++x) blk[x] = 0.0;
    int lsA = SA->pw[0][0] + SA->pw[0][1] + SA->pw[0][2];
    int lsB = SB->pw[0][0] + SB->pw[0][1] + SB->pw[0][2];
    int lsC = SC->pw[0][0] + SC->pw[0][1] + SC->pw[0][2];
    int lsD = SD->pw[0][0] + SD->pw[0][1] + SD->pw[0][2];
    int ME = (lsA + lsB > lsC + lsD) ? lsA + lsB : lsC + lsD;
    int NN = lsA + lsB + lsC + lsD;
    int ncomb = (lsA + 1) * (lsB + 1) * (lsC + 1) * (lsD + 1);
    const double *av = c->a, *Lc = c->L;
    const double *rA = SA->r, *rB = SB->r, *rC = SC->r, *rD = SD->r;
    double fac_const = 2.0 / sqrt(PI_D);
    for (int d = 0; d < ndp; ++d) fac_const *= Lc[d] * Lc[d];
    int n1 = SA->np, n2 = SB->np, n3 = SC->np, n4 = SD->np, nket = n3 * n4;
    int nw = c->ncap + ME + 2;
    int NE = NMC + 1;

    double *k_fac = malloc(sizeof(double) * nket), *k_cen = malloc(sizeof(double) * 3 * nket);
    double *k_q = malloc(sizeof(double) * nket);
    int *k_N = malloc(sizeof(int) * 3 * nket), *k_off = malloc(sizeof(int) * 3 * nket);
    double *k_E = calloc((size_t)NE * (lsC + 1) * (lsD + 1) * 3 * nket, sizeof(double));
#define KE(t, ic, id, d, kl) k_E[(t) + NE * ((ic) + (lsC + 1) * ((id) + (lsD + 1) * ((d) + 3 * (kl))))]
    double b_cen[3]; int b_N[3];
    double *b_E = calloc((size_t)NE * (lsA + 1) * (lsB + 1) * 3, sizeof(double));
#define BE(t, ia, ib, d) b_E[(t) + NE * ((ia) + (lsA + 1) * ((ib) + (lsB + 1) * (d)))]
    double *F = malloc(sizeof(double) * (nw + 1));
    size_t gsz = (size_t)(nw + 1) * (lsA + 1) * (lsB + 1) * (ndp > 0 ? ndp : 1);
    double *Gre = calloc(gsz, sizeof(double)), *Gim = calloc(gsz, sizeof(double));
#define GI(n, ia, ib, d) ((size_t)(n) + (size_t)(nw + 1) * ((ia) + (lsA + 1) * ((ib) + (lsB + 1) * (size_t)(d))))
    double *Idir = calloc((size_t)nq * ncomb * 3, sizeof(double));
#define ID(kq, cmb, d) Idir[(kq) + nq * ((cmb) + ncomb * (d))]
    double SNv[4 * NMC + 1];
    double *gt = malloc(sizeof(double) * (NN + 1) * nq);
    double *cph = malloc(sizeof(double) * (nw + 1)), *sph = malloc(sizeof(double) * (nw + 1));
    double *rD2 = malloc(sizeof(double) * nq), *rw = malloc(sizeof(double) * nq), *rs = malloc(sizeof(double) * nq);
    double *Iacc = malloc(sizeof(double) * nq);

    /* ---------------- ket pairs (:133-164) ---------------- */
    int kl = 0, off = 0;
    double ket_max = 0.0;
    for (int k = 0; k < n3; ++k)
        for (int l = 0; l < n4; ++l, ++kl) {
            double e1 = SC->e[k], e2 = SD->e[l], esum = e1 + e2;
            /* two exponent-0 functions (density-fitting dummies, df_toroidal.f90:837)
               are never paired by the reference: zero weight, no division by 0 */
            int nil = !(esum > 0.0);
            double mu = nil ? 0.0 : e1 * e2 / esum;
            k_q[kl] = esum;
            double cf = 1.0, pe, cen;
            for (int d = 0; d < 3; ++d) {
                if (d < ndp) {
                    orc_bary(e1, e2, rC[d], rD[d], Lc[d], av[d], &pe, &cen);
                    k_cen[d + 3 * kl] = cen;
                    cf *= exp(-2.0 * (esum - pe) / (av[d] * av[d]));
                    int est = orc_bessel_nmax_estimate(2.0 * pe / (av[d] * av[d]));
                    k_N[d + 3 * kl] = est < nw - ME - 2 ? est : nw - ME - 2;
                    k_off[d + 3 * kl] = off;
                    off += (k_N[d + 3 * kl] + 1) * (lsC + 1) * (lsD + 1);
                } else {
                    cen = nil ? rC[d] : (e1 * rC[d] + e2 * rD[d]) / esum;
                    k_cen[d + 3 * kl] = cen;
                    cf *= exp(-mu * (rC[d] - rD[d]) * (rC[d] - rD[d]));
                    for (int ic = 0; ic <= lsC; ++ic)
                        for (int id = 0; id <= lsD; ++id) {
                            if (nil) {
                                for (int t = 0; t <= 16; ++t) (&KE(0, ic, id, d, kl))[t] = 0.0;
                            } else {
                                orc_hermite_E_1D(ic, id, esum, cen - rC[d], cen - rD[d], &KE(0, ic, id, d, kl));
                            }
                        }
                }
            }
            if (nil) cf = 0.0;
            k_fac[kl] = cf;
            double mc = 0.0, md = 0.0;
            for (int x = 0; x < nC; ++x) if (fabs(SC->c[x][k]) > mc) mc = fabs(SC->c[x][k]);
            for (int x = 0; x < nD; ++x) if (fabs(SD->c[x][l]) > md) md = fabs(SD->c[x][l]);
            double v = fabs(cf) * mc * md;
            if (v > ket_max) ket_max = v;
        }
    size_t hsz = off > 1 ? (size_t)off : 1;
    double *Hre = calloc(hsz, sizeof(double)), *Him = calloc(hsz, sizeof(double));
    char *k_done = calloc((size_t)nket, 1);

    /* ---------------- bra pairs / quartets (:170-364) ---------------- */
    for (int i = 0; i < n1; ++i)
        for (int j = 0; j < n2; ++j) {
            double e1 = SA->e[i], e2 = SB->e[j], esum = e1 + e2, p = esum;
            int bnil = !(esum > 0.0);                  /* two exponent-0 dummies: never paired */
            double mu = bnil ? 0.0 : e1 * e2 / esum;
            double cAmax = 0.0, cBmax = 0.0;
            for (int x = 0; x < nA; ++x) if (fabs(SA->c[x][i]) > cAmax) cAmax = fabs(SA->c[x][i]);
            for (int x = 0; x < nB; ++x) if (fabs(SB->c[x][j]) > cBmax) cBmax = fabs(SB->c[x][j]);
            double bra_fac = fac_const, pe, cen, Aarg;
            for (int d = 0; d < 3; ++d) {
                if (d < ndp) {
                    orc_bary(e1, e2, rA[d], rB[d], Lc[d], av[d], &pe, &cen);
                    b_cen[d] = cen;
                    bra_fac *= exp(-2.0 * (esum - pe) / (av[d] * av[d]));
                    Aarg = 2.0 * pe / (av[d] * av[d]);
                    int est = orc_bessel_nmax_estimate(Aarg);
                    b_N[d] = est < nw - ME - 2 ? est : nw - ME - 2;
                } else {
                    cen = bnil ? rA[d] : (e1 * rA[d] + e2 * rB[d]) / esum;
                    b_cen[d] = cen;
                    bra_fac *= exp(-mu * (rA[d] - rB[d]) * (rA[d] - rB[d]));
                }
            }
            if (bnil) continue;
            if (!ps_noscreen && fabs(bra_fac) * cAmax * cBmax * ket_max <= screen_tol) continue;

            for (int d = 0; d < 3; ++d) {
                if (d < ndp) {
                    orc_bary(e1, e2, rA[d], rB[d], Lc[d], av[d], &pe, &cen);
                    Aarg = 2.0 * pe / (av[d] * av[d]);
                    for (int ia = 0; ia <= lsA; ++ia)
                        for (int ib = 0; ib <= lsB; ++ib)
                            PAIR_VECTOR(b_N[d], Aarg, ia, ib, av[d] * (cen - rA[d]), av[d] * (cen - rB[d]), -1,
                                            &Gre[GI(0, ia, ib, d)], &Gim[GI(0, ia, ib, d)]);
                } else {
                    for (int ia = 0; ia <= lsA; ++ia)
                        for (int ib = 0; ib <= lsB; ++ib)
                            orc_hermite_E_1D(ia, ib, p, b_cen[d] - rA[d], b_cen[d] - rB[d], &BE(0, ia, ib, d));
                }
            }

            kl = 0;
            for (int k = 0; k < n3; ++k)
                for (int l = 0; l < n4; ++l, ++kl) {
                    double fac = bra_fac * k_fac[kl];
                    double mc = 0.0, md = 0.0;
                    for (int x = 0; x < nC; ++x) if (fabs(SC->c[x][k]) > mc) mc = fabs(SC->c[x][k]);
                    for (int x = 0; x < nD; ++x) if (fabs(SD->c[x][l]) > md) md = fabs(SD->c[x][l]);
                    if (!ps_noscreen && fabs(fac) * cAmax * cBmax * mc * md <= screen_tol) continue;
                    if (ps_bra && ps_ket)
                        if (ps_bra[i + mp * j] * ps_ket[k + mp * l] < c->s.prim_thr) continue;
                    double q = k_q[kl];
                    if (!k_done[kl]) { /* build_ket :371-388 */
                        double f1 = SC->e[k], f2 = SD->e[l], kpe, kcen;
                        for (int d = 0; d < ndp; ++d) {
                            orc_bary(f1, f2, rC[d], rD[d], Lc[d], av[d], &kpe, &kcen);
                            double KA = 2.0 * kpe / (av[d] * av[d]);
                            int kN = k_N[d + 3 * kl];
                            for (int ic = 0; ic <= lsC; ++ic)
                                for (int id = 0; id <= lsD; ++id) {
                                    size_t o = (size_t)k_off[d + 3 * kl] + (size_t)(kN + 1) * (ic + (lsC + 1) * id);
                                    PAIR_VECTOR(kN, KA, ic, id, av[d] * (kcen - rC[d]), av[d] * (kcen - rD[d]), 1,
                                                    &Hre[o], &Him[o]);
                                }
                        }
                        k_done[kl] = 1;
                    }
                    /* ---- 1D factors for every power combination (:227-337) ---- */
                    if (ndp < 3)
                        for (int kq = 0; kq < nq; ++kq) {
                            double t2 = c->t_node[kq] * c->t_node[kq];
                            double D2 = 1.0 / (p * q + (p + q) * t2);
                            rD2[kq] = D2;
                            rw[kq] = p * q * t2 * D2;
                            rs[kq] = PI_D * sqrt(D2);
                        }
                    for (int d = 0; d < 3; ++d) {
                        if (d < ndp) {
                            int kN = k_N[d + 3 * kl];
                            int nm = b_N[d] < kN ? b_N[d] : kN;
                            double phi = av[d] * (b_cen[d] - k_cen[d + 3 * kl]);
                            double c1 = cos(phi), s1 = sin(phi), cn = 1.0, sn = 0.0, tmp;
                            for (int n = 0; n <= nm; ++n) {
                                if (n > 0) {
                                    if (n % 32 == 0) { cn = cos(n * phi); sn = sin(n * phi); }
                                    else { tmp = cn * c1 - sn * s1; sn = sn * c1 + cn * s1; cn = tmp; }
                                }
                                cph[n] = cn; sph[n] = sn;
                            }
                            for (int id = 0; id <= lsD; ++id)
                                for (int ic = 0; ic <= lsC; ++ic)
                                    for (int ib = 0; ib <= lsB; ++ib)
                                        for (int ia = 0; ia <= lsA; ++ia) {
                                            int cmb = ia + (lsA + 1) * (ib + (lsB + 1) * (ic + (lsC + 1) * id));
                                            size_t ho = (size_t)k_off[d + 3 * kl] + (size_t)(kN + 1) * (ic + (lsC + 1) * id);
                                            for (int n = 0; n <= nm; ++n) {
                                                double gr = Gre[GI(n, ia, ib, d)], gi = Gim[GI(n, ia, ib, d)];
                                                double hr = Hre[ho + n], hi = Him[ho + n];
                                                double ar = gr * hr - gi * hi, ai = gr * hi + gi * hr;
                                                F[n] = ar * cph[n] - ai * sph[n];
                                            }
                                            double sgn = pow(av[d], -(ia + ib + ic + id));
                                            if (ndp == 1) {
                                                for (int kq = 0; kq < nq; ++kq) {
                                                    int tn = c->t_nmax[kq + nq * d];
                                                    int nt = nm < tn ? nm : tn;
                                                    double val = F[0] * TB(c, 0, kq, d), dot = 0.0;
                                                    for (int n = 1; n <= nt; ++n) dot += F[n] * TB(c, n, kq, d);
                                                    if (nt >= 1) val += 2.0 * dot;
                                                    ID(kq, cmb, d) = val * sgn;
                                                }
                                            } else {
                                                int ne = nm < c->t_nmaxall[d] ? nm : c->t_nmaxall[d];
                                                double Fmx = 0.0;
                                                for (int n = 0; n <= ne; ++n) if (fabs(F[n]) > Fmx) Fmx = fabs(F[n]);
                                                while (ne > 0) { if (fabs(F[ne]) >= 1e-17 * Fmx) break; --ne; }
                                                int ns = ne < c->t_nsplit[d] ? ne : c->t_nsplit[d];
                                                for (int kq = 0; kq < nq; ++kq) Iacc[kq] = F[0] * TBT(c, kq, 0, d);
                                                for (int n = 1; n <= ns; ++n) {
                                                    int k0 = c->t_kfirst[n + (c->ncap + 1) * d];
                                                    for (int kq = k0; kq < nq; ++kq) Iacc[kq] += F[n] * TBT(c, kq, n, d);
                                                }
                                                if (ne > ns) {
                                                    for (int kq = c->t_kfirst[ns + 1 + (c->ncap + 1) * d]; kq < nq; ++kq) {
                                                        int tn = c->t_nmax[kq + nq * d];
                                                        int nt = ne < tn ? ne : tn;
                                                        if (nt > ns) {
                                                            double dot = 0.0;
                                                            for (int n = ns + 1; n <= nt; ++n) dot += F[n] * TB(c, n, kq, d);
                                                            Iacc[kq] += 2.0 * dot;
                                                        }
                                                    }
                                                }
                                                for (int kq = 0; kq < nq; ++kq) ID(kq, cmb, d) = Iacc[kq] * sgn;
                                            }
                                        }
                        } else {
                            double Rr = b_cen[d] - k_cen[d + 3 * kl];
                            for (int kq = 0; kq < nq; ++kq) {
                                double w = rw[kq];
                                gt[0 + (NN + 1) * kq] = (Rr == 0.0) ? rs[kq] : rs[kq] * exp(-w * Rr * Rr);
                                double gm1 = 0.0, g0 = gt[(NN + 1) * kq], gp1;
                                for (int n = 0; n <= NN - 1; ++n) {
                                    gp1 = 2.0 * w * Rr * g0 - 2.0 * (double)n * w * gm1;
                                    gt[n + 1 + (NN + 1) * kq] = gp1;
                                    gm1 = g0; g0 = gp1;
                                }
                            }
                            for (int id = 0; id <= lsD; ++id)
                                for (int ic = 0; ic <= lsC; ++ic)
                                    for (int ib = 0; ib <= lsB; ++ib)
                                        for (int ia = 0; ia <= lsA; ++ia) {
                                            int cmb = ia + (lsA + 1) * (ib + (lsB + 1) * (ic + (lsC + 1) * id));
                                            for (int x = 0; x <= NN; ++x) SNv[x] = 0.0;
                                            for (int n = 0; n <= ia + ib; ++n)
                                                for (int kk = 0; kk <= ic + id; ++kk)
                                                    SNv[n + kk] += ((n % 2 == 1) ? -1.0 : 1.0) * BE(n, ia, ib, d) * KE(kk, ic, id, d, kl);
                                            int tot = ia + ib + ic + id;
                                            for (int kq = 0; kq < nq; ++kq) {
                                                double s = 0.0;
                                                for (int x = 0; x <= tot; ++x) s += SNv[x] * gt[x + (NN + 1) * kq];
                                                ID(kq, cmb, d) = s;
                                            }
                                        }
                        }
                    }
                    for (int cmb = 0; cmb < ncomb; ++cmb)
                        for (int kq = 0; kq < nq; ++kq) ID(kq, cmb, 0) *= c->t_weight[kq];

                    /* ---- all component quartets (:343-359) ---- */
                    for (int cd = 0; cd < nD; ++cd)
                        for (int cc = 0; cc < nC; ++cc)
                            for (int cb = 0; cb < nB; ++cb)
                                for (int ca = 0; ca < nA; ++ca) {
                                    int cx = SA->pw[ca][0] + (lsA + 1) * (SB->pw[cb][0] + (lsB + 1) * (SC->pw[cc][0] + (lsC + 1) * SD->pw[cd][0]));
                                    int cy = SA->pw[ca][1] + (lsA + 1) * (SB->pw[cb][1] + (lsB + 1) * (SC->pw[cc][1] + (lsC + 1) * SD->pw[cd][1]));
                                    int cz = SA->pw[ca][2] + (lsA + 1) * (SB->pw[cb][2] + (lsB + 1) * (SC->pw[cc][2] + (lsC + 1) * SD->pw[cd][2]));
                                    double val = 0.0;
                                    for (int kq = 0; kq < nq; ++kq) val += ID(kq, cx, 0) * ID(kq, cy, 1) * ID(kq, cz, 2);
                                    blk[ca + nA * (cb + nB * (cc + nC * cd))] +=
                                        fac * SA->c[ca][i] * SB->c[cb][j] * SC->c[cc][k] * SD->c[cd][l] * val;
                                }
                }
        }
#undef KE
#undef BE
#undef GI
#undef ID
    free(k_fac); free(k_cen); free(k_q); free(k_N); free(k_off); free(k_E); free(b_E); free(F);
    free(Gre); free(Gim); free(Idir); free(gt); free(cph); free(sph); free(rD2); free(rw); free(rs);
    free(Iacc); free(Hre); free(Him); free(k_done);
}

/* ---- lattice helpers (ERI_toroidal.f90:142-156, :591-634) ---- */
static int mod_pos(int a, int m) { int r = a % m; return r < 0 ? r + m : r; }

static void translate_to_unit_cell(int p[4], int nblk, const int ncl[3]) /* :591-609, 0-based */
{
    int c = p[0] / nblk;
    int tx = c % ncl[0], ty = (c / ncl[0]) % ncl[1], tz = c / (ncl[0] * ncl[1]);
    for (int ii = 0; ii < 4; ++ii) {
        int cc = p[ii] / nblk, loc = p[ii] % nblk;
        int cx = mod_pos(cc % ncl[0] - tx, ncl[0]);
        int cy = mod_pos((cc / ncl[0]) % ncl[1] - ty, ncl[1]);
        int cz = mod_pos(cc / (ncl[0] * ncl[1]) - tz, ncl[2]);
        p[ii] = (cx + ncl[0] * (cy + ncl[1] * cz)) * nblk + loc;
    }
}

static const int iperm8[8][4] = {{0,1,2,3},{1,0,2,3},{0,1,3,2},{1,0,3,2},{2,3,0,1},{3,2,0,1},{2,3,1,0},{3,2,1,0}};

static int is_canonical(const orc_ctx *c, const int q4[4]) /* :356-373 (== canonical_quartet_toroidal) */
{
    int t4[4], r4[4];
    for (int ip = 1; ip < 8; ++ip) {
        for (int ii = 0; ii < 4; ++ii) t4[ii] = q4[iperm8[ip][ii]];
        for (int ii = 0; ii < 4; ++ii) r4[ii] = t4[ii];
        translate_to_unit_cell(r4, c->nshuc, c->ncl);
        for (int ii = 0; ii < 4; ++ii) {
            if (r4[ii] < q4[ii]) return 0;
            if (r4[ii] > q4[ii]) break;
        }
    }
    return 1;
}

static void shell_view(const orc_ctx *c, int S, shellv *v) { make_shell(c, c->sh_first[S], c->sh_n[S], v); }

static const double *ket_table(const orc_ctx *c, int SK, int SL) /* set_ps eri_direct.f90:249-257 */
{
    int ab[4] = {SK, SL, SK, SK};
    translate_to_unit_cell(ab, c->nshuc, c->ncl);
    return c->ps_qp + (size_t)c->mp * c->mp * ((size_t)ab[0] + (size_t)c->nshuc * ab[1]);
}

void orc_shell_block(orc_ctx *c, int S1, int S2, int S3, int S4, int mode, double *blk)
{
    shellv *v = malloc(4 * sizeof(shellv));
    shell_view(c, S1, &v[0]); shell_view(c, S2, &v[1]); shell_view(c, S3, &v[2]); shell_view(c, S4, &v[3]);
    const double *pb = NULL, *pk = NULL;
    if (mode == 1 && c->ps_qp && S1 < c->nshuc) {
        pb = c->ps_qp + (size_t)c->mp * c->mp * ((size_t)S1 + (size_t)c->nshuc * S2);
        pk = ket_table(c, S3, S4);
    }
    shell_block(c, &v[0], &v[1], &v[2], &v[3], mode == 2, pb, pk, c->mp, blk);
    free(v);
}

/* Blocks of n shell quartets (items4[4*i..4*i+3]), concatenated in item order,
 * each column-major as orc_shell_block; OpenMP over the quartets.  Returns the
 * number of doubles written. */
int64_t orc_shell_blocks(orc_ctx *c, int64_t n, const int32_t *items4, int mode, double *out)
{
    int64_t *off = malloc(sizeof(int64_t) * (size_t)(n + 1));
    off[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        const int32_t *q = items4 + 4 * i;
        off[i + 1] = off[i] + (int64_t)c->sh_n[q[0]] * c->sh_n[q[1]] * c->sh_n[q[2]] * c->sh_n[q[3]];
    }
    #pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < n; ++i) {
        const int32_t *q = items4 + 4 * i;
        orc_shell_block(c, q[0], q[1], q[2], q[3], mode, out + off[i]);
    }
    int64_t tot = off[n];
    free(off);
    return tot;
}

orc_ctx *orc_create(const orc_system *sys)
{
    init_clifford();
    orc_ctx *c = calloc(1, sizeof(orc_ctx));
    c->s = *sys;
    int nbas = c->nbas = sys->nbas, nfuc = c->nfuc = sys->nfuc, ndp = c->ndp = sys->ndp;
    for (int d = 0; d < 3; ++d) { c->L[d] = sys->L[d]; c->a[d] = (sys->L[d] > 0) ? 2.0 * PI_D / sys->L[d] : 0.0; }
    int np = sys->prim_off[nbas];
    c->ctr = malloc(sizeof(double) * 3 * nbas); memcpy(c->ctr, sys->ctr, sizeof(double) * 3 * nbas);
    c->lxyz = malloc(sizeof(int32_t) * 3 * nbas); memcpy(c->lxyz, sys->lxyz, sizeof(int32_t) * 3 * nbas);
    c->poff = malloc(sizeof(int32_t) * (nbas + 1)); memcpy(c->poff, sys->prim_off, sizeof(int32_t) * (nbas + 1));
    c->exps = malloc(sizeof(double) * np); memcpy(c->exps, sys->exps, sizeof(double) * np);
    c->coefs = malloc(sizeof(double) * np); memcpy(c->coefs, sys->coefs, sizeof(double) * np);

    /* t-table size (ERI_toroidal.f90:93-104) */
    int lmax = 0; double emax = 0.0;
    for (int f = 0; f < nbas; ++f) {
        for (int d = 0; d < ndp; ++d) if (c->lxyz[3 * f + d] > lmax) lmax = c->lxyz[3 * f + d];
        for (int p = c->poff[f]; p < c->poff[f + 1]; ++p) if (c->exps[p] > emax) emax = c->exps[p];
    }
    double amin = c->a[0];
    for (int d = 1; d < ndp; ++d) if (c->a[d] < amin) amin = c->a[d];
    c->ncap = orc_bessel_nmax_estimate(4.0 * emax / (amin * amin)) + 2 * lmax + 1;
    c->nq = sys->nquad;
    c->t_node = malloc(sizeof(double) * c->nq); c->t_weight = malloc(sizeof(double) * c->nq);
    if (sys->t_nodes) {
        memcpy(c->t_node, sys->t_nodes, sizeof(double) * c->nq);
        memcpy(c->t_weight, sys->t_weights, sizeof(double) * c->nq);
    } else orc_fast_quad_points(c->nq, c->t_node, c->t_weight);
    setup_t_tables(c);

    /* shells (:106-125) */
    c->sh_first = malloc(sizeof(int) * nbas); c->sh_n = malloc(sizeof(int) * nbas);
    int nsh = 0;
    for (int i = 0; i < nbas;) {
        int lt = c->lxyz[3 * i] + c->lxyz[3 * i + 1] + c->lxyz[3 * i + 2];
        int ncomp = (lt + 1) * (lt + 2) / 2;
        int same = (i + ncomp - 1 <= nbas - 1);
        if (same)
            for (int j = i + 1; j <= i + ncomp - 1; ++j) {
                int lj = c->lxyz[3 * j] + c->lxyz[3 * j + 1] + c->lxyz[3 * j + 2];
                int npj = c->poff[j + 1] - c->poff[j], npi = c->poff[i + 1] - c->poff[i];
                same = same && lj == lt && c->ctr[3 * j] == c->ctr[3 * i] && c->ctr[3 * j + 1] == c->ctr[3 * i + 1] &&
                       c->ctr[3 * j + 2] == c->ctr[3 * i + 2] && npj == npi;
                if (same)
                    for (int p = 0; p < npi; ++p) same = same && c->exps[c->poff[j] + p] == c->exps[c->poff[i] + p];
            }
        if (!same) ncomp = 1;
        c->sh_first[nsh] = i; c->sh_n[nsh] = ncomp; ++nsh;
        i += ncomp;
    }
    c->nsh = nsh;
    for (int d = 0; d < 3; ++d) c->ncl[d] = sys->ncell[d] > 1 ? sys->ncell[d] : 1;
    c->ncell = c->ncl[0] * c->ncl[1] * c->ncl[2];
    c->nshuc = 0;
    for (int S = 0; S < nsh; ++S) if (c->sh_first[S] < nfuc) ++c->nshuc;
    c->sym_ok = (nsh == c->nshuc * c->ncell) && (nbas == nfuc * c->ncell);
    if (c->sym_ok)
        for (int S = 0; S < nsh - c->nshuc; ++S)
            if (c->sh_n[S + c->nshuc] != c->sh_n[S] || c->sh_first[S + c->nshuc] != c->sh_first[S] + nfuc) c->sym_ok = 0;

    /* Schwarz (:200-236), sym_ok: SI in unit cell + lattice shifts */
    c->Q = calloc((size_t)nbas * nbas, sizeof(double));
    c->Qsh = calloc((size_t)nsh * nsh, sizeof(double));
    int nshuc = c->nshuc;
    if (c->sym_ok) {
        #pragma omp parallel for schedule(dynamic, 1) collapse(2)
        for (int SI = 0; SI < nshuc; ++SI)
            for (int SJ = 0; SJ < nsh; ++SJ) {
                int ni = c->sh_n[SI], nj = c->sh_n[SJ];
                double *blk = malloc(sizeof(double) * ni * nj * ni * nj);
                orc_shell_block(c, SI, SJ, SI, SJ, 0, blk);
                for (int a = 0; a < ni; ++a)
                    for (int b = 0; b < nj; ++b) {
                        int i = c->sh_first[SI] + a, j = c->sh_first[SJ] + b;
                        double qv = sqrt(fabs(blk[a + ni * (b + nj * (a + ni * b))]));
                        for (int ct = 0; ct < c->ncell; ++ct) {
                            int p[4] = {i, j, i, i};
                            /* shift both by the lattice vector of cell ct (shift_cell eri_direct.f90:228-236) */
                            int cx = ct % c->ncl[0], cy = (ct / c->ncl[0]) % c->ncl[1], cz = ct / (c->ncl[0] * c->ncl[1]);
                            for (int u = 0; u < 2; ++u) {
                                int cc = p[u] / nfuc, loc = p[u] % nfuc;
                                int x = mod_pos(cc % c->ncl[0] + cx, c->ncl[0]);
                                int y = mod_pos((cc / c->ncl[0]) % c->ncl[1] + cy, c->ncl[1]);
                                int z = mod_pos(cc / (c->ncl[0] * c->ncl[1]) + cz, c->ncl[2]);
                                p[u] = (x + c->ncl[0] * (y + c->ncl[1] * z)) * nfuc + loc;
                            }
                            c->Q[p[0] + (size_t)nbas * p[1]] = qv;
                            c->Q[p[1] + (size_t)nbas * p[0]] = qv;
                        }
                    }
                free(blk);
            }
    } else {
        #pragma omp parallel for schedule(dynamic, 1)
        for (int SI = 0; SI < nsh; ++SI)
            for (int SJ = SI; SJ < nsh; ++SJ) {
                int ni = c->sh_n[SI], nj = c->sh_n[SJ];
                double *blk = malloc(sizeof(double) * ni * nj * ni * nj);
                orc_shell_block(c, SI, SJ, SI, SJ, 0, blk);
                for (int a = 0; a < ni; ++a)
                    for (int b = 0; b < nj; ++b) {
                        int i = c->sh_first[SI] + a, j = c->sh_first[SJ] + b;
                        double qv = sqrt(fabs(blk[a + ni * (b + nj * (a + ni * b))]));
                        c->Q[i + (size_t)nbas * j] = qv; c->Q[j + (size_t)nbas * i] = qv;
                    }
                free(blk);
            }
    }
    c->Qmax = 0.0;
    for (int SI = 0; SI < nsh; ++SI)
        for (int SJ = 0; SJ < nsh; ++SJ) {
            double m = 0.0;
            for (int a = 0; a < c->sh_n[SI]; ++a)
                for (int b = 0; b < c->sh_n[SJ]; ++b) {
                    double v = c->Q[(c->sh_first[SI] + a) + (size_t)nbas * (c->sh_first[SJ] + b)];
                    if (v > m) m = v;
                }
            c->Qsh[SI + (size_t)nsh * SJ] = m;
            if (m > c->Qmax) c->Qmax = m;
        }

    /* primitive Schwarz table (:296-337), sym_ok only, prim_screen */
    c->mp = 0; c->ps_qp = NULL;
    if (c->sym_ok && sys->prim_screen) {
        int mp = 0;
        for (int S = 0; S < nsh; ++S) { int n = c->poff[c->sh_first[S] + 1] - c->poff[c->sh_first[S]]; if (n > mp) mp = n; }
        c->mp = mp;
        c->ps_qp = calloc((size_t)mp * mp * nshuc * nsh, sizeof(double));
        #pragma omp parallel for schedule(dynamic, 1) collapse(2)
        for (int SI = 0; SI < nshuc; ++SI)
            for (int SJ = 0; SJ < nsh; ++SJ) {
                shellv *v = malloc(4 * sizeof(shellv));
                shell_view(c, SI, &v[0]); shell_view(c, SJ, &v[1]);
                int ni = v[0].n, nj = v[1].n;
                double *blk = malloc(sizeof(double) * ni * nj * ni * nj);
                double *dst = c->ps_qp + (size_t)mp * mp * ((size_t)SI + (size_t)nshuc * SJ);
                for (int p1 = 0; p1 < v[0].np; ++p1)
                    for (int p2 = 0; p2 < v[1].np; ++p2) {
                        single_prim(&v[0], p1, &v[2]); single_prim(&v[1], p2, &v[3]);
                        shell_block(c, &v[2], &v[3], &v[2], &v[3], 1, NULL, NULL, mp, blk);
                        for (int a = 0; a < ni; ++a)
                            for (int b = 0; b < nj; ++b) {
                                double q = sqrt(fabs(blk[a + ni * (b + nj * (a + ni * b))]));
                                if (q > dst[p1 + mp * p2]) dst[p1 + mp * p2] = q;
                            }
                    }
                free(blk); free(v);
            }
    }

    if (c->sym_ok) { /* cell tables for the scatter */
        c->fcell = malloc(sizeof(int) * nbas); c->floc = malloc(sizeof(int) * nbas);
        for (int i = 0; i < nbas; ++i) { c->fcell[i] = i / nfuc; c->floc[i] = i % nfuc; }
    }
    return c;
}

void orc_destroy(orc_ctx *c)
{
    if (!c) return;
    free(c->ctr); free(c->lxyz); free(c->poff); free(c->exps); free(c->coefs);
    free(c->t_node); free(c->t_weight); free(c->t_bessel); free(c->t_bt); free(c->t_nmax); free(c->t_kfirst);
    free(c->sh_first); free(c->sh_n); free(c->Q); free(c->Qsh); free(c->ps_qp); free(c->fcell); free(c->floc);
    free(c);
}

int orc_nshells(const orc_ctx *c, int *nshuc, int *ncap) { if (nshuc) *nshuc = c->nshuc; if (ncap) *ncap = c->ncap; return c->nsh; }
void orc_shell_info(const orc_ctx *c, int s, int *first, int *n) { *first = c->sh_first[s]; *n = c->sh_n[s]; }
const double *orc_schwarz(const orc_ctx *c) { return c->Q; }
const double *orc_schwarz_shell(const orc_ctx *c) { return c->Qsh; }
const double *orc_prim_table(const orc_ctx *c, int *mp) { if (mp) *mp = c->mp; return c->ps_qp; }
void orc_t_tables(const orc_ctx *c, const double **node, const double **weight, const double **tb, const int **tn)
{ *node = c->t_node; *weight = c->t_weight; *tb = c->t_bessel; *tn = c->t_nmax; }

/* ---- stored ERIs: ERI_toroidal.f90:240-548 ---- */
int64_t orc_eri_stored(orc_ctx *c, double *eri)
{
    const double thr = c->s.schwarz_thr;
    int nbas = c->nbas, nfuc = c->nfuc, nsh = c->nsh, nshuc = c->nshuc;
    int esz = c->s.sao ? nfuc : nbas;
    size_t total = (size_t)esz * nbas * nbas * nbas;
    memset(eri, 0, total * sizeof(double));
    int64_t nq = 0;
    int phys = c->s.physicist;
#define EIDX(a, b, cc, d) ((size_t)(a) + (size_t)esz * ((size_t)(b) + (size_t)nbas * ((size_t)(cc) + (size_t)nbas * (size_t)(d))))
    if (c->sym_ok) {
        #pragma omp parallel for schedule(dynamic, 1) collapse(2) reduction(+ : nq)
        for (int SI = 0; SI < nshuc; ++SI)
            for (int SJ = 0; SJ < nsh; ++SJ) {
                if (SJ % nshuc < SI) continue;
                if (c->Qsh[SI + (size_t)nsh * SJ] * c->Qmax < thr) continue;
                for (int SK = 0; SK < nsh; ++SK) {
                    if (SK % nshuc < SI) continue;
                    for (int SL = 0; SL < nsh; ++SL) {
                        if (SL % nshuc < SI) continue;
                        if (c->Qsh[SI + (size_t)nsh * SJ] * c->Qsh[SK + (size_t)nsh * SL] < thr) continue;
                        int q4[4] = {SI, SJ, SK, SL};
                        if (!is_canonical(c, q4)) continue;
                        ++nq;
                        int n1 = c->sh_n[SI], n2 = c->sh_n[SJ], n3 = c->sh_n[SK], n4 = c->sh_n[SL];
                        double *blk = malloc(sizeof(double) * n1 * n2 * n3 * n4);
                        orc_shell_block(c, SI, SJ, SK, SL, c->ps_qp ? 1 : 0, blk);
                        for (int d = 0; d < n4; ++d)
                            for (int cc = 0; cc < n3; ++cc)
                                for (int b = 0; b < n2; ++b)
                                    for (int a = 0; a < n1; ++a) {
                                        int f[4] = {c->sh_first[SI] + a, c->sh_first[SJ] + b, c->sh_first[SK] + cc, c->sh_first[SL] + d};
                                        if (c->Q[f[0] + (size_t)nbas * f[1]] * c->Q[f[2] + (size_t)nbas * f[3]] < thr) continue;
                                        double val = blk[a + n1 * (b + n2 * (cc + n3 * d))];
                                        for (int ip = 0; ip < 8; ++ip) {
                                            int pp[4];
                                            for (int ii = 0; ii < 4; ++ii) pp[ii] = f[iperm8[ip][ii]];
                                            translate_to_unit_cell(pp, nfuc, c->ncl);
                                            if (phys) eri[EIDX(pp[0], pp[2], pp[1], pp[3])] = val;
                                            else eri[EIDX(pp[0], pp[1], pp[2], pp[3])] = val;
                                        }
                                    }
                        free(blk);
                    }
                }
            }
    } else { /* :473-546 */
        for (int SI = 0; SI < nsh; ++SI) {
            if (c->sh_first[SI] >= nfuc) continue;
            #pragma omp parallel for schedule(dynamic, 1) reduction(+ : nq)
            for (int SJ = SI; SJ < nsh; ++SJ)
                for (int SK = 0; SK < nsh; ++SK) {
                    if (c->sh_first[SI] > c->sh_first[SK] + c->sh_n[SK] - 1) continue;
                    for (int SL = SK; SL < nsh; ++SL) {
                        if (c->Qsh[SI + (size_t)nsh * SJ] * c->Qsh[SK + (size_t)nsh * SL] < thr) continue;
                        ++nq;
                        int n1 = c->sh_n[SI], n2 = c->sh_n[SJ], n3 = c->sh_n[SK], n4 = c->sh_n[SL];
                        double *blk = malloc(sizeof(double) * n1 * n2 * n3 * n4);
                        orc_shell_block(c, SI, SJ, SK, SL, 0, blk);
                        for (int d = 0; d < n4; ++d)
                            for (int cc = 0; cc < n3; ++cc)
                                for (int b = 0; b < n2; ++b)
                                    for (int a = 0; a < n1; ++a) {
                                        int i = c->sh_first[SI] + a, j = c->sh_first[SJ] + b, k = c->sh_first[SK] + cc, l = c->sh_first[SL] + d;
                                        if (i >= nfuc || j < i || l < k || i > k) continue;
                                        if (c->Q[i + (size_t)nbas * j] * c->Q[k + (size_t)nbas * l] < thr) continue;
                                        double val = blk[a + n1 * (b + n2 * (cc + n3 * d))];
                                        if (phys) {
                                            if (i < nfuc) eri[EIDX(i, k, j, l)] = val;
                                            if (j < nfuc) eri[EIDX(j, k, i, l)] = val;
                                            if (i < nfuc) eri[EIDX(i, l, j, k)] = val;
                                            if (j < nfuc) eri[EIDX(j, l, i, k)] = val;
                                            if (k < nfuc) eri[EIDX(k, i, l, j)] = val;
                                            if (l < nfuc) eri[EIDX(l, i, k, j)] = val;
                                            if (k < nfuc) eri[EIDX(k, j, l, i)] = val;
                                            if (l < nfuc) eri[EIDX(l, j, k, i)] = val;
                                        } else {
                                            if (i < nfuc) eri[EIDX(i, j, k, l)] = val;
                                            if (j < nfuc) eri[EIDX(j, i, k, l)] = val;
                                            if (i < nfuc) eri[EIDX(i, j, l, k)] = val;
                                            if (j < nfuc) eri[EIDX(j, i, l, k)] = val;
                                            if (k < nfuc) eri[EIDX(k, l, i, j)] = val;
                                            if (l < nfuc) eri[EIDX(l, k, i, j)] = val;
                                            if (k < nfuc) eri[EIDX(k, l, j, i)] = val;
                                            if (l < nfuc) eri[EIDX(l, k, j, i)] = val;
                                        }
                                    }
                        free(blk);
                    }
                }
        }
    }
#undef EIDX
    if (!c->s.sao) orc_sym_fill_eri(nbas, nfuc, c->ncl, eri);
    return nq;
}

/* symmetry_of_integrals_ERI symmetric_matrix.f90:62-131 (x fastest) */
void orc_sym_fill_eri(int nf, int fpuc, const int32_t ncl_in[3], double *eri)
{
    int nx = ncl_in[0] > 1 ? ncl_in[0] : 1, ny = ncl_in[1] > 1 ? ncl_in[1] : 1, nz = ncl_in[2] > 1 ? ncl_in[2] : 1;
    int *fi = malloc(sizeof(int) * nf), *ic = malloc(sizeof(int) * nf), *jc = malloc(sizeof(int) * nf), *kc = malloc(sizeof(int) * nf);
    for (int idx = 0; idx < nf; ++idx) {
        fi[idx] = idx % fpuc;
        int ii = idx / fpuc;
        ic[idx] = ii % nx; ii /= nx; jc[idx] = ii % ny; kc[idx] = ii / ny;
    }
    #pragma omp parallel for schedule(static)
    for (int i = fpuc; i < nf; ++i) {
        int *eqv = malloc(sizeof(int) * nf);
        for (int j = 0; j < nf; ++j) {
            int m = mod_pos(ic[j] - ic[i], nx), n = mod_pos(jc[j] - jc[i], ny), p = mod_pos(kc[j] - kc[i], nz);
            eqv[j] = (p * nx * ny + n * nx + m) * fpuc + fi[j];
        }
        for (int l = 0; l < nf; ++l)
            for (int k = 0; k < nf; ++k)
                for (int j = 0; j < nf; ++j)
                    eri[(size_t)i + (size_t)nf * ((size_t)j + (size_t)nf * ((size_t)k + (size_t)nf * l))] =
                        eri[(size_t)fi[i] + (size_t)nf * ((size_t)eqv[j] + (size_t)nf * ((size_t)eqv[k] + (size_t)nf * eqv[l]))];
        free(eqv);
    }
    free(fi); free(ic); free(jc); free(kc);
}

/* ---- hartree_exchange_potential.f90:30-202 (dense loop; the sparse loop is bitwise equal) ---- */
void orc_hartree_exchange(int n1, int nbas, int physicist, const double *P, const double *eri, double *J, double *K)
{
    memset(J, 0, sizeof(double) * nbas * nbas);
    memset(K, 0, sizeof(double) * nbas * nbas);
    double *Jloc = calloc((size_t)n1 * nbas, sizeof(double)), *kcol = malloc(sizeof(double) * n1);
    for (int d = 0; d < nbas; ++d) {
        for (int a = 0; a < n1; ++a) kcol[a] = 0.0;
        for (int c = 0; c < nbas; ++c)
            for (int b = 0; b < nbas; ++b) {
                const double *col = eri + (size_t)n1 * ((size_t)b + (size_t)nbas * ((size_t)c + (size_t)nbas * d));
                if (!physicist) {
                    double pcd = P[c + (size_t)nbas * d], pbc = P[b + (size_t)nbas * c];
                    for (int a = 0; a < n1; ++a) { Jloc[a + (size_t)n1 * b] += col[a] * pcd; kcol[a] += col[a] * pbc; }
                } else {
                    double pbd = P[b + (size_t)nbas * d], pcb = P[c + (size_t)nbas * b];
                    for (int a = 0; a < n1; ++a) { Jloc[a + (size_t)n1 * c] += col[a] * pbd; kcol[a] += col[a] * pcb; }
                }
            }
        for (int a = 0; a < n1; ++a) K[a + (size_t)nbas * d] = -0.5 * kcol[a];
    }
    for (int b = 0; b < nbas; ++b)
        for (int a = 0; a < n1; ++a) J[a + (size_t)nbas * b] += Jloc[a + (size_t)n1 * b];
    free(Jloc); free(kcol);
}

/* ---- direct_JK : eri_direct.f90:262-374 ---- */
int64_t orc_direct_jk(orc_ctx *c, const double *P, double *J, double *K)
{
    const double thr = c->s.schwarz_thr;
    int nbas = c->nbas, nfuc = c->nfuc, nsh = c->nsh, nshuc = c->nshuc;
    memset(J, 0, sizeof(double) * nbas * nbas);
    memset(K, 0, sizeof(double) * nbas * nbas);
    if (!c->sym_ok) return -1; /* error stop 'the shells must be the same in every cell' */
    int mx = 0;
    for (int S = 0; S < nsh; ++S) if (c->sh_n[S] > mx) mx = c->sh_n[S];
    int hs = 1;
    while (hs < 4 * 8 * mx * mx * mx * mx) hs *= 2;
    int nt = 0;
    int *tq = malloc(sizeof(int) * 2 * nshuc * nsh);
    for (int SI = 0; SI < nshuc; ++SI)
        for (int SJ = 0; SJ < nsh; ++SJ) {
            if (SJ % nshuc < SI) continue;
            if (c->Qsh[SI + (size_t)nsh * SJ] * c->Qmax < thr) continue;
            tq[2 * nt] = SI; tq[2 * nt + 1] = SJ; ++nt;
        }
    int64_t nq = 0;
    #pragma omp parallel reduction(+ : nq)
    {
        double *Jl = calloc((size_t)nfuc * nbas, sizeof(double)), *Kl = calloc((size_t)nfuc * nbas, sizeof(double));
        int64_t *hkey = malloc(sizeof(int64_t) * hs);
        int *used = malloc(sizeof(int) * 8 * mx * mx * mx * mx);
        for (int h = 0; h < hs; ++h) hkey[h] = -1;
        #pragma omp for schedule(dynamic, 1)
        for (int it = 0; it < nt; ++it) {
            int SI = tq[2 * it], SJ = tq[2 * it + 1];
            for (int SK = 0; SK < nsh; ++SK) {
                if (SK % nshuc < SI) continue;
                for (int SL = 0; SL < nsh; ++SL) {
                    if (SL % nshuc < SI) continue;
                    if (c->Qsh[SI + (size_t)nsh * SJ] * c->Qsh[SK + (size_t)nsh * SL] < thr) continue;
                    int q4[4] = {SI, SJ, SK, SL};
                    if (!is_canonical(c, q4)) continue;
                    ++nq;
                    int n1 = c->sh_n[SI], n2 = c->sh_n[SJ], n3 = c->sh_n[SK], n4 = c->sh_n[SL];
                    double *blk = malloc(sizeof(double) * n1 * n2 * n3 * n4);
                    orc_shell_block(c, SI, SJ, SK, SL, c->ps_qp ? 1 : 0, blk);
                    int ns = 0;
                    for (int d = 0; d < n4; ++d)
                        for (int cc = 0; cc < n3; ++cc)
                            for (int b = 0; b < n2; ++b)
                                for (int a = 0; a < n1; ++a) {
                                    int f[4] = {c->sh_first[SI] + a, c->sh_first[SJ] + b, c->sh_first[SK] + cc, c->sh_first[SL] + d};
                                    if (c->Q[f[0] + (size_t)nbas * f[1]] * c->Q[f[2] + (size_t)nbas * f[3]] < thr) continue;
                                    double val = blk[a + n1 * (b + n2 * (cc + n3 * d))];
                                    for (int ip = 0; ip < 8; ++ip) {
                                        int pp[4];
                                        for (int ii = 0; ii < 4; ++ii) pp[ii] = f[iperm8[ip][ii]];
                                        translate_to_unit_cell(pp, nfuc, c->ncl);
                                        int64_t key = (int64_t)pp[0] + (int64_t)nfuc * ((int64_t)pp[1] + (int64_t)nbas * ((int64_t)pp[2] + (int64_t)nbas * pp[3]));
                                        int h = (int)((key + (key >> 11) + (key >> 23) + (key >> 37)) & (hs - 1));
                                        while (hkey[h] != -1 && hkey[h] != key) h = (h + 1) & (hs - 1);
                                        if (hkey[h] == key) continue;
                                        hkey[h] = key; used[ns++] = h;
                                        Jl[pp[0] + (size_t)nfuc * pp[1]] += val * P[pp[2] + (size_t)nbas * pp[3]];
                                        Kl[pp[0] + (size_t)nfuc * pp[3]] -= 0.5 * val * P[pp[1] + (size_t)nbas * pp[2]];
                                    }
                                }
                    for (int x = 0; x < ns; ++x) hkey[used[x]] = -1;
                    free(blk);
                }
            }
        }
        #pragma omp critical
        {
            for (int b = 0; b < nbas; ++b)
                for (int a = 0; a < nfuc; ++a) {
                    J[a + (size_t)nbas * b] += Jl[a + (size_t)nfuc * b];
                    K[a + (size_t)nbas * b] += Kl[a + (size_t)nfuc * b];
                }
        }
        free(Jl); free(Kl); free(hkey); free(used);
    }
    free(tq);
    return nq;
}

/* ---- counts of the work the direct/stored drivers do ---- */
void orc_count(orc_ctx *c, int64_t *n_shell_q, int64_t *n_func_q, int64_t *n_prim_q)
{
    const double thr = c->s.schwarz_thr;
    int nbas = c->nbas, nsh = c->nsh, nshuc = c->nshuc;
    int64_t ns = 0, nf = 0, npq = 0;
    if (!c->sym_ok) { *n_shell_q = *n_func_q = *n_prim_q = -1; return; }
    #pragma omp parallel for schedule(dynamic, 1) collapse(2) reduction(+ : ns, nf, npq)
    for (int SI = 0; SI < nshuc; ++SI)
        for (int SJ = 0; SJ < nsh; ++SJ) {
            if (SJ % nshuc < SI) continue;
            if (c->Qsh[SI + (size_t)nsh * SJ] * c->Qmax < thr) continue;
            for (int SK = 0; SK < nsh; ++SK) {
                if (SK % nshuc < SI) continue;
                for (int SL = 0; SL < nsh; ++SL) {
                    if (SL % nshuc < SI) continue;
                    if (c->Qsh[SI + (size_t)nsh * SJ] * c->Qsh[SK + (size_t)nsh * SL] < thr) continue;
                    int q4[4] = {SI, SJ, SK, SL};
                    if (!is_canonical(c, q4)) continue;
                    ++ns;
                    int S[4] = {SI, SJ, SK, SL};
                    for (int a = 0; a < c->sh_n[SI]; ++a)
                        for (int b = 0; b < c->sh_n[SJ]; ++b)
                            for (int cc = 0; cc < c->sh_n[SK]; ++cc)
                                for (int d = 0; d < c->sh_n[SL]; ++d) {
                                    int f0 = c->sh_first[SI] + a, f1 = c->sh_first[SJ] + b, f2 = c->sh_first[SK] + cc, f3 = c->sh_first[SL] + d;
                                    if (c->Q[f0 + (size_t)nbas * f1] * c->Q[f2 + (size_t)nbas * f3] >= thr) ++nf;
                                }
                    if (c->ps_qp) {
                        const double *pb = c->ps_qp + (size_t)c->mp * c->mp * ((size_t)SI + (size_t)nshuc * SJ);
                        const double *pk = ket_table(c, SK, SL);
                        int np[4];
                        for (int u = 0; u < 4; ++u) np[u] = c->poff[c->sh_first[S[u]] + 1] - c->poff[c->sh_first[S[u]]];
                        for (int i = 0; i < np[0]; ++i)
                            for (int j = 0; j < np[1]; ++j)
                                for (int k = 0; k < np[2]; ++k)
                                    for (int l = 0; l < np[3]; ++l)
                                        if (pb[i + c->mp * j] * pk[k + c->mp * l] >= c->s.prim_thr) ++npq;
                    }
                }
            }
        }
    *n_shell_q = ns; *n_func_q = nf; *n_prim_q = npq;
}

/* ---- the unique shell quartets of the direct/stored drivers (ERI_toroidal.f90:342-401),
 *      in driver order; returns the count (items written while < cap) ---- */
int64_t orc_items(orc_ctx *c, int32_t *out4, int64_t cap)
{
    const double thr = c->s.schwarz_thr;
    int nsh = c->nsh, nshuc = c->nshuc;
    int64_t n = 0;
    if (!c->sym_ok) return -1;
    for (int SI = 0; SI < nshuc; ++SI)
        for (int SJ = 0; SJ < nsh; ++SJ) {
            if (SJ % nshuc < SI) continue;
            if (c->Qsh[SI + (size_t)nsh * SJ] * c->Qmax < thr) continue;
            for (int SK = 0; SK < nsh; ++SK) {
                if (SK % nshuc < SI) continue;
                for (int SL = 0; SL < nsh; ++SL) {
                    if (SL % nshuc < SI) continue;
                    if (c->Qsh[SI + (size_t)nsh * SJ] * c->Qsh[SK + (size_t)nsh * SL] < thr) continue;
                    int q4[4] = {SI, SJ, SK, SL};
                    if (!is_canonical(c, q4)) continue;
                    if (n < cap) { out4[4 * n] = SI; out4[4 * n + 1] = SJ; out4[4 * n + 2] = SK; out4[4 * n + 3] = SL; }
                    ++n;
                }
            }
        }
    return n;
}

/* ---- direct_JK restricted to an explicit list of unique shell quartets
 *      (same contraction and once-per-element rule as orc_direct_jk);
 *      J/K are accumulated (not zeroed); returns the function quartets done ---- */
int64_t orc_direct_jk_items(orc_ctx *c, const int32_t *items4, int64_t nitems, const double *P, double *J, double *K)
{
    const double thr = c->s.schwarz_thr;
    int nbas = c->nbas, nfuc = c->nfuc, nsh = c->nsh;
    int mx = 0;
    for (int S = 0; S < nsh; ++S) if (c->sh_n[S] > mx) mx = c->sh_n[S];
    int hs = 1;
    while (hs < 4 * 8 * mx * mx * mx * mx) hs *= 2;
    int64_t nf = 0;
    #pragma omp parallel reduction(+ : nf)
    {
        double *Jl = calloc((size_t)nfuc * nbas, sizeof(double)), *Kl = calloc((size_t)nfuc * nbas, sizeof(double));
        int64_t *hkey = malloc(sizeof(int64_t) * hs);
        int *used = malloc(sizeof(int) * 8 * mx * mx * mx * mx);
        for (int h = 0; h < hs; ++h) hkey[h] = -1;
        #pragma omp for schedule(dynamic, 1)
        for (int64_t it = 0; it < nitems; ++it) {
            int SI = items4[4 * it], SJ = items4[4 * it + 1], SK = items4[4 * it + 2], SL = items4[4 * it + 3];
            int n1 = c->sh_n[SI], n2 = c->sh_n[SJ], n3 = c->sh_n[SK], n4 = c->sh_n[SL];
            double *blk = malloc(sizeof(double) * n1 * n2 * n3 * n4);
            orc_shell_block(c, SI, SJ, SK, SL, c->ps_qp ? 1 : 0, blk);
            int ns = 0;
            for (int d = 0; d < n4; ++d)
                for (int cc = 0; cc < n3; ++cc)
                    for (int b = 0; b < n2; ++b)
                        for (int a = 0; a < n1; ++a) {
                            int f[4] = {c->sh_first[SI] + a, c->sh_first[SJ] + b, c->sh_first[SK] + cc, c->sh_first[SL] + d};
                            if (c->Q[f[0] + (size_t)nbas * f[1]] * c->Q[f[2] + (size_t)nbas * f[3]] < thr) continue;
                            ++nf;
                            double val = blk[a + n1 * (b + n2 * (cc + n3 * d))];
                            for (int ip = 0; ip < 8; ++ip) {
                                int pp[4];
                                for (int ii = 0; ii < 4; ++ii) pp[ii] = f[iperm8[ip][ii]];
                                translate_to_unit_cell(pp, nfuc, c->ncl);
                                int64_t key = (int64_t)pp[0] + (int64_t)nfuc * ((int64_t)pp[1] + (int64_t)nbas * ((int64_t)pp[2] + (int64_t)nbas * pp[3]));
                                int h = (int)((key + (key >> 11) + (key >> 23) + (key >> 37)) & (hs - 1));
                                while (hkey[h] != -1 && hkey[h] != key) h = (h + 1) & (hs - 1);
                                if (hkey[h] == key) continue;
                                hkey[h] = key; used[ns++] = h;
                                Jl[pp[0] + (size_t)nfuc * pp[1]] += val * P[pp[2] + (size_t)nbas * pp[3]];
                                Kl[pp[0] + (size_t)nfuc * pp[3]] -= 0.5 * val * P[pp[1] + (size_t)nbas * pp[2]];
                            }
                        }
            for (int x = 0; x < ns; ++x) hkey[used[x]] = -1;
            free(blk);
        }
        #pragma omp critical
        {
            for (int b = 0; b < nbas; ++b)
                for (int a = 0; a < nfuc; ++a) {
                    J[a + (size_t)nbas * b] += Jl[a + (size_t)nfuc * b];
                    K[a + (size_t)nbas * b] += Kl[a + (size_t)nfuc * b];
                }
        }
        free(Jl); free(Kl); free(hkey); free(used);
    }
    return nf;
}

/* =====================================================================
 * one-electron matrices for the SCF consumer (inputs of RHF_SAO)
 * ===================================================================== */

/* kinetic_1D_clifford clifford_tools.f90:305-330 */
static double kinetic_1D_clifford(int i, int l, double beta, double ax, double spa, double cpa, double spb,
                                  double cpb, double R[NMC + 1][NMC + 1], double L)
{
    double inv_ax = 1.0 / ax, acc = 0.0;
    if (l >= 2) acc += (double)(l * (l - 1)) * overlap_1D_clifford_ext(i, l - 2, 0, 0, spa, cpa, spb, cpb, inv_ax, R, L);
    if (l >= 1) acc -= (double)(l * l) * ax * ax * overlap_1D_clifford_ext(i, l, 0, 0, spa, cpa, spb, cpb, inv_ax, R, L);
    double cosu = cpb * overlap_1D_clifford_ext(i, l, 0, 1, spa, cpa, spb, cpb, inv_ax, R, L) -
                  spb * overlap_1D_clifford_ext(i, l, 1, 0, spa, cpa, spb, cpb, inv_ax, R, L);
    acc -= 2.0 * beta * (double)(2 * l + 1) * cosu;
    acc += 4.0 * beta * beta * overlap_1D_clifford_ext(i, l + 2, 0, 0, spa, cpa, spb, cpb, inv_ax, R, L);
    return acc;
}

/* kinetic_1D_real clifford_tools.f90:368-379 */
static double kinetic_1D_real(int j, int m, double beta, double p, double pa, double pb)
{
    double acc = -2.0 * beta * (double)(2 * m + 1) * overlap_1D_real(j, m, p, pa, pb) +
                 4.0 * beta * beta * overlap_1D_real(j, m + 2, p, pa, pb);
    if (m >= 2) acc += (double)(m * (m - 1)) * overlap_1D_real(j, m - 2, p, pa, pb);
    return acc;
}

/* kinetic_integral_toroidal_{1,2,3}D (1D_Kinetic_toroidal.f90:18-97, 3D_Kinetic_toroidal.f90) */
double orc_kinetic_pair(int ndp, const double L[3], const int32_t l1[3], const int32_t l2[3], const double r1[3],
                        const double r2[3], int n1, const double *e1, const double *c1, int n2, const double *e2,
                        const double *c2)
{
    init_clifford();
    double K = 0.0, R[NMC + 1][NMC + 1];
    for (int i = 0; i < n1; ++i)
        for (int j = 0; j < n2; ++j) {
            double al = e1[i], be = e2[j], sd[3], dd[3];
            for (int d = 0; d < 3; ++d) {
                if (d < ndp) {
                    double a = 2.0 * PI_D / L[d], pe, cen;
                    orc_bary(al, be, r1[d], r2[d], L[d], a, &pe, &cen);
                    double A = 2.0 * pe / (a * a), kd = exp(-2.0 * (al + be - pe) / (a * a));
                    double spa = sin(a * (cen - r1[d])), cpa = cos(a * (cen - r1[d]));
                    double spb = sin(a * (cen - r2[d])), cpb = cos(a * (cen - r2[d]));
                    int nmax = l1[d] + l2[d] + 2 < NMC ? l1[d] + l2[d] + 2 : NMC;
                    clifford_bessel_ratios(nmax, A, R);
                    sd[d] = kd * overlap_1D_clifford_ext(l1[d], l2[d], 0, 0, spa, cpa, spb, cpb, 1.0 / a, R, L[d]);
                    dd[d] = kd * kinetic_1D_clifford(l1[d], l2[d], be, a, spa, cpa, spb, cpb, R, L[d]);
                } else {
                    double es = al + be, mu = al * be / es, P = (al * r1[d] + be * r2[d]) / es;
                    double k = exp(-mu * (r1[d] - r2[d]) * (r1[d] - r2[d]));
                    sd[d] = k * overlap_1D_real(l1[d], l2[d], es, P - r1[d], P - r2[d]);
                    dd[d] = k * kinetic_1D_real(l1[d], l2[d], be, es, P - r1[d], P - r2[d]);
                }
            }
            K -= 0.5 * c1[i] * c2[j] * (dd[0] * sd[1] * sd[2] + sd[0] * dd[1] * sd[2] + sd[0] * sd[1] * dd[2]);
        }
    return K;
}

/* nuclear_attraction_integral_toroidal_{1,2,3}D (1D_Nuclear_attraction_toroidal.f90:26-163,
 * 3D_Nuclear_attraction_toroidal.f90:18-113): periodic directions by the Fourier/Bessel
 * t-quadrature, real directions by the Gaussian product with the nucleus. */
static double nuclear_pair(const orc_ctx *c, const int32_t l1[3], const int32_t l2[3], const double r1[3],
                           const double r2[3], int n1, const double *e1, const double *c1, int n2, const double *e2,
                           const double *c2, int natoms, const double *geo, const int32_t *Z)
{
    const int ndp = c->ndp, nq = c->nq;
    int M[3], Mmax = 0;
    for (int d = 0; d < 3; ++d) { M[d] = l1[d] + l2[d]; if (d < ndp && M[d] > Mmax) Mmax = M[d]; }
    int nw = c->ncap + Mmax + 2;
    double *Iv = malloc(sizeof(double) * (nw + 64));
    double *Gre = malloc(sizeof(double) * (nw + 1) * 3), *Gim = malloc(sizeof(double) * (nw + 1) * 3);
    double *F = malloc(sizeof(double) * (nw + 1) * 3);
    double V = 0.0;
    for (int i = 0; i < n1; ++i)
        for (int j = 0; j < n2; ++j) {
            double al = e1[i], be = e2[j], es = al + be, mu = al * be / es;
            double pref = c1[i] * c2[j] * 2.0 / sqrt(PI_D);
            double cen[3];
            int Np[3] = {0, 0, 0};
            for (int d = 0; d < 3; ++d) {
                if (d < ndp) {
                    double a = c->a[d], pe;
                    orc_bary(al, be, r1[d], r2[d], c->L[d], a, &pe, &cen[d]);
                    double A = 2.0 * pe / (a * a);
                    pref *= exp(-2.0 * (es - pe) / (a * a)) * c->L[d] / pow(a, M[d]);
                    int est = orc_bessel_nmax_estimate(A);
                    Np[d] = est < nw - Mmax - 2 ? est : nw - Mmax - 2;
                    double dre[2 * NMC + 1], dim[2 * NMC + 1];
                    orc_fourier_sin_product(l1[d], l2[d], a * (cen[d] - r1[d]), a * (cen[d] - r2[d]), dre, dim);
                    orc_bessel_scaled_vector_fast(Np[d] + M[d], A, Iv);
                    for (int n = 0; n <= Np[d]; ++n) {
                        double ar = 0.0, ai = 0.0;
                        for (int kk = -M[d]; kk <= M[d]; ++kk) {
                            double b = Iv[abs(n + kk)];
                            ar += dre[kk + M[d]] * b; ai += dim[kk + M[d]] * b;
                        }
                        Gre[n + (nw + 1) * d] = ar; Gim[n + (nw + 1) * d] = ai;
                    }
                } else {
                    cen[d] = (al * r1[d] + be * r2[d]) / es;
                    pref *= exp(-mu * (r1[d] - r2[d]) * (r1[d] - r2[d]));
                }
            }
            for (int at = 0; at < natoms; ++at) {
                const double *C = geo + 3 * at;
                for (int d = 0; d < ndp; ++d) {
                    double phi = c->a[d] * (cen[d] - C[d]);
                    double cs1 = cos(phi), sn1 = sin(phi), cn = 1.0, sn = 0.0, tmp;
                    for (int n = 0; n <= Np[d]; ++n) {
                        if (n > 0) {
                            if (n % 32 == 0) { cn = cos(n * phi); sn = sin(n * phi); }
                            else { tmp = cn * cs1 - sn * sn1; sn = sn * cs1 + cn * sn1; cn = tmp; }
                        }
                        F[n + (nw + 1) * d] = Gre[n + (nw + 1) * d] * cn - Gim[n + (nw + 1) * d] * sn;
                    }
                }
                double res = 0.0;
                for (int k = 0; k < nq; ++k) {
                    double prod = 1.0, t2 = c->t_node[k] * c->t_node[k];
                    for (int d = 0; d < 3; ++d) {
                        if (d < ndp) {
                            int tn = c->t_nmax[k + nq * d], nt = Np[d] < tn ? Np[d] : tn;
                            double sdv = F[(nw + 1) * d] * TB(c, 0, k, d), dot = 0.0;
                            for (int n = 1; n <= nt; ++n) dot += F[n + (nw + 1) * d] * TB(c, n, k, d);
                            if (nt >= 1) sdv += 2.0 * dot;
                            prod *= sdv;
                        } else {
                            double ppt = es + t2, eta = t2 / ppt, pc = cen[d] - C[d];
                            double ed = exp(-es * eta * pc * pc);
                            double sdv = overlap_1D_real(l1[d], l2[d], ppt, (cen[d] - r1[d]) - eta * pc, (cen[d] - r2[d]) - eta * pc);
                            prod *= ed * sdv;
                        }
                    }
                    res += c->t_weight[k] * prod;
                }
                V -= (double)Z[at] * pref * res;
            }
        }
    free(Iv); free(Gre); free(Gim); free(F);
    return V;
}

/* fill_with_symmetry symmetric_matrix.f90:1-52: rows i >= nfuc from the first nfuc rows */
static void fill_with_symmetry(int nbas, int nfuc, const int ncl[3], double *M)
{
    int nx = ncl[0], ny = ncl[1], nz = ncl[2];
    for (int i = nfuc; i < nbas; ++i) {
        int Ri = i / nfuc, a = i % nfuc;
        int Rzi = Ri / (nx * ny), Ryi = (Ri / nx) % ny, Rxi = Ri % nx;
        for (int j = 0; j < nbas; ++j) {
            int Rj = j / nfuc, b = j % nfuc;
            int Rzj = Rj / (nx * ny), Ryj = (Rj / nx) % ny, Rxj = Rj % nx;
            int dx = mod_pos(Rxj - Rxi, nx), dy = mod_pos(Ryj - Ryi, ny), dz = mod_pos(Rzj - Rzi, nz);
            int src = dz * nx * ny + dy * nx + dx;
            M[i + (size_t)nbas * j] = M[a + (size_t)nbas * (b + src * nfuc)];
        }
    }
}

/* overlap / kinetic / nuclear-attraction matrices (rows < nfuc computed, |x| < 1e-14
 * set to zero, the rest by translation), e.g. overlap_matrix_toroidal_1D
 * 1D_Overlap_toroidal.f90:23-81 */
void orc_one_electron(orc_ctx *c, int natoms, const double *geo, const int32_t *Z, double *S, double *T, double *V)
{
    int nbas = c->nbas, nfuc = c->nfuc;
    init_clifford();   /* shared tables: fill them before the parallel region */
    memset(S, 0, sizeof(double) * nbas * nbas);
    memset(T, 0, sizeof(double) * nbas * nbas);
    memset(V, 0, sizeof(double) * nbas * nbas);
    #pragma omp parallel for schedule(dynamic, 4) collapse(2)
    for (int i = 0; i < nfuc; ++i)
        for (int j = 0; j < nbas; ++j) {
            int pi = c->poff[i], ni = c->poff[i + 1] - pi, pj = c->poff[j], nj = c->poff[j + 1] - pj;
            const int32_t *li = c->lxyz + 3 * i, *lj = c->lxyz + 3 * j;
            const double *ri = c->ctr + 3 * i, *rj = c->ctr + 3 * j;
            double s = orc_overlap_pair(c->ndp, c->L, li, lj, ri, rj, ni, c->exps + pi, c->coefs + pi, nj, c->exps + pj, c->coefs + pj);
            double t = orc_kinetic_pair(c->ndp, c->L, li, lj, ri, rj, ni, c->exps + pi, c->coefs + pi, nj, c->exps + pj, c->coefs + pj);
            double v = nuclear_pair(c, li, lj, ri, rj, ni, c->exps + pi, c->coefs + pi, nj, c->exps + pj, c->coefs + pj, natoms, geo, Z);
            S[i + (size_t)nbas * j] = fabs(s) < 1e-14 ? 0.0 : s;
            T[i + (size_t)nbas * j] = fabs(t) < 1e-14 ? 0.0 : t;
            V[i + (size_t)nbas * j] = fabs(v) < 1e-14 ? 0.0 : v;
        }
    fill_with_symmetry(nbas, nfuc, c->ncl, S);
    fill_with_symmetry(nbas, nfuc, c->ncl, T);
    fill_with_symmetry(nbas, nfuc, c->ncl, V);
}

/* NRE Nuclear_repulsion.f90:1-59: chord distance along the periodic directions */
double orc_nuclear_repulsion(int ndp, const double L[3], int natoms, const double *geo, const int32_t *Z)
{
    double E = 0.0;
    for (int i = 0; i < natoms - 1; ++i)
        for (int j = i + 1; j < natoms; ++j) {
            double dd[3];
            for (int d = 0; d < 3; ++d) {
                dd[d] = geo[3 * i + d] - geo[3 * j + d];
                if (d < ndp) {
                    double a = 2.0 * PI_D / L[d];
                    dd[d] = sqrt(2.0 * (1.0 - cos(a * dd[d])) / (a * a));
                }
            }
            E += (double)Z[i] * (double)Z[j] / sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
        }
    return E;
}
