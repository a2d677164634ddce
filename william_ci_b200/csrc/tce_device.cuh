// tce_device.cuh -- device-side data layout and math primitives of the
// toroidal ERI engine (sm_100a).
//
// Layout (all in HBM, built once per tce_create):
//   shells      : first function, component count, l, primitive count,
//                 exponents, per-component coefficients, max |coef|.
//   unit pairs  : every shell pair (S1 in the unit cell, S2 anywhere).  A ket
//                 pair (SK,SL) is the unit pair of its translate with SK in
//                 the unit cell plus a lattice shift of the centre.
//   pair prims  : per primitive pair: esum, prefactor, barycentre, Bessel
//                 truncation order N_d, primitive Schwarz value.
//   pair vectors: Fourier vectors V_n = sum_k d_k I~_{|n - s k|}(A) per
//                 (direction, power ia, power ib, sign s), stored n-major with
//                 the primitive pairs of the shell pair contiguous, so that the
//                 32 lanes of a warp working on one shell quartet read one
//                 line per n.
//   T table     : c_n e^{-C_k} I_n(C_k) for the t nodes (c_0 = 1, c_n = 2),
//                 zero beyond the node's truncation order, n-major with the
//                 nodes contiguous.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define TCE_LMAX 2            // s, p, d shells
#define TCE_NCOMP_MAX 6       // Cartesian components of a d shell
#define TCE_NMC 16            // NMAX_CLIFF (clifford_tools.f90:82)
#define TCE_ECO 5             // Hermite E entries kept per (ia,ib): t <= 2*TCE_LMAX
#define TCE_MAXG 16           // node groups of 8 (nq <= 128)

struct UnitPair {
    int S1, S2, l1, l2, np1, np2, npp, Nlen;   // Nlen = padded vector length
    long long pp_off;    // first PairPrim
    long long vec_off;   // first double2 of the vector slabs
    long long e_off;     // first double of the Hermite E table
    double ket_max;      // max_pp |pfac| cmax1 cmax2 (the kernel's ket_max)
};

struct PairPrim {
    double esum;         // e1 + e2
    double pfac;         // prod_d prefactor (no 2/sqrt(pi) L^2 constant)
    double cmax12;       // max|c1| * max|c2| over components
    double ps;           // primitive Schwarz value (prim_screen table)
    double cen[3];       // barycentre (absolute, S1 in the unit cell)
    double A[3];         // Bessel arguments 2 pe / a^2 (periodic d)
    int N[3];            // truncation orders (periodic d)
    int pad;
};

struct DevSys {
    int ndp, nq, ncap, nbas, nfuc, nsh, nshuc, ncell;
    int ncl[3];
    double a[3], L[3], fac_const;
    double thr, prim_thr;
    // shells
    const int *sh_first, *sh_n, *sh_l, *sh_np, *sh_eoff, *sh_coff;
    const double *sh_r;       // [3*nsh]
    const double *sh_exp;     // exponents, sh_eoff
    const double *sh_coef;    // [sh_coff + comp*np + p]
    const double *sh_cmax;    // [sh_eoff + p]
    const int *fn_pw;         // [3*nbas]
    const int4 *fn_cell;      // [nbas]: cell coordinates (x, y, z) and index in the unit cell
    // pairs
    const UnitPair *up;
    const PairPrim *pp;
    const double2 *vec;
    const double *ecoef;
    // t tables
    const double *tnode, *tweight, *Tt;   // Tt[(d*(ncap+1)+n)*nq + k]
    int gmax[3][TCE_MAXG];                // per 8-node group: last n with a nonzero entry
    // Schwarz
    const double *Q;
};

// One rule of the learned-grid dictionary: a mapped Gauss-Kronrod rule padded
// to nq = 32 or 64 nodes (zero weights past nn), its T table [d][n][nq] at
// T_off and the per-8-node-group truncation orders gmax[d*TCE_MAXG + g].
struct RuleDev {
    long long T_off;
    int node_off;      // nodes / Kronrod / Gauss weights at node_off .. node_off+nq-1
    int nn;            // real nodes (2n+1 of the Kronrod rule)
    int nq;            // padded node count: 32 or 64
    int gmax[3 * TCE_MAXG];
};

// ---------------------------------------------------------------------------
// e^{-x} I_0(x): the v = 0 branches of iv_log (bessel_iv_log.f90:43-318):
//   x > 1400   : mu-series, 3 terms   (method 1)
//   x > 30     : mu-series, 20 terms  (method 2)
//   otherwise  : power series in log form with peak normalisation (method 7)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double tce_iv0_scaled(double x)
{
    const double LOG_INV_SQRT_2PI = -0.91893853320467267;
    if (x <= 0.0) return 1.0;
    double log_x = log(x);
    if (x > 1.4e3 || x > 30.0) {
        int kmax = (x > 1.4e3) ? 5 : 39;
        double cur = 1.0, sum = 1.0;
        for (int k = 1, c = 1; k <= kmax; k += 2, ++c) {
            cur = cur * ((double)(k * k) / ((double)c * 8.0 * x));
            sum += cur;
        }
        return exp(LOG_INV_SQRT_2PI - 0.5 * log_x + log(fabs(sum)));
    }
    // method 7 with v = 0: terms[k] = log((x^2/4)^k / (k!)^2)
    double inv = 4.0 / (x * x);
    int peak = (int)floor(x / 2.0);
    if (peak > 40) peak = 40;
    double tk = 0.0, tpeak = 0.0;
    for (int k = 1; k <= peak; ++k) tk -= log((double)k * ((double)k * inv));
    tpeak = tk;
    double s = 0.0;
    tk = 0.0;
    for (int k = 0; k <= 40; ++k) {
        if (k > 0) tk -= log((double)k * ((double)k * inv));
        s += exp(tk - tpeak);
    }
    return exp(tpeak + log(s) - x);
}

// bessel_nmax_estimate (clifford_tools.f90:566-572)
__device__ __forceinline__ int tce_nmax_estimate(double A)
{
    return 20 + (int)ceil(9.0 * sqrt(A > 0.0 ? A : 0.0));
}

// Product of two Clifford primitives along one periodic direction:
// bary_exponent_* and bary_center_toroidal_* (tools.f90:1-264).
__device__ __forceinline__ void tce_bary(double e1, double e2, double x1, double x2, double L, double a,
                                         double &pe, double &cen)
{
    const double eps = 1e-6;
    double x = x1 - x2, p;
    if (fabs(x) > 0.5 * L - eps && fabs(x) < 0.5 * L + eps)
        p = (fabs(e1 - e2) < 1e-8) ? 0.0 : fabs(e1 - e2);
    else
        p = sqrt(fabs(e1 * e1 + e2 * e2 + 2.0 * e1 * e2 * cos(a * x)));
    if (p > e1 + e2) p = e1 + e2;
    if (e1 + e2 - p < 1e-14) p = e1 + e2;
    pe = p;
    double d = fabs(x1 - x2);
    if (d < 0.5 * L + eps && d > 0.5 * L - eps) {
        if (fabs(e1 - e2) < 1e-10) cen = 0.5 * (x1 + x2);
        else if (e1 > e2) cen = x1;
        else if (e2 > e1) cen = x2;
        else cen = 0.5 * (x1 + x2);
    } else if (fabs(e1 - e2) < 1e-10) {
        cen = (d > 0.5 * L + eps) ? 0.5 * (x1 + x2) - 0.5 * L : 0.5 * (x1 + x2);
    } else {
        double val = e1 * cos(a * x1) + e2 * cos(a * x2);
        double H = (-val >= 0.0) ? 1.0 : 0.0;
        cen = atan((e1 * sin(a * x1) + e2 * sin(a * x2)) / val) / a + 0.5 * L * H;
    }
}

// McMurchie-Davidson E_t for a real direction (hermite_E_1D, clifford_tools.f90:757-785),
// t = 0..i+j (i, j <= 2 here); E has TCE_ECO entries.
__device__ __forceinline__ void tce_hermite_E(int i, int j, double p, double PA, double PB, double *E)
{
    double Eo[TCE_ECO + 2], En[TCE_ECO + 2];   // Eo[t+1] = E_t, t = -1..
#pragma unroll
    for (int t = 0; t < TCE_ECO + 2; ++t) { Eo[t] = 0.0; En[t] = 0.0; }
    Eo[1] = 1.0;
    double inv2p = 0.5 / p;
    int deg = 0;
    for (int m = 1; m <= i + j; ++m) {
        double X = (m <= i) ? PA : PB;
        for (int t = 0; t <= deg + 1; ++t)
            En[t] = inv2p * Eo[t] + X * Eo[t + 1] + (double)(t + 1) * Eo[t + 2 < TCE_ECO + 2 ? t + 2 : TCE_ECO + 1];
        deg += 1;
        for (int t = 0; t <= deg; ++t) Eo[t + 1] = En[t];
        if (deg + 2 < TCE_ECO + 2) Eo[deg + 2] = 0.0;
    }
#pragma unroll
    for (int t = 0; t < TCE_ECO; ++t) E[t] = (t <= deg) ? Eo[t + 1] : 0.0;
}

// Fourier coefficients of sin^i(u+phA) sin^l(u+phB) (fourier_sin_product,
// clifford_tools.f90:578-607); d[k + M], M = i + l <= 4.
__device__ __forceinline__ void tce_fourier_sin(int i, int l, double phA, double phB, double *dre, double *dim)
{
    const int MM = 2 * TCE_LMAX;
    int M = i + l, deg = 0;
    double tre[2 * MM + 3], tim[2 * MM + 3];
    for (int k = 0; k <= 2 * MM; ++k) { dre[k] = 0.0; dim[k] = 0.0; }
    dre[M] = 1.0;
    for (int m = 1; m <= M; ++m) {
        double ph = (m <= i) ? phA : phB;
        double s, c;
        sincos(ph, &s, &c);
        double cpr = 0.5 * s, cpi = -0.5 * c, cmr = 0.5 * s, cmi = 0.5 * c;
        for (int k = 0; k < 2 * MM + 3; ++k) { tre[k] = 0.0; tim[k] = 0.0; }
        for (int k = -deg; k <= deg; ++k) {
            double ar = dre[k + M], ai = dim[k + M];
            tre[k + 2 + M] += cpr * ar - cpi * ai;
            tim[k + 2 + M] += cpr * ai + cpi * ar;
            tre[k + M] += cmr * ar - cmi * ai;
            tim[k + M] += cmr * ai + cmi * ar;
        }
        deg += 1;
        for (int k = -deg; k <= deg; ++k) { dre[k + M] = tre[k + M + 1]; dim[k + M] = tim[k + M + 1]; }
    }
}

__device__ __forceinline__ double tce_warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int tce_mod(int a, int m) { int r = a % m; return r < 0 ? r + m : r; }

// Shift an index (function or shell, nblk per cell, cells x fastest) by the
// lattice vector -(cell of ref).  translate_to_unit_cell (ERI_toroidal.f90:591-609).
__device__ __forceinline__ int tce_shift_to(int idx, int refcell, int nblk, const int *ncl)
{
    int tx = refcell % ncl[0], ty = (refcell / ncl[0]) % ncl[1], tz = refcell / (ncl[0] * ncl[1]);
    int c = idx / nblk, loc = idx - c * nblk;
    int cx = tce_mod(c % ncl[0] - tx, ncl[0]);
    int cy = tce_mod((c / ncl[0]) % ncl[1] - ty, ncl[1]);
    int cz = tce_mod(c / (ncl[0] * ncl[1]) - tz, ncl[2]);
    return (cx + ncl[0] * (cy + ncl[1] * cz)) * nblk + loc;
}

// tce_shift_to for functions, without integer division: the function's cell
// coordinates come from the table fn_cell, the reference cell's are given.
__device__ __forceinline__ int tce_shift_fn(const DevSys &S, int f, int rx, int ry, int rz)
{
    const int4 c = __ldg(S.fn_cell + f);
    int cx = c.x - rx, cy = c.y - ry, cz = c.z - rz;
    cx += cx < 0 ? S.ncl[0] : 0;
    cy += cy < 0 ? S.ncl[1] : 0;
    cz += cz < 0 ? S.ncl[2] : 0;
    return (cx + S.ncl[0] * (cy + S.ncl[1] * cz)) * S.nfuc + c.w;
}

// J/K contributions of one function quartet f = (i,j|k,l) of the block of
// shell quartet (fI..|..), every stored element (p1 in the unit cell) once:
// J(p1,p2) += E P(p3,p4), K(p1,p4) += -1/2 E P(p2,p3) (eri_direct.f90:331-357).
// The element set of f is its 8 permutations translated to the unit cell; f
// contributes only if it is the smallest member of that set inside the block,
// and each distinct element once (the reference dedupes with a hash).
__device__ __forceinline__ void tce_scatter_jk(const DevSys &S, const double *__restrict__ P, double *J, double *K,
                                               const int f[4], double val, int fI, int nA, int fJ, int nB, int fK,
                                               int nC, int fL, int nD)
{
    const int perm[8][4] = {{0,1,2,3},{1,0,2,3},{0,1,3,2},{1,0,3,2},{2,3,0,1},{3,2,0,1},{2,3,1,0},{3,2,1,0}};
    int img[8][4];
    for (int ip = 0; ip < 8; ++ip) {
        int t[4];
#pragma unroll
        for (int ii = 0; ii < 4; ++ii) t[ii] = f[perm[ip][ii]];
        const int4 rc = __ldg(S.fn_cell + t[0]);
#pragma unroll
        for (int ii = 0; ii < 4; ++ii) img[ip][ii] = tce_shift_fn(S, t[ii], rc.x, rc.y, rc.z);
        const int *g = img[ip];
        bool inblk = g[0] >= fI && g[0] < fI + nA && g[1] >= fJ && g[1] < fJ + nB && g[2] >= fK && g[2] < fK + nC &&
                     g[3] >= fL && g[3] < fL + nD;
        if (inblk) {
            for (int ii = 0; ii < 4; ++ii) {
                if (g[ii] < f[ii]) return;
                if (g[ii] > f[ii]) break;
            }
        }
    }
    for (int ip = 0; ip < 8; ++ip) {
        const int *g = img[ip];
        bool dup = false;
        for (int jp = 0; jp < ip && !dup; ++jp)
            dup = img[jp][0] == g[0] && img[jp][1] == g[1] && img[jp][2] == g[2] && img[jp][3] == g[3];
        if (dup) continue;
        atomicAdd(J + g[0] + (long long)S.nfuc * g[1], val * P[g[2] + (long long)S.nbas * g[3]]);
        atomicAdd(K + g[0] + (long long)S.nfuc * g[3], -0.5 * val * P[g[1] + (long long)S.nbas * g[2]]);
    }
}

