// tce_onee.cu -- nuclear attraction matrix on the device.
//
// NA(i, j) = -sum_atoms Z_C <i| 1/|r - C| |j> for i in the unit cell, j in
// the supercell: nuclear_attraction_integral_toroidal_{1,2,3}D
// (1D_Nuclear_attraction_toroidal.f90:26-163, 3D_Nuclear_attraction_toroidal.f90
// :18-111) with the handle's t-rule and T table, then |NA| < 1e-14 set to
// zero and the other cells' rows by translation (nuclear_attraction_matrix_
// toroidal_1D, :169-276; fill_with_symmetry, symmetric_matrix.f90:1-52).
//
// Per primitive pair the integral is
//   (2/sqrt(pi)) c1 c2 prod_periodic[e^{-2(p - pe)/a^2} L / a^M] prod_real e^{-mu R^2}
//   x sum_k w_k prod_d X_d(t_k),
// periodic d: X_d = sum_n F_n T[n][k], F_n = Re[(G_n) e^{i n phi_C}], G_n the
// pair's Fourier-Bessel vector sum_j d_j e^{-A} I_{|n+j|}(A), phi_C = a (P - C);
// real d: X_d = e^{-p eta (P - C)^2} S_1D(l1, l2, p + t^2, PA - eta PC, PB - eta PC),
// eta = t^2 / (p + t^2).
//
// One warp per function pair (i, j).  Lane 0 runs the Miller recurrence of
// e^{-A} I_n(A) (bessel_scaled_vector_fast, clifford_tools.f90:429-461) into
// shared memory; the lanes build G_n over n, then per atom F_n over n (a
// rotation by e^{32 i phi} per step of the lane's n) and finally the node
// sums over k (lanes over nodes, F broadcast from shared memory, T rows
// coalesced), reduced over the warp.
#include <algorithm>
#include <cmath>
#include <vector>

#include "tce_handle.h"

namespace {

constexpr double PI_D = 3.14159265358979323846;
constexpr int NA_WARPS_MAX = 8;
constexpr int NA_MEXTRA = 4 * TCE_LMAX + 4;   // Bessel orders past N for the Fourier product

// 1D overlap of x^j e^{-p (x - PA')...}: sum_k sum_q C(j,k) C(m,q) pa^{j-k} pb^{m-q}
// <x^{k+q}>, moments (n-1)!! / (2p)^{n/2} sqrt(pi/p) (overlap_1D_real, :336-361)
__device__ double na_overlap_1d(int j, int m, double p, double pa, double pb)
{
    double mom[2 * TCE_LMAX + 1];
    mom[0] = sqrt(PI_D / p);
    if (j + m >= 1) mom[1] = 0.0;
    for (int n = 2; n <= j + m; ++n) mom[n] = (n & 1) ? 0.0 : mom[n - 2] * (double)(n - 1) / (2.0 * p);
    double acc = 0.0, bj = 1.0;
    for (int k = 0; k <= j; ++k) {
        double bm = 1.0;
        for (int q = 0; q <= m; ++q) {
            if (((k + q) & 1) == 0) acc += bj * bm * pow(pa, (double)(j - k)) * pow(pb, (double)(m - q)) * mom[k + q];
            bm = bm * (double)(m - q) / (double)(q + 1);
        }
        bj = bj * (double)(j - k) / (double)(k + 1);
    }
    return acc;
}

struct NaArgs {
    const int2 *fsh;     // per function: shell, component
    const int2 *plist;   // (i, j) of each element, or null: every i < nfuc, j < nbas
    long long npairs;
    int natoms;
    const double *geo;   // [natoms + natoms * d] (Fortran geometry(natoms, 3))
    const int *Z;
    double *V;           // rows of the unit cell V[i + nfuc * j], or V[p] for a pair list
    int wdoubles;        // shared doubles per warp
};

__global__ void __launch_bounds__(NA_WARPS_MAX * 32) k_nuclear(DevSys S, NaArgs A)
{
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long pair = (long long)blockIdx.x * (blockDim.x >> 5) + wib;
    if (pair >= A.npairs) return;
    const int fi = A.plist ? A.plist[pair].x : (int)(pair % S.nfuc);
    const int fj = A.plist ? A.plist[pair].y : (int)(pair / S.nfuc);
    const int NW = S.ncap + 1;
    double *Iv = smem + (size_t)wib * A.wdoubles;            // NW + NA_MEXTRA
    double *Gre = Iv + NW + NA_MEXTRA;                        // [ndp][NW] each
    double *Gim = Gre + S.ndp * NW;
    double *F = Gim + S.ndp * NW;
    const int2 a1 = A.fsh[fi], a2 = A.fsh[fj];
    const int S1 = a1.x, S2 = a2.x;
    int l1[3], l2[3], M[3];
    for (int d = 0; d < 3; ++d) {
        l1[d] = S.fn_pw[3 * fi + d];
        l2[d] = S.fn_pw[3 * fj + d];
        M[d] = l1[d] + l2[d];
    }
    const double *r1 = S.sh_r + 3 * S1, *r2 = S.sh_r + 3 * S2;
    const int n1 = S.sh_np[S1], n2 = S.sh_np[S2];
    double V = 0.0;
    for (int pi = 0; pi < n1; ++pi)
        for (int pj = 0; pj < n2; ++pj) {
            const double al = S.sh_exp[S.sh_eoff[S1] + pi], be = S.sh_exp[S.sh_eoff[S2] + pj];
            const double es = al + be, mu = al * be / es;
            double pref = S.sh_coef[S.sh_coff[S1] + a1.y * n1 + pi] * S.sh_coef[S.sh_coff[S2] + a2.y * n2 + pj] * 2.0 /
                          sqrt(PI_D);
            double cen[3];
            int Np[3] = {0, 0, 0};
            for (int d = 0; d < 3; ++d) {
                if (d < S.ndp) {
                    const double a = S.a[d];
                    double pe;
                    tce_bary(al, be, r1[d], r2[d], S.L[d], a, pe, cen[d]);
                    const double Aa = 2.0 * pe / (a * a);
                    pref *= exp(-2.0 * (es - pe) / (a * a)) * S.L[d] / pow(a, (double)M[d]);
                    const int est = tce_nmax_estimate(Aa);
                    Np[d] = est < S.ncap ? est : S.ncap;
                    const int N = Np[d] + M[d];
                    if (lane == 0) {   // e^{-A} I_n(A), n = 0..N, Miller from N
                        if (Aa < 1e-10) {
                            for (int k = 0; k <= N; ++k) Iv[k] = 0.0;
                            Iv[0] = 1.0;
                        } else if (N < 2) {
                            for (int k = 0; k <= N; ++k) Iv[k] = 0.0;
                            Iv[0] = tce_iv0_scaled(Aa);
                        } else {
                            const double inv_A2 = 2.0 / Aa;
                            Iv[N] = 1e-280;
                            Iv[N - 1] = Iv[N] * (double)N * inv_A2;
                            for (int k = N - 1; k >= 1; --k) {
                                Iv[k - 1] = Iv[k + 1] + (double)k * inv_A2 * Iv[k];
                                if (Iv[k - 1] > 1e250)
                                    for (int m = k - 1; m <= N; ++m) Iv[m] *= 1e-250;
                            }
                            const double s = tce_iv0_scaled(Aa) / Iv[0];
                            for (int k = 0; k <= N; ++k) Iv[k] *= s;
                        }
                    }
                    __syncwarp();
                    double dre[4 * TCE_LMAX + 1], dim[4 * TCE_LMAX + 1];
                    if (M[d] > 0) tce_fourier_sin(l1[d], l2[d], a * (cen[d] - r1[d]), a * (cen[d] - r2[d]), dre, dim);
                    for (int n = lane; n <= Np[d]; n += 32) {
                        double gr = 0.0, gi = 0.0;
                        if (M[d] == 0) {
                            gr = Iv[n];
                        } else {
                            for (int kk = -M[d]; kk <= M[d]; ++kk) {
                                const int idx = n + kk;
                                const double b = Iv[idx < 0 ? -idx : idx];
                                gr += dre[kk + M[d]] * b;
                                gi += dim[kk + M[d]] * b;
                            }
                        }
                        Gre[d * NW + n] = gr;
                        Gim[d * NW + n] = gi;
                    }
                    __syncwarp();
                } else {
                    cen[d] = (al * r1[d] + be * r2[d]) / es;
                    pref *= exp(-mu * (r1[d] - r2[d]) * (r1[d] - r2[d]));
                }
            }
            for (int at = 0; at < A.natoms; ++at) {
                double Cc[3];
                for (int d = 0; d < 3; ++d) Cc[d] = A.geo[at + (size_t)A.natoms * d];
                for (int d = 0; d < S.ndp; ++d) {
                    const double phi = S.a[d] * (cen[d] - Cc[d]);
                    double sn, cn, s32, c32;
                    sincos((double)lane * phi, &sn, &cn);
                    sincos(32.0 * phi, &s32, &c32);
                    for (int n = lane; n <= Np[d]; n += 32) {
                        F[d * NW + n] = Gre[d * NW + n] * cn - Gim[d * NW + n] * sn;
                        const double t = cn * c32 - sn * s32;
                        sn = sn * c32 + cn * s32;
                        cn = t;
                    }
                }
                __syncwarp();
                double res = 0.0;
                for (int k = lane; k < S.nq; k += 32) {
                    const double t2 = S.tnode[k] * S.tnode[k];
                    double prod = 1.0;
                    for (int d = 0; d < 3; ++d) {
                        if (d < S.ndp) {
                            const double *Tk = S.Tt + (size_t)d * NW * S.nq + k;
                            const double *Fd = F + d * NW;
                            double d0 = 0.0, d1 = 0.0, d2 = 0.0, d3 = 0.0;   // four chains
                            int n = 0;
                            for (; n + 3 <= Np[d]; n += 4) {
                                d0 = fma(Fd[n], Tk[(size_t)n * S.nq], d0);
                                d1 = fma(Fd[n + 1], Tk[(size_t)(n + 1) * S.nq], d1);
                                d2 = fma(Fd[n + 2], Tk[(size_t)(n + 2) * S.nq], d2);
                                d3 = fma(Fd[n + 3], Tk[(size_t)(n + 3) * S.nq], d3);
                            }
                            for (; n <= Np[d]; ++n) d0 = fma(Fd[n], Tk[(size_t)n * S.nq], d0);
                            prod *= (d0 + d1) + (d2 + d3);
                        } else {
                            const double ppt = es + t2, eta = t2 / ppt, pc = cen[d] - Cc[d];
                            const double ed = exp(-es * eta * pc * pc);
                            prod *= ed * na_overlap_1d(l1[d], l2[d], ppt, (cen[d] - r1[d]) - eta * pc,
                                                        (cen[d] - r2[d]) - eta * pc);
                        }
                    }
                    res = fma(S.tweight[k], prod, res);
                }
                res = tce_warp_sum(res);
                V -= (double)A.Z[at] * pref * res;
                __syncwarp();
            }
        }
    if (lane == 0) A.V[A.plist ? pair : fi + (long long)S.nfuc * fj] = fabs(V) < 1e-14 ? 0.0 : V;
}

__device__ __forceinline__ void na_dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// One periodic direction, 32- or 64-node rule: per primitive pair the node
// sums of every atom, X(atom, k) = sum_n F_n(atom) T[n][k], are an
// (atoms x orders) x (orders x nodes) product done as FP64 mma.sync.m8n8k4
// tiles: 16 atoms x 32 nodes per pass, lane l owns atom rows 8 m + l/4 and
// order 4 s + l%4, cos / sin(n phi_atom) by the three-term recurrence in
// steps of four (re-seeded every 32 orders), B fragments T[4 s + l%4][8 g + l/4].
// The epilogue multiplies each (atom, node) by its real-direction factors,
// weight and charge.  G vectors, prefactor and the rest as k_nuclear.
template <int NQ>
__global__ void __launch_bounds__(NA_WARPS_MAX * 32, 1) k_nuclear_tc(DevSys S, NaArgs A)
{
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int rq = lane >> 2, cq = lane & 3;
    const long long pair = (long long)blockIdx.x * (blockDim.x >> 5) + wib;
    if (pair >= A.npairs) return;
    const int fi = A.plist ? A.plist[pair].x : (int)(pair % S.nfuc);
    const int fj = A.plist ? A.plist[pair].y : (int)(pair / S.nfuc);
    const int NW = S.ncap + 1;
    double *Iv = smem + (size_t)wib * A.wdoubles;
    double *Gre = Iv + NW + NA_MEXTRA;
    double *Gim = Gre + NW;
    const int2 a1 = A.fsh[fi], a2 = A.fsh[fj];
    const int S1 = a1.x, S2 = a2.x;
    int l1[3], l2[3], M[3];
    for (int d = 0; d < 3; ++d) {
        l1[d] = S.fn_pw[3 * fi + d];
        l2[d] = S.fn_pw[3 * fj + d];
        M[d] = l1[d] + l2[d];
    }
    const double *r1 = S.sh_r + 3 * S1, *r2 = S.sh_r + 3 * S2;
    const int n1 = S.sh_np[S1], n2 = S.sh_np[S2];
    const double a = S.a[0];
    double V = 0.0;
    for (int pi = 0; pi < n1; ++pi)
        for (int pj = 0; pj < n2; ++pj) {
            const double al = S.sh_exp[S.sh_eoff[S1] + pi], be = S.sh_exp[S.sh_eoff[S2] + pj];
            const double es = al + be, mu = al * be / es;
            double pref = S.sh_coef[S.sh_coff[S1] + a1.y * n1 + pi] * S.sh_coef[S.sh_coff[S2] + a2.y * n2 + pj] * 2.0 /
                          sqrt(PI_D);
            double cen[3], pe;
            tce_bary(al, be, r1[0], r2[0], S.L[0], a, pe, cen[0]);
            const double Aa = 2.0 * pe / (a * a);
            pref *= exp(-2.0 * (es - pe) / (a * a)) * S.L[0] / pow(a, (double)M[0]);
            const int est = tce_nmax_estimate(Aa);
            const int Np = est < S.ncap ? est : S.ncap;
            const int N = Np + M[0];
            for (int d = 1; d < 3; ++d) {
                cen[d] = (al * r1[d] + be * r2[d]) / es;
                pref *= exp(-mu * (r1[d] - r2[d]) * (r1[d] - r2[d]));
            }
            if (lane == 0) {   // e^{-A} I_n(A), n = 0..N
                if (Aa < 1e-10) {
                    for (int k = 0; k <= N; ++k) Iv[k] = 0.0;
                    Iv[0] = 1.0;
                } else if (N < 2) {
                    for (int k = 0; k <= N; ++k) Iv[k] = 0.0;
                    Iv[0] = tce_iv0_scaled(Aa);
                } else {
                    const double inv_A2 = 2.0 / Aa;
                    Iv[N] = 1e-280;
                    Iv[N - 1] = Iv[N] * (double)N * inv_A2;
                    for (int k = N - 1; k >= 1; --k) {
                        Iv[k - 1] = Iv[k + 1] + (double)k * inv_A2 * Iv[k];
                        if (Iv[k - 1] > 1e250)
                            for (int m = k - 1; m <= N; ++m) Iv[m] *= 1e-250;
                    }
                    const double sc = tce_iv0_scaled(Aa) / Iv[0];
                    for (int k = 0; k <= N; ++k) Iv[k] *= sc;
                }
            }
            __syncwarp();
            double dre[4 * TCE_LMAX + 1], dim[4 * TCE_LMAX + 1];
            if (M[0] > 0) tce_fourier_sin(l1[0], l2[0], a * (cen[0] - r1[0]), a * (cen[0] - r2[0]), dre, dim);
            for (int n = lane; n <= Np; n += 32) {
                double gr = 0.0, gi = 0.0;
                if (M[0] == 0) {
                    gr = Iv[n];
                } else {
                    for (int kk = -M[0]; kk <= M[0]; ++kk) {
                        const int idx = n + kk;
                        const double bv = Iv[idx < 0 ? -idx : idx];
                        gr += dre[kk + M[0]] * bv;
                        gi += dim[kk + M[0]] * bv;
                    }
                }
                Gre[n] = gr;
                Gim[n] = gi;
            }
            __syncwarp();
            double vsum = 0.0;
            for (int at0 = 0; at0 < A.natoms; at0 += 16) {
                double phr[2];
                bool valid[2];
#pragma unroll
                for (int m = 0; m < 2; ++m) {
                    const int at = at0 + 8 * m + rq;
                    valid[m] = at < A.natoms;
                    phr[m] = valid[m] ? a * (cen[0] - A.geo[at]) : 0.0;
                }
#pragma unroll 1
                for (int g0 = 0; g0 < NQ / 8; g0 += 4) {
                    double acc[16];
#pragma unroll
                    for (int x = 0; x < 16; ++x) acc[x] = 0.0;
                    double cc[2], cp[2], sc[2], sp[2], c4[2];
#pragma unroll
                    for (int m = 0; m < 2; ++m) {
                        sincos((double)cq * phr[m], &sc[m], &cc[m]);
                        sincos((double)(cq - 4) * phr[m], &sp[m], &cp[m]);
                        c4[m] = 2.0 * cos(4.0 * phr[m]);
                    }
                    for (int s4 = 0; s4 <= Np; s4 += 4) {
                        const int n = s4 + cq, n1 = n + 4;
                        const bool inr = n <= Np;
                        const double gr = inr ? Gre[n] : 0.0, gi = inr ? Gim[n] : 0.0;
                        double F[2];
#pragma unroll
                        for (int m = 0; m < 2; ++m) F[m] = valid[m] ? gr * cc[m] - gi * sc[m] : 0.0;
                        double Tb[4];
#pragma unroll
                        for (int t = 0; t < 4; ++t)
                            Tb[t] = (n <= S.ncap) ? __ldg(S.Tt + (size_t)n * S.nq + 8 * (g0 + t) + rq) : 0.0;
                        if (((s4 + 4) & 31) == 0) {
#pragma unroll
                            for (int m = 0; m < 2; ++m) {
                                sincos((double)n * phr[m], &sp[m], &cp[m]);
                                sincos((double)n1 * phr[m], &sc[m], &cc[m]);
                            }
                        } else {
#pragma unroll
                            for (int m = 0; m < 2; ++m) {
                                const double tc_ = c4[m] * cc[m] - cp[m], ts_ = c4[m] * sc[m] - sp[m];
                                cp[m] = cc[m];
                                cc[m] = tc_;
                                sp[m] = sc[m];
                                sc[m] = ts_;
                            }
                        }
#pragma unroll
                        for (int t = 0; t < 4; ++t)
#pragma unroll
                            for (int m = 0; m < 2; ++m) na_dmma(acc[(m * 4 + t) * 2], acc[(m * 4 + t) * 2 + 1], F[m], Tb[t]);
                    }
                    // epilogue: acc[(m 4 + t) 2 + i] = X(atom 8 m + rq, node 8 (g0 + t) + 2 cq + i)
#pragma unroll
                    for (int m = 0; m < 2; ++m) {
                        if (!valid[m]) continue;
                        const int at = at0 + 8 * m + rq;
                        double Cc[3];
                        for (int d = 1; d < 3; ++d) Cc[d] = A.geo[at + (size_t)A.natoms * d];
                        double part = 0.0;
#pragma unroll
                        for (int t = 0; t < 4; ++t)
#pragma unroll
                            for (int i = 0; i < 2; ++i) {
                                const int k = 8 * (g0 + t) + 2 * cq + i;
                                const double t2 = S.tnode[k] * S.tnode[k];
                                double prod = acc[(m * 4 + t) * 2 + i];
                                for (int d = 1; d < 3; ++d) {
                                    const double ppt = es + t2, eta = t2 / ppt, pc = cen[d] - Cc[d];
                                    const double ed = exp(-es * eta * pc * pc);
                                    prod *= ed * na_overlap_1d(l1[d], l2[d], ppt, (cen[d] - r1[d]) - eta * pc,
                                                                (cen[d] - r2[d]) - eta * pc);
                                }
                                part = fma(S.tweight[k], prod, part);
                            }
                        vsum = fma((double)A.Z[at], part, vsum);
                    }
                }
            }
            vsum = tce_warp_sum(vsum);
            V -= pref * vsum;
            __syncwarp();
        }
    if (lane == 0) A.V[A.plist ? pair : fi + (long long)S.nfuc * fj] = fabs(V) < 1e-14 ? 0.0 : V;
}

}  // namespace

using namespace tcehost;

// Elements of the nuclear attraction matrix on the device: every i < nfuc,
// j < nbas (plist empty; out[i + nfuc j]) or the listed (i, j) (out[p]).
static int nuclear_elements(Handle *h, int natoms, const double *geo, const int32_t *Z, const std::vector<int2> &plist,
                            std::vector<double> &out)
{
    const int nbas = h->nbas, nfuc = h->nfuc;
    std::vector<int2> fsh((size_t)nbas, make_int2(-1, 0));
    for (int s = 0; s < (int)h->sh_first.size(); ++s)
        for (int c = 0; c < h->sh_n[s]; ++c) fsh[(size_t)h->sh_first[s] + c] = make_int2(s, c);
    for (int f = 0; f < nbas; ++f)
        if (fsh[(size_t)f].x < 0) return fail(h, TCE_ERR_STATE, "function without a shell");
    for (const int2 &p : plist)
        if (p.x < 0 || p.x >= nfuc || p.y < 0 || p.y >= nbas) return fail(h, TCE_ERR_ARG, "element outside the unit-cell rows");
    const long long npairs = plist.empty() ? (long long)nfuc * nbas : (long long)plist.size();
    std::vector<double> g(geo, geo + (size_t)natoms * 3);
    std::vector<int> z(Z, Z + natoms);
    int2 *d_fsh = nullptr, *d_pl = nullptr;
    double *d_geo = nullptr, *d_V = nullptr;
    int *d_Z = nullptr;
    int s;
    auto cleanup = [&]() {
        dfree(h, d_fsh);
        dfree(h, d_pl);
        dfree(h, d_geo);
        dfree(h, d_Z);
        dfree(h, d_V);
    };
    if ((s = upload(h, &d_fsh, fsh)) || (!plist.empty() && (s = upload(h, &d_pl, plist))) ||
        (s = upload(h, &d_geo, g)) || (s = upload(h, &d_Z, z)) || (s = dalloc(h, &d_V, (size_t)npairs))) {
        cleanup();
        return s;
    }
    NaArgs A;
    A.fsh = d_fsh;
    A.plist = plist.empty() ? nullptr : d_pl;
    A.npairs = npairs;
    A.natoms = natoms;
    A.geo = d_geo;
    A.Z = d_Z;
    A.V = d_V;
    const int NW = h->ncap + 1;
    A.wdoubles = (NW + NA_MEXTRA + 3 * h->ndp * NW + 31) / 32 * 32;
    const size_t wbytes = (size_t)A.wdoubles * sizeof(double);
    int warps = NA_WARPS_MAX;
    while (warps > 1 && wbytes * warps > 200 * 1024) --warps;
    if (wbytes > 200 * 1024) {
        cleanup();
        return fail(h, TCE_ERR_UNSUPPORTED, "truncation order too large for the nuclear-attraction kernel");
    }
    const size_t smem = wbytes * (size_t)warps;
    // one periodic direction with a 32- or 64-node rule: the tensor-core form
    const unsigned grid = (unsigned)((npairs + warps - 1) / warps);
    if (h->use_tc && h->ndp == 1 && (h->nq == 32 || h->nq == 64)) {
        auto kern = h->nq == 32 ? k_nuclear_tc<32> : k_nuclear_tc<64>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, 32 * warps, smem, h->st>>>(h->S, A);
    } else {
        cudaFuncSetAttribute(k_nuclear, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_nuclear<<<grid, 32 * warps, smem, h->st>>>(h->S, A);
    }
    cudaError_t e = cudaGetLastError();
    out.assign((size_t)npairs, 0.0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out.data(), d_V, sizeof(double) * out.size(), cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    cleanup();
    if (e != cudaSuccess) return fail(h, TCE_ERR_CUDA, std::string("nuclear attraction: ") + cudaGetErrorString(e));
    return TCE_OK;
}

extern "C" int tce_nuclear_attraction(void *handle, int32_t natoms, const double *geo, const int32_t *Z, double *V)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !geo || !Z || !V || natoms < 1) return fail(h, TCE_ERR_ARG, "bad argument");
    const int nbas = h->nbas, nfuc = h->nfuc;
    std::vector<double> rows;
    int s = nuclear_elements(h, natoms, geo, Z, {}, rows);
    if (s) return s;
    // rows of the unit cell, the rest by translation (fill_with_symmetry)
    const int nx = h->ncl[0], ny = h->ncl[1], nz = h->ncl[2];
    for (int i = 0; i < nbas; ++i) {
        const int Ri = i / nfuc, a = i % nfuc;
        const int Rxi = Ri % nx, Ryi = (Ri / nx) % ny, Rzi = Ri / (nx * ny);
        for (int j = 0; j < nbas; ++j) {
            const int Rj = j / nfuc, b = j % nfuc;
            const int Rxj = Rj % nx, Ryj = (Rj / nx) % ny, Rzj = Rj / (nx * ny);
            const int dx = ((Rxj - Rxi) % nx + nx) % nx, dy = ((Ryj - Ryi) % ny + ny) % ny;
            const int dz = ((Rzj - Rzi) % nz + nz) % nz;
            const int src = (dz * ny + dy) * nx + dx;
            V[i + (size_t)nbas * j] = rows[a + (size_t)nfuc * (b + (size_t)src * nfuc)];
        }
    }
    return TCE_OK;
}

// The nuclear-attraction half of fast_quad_self_check (fast_quad_self_check.f90
// :135-172, 189): after the ERI sample (tce_quad_self_check, whose 50 random
// quartets take 200 draws of the generator next() :228-231, seed 12345), the
// diagonal V(i,i) of the first function of every unit-cell shell, 20 random
// pairs inside the unit cell and 20 with j anywhere, each with both handles'
// rules; the fast rule stays when both largest differences are <= 1e-10.
extern "C" int tce_quad_self_check_nuc(void *fast, void *full, int32_t natoms, const double *geo, const int32_t *Z,
                                       double *dmax, double *dV, int32_t *nq, int32_t *nv)
{
    Handle *hf = static_cast<Handle *>(fast), *hg = static_cast<Handle *>(full);
    if (!hf || !hg || !geo || !Z || !dmax || !dV || !nq || !nv || natoms < 1) return fail(hf, TCE_ERR_ARG, "bad argument");
    if (hf->nbas != hg->nbas || hf->nfuc != hg->nfuc) return fail(hf, TCE_ERR_ARG, "handles of different systems");
    int s = tce_quad_self_check(fast, full, dmax, nq);
    if (s) return s;
    const int nfuc = hf->nfuc, nbas = hf->nbas;
    long long seed = 12345;
    auto next = [&]() {
        seed = (seed * 1103515245LL + 12345LL) % 2147483648LL;
        return seed / 16;
    };
    for (int k = 0; k < 4 * 50; ++k) next();   // the ERI sample's draws
    std::vector<int2> pl;
    for (size_t sh = 0; sh < hf->sh_first.size(); ++sh)
        if (hf->sh_first[sh] < nfuc) pl.push_back(make_int2(hf->sh_first[sh], hf->sh_first[sh]));
    if (pl.empty()) pl.push_back(make_int2(0, 0));
    for (int r = 0; r < 40; ++r) {
        const int i = (int)(next() % nfuc);
        const int j = (int)(next() % (r < 20 ? nfuc : nbas));
        pl.push_back(make_int2(i, j));
    }
    std::vector<double> v1, v2;
    if ((s = nuclear_elements(hf, natoms, geo, Z, pl, v1))) return s;
    if ((s = nuclear_elements(hg, natoms, geo, Z, pl, v2))) return fail(hf, s, hg->err);
    double m = 0.0;
    for (size_t p = 0; p < pl.size(); ++p) m = std::max(m, std::fabs(v1[p] - v2[p]));
    *dV = m;
    *nv = (int32_t)pl.size();
    return TCE_OK;
}
