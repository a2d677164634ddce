// tce_kernels_tc.cuh -- pieces shared by the FP64 tensor-core kernels of one
// periodic direction (learned grid): the mma.sync.m8n8k4 (FP64) wrapper, the
// primitive pool fill, the launch helpers, and the s/p kernel
// k_quartets_sp_tc (one or two p shells), instantiated per class in
// tce_kernels_tc.cu (one p) and tce_kernels_sp2.cu (two p).
#pragma once
#include "tce_kernels_s.cuh"

__device__ __forceinline__ void tce_dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Screen the primitive quartets base + lane of a shell quartet (as
// k_quartets_s) and append the kept ones to the warp's pool: pair indices,
// factor (FOLD: with the four contraction coefficients of s shells folded in)
// and the truncation order min(N_bra, N_ket) of the periodic direction.
// Returns the pool's new fill.
template <bool FOLD>
__device__ __forceinline__ int tce_pool_add(const DevSys &S, const SArgs &A, const UnitPair &Ub, const UnitPair &Uk,
                                            const int4 &q, long long base, long long total, int lane,
                                            const PrimPool &Pool, int np)
{
    const int nppk = Uk.npp;
    const long long idx = base + lane;
    bool keep = idx < total;
    int ipb = 0, ipk = 0, key = 0;
    double fac = 0.0;
    if (keep) {
        ipb = (int)(idx / nppk);
        ipk = (int)(idx - (long long)ipb * nppk);
        const PairPrim &Pb = S.pp[Ub.pp_off + ipb];
        const PairPrim &Pk = S.pp[Uk.pp_off + ipk];
        fac = S.fac_const * Pb.pfac * Pk.pfac;
        const double bra = fabs(S.fac_const * Pb.pfac) * Pb.cmax12;
        if (bra * Uk.ket_max <= 2.22e-16) keep = false;
        else if (fabs(fac) * Pb.cmax12 * Pk.cmax12 <= 2.22e-16) keep = false;
        else if (A.prim_screen && Pb.ps * Pk.ps < S.prim_thr) keep = false;
        if (keep) {
            if (FOLD)
                fac *= S.sh_coef[S.sh_coff[q.x] + ipb / Ub.np2] * S.sh_coef[S.sh_coff[q.y] + ipb % Ub.np2] *
                       S.sh_coef[S.sh_coff[q.z] + ipk / Uk.np2] * S.sh_coef[S.sh_coff[q.w] + ipk % Uk.np2];
            key = Pb.N[0] < Pk.N[0] ? Pb.N[0] : Pk.N[0];
        }
    }
    const unsigned msk = __ballot_sync(0xffffffffu, keep);
    const int pos = __popc(msk & ((1u << lane) - 1u));
    if (keep) {
        Pool.pq[np + pos] = make_int2(ipb, ipk);
        Pool.fac[np + pos] = fac;
        Pool.key[np + pos] = key;
    }
    __syncwarp();
    return np + __popc(msk);
}

static inline void tc_args(SArgs &A, const SArgsHost &h)
{
    A.items = h.items;
    A.nitems = h.nitems;
    A.prim_screen = h.prim_screen;
    A.next = h.next;
    A.P = h.P;
    A.J = h.J;
    A.K = h.K;
    A.item_rule = h.item_rule;
    A.rules = h.rules;
    A.rule_T = h.rule_T;
    A.rule_t = h.rule_t;
    A.rule_wk = h.rule_wk;
    A.rule_wg = h.rule_wg;
    A.judge_tol = h.judge_tol;
    A.fb_items = h.fb_items;
    A.fb_count = h.fb_count;
}

// persistent launch: as many 256-thread blocks as fit on every SM; shared
// memory = the eight warps' pools plus, for ncq components, their per-lane
// Kronrod and Gauss block accumulators
template <class Kern>
static void tc_launch(Kern kern, const DevSys &S, const SArgs &A, int nsm, cudaStream_t st, int ncq = 0)
{
    const size_t smem = 8 * ((size_t)TCE_POOL_BYTES + 2 * (size_t)ncq * 32 * sizeof(double));
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, smem);
    if (per < 1) per = 1;
    kern<<<nsm * per, 256, smem, st>>>(S, A);
}

// ============================================================================
// s/p classes with one or two p shells, one periodic direction
// (compile-time class LA, LB | LC, LD in {0, 1}), learned grid: the quartet of
// ERI_shell_block_toroidal.f90:28-366 for these classes, scattered like
// direct_JK (eri_direct.f90:331-357), with the node sums on the tensor cores.
//
// Power combinations.  The periodic direction has one row per x-power
// combination (ia, ib | ic, id) of the p shells (2^NP of them):
//     I_cmb[pq][k] = sum_n Re[G^(ia,ib)_n H^(ic,id)_n e^{i n phi}] T[n][k],
// all of them in the same step loop: the zero-power vectors G^(0,0), H^(0,0)
// are real and loaded once for every combination, and cos(n phi), sin(n phi)
// come from one three-term recurrence in steps of four (re-seeded every 32
// orders).  The A fragments are F = Re(G H) cos(n phi) - Im(G H) sin(n phi)
// with the products of real factors left out.
//
// Epilogue by moments.  The real directions add, per node k and component c
// (x powers = combination cmb), w_k I_cmb I_y I_z with the McMurchie-Davidson
// sums of ERI_shell_block_toroidal.f90:302-335:
//     I_d = sum_{u,v} (-1)^u E_u E'_v g_d[u + v],
//     g_d[m] = pi sqrt(D2) e^{-w R_d^2} h_m(w),  D2 = 1 / (pq + (p + q) t_k^2),
//     w = pq t_k^2 D2,  h_0 = 1,  h_{m+1} = 2 w R_d h_m - 2 m w h_{m-1}.
// So I_y I_z = pi^2 D2 e^{-w R^2} P_c(w) (R^2 = R_y^2 + R_z^2), P_c a
// polynomial in w of degree <= the component's y and z powers whose
// coefficients depend on the primitive quartet only.  Each lane sums, over its
// nodes, the moments
//     M_cmb,j = sum_k I_cmb[pq][k] D2 e^{-w R^2} w^j   (Kronrod and Gauss weights)
// and each component follows once per row: pi^2 a^-xs sum_j P_c[j] M_cmb,j.
//
// A batch is 8 MT primitive quartets (rows, sorted by truncation order), a pass
// NT node tiles of 8; per pass and step of four orders a warp issues
// 2^NP MT NT mma.sync.m8n8k4.  Shapes with 16 or more accumulator tiles per warp
// keep them in up to 255 registers (8 warps per SM), the others in 128 (16).
// ============================================================================
template <int NQ, int LA, int LB, int LC, int LD, int MTP, int NTP,
          int MINB = ((1 << (LA + LB + LC + LD)) * MTP * ((NQ / 8) < NTP ? (NQ / 8) : NTP) >= 16 ? 1 : 2)>
__global__ void __launch_bounds__(256, MINB) k_quartets_sp_tc(DevSys S, SArgs A)
{
    constexpr int NP = LA + LB + LC + LD;
    static_assert(NP >= 1 && NP <= 2, "one or two p shells");
    constexpr int MT = MTP, BT = 8 * MTP;
    constexpr int NT = (NQ / 8) < NTP ? (NQ / 8) : NTP;   // node tiles per pass
    constexpr int NA = LA == 0 ? 1 : 3, NB = LB == 0 ? 1 : 3, NC = LC == 0 ? 1 : 3, ND = LD == 0 ? 1 : 3;
    constexpr int NCQ = NA * NB * NC * ND;
    constexpr int NCOMB = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
    constexpr int NGV = (LA + 1) * (LB + 1), NHV = (LC + 1) * (LD + 1);
    constexpr int NN = NP;                                // largest y + z power of a component
    constexpr int EB = tce_ecount(LA, LB), EK = tce_ecount(LC, LD);
    constexpr int AT = 2 * MT * NT;                       // accumulators per combination and lane
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int rq = lane >> 2, cq = lane & 3;   // fragment row in an 8-row tile, fragment column
    const PrimPool Pool = tce_pool(smem, wib);
    // per-lane Kronrod / Gauss block accumulators of the components (shared
    // memory, after the eight pools): [c][lane] and [NCQ + c][lane]
    double *bacc = reinterpret_cast<double *>(reinterpret_cast<char *>(smem) + 8 * (size_t)TCE_POOL_BYTES) +
                   (size_t)wib * 2 * NCQ * 32;
    const double PI2 = PI_D * PI_D, ainv = 1.0 / S.a[0];
    // x-power sum of a combination
    auto xsum = [](int cmb) {
        return cmb % (LA + 1) + (cmb / (LA + 1)) % (LB + 1) + (cmb / NGV) % (LC + 1) + cmb / (NGV * (LC + 1));
    };

    while (true) {
        int it = 0;
        if (lane == 0) it = (int)atomicAdd(A.next, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.nitems) break;
        const int4 q = A.items[it];
        const RuleDev *D = A.rules + A.item_rule[it];
        const double *Tg = A.rule_T + D->T_off;
        const int *gm = D->gmax;
        const double *tn = A.rule_t + D->node_off, *wk = A.rule_wk + D->node_off, *wg = A.rule_wg + D->node_off;
        const int cK = q.z / S.nshuc;
        const int SK0 = q.z - cK * S.nshuc;
        const int SLp = tce_shift_to(q.w, cK, S.nshuc, S.ncl);
        const UnitPair Ub = S.up[(long long)q.x * S.nsh + q.y];
        const UnitPair Uk = S.up[(long long)SK0 * S.nsh + SLp];
        const double Tx = S.sh_r[3 * q.z] - S.sh_r[3 * SK0];
        const int nppb = Ub.npp, nppk = Uk.npp;
        const int npA = S.sh_np[q.x], npB = S.sh_np[q.y], npC = S.sh_np[q.z], npD = S.sh_np[q.w];
        const long long total = (long long)nppb * nppk;
        // power vectors of the periodic direction: bra g = ia + (LA + 1) ib at
        // Gv + 2 g gl, ket h = ic + (LC + 1) id at Hv + 2 h hl
        const long long gl = (long long)Ub.Nlen * nppb, hl = (long long)Uk.Nlen * nppk;
        const double2 *Gv = S.vec + Ub.vec_off, *Hv = S.vec + Uk.vec_off + hl;
        const double *G0 = reinterpret_cast<const double *>(Gv), *H0 = reinterpret_cast<const double *>(Hv);
#pragma unroll
        for (int c = 0; c < 2 * NCQ; ++c) bacc[c * 32 + lane] = 0.0;
        int np = 0;
        for (long long base = 0; base < total; base += 32) {
            np = tce_pool_add<false>(S, A, Ub, Uk, q, base, total, lane, Pool, np);
            const bool last = base + 32 >= total;
            if (!(np > TCE_POOL - 32 || (last && np > 0))) continue;
            if (np > BT) tce_pool_sort(Pool, np, lane);
            const int nproc = last ? np : (np & ~(BT - 1));
            for (int b0 = 0; b0 < nproc; b0 += BT) {
                const int nb = nproc - b0 < BT ? nproc - b0 : BT;
                const int nmax = Pool.key[b0];   // largest truncation order of the batch (sorted)
                int nmr[MT], go[MT], ho[MT];
#pragma unroll
                for (int m = 0; m < MT; ++m) {
                    const int r = 8 * m + rq;
                    nmr[m] = -1;
                    go[m] = ho[m] = 0;
                    if (r < nb) {
                        const int2 pq = Pool.pq[b0 + r];
                        nmr[m] = Pool.key[b0 + r];
                        go[m] = pq.x;
                        ho[m] = pq.y;
                    }
                }
                auto phase = [&](int m) {
                    const int r = 8 * m + rq;
                    if (r >= nb) return 0.0;
                    const int2 pq = Pool.pq[b0 + r];
                    return S.a[0] * (S.pp[Ub.pp_off + pq.x].cen[0] - (S.pp[Uk.pp_off + pq.y].cen[0] + Tx));
                };
                // the vectors of order n of row m (zero past the row's truncation order)
                double g0N[MT], h0N[MT];
                double2 gN[NGV - 1 > 0 ? NGV - 1 : 1][MT], hN[NHV - 1 > 0 ? NHV - 1 : 1][MT];
                auto load = [&](int m, int n) {
                    const bool ok = n <= nmr[m];
                    g0N[m] = ok ? __ldg(G0 + 2 * ((size_t)go[m] + (size_t)n * nppb)) : 0.0;
                    h0N[m] = ok ? __ldg(H0 + 2 * ((size_t)ho[m] + (size_t)n * nppk)) : 0.0;
#pragma unroll
                    for (int g = 1; g < NGV; ++g)
                        gN[g - 1][m] = ok ? __ldg(Gv + 2 * g * gl + go[m] + (size_t)n * nppb) : make_double2(0.0, 0.0);
#pragma unroll
                    for (int h = 1; h < NHV; ++h)
                        hN[h - 1][m] = ok ? __ldg(Hv + 2 * h * hl + ho[m] + (size_t)n * nppk) : make_double2(0.0, 0.0);
                };
#pragma unroll 1
                for (int g0 = 0; g0 < NQ / 8; g0 += NT) {
                    int gmb[NT], nend = -1;
#pragma unroll
                    for (int t = 0; t < NT; ++t) {
                        gmb[t] = gm[g0 + t];
                        nend = gmb[t] > nend ? gmb[t] : nend;
                    }
                    nend = nend < nmax ? nend : nmax;
                    double acc[NCOMB][AT];
#pragma unroll
                    for (int cmb = 0; cmb < NCOMB; ++cmb)
#pragma unroll
                        for (int x = 0; x < AT; ++x) acc[cmb][x] = 0.0;
                    // cos / sin of n phi and (n - 4) phi, 2 cos(4 phi)
                    double cc[MT], cp[MT], sc[MT], sp[MT], c4[MT];
#pragma unroll
                    for (int m = 0; m < MT; ++m) {
                        const double ph = phase(m);
                        sincos((double)cq * ph, &sc[m], &cc[m]);
                        sincos((double)(cq - 4) * ph, &sp[m], &cp[m]);
                        c4[m] = 2.0 * cos(4.0 * ph);
                        load(m, cq);
                    }
                    double tN[NT];
#pragma unroll
                    for (int t = 0; t < NT; ++t)
                        tN[t] = (0 <= gmb[t] && cq <= S.ncap) ? __ldg(Tg + (size_t)cq * NQ + 8 * (g0 + t) + rq) : 0.0;
#pragma unroll 2
                    for (int s4 = 0; s4 <= nend; s4 += 4) {
                        const int n = s4 + cq, n1 = n + 4;
                        double F[NCOMB][MT], Tb[NT];
#pragma unroll
                        for (int m = 0; m < MT; ++m) {
#pragma unroll
                            for (int cmb = 0; cmb < NCOMB; ++cmb) {
                                const int gi = cmb % NGV, hi = cmb / NGV;
                                if (gi == 0 && hi == 0) {
                                    F[cmb][m] = g0N[m] * h0N[m] * cc[m];
                                } else if (gi == 0) {
                                    const double2 hv = hN[hi > 0 ? hi - 1 : 0][m];
                                    F[cmb][m] = g0N[m] * (hv.x * cc[m] - hv.y * sc[m]);
                                } else if (hi == 0) {
                                    const double2 gv = gN[gi > 0 ? gi - 1 : 0][m];
                                    F[cmb][m] = h0N[m] * (gv.x * cc[m] - gv.y * sc[m]);
                                } else {
                                    const double2 gv = gN[gi - 1][m], hv = hN[hi - 1][m];
                                    const double ar = gv.x * hv.x - gv.y * hv.y, ai = gv.x * hv.y + gv.y * hv.x;
                                    F[cmb][m] = ar * cc[m] - ai * sc[m];
                                }
                            }
                            load(m, n1);
                        }
#pragma unroll
                        for (int t = 0; t < NT; ++t) {
                            Tb[t] = tN[t];
                            tN[t] = (s4 + 4 <= gmb[t] && n1 <= S.ncap)
                                        ? __ldg(Tg + (size_t)n1 * NQ + 8 * (g0 + t) + rq) : 0.0;
                        }
                        if (((s4 + 4) & 31) == 0) {   // re-seed the recurrences
#pragma unroll
                            for (int m = 0; m < MT; ++m) {
                                const double ph = phase(m);
                                sincos((double)n * ph, &sp[m], &cp[m]);
                                sincos((double)n1 * ph, &sc[m], &cc[m]);
                            }
                        } else {
#pragma unroll
                            for (int m = 0; m < MT; ++m) {
                                const double tc_ = c4[m] * cc[m] - cp[m], ts_ = c4[m] * sc[m] - sp[m];
                                cp[m] = cc[m];
                                cc[m] = tc_;
                                sp[m] = sc[m];
                                sc[m] = ts_;
                            }
                        }
#pragma unroll
                        for (int t = 0; t < NT; ++t)
                            if (s4 <= gmb[t]) {
#pragma unroll
                                for (int m = 0; m < MT; ++m)
#pragma unroll
                                    for (int cmb = 0; cmb < NCOMB; ++cmb) {
                                        const int x = (m * NT + t) * 2;
                                        tce_dmma(acc[cmb][x], acc[cmb][x + 1], F[cmb][m], Tb[t]);
                                    }
                            }
                    }
                    // epilogue per fragment row: acc[cmb][2 (m NT + t) + i] = I_cmb[8 m + rq][8 (g0 + t) + 2 cq + i]
#pragma unroll
                    for (int m = 0; m < MT; ++m) {
                        const int r = 8 * m + rq;
                        if (r >= nb) continue;
                        const int2 pq = Pool.pq[b0 + r];
                        const PairPrim &Pb = S.pp[Ub.pp_off + pq.x];
                        const PairPrim &Pk = S.pp[Uk.pp_off + pq.y];
                        const double p = Pb.esum, qq = Pk.esum, pq_ = p * qq, ps = p + qq;
                        const double Ry = Pb.cen[1] - Pk.cen[1], Rz = Pb.cen[2] - Pk.cen[2];
                        const double R2 = Ry * Ry + Rz * Rz;
                        // moments [cmb][j][Kronrod, Gauss], j <= NN - xsum(cmb)
                        double Mo[NCOMB][NN + 1][2];
#pragma unroll
                        for (int cmb = 0; cmb < NCOMB; ++cmb)
#pragma unroll
                            for (int j = 0; j <= NN; ++j) Mo[cmb][j][0] = Mo[cmb][j][1] = 0.0;
#pragma unroll
                        for (int t = 0; t < NT; ++t) {
                            if (gmb[t] < 0) continue;   // padding nodes
#pragma unroll
                            for (int i = 0; i < 2; ++i) {
                                const int k = 8 * (g0 + t) + 2 * cq + i;
                                const double t2 = tn[k] * tn[k];
                                const double D2 = 1.0 / (pq_ + ps * t2);
                                const double w = pq_ * t2 * D2;
                                const double bse = (R2 == 0.0) ? D2 : D2 * exp(-w * R2);
                                const double wkk = wk[k], wgk = wg[k];
#pragma unroll
                                for (int cmb = 0; cmb < NCOMB; ++cmb) {
                                    const double b = acc[cmb][(m * NT + t) * 2 + i] * bse;
                                    double bk = b * wkk, bg = b * wgk;
#pragma unroll
                                    for (int j = 0; j <= NN - xsum(cmb); ++j) {
                                        Mo[cmb][j][0] += bk;
                                        Mo[cmb][j][1] += bg;
                                        bk *= w;
                                        bg *= w;
                                    }
                                }
                            }
                        }
                        // Hermite E coefficients of the real directions y (dr = 0), z (dr = 1)
                        double eb[2][EB], ek[2][EK];
                        const double *Ebp = S.ecoef + Ub.e_off + (long long)pq.x * 2 * (LA + 1) * (LB + 1) * TCE_ECO;
                        const double *Ekp = S.ecoef + Uk.e_off + (long long)pq.y * 2 * (LC + 1) * (LD + 1) * TCE_ECO;
#pragma unroll
                        for (int dr = 0; dr < 2; ++dr) {
#pragma unroll
                            for (int a = 0; a <= LA; ++a)
#pragma unroll
                                for (int b = 0; b <= LB; ++b)
#pragma unroll
                                    for (int u = 0; u <= a + b; ++u)
                                        eb[dr][tce_eoff(LB, a, b) + u] = Ebp[((dr * (LA + 1) + a) * (LB + 1) + b) * TCE_ECO + u];
#pragma unroll
                            for (int a = 0; a <= LC; ++a)
#pragma unroll
                                for (int b = 0; b <= LD; ++b)
#pragma unroll
                                    for (int u = 0; u <= a + b; ++u)
                                        ek[dr][tce_eoff(LD, a, b) + u] = Ekp[((dr * (LC + 1) + a) * (LD + 1) + b) * TCE_ECO + u];
                        }
                        // coefficients in w of h_m(w) per real direction: hc[dr][m][j]
                        double hc[2][NN + 1][NN + 1];
#pragma unroll
                        for (int dr = 0; dr < 2; ++dr) {
                            const double R = dr == 0 ? Ry : Rz;
#pragma unroll
                            for (int mm = 0; mm <= NN; ++mm)
#pragma unroll
                                for (int j = 0; j <= NN; ++j) hc[dr][mm][j] = (mm == 0 && j == 0) ? 1.0 : 0.0;
#pragma unroll
                            for (int mm = 0; mm < NN; ++mm)
#pragma unroll
                                for (int j = 1; j <= NN; ++j)
                                    hc[dr][mm + 1][j] = 2.0 * R * hc[dr][mm][j - 1] - (mm > 0 ? 2.0 * mm * hc[dr][mm - 1][j - 1] : 0.0);
                        }
                        const double fac = Pool.fac[b0 + r] * PI2;
                        const int i0 = pq.x / Ub.np2, j0 = pq.x - i0 * Ub.np2;
                        const int k0 = pq.y / Uk.np2, l0 = pq.y - k0 * Uk.np2;
#pragma unroll
                        for (int c = 0; c < NCQ; ++c) {
                            const int ca = c % NA, cb = (c / NA) % NB, cc_ = (c / (NA * NB)) % NC, cd = c / (NA * NB * NC);
                            const int cmb = tce_pw(LA, ca, 0) + (LA + 1) * (tce_pw(LB, cb, 0) + (LB + 1) * (tce_pw(LC, cc_, 0) + (LC + 1) * tce_pw(LD, cd, 0)));
                            const int xs = xsum(cmb);
                            // P_d(w) = sum_{u,v} (-1)^u E_u E'_v h_{u+v}(w) per real direction
                            double Pd[2][NN + 1];
#pragma unroll
                            for (int dr = 0; dr < 2; ++dr) {
                                const int pa = tce_pw(LA, ca, dr + 1), pb = tce_pw(LB, cb, dr + 1);
                                const int pc = tce_pw(LC, cc_, dr + 1), pd = tce_pw(LD, cd, dr + 1);
#pragma unroll
                                for (int j = 0; j <= NN; ++j) Pd[dr][j] = 0.0;
#pragma unroll
                                for (int u = 0; u <= pa + pb; ++u)
#pragma unroll
                                    for (int v = 0; v <= pc + pd; ++v) {
                                        const double e1 = eb[dr][tce_eoff(LB, pa, pb) + u];
                                        const double ee = ((u & 1) ? -e1 : e1) * ek[dr][tce_eoff(LD, pc, pd) + v];
#pragma unroll
                                        for (int j = 0; j <= u + v; ++j) Pd[dr][j] = fma(ee, hc[dr][u + v][j], Pd[dr][j]);
                                    }
                            }
                            double vK = 0.0, vG = 0.0;
#pragma unroll
                            for (int j = 0; j <= NN - xs; ++j) {
                                double cj = 0.0;
#pragma unroll
                                for (int j1 = 0; j1 <= j; ++j1) cj = fma(Pd[0][j1], Pd[1][j - j1], cj);
                                vK = fma(cj, Mo[cmb][j][0], vK);
                                vG = fma(cj, Mo[cmb][j][1], vG);
                            }
                            const double sg = xs == 0 ? 1.0 : xs == 1 ? ainv : ainv * ainv;
                            const double cf = S.sh_coef[S.sh_coff[q.x] + ca * npA + i0] * S.sh_coef[S.sh_coff[q.y] + cb * npB + j0] *
                                              S.sh_coef[S.sh_coff[q.z] + cc_ * npC + k0] * S.sh_coef[S.sh_coff[q.w] + cd * npD + l0];
                            const double f = fac * cf * sg;
                            bacc[c * 32 + lane] = fma(f, vK, bacc[c * 32 + lane]);
                            bacc[(NCQ + c) * 32 + lane] = fma(f, vG, bacc[(NCQ + c) * 32 + lane]);
                        }
                    }
                }
            }
            __syncwarp();
            if (np > nproc) tce_pool_carry(Pool, nproc, np - nproc, lane);
            np -= nproc;
        }
        const int fI = S.sh_first[q.x], fJ = S.sh_first[q.y], fK = S.sh_first[q.z], fL = S.sh_first[q.w];
        double e = 0.0, M = 0.0;
        double blk[NCQ];
#pragma unroll
        for (int c = 0; c < NCQ; ++c) {
            blk[c] = tce_warp_sum(bacc[c * 32 + lane]);
            const double vg = tce_warp_sum(bacc[(NCQ + c) * 32 + lane]);
            e = fmax(e, fabs(blk[c] - vg));
            M = fmax(M, fabs(blk[c]));
        }
        if (!tce_judge_accepts(e, M, A.judge_tol)) {
            if (lane == 0) tce_queue_fallback(A, q);
            __syncwarp();
            continue;
        }
#pragma unroll
        for (int c = 0; c < NCQ; ++c) {
            const double v = blk[c];
            if (lane == (c & 31)) {
                const int ca = c % NA, cb = (c / NA) % NB, cc_ = (c / (NA * NB)) % NC, cd = c / (NA * NB * NC);
                const int f[4] = {fI + ca, fJ + cb, fK + cc_, fL + cd};
                if (S.Q[f[0] + (long long)S.nbas * f[1]] * S.Q[f[2] + (long long)S.nbas * f[3]] >= S.thr)
                    tce_scatter_jk(S, A.P, A.J, A.K, f, v, fI, NA, fJ, NB, fK, NC, fL, ND);
            }
        }
        __syncwarp();
    }
}

// one class of the s/p kernel in tile shape (MT, NT): ncq components
template <int NQ, int LA, int LB, int LC, int LD, int MT, int NT>
static void sp_tc_launch(const DevSys &S, const SArgs &A, int nsm, cudaStream_t st)
{
    constexpr int ncq = (LA ? 3 : 1) * (LB ? 3 : 1) * (LC ? 3 : 1) * (LD ? 3 : 1);
    tc_launch(k_quartets_sp_tc<NQ, LA, LB, LC, LD, MT, NT>, S, A, nsm, st, ncq);
}

// the classes with two p shells (tce_kernels_sp2.cu), as sp1_launch in
// tce_kernels_tc.cu: shape 1: 8 rows x 16 nodes per pass, 2: 8 x 32, 3: 8 x 64
int tce_sp2_launch(const DevSys &S, int cls, const SArgs &A, int nq, int shape, int nsm, cudaStream_t st);
