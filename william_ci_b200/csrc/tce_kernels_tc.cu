// tce_kernels_tc.cu -- all-s shell quartets of one periodic direction with
// per-quartet learned-grid rules, the node sums on the FP64 tensor cores.
//
// The quartet is the one k_quartets_s evaluates (ERI_shell_block_toroidal.f90
// :28-366 for s functions, scattered like direct_JK, eri_direct.f90:331-357).
// For a batch of up to 16 primitive quartets pq (sorted by truncation order)
// the periodic direction needs, per node k of the quartet's rule,
//     I[pq][k] = sum_n F[pq][n] T[n][k],   F[pq][n] = G_n H_n cos(n phi_pq)
// (n <= min(N_bra, N_ket); T[n][k] = c_n e^{-C_k} I_n(C_k), rows past the node
// group's truncation order skipped).  Per pass of 32 nodes this is a
// (16 x N) x (N x 32) product: one warp holds it as 2 x 4 tiles of 8 x 8 and
// issues mma.sync.m8n8k4 (FP64) per tile and step of four orders n.  A
// fragments (F) are built in registers by the lanes that own them: lane l
// holds rows 8 m + l/4 (m = 0, 1) and order 4 s + l%4, with cos(n phi) from
// the three-term recurrence in steps of four (re-seeded every 32 orders).
// B fragments are T[4 s + l%4][8 g + l/4], one load per tile column.  The
// G, H and T values of the next step are loaded before the current step's
// mma instructions are issued.  The
// epilogue (real directions, weights, Kronrod and Gauss sums, the judge and
// the J/K scatter) is the one of k_quartets_s.
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

// MT row tiles of 8 per warp: batches of 8 MT primitive quartets; acc holds
// the batch's 8 MT rows x 8 NT nodes of one pass (MT x NT tiles, 2 per lane).
// The one-p kernel uses MT = 2; the all-s kernel takes (MT, NT) as template
// parameters, its tile shape (TCE_TC_SHAPES) chosen per work list by
// tce_lg_autotune.
constexpr int TCE_TC_MT = 2;
constexpr int TCE_TC_BATCH = 8 * TCE_TC_MT;
// node tiles of 8 per pass of the one-p kernel and of the all-s default (4: 32 nodes per pass)
constexpr int TCE_TC_NT = 4;

template <int NQ, int MTP, int NTP>
__global__ void __launch_bounds__(256, 2) k_quartets_s_tc(DevSys S, SArgs A)
{
    constexpr int MT = MTP, BT = 8 * MTP;
    constexpr int NT = (NQ / 8) < NTP ? (NQ / 8) : NTP;   // node tiles per pass
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int rq = lane >> 2, cq = lane & 3;   // fragment row in an 8-row tile, fragment column
    const PrimPool Pool = tce_pool(smem, wib);
    const double PI2 = PI_D * PI_D;

    while (true) {
        int it = 0;
        if (lane == 0) it = (int)atomicAdd(A.next, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.nitems) break;
        const int4 q = A.items[it];
        const RuleDev *D = A.rules + A.item_rule[it];
        const double *Tg = A.rule_T + D->T_off;   // direction 0: (ncap + 1) rows of NQ nodes
        const int *gm = D->gmax;
        const double *tn = A.rule_t + D->node_off, *wk = A.rule_wk + D->node_off, *wg = A.rule_wg + D->node_off;
        const int cK = q.z / S.nshuc;
        const int SK0 = q.z - cK * S.nshuc;
        const int SLp = tce_shift_to(q.w, cK, S.nshuc, S.ncl);
        const UnitPair Ub = S.up[(long long)q.x * S.nsh + q.y];
        const UnitPair Uk = S.up[(long long)SK0 * S.nsh + SLp];
        double Tsh[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) Tsh[d] = S.sh_r[3 * q.z + d] - S.sh_r[3 * SK0 + d];
        const int nppb = Ub.npp, nppk = Uk.npp;
        const long long total = (long long)nppb * nppk;
        const double *Gbase = reinterpret_cast<const double *>(S.vec + Ub.vec_off);
        const double *Hbase = reinterpret_cast<const double *>(S.vec + Uk.vec_off + (long long)Uk.Nlen * nppk);
        double blk = 0.0, blkG = 0.0;
        int np = 0;
        for (long long base = 0; base < total; base += 32) {
            np = tce_pool_add<true>(S, A, Ub, Uk, q, base, total, lane, Pool, np);
            const bool last = base + 32 >= total;
            if (!(np > TCE_POOL - 32 || (last && np > 0))) continue;
            if (np > BT) tce_pool_sort(Pool, np, lane);
            const int nproc = last ? np : (np & ~(BT - 1));
            for (int b0 = 0; b0 < nproc; b0 += BT) {
                const int nb = nproc - b0 < BT ? nproc - b0 : BT;
                const int nmax = Pool.key[b0];   // largest truncation order of the batch (sorted)
                // this lane's fragment rows: primitive quartets 8 m + rq of the batch
                int goff[MT], hoff[MT], nmr[MT];
#pragma unroll
                for (int m = 0; m < MT; ++m) {
                    const int r = 8 * m + rq;
                    nmr[m] = -1;
                    goff[m] = hoff[m] = 0;
                    if (r < nb) {
                        const int2 pq = Pool.pq[b0 + r];
                        nmr[m] = Pool.key[b0 + r];
                        goff[m] = 2 * pq.x;
                        hoff[m] = 2 * pq.y;
                    }
                }
                // phase of row m, from the pool entry (read again where the recurrence is re-seeded)
                auto phase = [&](int m) {
                    const int r = 8 * m + rq;
                    if (r >= nb) return 0.0;
                    const int2 pq = Pool.pq[b0 + r];
                    return S.a[0] * (S.pp[Ub.pp_off + pq.x].cen[0] - (S.pp[Uk.pp_off + pq.y].cen[0] + Tsh[0]));
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
                    double acc[2 * MT * NT];
#pragma unroll
                    for (int x = 0; x < 2 * MT * NT; ++x) acc[x] = 0.0;
                    double cc[MT], cp[MT], c4[MT];   // cos(n phi), cos((n - 4) phi), 2 cos(4 phi)
                    double gN[MT], hN[MT];           // G_n, H_n of the next step (prefetched)
#pragma unroll
                    for (int m = 0; m < MT; ++m) {
                        const double ph = phase(m);
                        cc[m] = cos((double)cq * ph);
                        cp[m] = cos((double)(cq - 4) * ph);
                        c4[m] = 2.0 * cos(4.0 * ph);
                        const bool ok = cq <= nmr[m];
                        gN[m] = ok ? __ldg(Gbase + goff[m] + 2 * (size_t)cq * nppb) : 0.0;
                        hN[m] = ok ? __ldg(Hbase + hoff[m] + 2 * (size_t)cq * nppk) : 0.0;
                    }
                    double tN[NT];                    // T fragments of the next step
#pragma unroll
                    for (int t = 0; t < NT; ++t)
                        tN[t] = (0 <= gmb[t] && cq <= S.ncap) ? __ldg(Tg + (size_t)cq * NQ + 8 * (g0 + t) + rq) : 0.0;
                    for (int s4 = 0; s4 <= nend; s4 += 4) {
                        const int n = s4 + cq, n1 = n + 4;
                        double F[MT], Tb[NT];
#pragma unroll
                        for (int m = 0; m < MT; ++m) {
                            F[m] = gN[m] * hN[m] * cc[m];
                            const bool ok = n1 <= nmr[m];
                            gN[m] = ok ? __ldg(Gbase + goff[m] + 2 * (size_t)n1 * nppb) : 0.0;
                            hN[m] = ok ? __ldg(Hbase + hoff[m] + 2 * (size_t)n1 * nppk) : 0.0;
                        }
#pragma unroll
                        for (int t = 0; t < NT; ++t) {
                            Tb[t] = tN[t];
                            tN[t] = (s4 + 4 <= gmb[t] && n1 <= S.ncap)
                                        ? __ldg(Tg + (size_t)n1 * NQ + 8 * (g0 + t) + rq) : 0.0;
                        }
                        if (((s4 + 4) & 31) == 0) {   // re-seed the recurrence
#pragma unroll
                            for (int m = 0; m < MT; ++m) {
                                const double ph = phase(m);
                                cp[m] = cos((double)n * ph);
                                cc[m] = cos((double)n1 * ph);
                            }
                        } else {
#pragma unroll
                            for (int m = 0; m < MT; ++m) {
                                const double t = c4[m] * cc[m] - cp[m];
                                cp[m] = cc[m];
                                cc[m] = t;
                            }
                        }
#pragma unroll
                        for (int t = 0; t < NT; ++t)
                            if (s4 <= gmb[t]) {
#pragma unroll
                                for (int m = 0; m < MT; ++m) tce_dmma(acc[(m * NT + t) * 2], acc[(m * NT + t) * 2 + 1], F[m], Tb[t]);
                            }
                    }
                    // epilogue: acc[2 (m NT + t) + i] = I[8 m + rq][8 (g0 + t) + 2 cq + i]
#pragma unroll
                    for (int m = 0; m < MT; ++m) {
                        const int r = 8 * m + rq;
                        if (r >= nb) continue;
                        const int2 pq = Pool.pq[b0 + r];
                        const PairPrim &Pb = S.pp[Ub.pp_off + pq.x];
                        const PairPrim &Pk = S.pp[Uk.pp_off + pq.y];
                        const double p = Pb.esum, qq = Pk.esum, pq_ = p * qq, ps = p + qq;
                        double R2 = 0.0;
#pragma unroll
                        for (int dd = 1; dd < 3; ++dd) {
                            const double R = Pb.cen[dd] - (Pk.cen[dd] + Tsh[dd]);
                            R2 += R * R;
                        }
                        double vK = 0.0, vG = 0.0;
#pragma unroll
                        for (int t = 0; t < NT; ++t) {
                            if (gmb[t] < 0) continue;   // padding nodes
#pragma unroll
                            for (int i = 0; i < 2; ++i) {
                                const int k = 8 * (g0 + t) + 2 * cq + i;
                                const double t2 = tn[k] * tn[k];
                                const double D2 = 1.0 / (pq_ + ps * t2);
                                const double e = (R2 == 0.0) ? 1.0 : exp(-(pq_ * t2 * D2) * R2);
                                const double bse = acc[(m * NT + t) * 2 + i] * (PI2 * D2 * e);
                                vK = fma(bse, wk[k], vK);
                                vG = fma(bse, wg[k], vG);
                            }
                        }
                        const double f = Pool.fac[b0 + r];
                        blk = fma(f, vK, blk);
                        blkG = fma(f, vG, blkG);
                    }
                }
            }
            __syncwarp();
            if (np > nproc) tce_pool_carry(Pool, nproc, np - nproc, lane);
            np -= nproc;
        }
        blk = tce_warp_sum(blk);
        blkG = tce_warp_sum(blkG);
        if (!tce_judge_accepts(fabs(blk - blkG), fabs(blk), A.judge_tol)) {
            if (lane == 0) tce_queue_fallback(A, q);
            __syncwarp();
            continue;
        }
        if (lane == 0) {
            const int fI = S.sh_first[q.x], fJ = S.sh_first[q.y], fK = S.sh_first[q.z], fL = S.sh_first[q.w];
            const int f[4] = {fI, fJ, fK, fL};
            if (S.Q[fI + (long long)S.nbas * fJ] * S.Q[fK + (long long)S.nbas * fL] >= S.thr)
                tce_scatter_jk(S, A.P, A.J, A.K, f, blk, fI, 1, fJ, 1, fK, 1, fL, 1);
        }
        __syncwarp();
    }
}

// ============================================================================
// s/p classes of one periodic direction (compile-time class LA, LB | LC, LD),
// learned grid, the k_quartets_r1 quartet with the node sums on the tensor
// cores.  Per power combination (ia, ib | ic, id) of the periodic direction
// the row is I[pq][k] = sgn sum_n Re[G_n H_n e^{i n phi}] T[n][k]: the A
// fragments are F = Re(G H) cos(n phi) - Im(G H) sin(n phi), cos and sin by
// the same three-term recurrence in steps of four.  The epilogue adds, per
// node and component whose x powers are the combination, w_k I_x I_y I_z with
// the McMurchie-Davidson sums of the real directions
// (ERI_shell_block_toroidal.f90:302-335), as k_quartets_r1.
// ============================================================================
template <int NQ, int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(256, 2) k_quartets_r1_tc(DevSys S, SArgs A)
{
    constexpr int MT = TCE_TC_MT, BT = TCE_TC_BATCH;
    constexpr int NA = LA == 0 ? 1 : 3, NB = LB == 0 ? 1 : 3, NC = LC == 0 ? 1 : 3, ND = LD == 0 ? 1 : 3;
    constexpr int NCQ = NA * NB * NC * ND;
    constexpr int NCOMB = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
    constexpr int NN = LA + LB + LC + LD;
    constexpr int EB = tce_ecount(LA, LB), EK = tce_ecount(LC, LD);
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int rq = lane >> 2, cq = lane & 3;
    const PrimPool Pool = tce_pool(smem, wib);
    // per-lane Kronrod / Gauss block accumulators of the components (shared
    // memory, after the eight pools): [c][lane] and [NCQ + c][lane]
    double *bacc = reinterpret_cast<double *>(reinterpret_cast<char *>(smem) + 8 * (size_t)TCE_POOL_BYTES) +
                   (size_t)wib * 2 * NCQ * 32;

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
                const int nmax = Pool.key[b0];
                int nmr[MT];
#pragma unroll
                for (int m = 0; m < MT; ++m) nmr[m] = (8 * m + rq < nb) ? Pool.key[b0 + 8 * m + rq] : -1;
                auto phase = [&](int m) {
                    const int r = 8 * m + rq;
                    if (r >= nb) return 0.0;
                    const int2 pq = Pool.pq[b0 + r];
                    return S.a[0] * (S.pp[Ub.pp_off + pq.x].cen[0] - (S.pp[Uk.pp_off + pq.y].cen[0] + Tx));
                };
#pragma unroll 1
                for (int g0 = 0; g0 < NQ / 8; g0 += 4) {
                    int gmb[4], nend = -1;
#pragma unroll
                    for (int t = 0; t < 4; ++t) {
                        gmb[t] = gm[g0 + t];
                        nend = gmb[t] > nend ? gmb[t] : nend;
                    }
                    nend = nend < nmax ? nend : nmax;
#pragma unroll 1
                    for (int cmb = 0; cmb < NCOMB; ++cmb) {
                        const int ia = cmb % (LA + 1), ib = (cmb / (LA + 1)) % (LB + 1);
                        const int ic = (cmb / ((LA + 1) * (LB + 1))) % (LC + 1);
                        const int id = cmb / ((LA + 1) * (LB + 1) * (LC + 1));
                        const bool cplx = (ia + ib + ic + id) > 0;
                        const double2 *Gb = S.vec + Ub.vec_off + (((long long)ia * (LB + 1) + ib) * 2 + 0) * Ub.Nlen * nppb;
                        const double2 *Hb = S.vec + Uk.vec_off + (((long long)ic * (LD + 1) + id) * 2 + 1) * Uk.Nlen * nppk;
                        int goff[MT], hoff[MT];
#pragma unroll
                        for (int m = 0; m < MT; ++m) {
                            goff[m] = hoff[m] = 0;
                            if (nmr[m] >= 0) {
                                const int2 pq = Pool.pq[b0 + 8 * m + rq];
                                goff[m] = pq.x;
                                hoff[m] = pq.y;
                            }
                        }
                        double acc[8 * MT];
#pragma unroll
                        for (int x = 0; x < 8 * MT; ++x) acc[x] = 0.0;
                        // cos / sin of n phi and (n - 4) phi, 2 cos(4 phi); G_n, H_n of the next step
                        double cc[MT], cp[MT], sc[MT], sp[MT], c4[MT];
                        double2 gN[MT], hN[MT];
#pragma unroll
                        for (int m = 0; m < MT; ++m) {
                            const double ph = phase(m);
                            sincos((double)cq * ph, &sc[m], &cc[m]);
                            sincos((double)(cq - 4) * ph, &sp[m], &cp[m]);
                            c4[m] = 2.0 * cos(4.0 * ph);
                            const bool ok = cq <= nmr[m];
                            gN[m] = ok ? __ldg(Gb + goff[m] + (size_t)cq * nppb) : make_double2(0.0, 0.0);
                            hN[m] = ok ? __ldg(Hb + hoff[m] + (size_t)cq * nppk) : make_double2(0.0, 0.0);
                        }
                        double tN[4];
#pragma unroll
                        for (int t = 0; t < 4; ++t)
                            tN[t] = (0 <= gmb[t] && cq <= S.ncap) ? __ldg(Tg + (size_t)cq * NQ + 8 * (g0 + t) + rq) : 0.0;
                        for (int s4 = 0; s4 <= nend; s4 += 4) {
                            const int n = s4 + cq, n1 = n + 4;
                            double F[MT], Tb[4];
#pragma unroll
                            for (int m = 0; m < MT; ++m) {
                                const double2 gv = gN[m], hv = hN[m];
                                if (cplx) {
                                    const double ar = gv.x * hv.x - gv.y * hv.y, ai = gv.x * hv.y + gv.y * hv.x;
                                    F[m] = ar * cc[m] - ai * sc[m];
                                } else {
                                    F[m] = gv.x * hv.x * cc[m];
                                }
                                const bool ok = n1 <= nmr[m];
                                gN[m] = ok ? __ldg(Gb + goff[m] + (size_t)n1 * nppb) : make_double2(0.0, 0.0);
                                hN[m] = ok ? __ldg(Hb + hoff[m] + (size_t)n1 * nppk) : make_double2(0.0, 0.0);
                            }
#pragma unroll
                            for (int t = 0; t < 4; ++t) {
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
                            for (int t = 0; t < 4; ++t)
                                if (s4 <= gmb[t]) {
#pragma unroll
                                    for (int m = 0; m < MT; ++m)
                                        tce_dmma(acc[8 * m + 2 * t], acc[8 * m + 2 * t + 1], F[m], Tb[t]);
                                }
                        }
                        const double sgn = cplx ? pow(S.a[0], -(double)(ia + ib + ic + id)) : 1.0;
                        // epilogue per fragment row: components whose x powers are this combination
#pragma unroll
                        for (int m = 0; m < MT; ++m) {
                            if (nmr[m] < 0) continue;
                            const int r = 8 * m + rq;
                            const int2 pq = Pool.pq[b0 + r];
                            const PairPrim &Pb = S.pp[Ub.pp_off + pq.x];
                            const PairPrim &Pk = S.pp[Uk.pp_off + pq.y];
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
                                        for (int t = 0; t <= a + b; ++t)
                                            eb[dr][tce_eoff(LB, a, b) + t] = Ebp[((dr * (LA + 1) + a) * (LB + 1) + b) * TCE_ECO + t];
#pragma unroll
                                for (int a = 0; a <= LC; ++a)
#pragma unroll
                                    for (int b = 0; b <= LD; ++b)
#pragma unroll
                                        for (int t = 0; t <= a + b; ++t)
                                            ek[dr][tce_eoff(LD, a, b) + t] = Ekp[((dr * (LC + 1) + a) * (LD + 1) + b) * TCE_ECO + t];
                            }
                            const double p = Pb.esum, qq = Pk.esum, pq_ = p * qq, ps = p + qq;
                            const double Ry = Pb.cen[1] - Pk.cen[1], Rz = Pb.cen[2] - Pk.cen[2];
                            double val[NCQ], valG[NCQ];
#pragma unroll
                            for (int c = 0; c < NCQ; ++c) val[c] = valG[c] = 0.0;
#pragma unroll
                            for (int t = 0; t < 4; ++t) {
                                if (gmb[t] < 0) continue;
#pragma unroll
                                for (int i = 0; i < 2; ++i) {
                                    const int k = 8 * (g0 + t) + 2 * cq + i;
                                    const double t2 = tn[k] * tn[k];
                                    const double rr = rsqrt(pq_ + ps * t2), D2 = rr * rr;
                                    const double w = pq_ * t2 * D2, rs = PI_D * rr;
                                    double gy[NN + 1], gz[NN + 1];
                                    gy[0] = (Ry == 0.0) ? rs : rs * exp(-w * Ry * Ry);
                                    gz[0] = (Rz == 0.0) ? rs : rs * exp(-w * Rz * Rz);
#pragma unroll
                                    for (int u = 0; u < NN; ++u) {
                                        gy[u + 1] = 2.0 * w * Ry * gy[u] - (u > 0 ? 2.0 * u * w * gy[u - 1] : 0.0);
                                        gz[u + 1] = 2.0 * w * Rz * gz[u] - (u > 0 ? 2.0 * u * w * gz[u - 1] : 0.0);
                                    }
                                    const double xv = acc[8 * m + 2 * t + i] * sgn;
                                    const double xk = xv * wk[k], xkG = xv * wg[k];
#pragma unroll
                                    for (int c = 0; c < NCQ; ++c) {
                                        const int ca = c % NA, cb = (c / NA) % NB, cc_ = (c / (NA * NB)) % NC, cd = c / (NA * NB * NC);
                                        const int cx = tce_pw(LA, ca, 0) + (LA + 1) * (tce_pw(LB, cb, 0) + (LB + 1) * (tce_pw(LC, cc_, 0) + (LC + 1) * tce_pw(LD, cd, 0)));
                                        if (cx != cmb) continue;
                                        double I[2];
#pragma unroll
                                        for (int dr = 0; dr < 2; ++dr) {
                                            const int pa = tce_pw(LA, ca, dr + 1), pb = tce_pw(LB, cb, dr + 1);
                                            const int pc = tce_pw(LC, cc_, dr + 1), pd = tce_pw(LD, cd, dr + 1);
                                            const double *gg = dr == 0 ? gy : gz;
                                            double sacc = 0.0;
#pragma unroll
                                            for (int u = 0; u <= pa + pb; ++u)
#pragma unroll
                                                for (int v = 0; v <= pc + pd; ++v) {
                                                    const double e1 = eb[dr][tce_eoff(LB, pa, pb) + u];
                                                    const double e2 = ek[dr][tce_eoff(LD, pc, pd) + v];
                                                    sacc += ((u & 1) ? -e1 : e1) * e2 * gg[u + v];
                                                }
                                            I[dr] = sacc;
                                        }
                                        val[c] = fma(xk, I[0] * I[1], val[c]);
                                        valG[c] = fma(xkG, I[0] * I[1], valG[c]);
                                    }
                                }
                            }
                            const double fac = Pool.fac[b0 + r];
                            const int i0 = pq.x / Ub.np2, j0 = pq.x - i0 * Ub.np2;
                            const int k0 = pq.y / Uk.np2, l0 = pq.y - k0 * Uk.np2;
#pragma unroll
                            for (int c = 0; c < NCQ; ++c) {
                                const int ca = c % NA, cb = (c / NA) % NB, cc_ = (c / (NA * NB)) % NC, cd = c / (NA * NB * NC);
                                const int cx = tce_pw(LA, ca, 0) + (LA + 1) * (tce_pw(LB, cb, 0) + (LB + 1) * (tce_pw(LC, cc_, 0) + (LC + 1) * tce_pw(LD, cd, 0)));
                                if (cx != cmb) continue;
                                const double cf = S.sh_coef[S.sh_coff[q.x] + ca * npA + i0] * S.sh_coef[S.sh_coff[q.y] + cb * npB + j0] *
                                                  S.sh_coef[S.sh_coff[q.z] + cc_ * npC + k0] * S.sh_coef[S.sh_coff[q.w] + cd * npD + l0];
                                bacc[c * 32 + lane] = fma(fac * cf, val[c], bacc[c * 32 + lane]);
                                bacc[(NCQ + c) * 32 + lane] = fma(fac * cf, valG[c], bacc[(NCQ + c) * 32 + lane]);
                            }
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

static void tc_args(SArgs &A, const SArgsHost &h)
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

int tce_launch_quartets_r1_tc(const DevSys &S, int cls, const SArgsHost &h, int nq, cudaStream_t st)
{
    if (!h.item_rule || !h.rules || !h.rule_T || !h.fb_items || !h.fb_count) return TCE_ERR_ARG;
    if (S.ndp != 1 || (nq != 32 && nq != 64)) return TCE_ERR_UNSUPPORTED;
    SArgs A{};
    tc_args(A, h);
    cudaMemsetAsync(h.next, 0, sizeof(unsigned int), st);
    const int nsm = h.num_sms > 0 ? h.num_sms : 148;
#define TCE_R1_TC(NQv)                                                                     \
    switch (cls) {                                                                         \
    case 1: tc_launch(k_quartets_r1_tc<NQv, 1, 0, 0, 0>, S, A, nsm, st, 3); break;            \
    case 2: tc_launch(k_quartets_r1_tc<NQv, 0, 1, 0, 0>, S, A, nsm, st, 3); break;            \
    case 4: tc_launch(k_quartets_r1_tc<NQv, 0, 0, 1, 0>, S, A, nsm, st, 3); break;            \
    case 8: tc_launch(k_quartets_r1_tc<NQv, 0, 0, 0, 1>, S, A, nsm, st, 3); break;            \
    default: return TCE_ERR_UNSUPPORTED;                                                   \
    }
    if (nq == 32) {
        TCE_R1_TC(32)
    } else {
        TCE_R1_TC(64)
    }
#undef TCE_R1_TC
    return cudaGetLastError() == cudaSuccess ? TCE_OK : TCE_ERR_CUDA;
}

int tce_tc_shapes_s(int nq)
{
    return (nq == 32 || nq == 64) ? 4 : 0;
}

// shape 1: 16 rows x 32 nodes per pass (the default), 2: 32 x 16, 3: 16 x 16,
// 4: 8 rows x 64 nodes (x 32 for 32-node rules)
int tce_launch_quartets_s_tc(const DevSys &S, const SArgsHost &h, int nq, int shape, cudaStream_t st)
{
    if (!h.item_rule || !h.rules || !h.rule_T || !h.fb_items || !h.fb_count) return TCE_ERR_ARG;
    if (S.ndp != 1 || (nq != 32 && nq != 64)) return TCE_ERR_UNSUPPORTED;
    if (shape < 1 || shape > tce_tc_shapes_s(nq)) return TCE_ERR_ARG;
    SArgs A{};
    tc_args(A, h);
    if (cudaMemsetAsync(h.next, 0, sizeof(unsigned int), st) != cudaSuccess) return TCE_ERR_CUDA;
    const int nsm = h.num_sms > 0 ? h.num_sms : 148;
#define TCE_S_TC(NQv)                                                              \
    switch (shape) {                                                               \
    case 1: tc_launch(k_quartets_s_tc<NQv, 2, 4>, S, A, nsm, st); break;           \
    case 2: tc_launch(k_quartets_s_tc<NQv, 4, 2>, S, A, nsm, st); break;           \
    case 3: tc_launch(k_quartets_s_tc<NQv, 2, 2>, S, A, nsm, st); break;           \
    default: tc_launch(k_quartets_s_tc<NQv, 1, 8>, S, A, nsm, st); break;          \
    }
    if (nq == 32) {
        TCE_S_TC(32)
    } else {
        TCE_S_TC(64)
    }
#undef TCE_S_TC
    return cudaGetLastError() == cudaSuccess ? TCE_OK : TCE_ERR_CUDA;
}
