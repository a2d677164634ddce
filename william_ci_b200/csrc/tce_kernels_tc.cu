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
//
// Also here: the launch of the s/p tensor-core kernel (k_quartets_sp_tc,
// tce_kernels_tc.cuh) for the classes with one p shell; those with two are
// instantiated in tce_kernels_sp2.cu.
#include "tce_kernels_tc.cuh"

// MT row tiles of 8 per warp: batches of 8 MT primitive quartets; acc holds
// the batch's 8 MT rows x 8 NT nodes of one pass (MT x NT tiles, 2 per lane).
// The all-s and the s/p kernels take (MT, NT) as template parameters, their
// tile shapes (tce_tc_shapes_s, tce_tc_shapes_sp) chosen per work list by
// tce_lg_autotune.

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
#pragma unroll 2
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

int tce_tc_shapes_sp(int nq)
{
    return nq == 64 ? 3 : nq == 32 ? 2 : 0;
}

// one p shell.  shape 1: 8 rows x 32 nodes per pass, 2: 16 x 32, 3: 8 x 64
static int sp1_launch(const DevSys &S, int cls, const SArgs &A, int nq, int shape, int nsm, cudaStream_t st)
{
#define TCE_SP1(NQv, MTv, NTv)                                                     \
    switch (cls) {                                                                 \
    case 1: sp_tc_launch<NQv, 1, 0, 0, 0, MTv, NTv>(S, A, nsm, st); break;         \
    case 2: sp_tc_launch<NQv, 0, 1, 0, 0, MTv, NTv>(S, A, nsm, st); break;         \
    case 4: sp_tc_launch<NQv, 0, 0, 1, 0, MTv, NTv>(S, A, nsm, st); break;         \
    case 8: sp_tc_launch<NQv, 0, 0, 0, 1, MTv, NTv>(S, A, nsm, st); break;         \
    default: return TCE_ERR_UNSUPPORTED;                                           \
    }
    if (nq == 32) {
        if (shape == 1) { TCE_SP1(32, 1, 4) } else { TCE_SP1(32, 2, 4) }
    } else {
        if (shape == 1) { TCE_SP1(64, 1, 4) } else if (shape == 2) { TCE_SP1(64, 2, 4) } else { TCE_SP1(64, 1, 8) }
    }
#undef TCE_SP1
    return TCE_OK;
}

int tce_launch_quartets_sp_tc(const DevSys &S, int cls, const SArgsHost &h, int nq, int shape, cudaStream_t st)
{
    if (!h.item_rule || !h.rules || !h.rule_T || !h.fb_items || !h.fb_count) return TCE_ERR_ARG;
    if (S.ndp != 1 || (nq != 32 && nq != 64)) return TCE_ERR_UNSUPPORTED;
    if (shape < 1 || shape > tce_tc_shapes_sp(nq)) return TCE_ERR_ARG;
    const int np = __builtin_popcount(cls & 15);
    if (cls < 1 || cls > 15 || np > 2) return TCE_ERR_UNSUPPORTED;
    SArgs A{};
    tc_args(A, h);
    if (cudaMemsetAsync(h.next, 0, sizeof(unsigned int), st) != cudaSuccess) return TCE_ERR_CUDA;
    const int nsm = h.num_sms > 0 ? h.num_sms : 148;
    const int s = np == 1 ? sp1_launch(S, cls, A, nq, shape, nsm, st) : tce_sp2_launch(S, cls, A, nq, shape, nsm, st);
    if (s != TCE_OK) return s;
    return cudaGetLastError() == cudaSuccess ? TCE_OK : TCE_ERR_CUDA;
}

int tce_tc_shapes_s(int nq)
{
    return (nq == 32 || nq == 64) ? 5 : 0;
}

// shape 1: 16 rows x 32 nodes per pass (the default), 2: 32 x 16, 3: 16 x 16,
// 4: 8 rows x 64 nodes (x 32 for 32-node rules), 5: 8 x 32
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
    case 4: tc_launch(k_quartets_s_tc<NQv, 1, 8>, S, A, nsm, st); break;           \
    default: tc_launch(k_quartets_s_tc<NQv, 1, 4>, S, A, nsm, st); break;          \
    }
    if (nq == 32) {
        TCE_S_TC(32)
    } else {
        TCE_S_TC(64)
    }
#undef TCE_S_TC
    return cudaGetLastError() == cudaSuccess ? TCE_OK : TCE_ERR_CUDA;
}
