// tce_quartets.cu -- the generic quartet kernel (sm_100a): every class up to
// d shells, one warp per shell quartet.  ERI_shell_block_toroidal
// (ERI_shell_block_toroidal.f90:28-366) evaluated with a t-quadrature rule
// given as a RuleView (nodes, weights, optional judge weights, the table
// c_n e^{-C_k} I_n(C_k) of the nodes), so the same code serves
//   * the reference rule (32/40-node mapped Gauss-Legendre or a 64/128 table),
//   * the learned grid: a per-quartet mapped Gauss-Kronrod rule picked by the
//     network; the embedded Gauss weights give a second estimate, and the
//     quartet is accepted when the error estimate of its block (block_judge)
//     is <= tol, otherwise it is queued for
//   * the plain method: adaptive bisection of u in [0,1] with a 15-point
//     Kronrod / 7-point Gauss pair per panel, the Bessel columns of each
//     panel's nodes computed on the fly (Miller recurrence as setup_t_tables,
//     clifford_tools.f90:620-709, or Debye-seeded downward recurrence).
// Consumers of a block: Schwarz / parity blocks, the primitive Schwarz table,
// the J/K scatter (direct_JK, eri_direct.f90:331-357) and the stored-ERI
// scatter (ERI_toroidal.f90:416-454).
#include <map>
#include <mutex>
#include <vector>

#include "tce_device.cuh"
#include "tce_kernels.h"

#define PI_D 3.14159265358979323846
#define PLAIN_PMAX 24

struct RuleView {
    const double *T;          // direction d at T + d * strideD, row n at + n * NQ
    long long strideD;
    const double *t, *wk, *wg;   // nodes, weights, judge weights (nullptr: no judge)
    const int *gmax;          // gmax[d * TCE_MAXG + g]: last n with a nonzero entry in node group g
};

struct QuartetArgs {
    const int4 *items;
    const int *prim_sel;
    int nitems;
    const unsigned int *nitems_dev;   // when set, the item count is read on the device
    int mode, method;
    int prim_screen;
    unsigned int *next;
    double *blk_out, *blk_out2;
    const long long *blk_off;
    const double *P;
    double *J, *K;
    double *eri;
    int eri_size, physicist;
    PairPrim *pp_rw;
    int rowcap, cstride, blkcap, warp_smem_doubles;
    int use_tc;
    const int *fixed_gmax;
    // learned grid
    const RuleDev *rules;
    const double *rule_T, *rule_t, *rule_wk, *rule_wg;
    const int *item_rule;
    int rule_override;
    double judge_tol;
    int4 *fb_items;
    int *fb_index;
    unsigned int *fb_count;
    // plain
    double *scratch;
    long long scratch_per_warp, T_doubles;
    double plain_tol, plain_scale;
    int plain_max_panels;
    const double *gk_u, *gk_wk, *gk_wg;
    unsigned long long *node_evals;
};

template <bool RO>
__device__ __forceinline__ double ldT(const double *p)
{
    if (RO) return __ldg(p);
    return *p;
}

// One row I_r(t_k) = sgn sum_n F_n T[n][k] of the nodes of one chunk: the
// 8-node groups g0 .. g0 + 3 (32 nodes, fewer at the end of the rule), out[x]
// for node 8 g0 + x.
template <int NQ, bool RO>
__device__ __forceinline__ void row_dot(const RuleView &R, int d, const double2 *__restrict__ G, int nppb, int ib_,
                                        const double2 *__restrict__ H, int nppk, int ik_, int nm, double phi,
                                        double sgn, int g0, double *out)
{
    constexpr int NG = NQ / 8;
    const double *T = R.T + (size_t)d * R.strideD;
    const int *gm = R.gmax + d * TCE_MAXG;
    double c1, s1;
    sincos(phi, &s1, &c1);
    double acc[32];
#pragma unroll
    for (int x = 0; x < 32; ++x) acc[x] = 0.0;
    double cn = 1.0, sn = 0.0;
    int n = 0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        if (g0 + s >= NG) break;
        int nend = gm[g0 + s];
        nend = nend < nm ? nend : nm;
        for (; n <= nend; ++n) {
            if (n > 0) {
                if ((n & 31) == 0) {
                    sincos((double)n * phi, &sn, &cn);
                } else {
                    double tmp = cn * c1 - sn * s1;
                    sn = sn * c1 + cn * s1;
                    cn = tmp;
                }
            }
            double2 g = __ldg(G + (size_t)n * nppb + ib_);
            double2 h = __ldg(H + (size_t)n * nppk + ik_);
            double ar = g.x * h.x - g.y * h.y, ai = g.x * h.y + g.y * h.x;
            double F = ar * cn - ai * sn;
            const double *Tn = T + (size_t)n * NQ + 8 * g0;
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                if (g >= s && g0 + g < NG) {
#pragma unroll
                    for (int kk = 0; kk < 8; ++kk)
                        acc[8 * g + kk] = fma(F, ldT<RO>(Tn + 8 * g + kk), acc[8 * g + kk]);
                }
            }
        }
    }
#pragma unroll
    for (int x = 0; x < 32; ++x)
        if (8 * g0 + x < NQ) out[x] = acc[x] * sgn;
}

struct QCtx {
    int SI, SJ, SK, SL, nA, nB, nC, nD, lsA, lsB, lsC, lsD, ncomb, ncq, NN, R;
    int cqg;   // lanes per component in the component contraction (power of two)
    UnitPair Ub, Uk;
    double Tsh[3];
};

// per-warp shared memory: [qlist rowcap int2][qfac rowcap][rows rowcap*RS]
// [real nreal*cstride*RS][blkK blkcap][blkG blkcap][extra]; RS = 33 (rows of a
// chunk of 32 nodes plus padding), 17 for the plain method's 16-node panels
struct WarpBuf {
    int2 *qlist;
    double *qfac, *rows, *realb, *blkK, *blkG, *extra;
};

__device__ __forceinline__ WarpBuf warp_buf(const QuartetArgs &A, double *ws, int nreal, int RS)
{
    WarpBuf b;
    b.qlist = reinterpret_cast<int2 *>(ws);
    b.qfac = ws + A.rowcap;
    b.rows = ws + 2 * A.rowcap;
    b.realb = b.rows + (size_t)A.rowcap * RS;
    b.blkK = b.realb + (size_t)nreal * A.cstride * RS;
    b.blkG = b.blkK + A.blkcap;
    b.extra = b.blkG + A.blkcap;
    return b;
}

__device__ __forceinline__ void tce_dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// The rows of row_dot for a batch and periodic direction d on the FP64 tensor
// cores: the batch's nb * ncomb rows of direction d (primitive quartet x power
// combination) in chunks of 32 are the A operand (32 x N, F = Re[G_n H_n
// e^{i n phi}]), the rule's T table of direction d the B operand (N x 32
// nodes per pass);
// mma.sync.m8n8k4 per 8 x 8 tile and step of four orders.  Lane l builds the
// A fragments of rows 8 m + l/4 (m = 0..3) at order 4 s + l%4, cos and sin
// of n phi by the three-term recurrence in steps of four (re-seeded every 32
// orders), and loads the next step's G, H and T before the current step's
// mma instructions.  Nodes of one chunk (8-node groups g0c .. g0c + 3); output
// as row_dot: rows[r * 33 + x] = sgn I_r(t_{8 g0c + x}).
template <int NQ>
__device__ void tc_rows(const DevSys &S, const RuleView &Rv, const QCtx &Q, int nb, const WarpBuf &b, int lane,
                        int g0c, int d)
{
    constexpr int RS = 32 + 1;
    const int rq = lane >> 2, cq = lane & 3;
    const int lsA = Q.lsA, lsB = Q.lsB, lsC = Q.lsC, lsD = Q.lsD, R = Q.R, nd = Q.ncomb;
    const int nppb = Q.Ub.npp, nppk = Q.Uk.npp;
    const int nrows = nb * nd;                 // the batch's rows of direction d
    const double *T = Rv.T + (size_t)d * Rv.strideD;
    const int *gm = Rv.gmax + d * TCE_MAXG;
    // row rr = (primitive quartet p, combination cmb) of direction d -> its place in b.rows
    auto orow = [&](int rr) {
        const int p = rr / nd;
        return p * R + d * nd + (rr - p * nd);
    };
    for (int r0 = 0; r0 < nrows; r0 += 32) {
        int goff[4], hoff[4], nmr[4];
        double sg[4];
        int nmax = -1;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const int r = r0 + 8 * m + rq;
            nmr[m] = -1;
            goff[m] = hoff[m] = 0;
            sg[m] = 0.0;
            if (r < nrows) {
                const int p = r / nd, cmb = r - p * nd;
                const int ia = cmb % (lsA + 1), t1 = cmb / (lsA + 1);
                const int ib = t1 % (lsB + 1), t2 = t1 / (lsB + 1);
                const int ic = t2 % (lsC + 1), id = t2 / (lsC + 1);
                const int2 pq = b.qlist[p];
                const PairPrim &Pb = S.pp[Q.Ub.pp_off + pq.x];
                const PairPrim &Pk = S.pp[Q.Uk.pp_off + pq.y];
                nmr[m] = Pb.N[d] < Pk.N[d] ? Pb.N[d] : Pk.N[d];
                goff[m] = (int)(((((long long)d * (lsA + 1) + ia) * (lsB + 1) + ib) * 2 + 0) * Q.Ub.Nlen * nppb + pq.x);
                hoff[m] = (int)(((((long long)d * (lsC + 1) + ic) * (lsD + 1) + id) * 2 + 1) * Q.Uk.Nlen * nppk + pq.y);
                sg[m] = pow(S.a[d], -(double)(ia + ib + ic + id));
                nmax = nmr[m] > nmax ? nmr[m] : nmax;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) nmax = max(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
        auto phase = [&](int m) {
            const int r = r0 + 8 * m + rq;
            if (r >= nrows) return 0.0;
            const int2 pq = b.qlist[r / nd];
            return S.a[d] * (S.pp[Q.Ub.pp_off + pq.x].cen[d] - (S.pp[Q.Uk.pp_off + pq.y].cen[d] + Q.Tsh[d]));
        };
        const double2 *Gv = S.vec + Q.Ub.vec_off, *Hv = S.vec + Q.Uk.vec_off;
        {
            const int g0 = g0c;
            int gmb[4], nend = -1;
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                gmb[t] = gm[g0 + t];
                nend = gmb[t] > nend ? gmb[t] : nend;
            }
            nend = nend < nmax ? nend : nmax;
            double acc[32];
#pragma unroll
            for (int x = 0; x < 32; ++x) acc[x] = 0.0;
            double cc[4], cp[4], sc[4], sp[4], c4[4];
            double2 gN[4], hN[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const double ph = phase(m);
                sincos((double)cq * ph, &sc[m], &cc[m]);
                sincos((double)(cq - 4) * ph, &sp[m], &cp[m]);
                c4[m] = 2.0 * cos(4.0 * ph);
                const bool ok = cq <= nmr[m];
                gN[m] = ok ? __ldg(Gv + goff[m] + (size_t)cq * nppb) : make_double2(0.0, 0.0);
                hN[m] = ok ? __ldg(Hv + hoff[m] + (size_t)cq * nppk) : make_double2(0.0, 0.0);
            }
            double tN[4];
#pragma unroll
            for (int t = 0; t < 4; ++t)
                tN[t] = (0 <= gmb[t] && cq <= S.ncap) ? __ldg(T + (size_t)cq * NQ + 8 * (g0 + t) + rq) : 0.0;
            for (int s4 = 0; s4 <= nend; s4 += 4) {
                const int n = s4 + cq, n1 = n + 4;
                double F[4], Tb[4];
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const double2 gv = gN[m], hv = hN[m];
                    const double ar = gv.x * hv.x - gv.y * hv.y, ai = gv.x * hv.y + gv.y * hv.x;
                    F[m] = ar * cc[m] - ai * sc[m];
                    const bool ok = n1 <= nmr[m];
                    gN[m] = ok ? __ldg(Gv + goff[m] + (size_t)n1 * nppb) : make_double2(0.0, 0.0);
                    hN[m] = ok ? __ldg(Hv + hoff[m] + (size_t)n1 * nppk) : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    Tb[t] = tN[t];
                    tN[t] = (s4 + 4 <= gmb[t] && n1 <= S.ncap) ? __ldg(T + (size_t)n1 * NQ + 8 * (g0 + t) + rq) : 0.0;
                }
                if (((s4 + 4) & 31) == 0) {
#pragma unroll
                    for (int m = 0; m < 4; ++m) {
                        const double ph = phase(m);
                        sincos((double)n * ph, &sp[m], &cp[m]);
                        sincos((double)n1 * ph, &sc[m], &cc[m]);
                    }
                } else {
#pragma unroll
                    for (int m = 0; m < 4; ++m) {
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
                        for (int m = 0; m < 4; ++m) tce_dmma(acc[8 * m + 2 * t], acc[8 * m + 2 * t + 1], F[m], Tb[t]);
                    }
            }
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const int r = r0 + 8 * m + rq;
                if (r >= nrows) continue;
#pragma unroll
                for (int t = 0; t < 4; ++t)
#pragma unroll
                    for (int i = 0; i < 2; ++i)
                        b.rows[(size_t)orow(r) * RS + 8 * t + 2 * cq + i] = acc[8 * m + 2 * t + i] * sg[m];
            }
        }
    }
}

// Phases 1+2 for a batch of nb primitive quartets, accumulating into blkK (and blkG)
template <int NQ, bool RO>
__device__ void process_batch(const DevSys &S, const RuleView &Rv, const QCtx &Q, int nb, const WarpBuf &b, int lane,
                              int cstride, bool tc)
{
    // The rule's nodes in chunks of NC (32): the rows of one chunk, then its
    // share of every component's node sum.  The row dots restart their order
    // loop per 32 nodes anyway, so chunking costs no extra arithmetic and the
    // per-warp row buffer holds 32 nodes instead of NQ (more warps per SM).
    constexpr int NC = NQ < 32 ? NQ : 32;
    constexpr int RS = NC + 1;
    const int ndp = S.ndp, nreal = 3 - ndp;
    const int lsA = Q.lsA, lsB = Q.lsB, lsC = Q.lsC, lsD = Q.lsD, ncomb = Q.ncomb, R = Q.R;
    const int nppb = Q.Ub.npp, nppk = Q.Uk.npp;
    const int nrows = nb * R;
    const int npA = S.sh_np[Q.SI], npB = S.sh_np[Q.SJ], npC = S.sh_np[Q.SK], npD = S.sh_np[Q.SL];
    const bool judge = Rv.wg != nullptr;
#pragma unroll 1
    for (int k0 = 0; k0 < NQ; k0 += NC) {
        const int g0c = k0 / 8, kn = NQ - k0 < NC ? NQ - k0 : NC;
        bool rows_done = false;
        // tensor-core rows when the launch asks for them (32- and 64-node rules)
        if constexpr (RO && (NQ == 32 || NQ == 64)) {
            if (tc) {
                for (int d = 0; d < ndp; ++d) tc_rows<NQ>(S, Rv, Q, nb, b, lane, g0c, d);
                rows_done = true;
            }
        }
        for (int r = lane; r < (rows_done ? 0 : nrows); r += 32) {
            int p = r / R, rem = r - p * R;
            int d = rem / ncomb, cmb = rem - d * ncomb;
            int ia = cmb % (lsA + 1), t1 = cmb / (lsA + 1);
            int ib = t1 % (lsB + 1), t2 = t1 / (lsB + 1);
            int ic = t2 % (lsC + 1), id = t2 / (lsC + 1);
            int2 pq = b.qlist[p];
            const PairPrim &Pb = S.pp[Q.Ub.pp_off + pq.x];
            const PairPrim &Pk = S.pp[Q.Uk.pp_off + pq.y];
            const double2 *G = S.vec + Q.Ub.vec_off +
                               ((((long long)d * (lsA + 1) + ia) * (lsB + 1) + ib) * 2 + 0) * (long long)Q.Ub.Nlen * nppb;
            const double2 *H = S.vec + Q.Uk.vec_off +
                               ((((long long)d * (lsC + 1) + ic) * (lsD + 1) + id) * 2 + 1) * (long long)Q.Uk.Nlen * nppk;
            int nm = Pb.N[d] < Pk.N[d] ? Pb.N[d] : Pk.N[d];
            double phi = S.a[d] * (Pb.cen[d] - (Pk.cen[d] + Q.Tsh[d]));
            double sgn = pow(S.a[d], -(double)(ia + ib + ic + id));
            row_dot<NQ, RO>(Rv, d, G, nppb, pq.x, H, nppk, pq.y, nm, phi, sgn, g0c, b.rows + (size_t)r * RS);
        }
        __syncwarp();
        for (int p = 0; p < nb; ++p) {
            int2 pq = b.qlist[p];
            const PairPrim &Pb = S.pp[Q.Ub.pp_off + pq.x];
            const PairPrim &Pk = S.pp[Q.Uk.pp_off + pq.y];
            const double pp_ = Pb.esum, qq = Pk.esum;
            if (nreal > 0) {
                const double *Eb = S.ecoef + Q.Ub.e_off + (long long)pq.x * nreal * (lsA + 1) * (lsB + 1) * TCE_ECO;
                const double *Ek = S.ecoef + Q.Uk.e_off + (long long)pq.y * nreal * (lsC + 1) * (lsD + 1) * TCE_ECO;
                for (int k = lane; k < kn; k += 32) {
                    double t = Rv.t[k0 + k], t2 = t * t;
                    const double rr = rsqrt(pp_ * qq + (pp_ + qq) * t2), D2 = rr * rr;
                    double w = pp_ * qq * t2 * D2, rs = PI_D * rr;
                    for (int dr = 0; dr < nreal; ++dr) {
                        int d = ndp + dr;
                        double Rr = Pb.cen[d] - (Pk.cen[d] + Q.Tsh[d]);
                        double gt[4 * TCE_LMAX + 2];
                        gt[0] = (Rr == 0.0) ? rs : rs * exp(-w * Rr * Rr);
                        double gm1 = 0.0, g0 = gt[0];
                        for (int n = 0; n < Q.NN; ++n) {
                            double gp1 = 2.0 * w * Rr * g0 - 2.0 * (double)n * w * gm1;
                            gt[n + 1] = gp1;
                            gm1 = g0;
                            g0 = gp1;
                        }
                        for (int cmb = 0; cmb < ncomb; ++cmb) {
                            int ia = cmb % (lsA + 1), u1 = cmb / (lsA + 1);
                            int ib = u1 % (lsB + 1), u2 = u1 / (lsB + 1);
                            int ic = u2 % (lsC + 1), id = u2 / (lsC + 1);
                            const double *eb = Eb + ((dr * (lsA + 1) + ia) * (lsB + 1) + ib) * TCE_ECO;
                            const double *ek = Ek + ((dr * (lsC + 1) + ic) * (lsD + 1) + id) * TCE_ECO;
                            double val = 0.0;
                            for (int n = 0; n <= ia + ib; ++n) {
                                double sb = (n & 1) ? -eb[n] : eb[n];
                                for (int kk = 0; kk <= ic + id; ++kk) val += sb * ek[kk] * gt[n + kk];
                            }
                            b.realb[((size_t)dr * cstride + cmb) * RS + k] = val;
                        }
                    }
                }
                __syncwarp();
            }
            const double fac = b.qfac[p];
            const double *rowp = b.rows + (size_t)p * R * RS;
            const int i = pq.x / Q.Ub.np2, j = pq.x % Q.Ub.np2;
            const int kp = pq.y / Q.Uk.np2, lp = pq.y % Q.Uk.np2;
            // The component quartets: sum_k w_k I_x I_y I_z per component.  G lanes
            // share one component and split its nodes (G = 32 / next power of two of
            // the component count, at most NQ), so that the warp holds 32 / G
            // components at once and each needs log2(G) shuffles instead of a full
            // warp reduction; each component's block entry has one owning lane.
            const int G = Q.cqg < NC ? Q.cqg : NC;
            const int slots = 32 / G, slot = lane / G, sub = lane - slot * G;
            for (int c0 = 0; c0 < Q.ncq; c0 += slots) {
                const int cq = c0 + slot;
                double vK = 0.0, vG = 0.0;
                int ca = 0, cb = 0, cc = 0, cd = 0;
                if (cq < Q.ncq) {
                    ca = cq % Q.nA;
                    const int r1 = cq / Q.nA;
                    cb = r1 % Q.nB;
                    const int r2 = r1 / Q.nB;
                    cc = r2 % Q.nC;
                    cd = r2 / Q.nC;
                    const int *pa = S.fn_pw + 3 * (S.sh_first[Q.SI] + ca);
                    const int *pb = S.fn_pw + 3 * (S.sh_first[Q.SJ] + cb);
                    const int *pc = S.fn_pw + 3 * (S.sh_first[Q.SK] + cc);
                    const int *pd = S.fn_pw + 3 * (S.sh_first[Q.SL] + cd);
                    const double *rw[3];
    #pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const int cm = pa[d] + (lsA + 1) * (pb[d] + (lsB + 1) * (pc[d] + (lsC + 1) * pd[d]));
                        rw[d] = (d < ndp) ? rowp + ((size_t)d * ncomb + cm) * RS
                                          : b.realb + ((size_t)(d - ndp) * cstride + cm) * RS;
                    }
                    // two partial sums per estimate: shorter dependent FMA chains
                    double vK1 = 0.0, vG1 = 0.0;
                    int k = sub;
                    for (; k + G < kn; k += 2 * G) {
                        const double p0 = rw[0][k] * rw[1][k] * rw[2][k];
                        const double p1 = rw[0][k + G] * rw[1][k + G] * rw[2][k + G];
                        vK = fma(Rv.wk[k0 + k], p0, vK);
                        vK1 = fma(Rv.wk[k0 + k + G], p1, vK1);
                        if (judge) {
                            vG = fma(Rv.wg[k0 + k], p0, vG);
                            vG1 = fma(Rv.wg[k0 + k + G], p1, vG1);
                        }
                    }
                    if (k < kn) {
                        const double p0 = rw[0][k] * rw[1][k] * rw[2][k];
                        vK = fma(Rv.wk[k0 + k], p0, vK);
                        if (judge) vG = fma(Rv.wg[k0 + k], p0, vG);
                    }
                    vK += vK1;
                    vG += vG1;
                }
                for (int o = G >> 1; o > 0; o >>= 1) {
                    vK += __shfl_xor_sync(0xffffffffu, vK, o);
                    if (judge) vG += __shfl_xor_sync(0xffffffffu, vG, o);
                }
                if (cq < Q.ncq && sub == 0) {
                    const double cf = S.sh_coef[S.sh_coff[Q.SI] + ca * npA + i] * S.sh_coef[S.sh_coff[Q.SJ] + cb * npB + j] *
                                      S.sh_coef[S.sh_coff[Q.SK] + cc * npC + kp] * S.sh_coef[S.sh_coff[Q.SL] + cd * npD + lp];
                    b.blkK[cq] += fac * cf * vK;
                    if (judge) b.blkG[cq] += fac * cf * vG;
                }
            }
            __syncwarp();
        }
    }
}

__device__ __forceinline__ void make_ctx(const DevSys &S, int4 q, QCtx &Q)
{
    Q.SI = q.x; Q.SJ = q.y; Q.SK = q.z; Q.SL = q.w;
    Q.nA = S.sh_n[Q.SI]; Q.nB = S.sh_n[Q.SJ]; Q.nC = S.sh_n[Q.SK]; Q.nD = S.sh_n[Q.SL];
    Q.lsA = S.sh_l[Q.SI]; Q.lsB = S.sh_l[Q.SJ]; Q.lsC = S.sh_l[Q.SK]; Q.lsD = S.sh_l[Q.SL];
    Q.ncomb = (Q.lsA + 1) * (Q.lsB + 1) * (Q.lsC + 1) * (Q.lsD + 1);
    Q.ncq = Q.nA * Q.nB * Q.nC * Q.nD;
    {
        int p2 = 1;
        while (p2 < Q.ncq) p2 <<= 1;
        Q.cqg = p2 >= 32 ? 1 : 32 / p2;
    }
    Q.NN = Q.lsA + Q.lsB + Q.lsC + Q.lsD;
    Q.R = Q.ncomb * S.ndp;
    const int cK = Q.SK / S.nshuc;
    const int SK0 = Q.SK - cK * S.nshuc;
    const int SLp = tce_shift_to(Q.SL, cK, S.nshuc, S.ncl);
    Q.Ub = S.up[(long long)Q.SI * S.nsh + Q.SJ];
    Q.Uk = S.up[(long long)SK0 * S.nsh + SLp];
#pragma unroll
    for (int d = 0; d < 3; ++d) Q.Tsh[d] = S.sh_r[3 * Q.SK + d] - S.sh_r[3 * SK0 + d];
}

// The block of one shell quartet with rule Rv: screen and batch the primitive
// quartets, accumulate into b.blkK (and b.blkG); both are zeroed first.
template <int NQ, bool RO>
__device__ void eval_block(const DevSys &S, const QuartetArgs &A, const RuleView &Rv, const QCtx &Q, const WarpBuf &b,
                           int lane, int want)
{
    for (int c = lane; c < Q.ncq; c += 32) {
        b.blkK[c] = 0.0;
        b.blkG[c] = 0.0;
    }
    __syncwarp();
    int B = A.rowcap / Q.R;
    if (B < 1) B = 1;
    const int nppb = Q.Ub.npp, nppk = Q.Uk.npp;
    const long long total = (long long)nppb * nppk;
    int nb = 0;
    for (long long base = 0; base < total; base += 32) {
        long long idx = base + lane;
        bool keep = idx < total;
        int ipb = 0, ipk = 0;
        double fac = 0.0;
        if (keep) {
            ipb = (int)(idx / nppk);
            ipk = (int)(idx - (long long)ipb * nppk);
            const PairPrim &Pb = S.pp[Q.Ub.pp_off + ipb];
            const PairPrim &Pk = S.pp[Q.Uk.pp_off + ipk];
            fac = S.fac_const * Pb.pfac * Pk.pfac;
            if (A.mode == TCE_MODE_PRIMTAB) {
                keep = (ipb == want) && (ipk == want);
            } else if (A.mode != TCE_MODE_NOSCREEN) {
                // prefactor screens (ERI_shell_block_toroidal.f90:191,216) and the
                // primitive Schwarz screen (:217-219)
                double bra = fabs(S.fac_const * Pb.pfac) * Pb.cmax12;
                if (bra * Q.Uk.ket_max <= 2.22e-16) keep = false;
                else if (fabs(fac) * Pb.cmax12 * Pk.cmax12 <= 2.22e-16) keep = false;
                else if (A.prim_screen && Pb.ps * Pk.ps < S.prim_thr) keep = false;
            }
        }
        const unsigned msk = __ballot_sync(0xffffffffu, keep);
        const int pos = __popc(msk & ((1u << lane) - 1u));
        const int cnt = __popc(msk);
        int done = 0;
        while (done < cnt) {
            int take = B - nb;
            if (take > cnt - done) take = cnt - done;
            if (keep && pos >= done && pos < done + take) {
                b.qlist[nb + pos - done] = make_int2(ipb, ipk);
                b.qfac[nb + pos - done] = fac;
            }
            nb += take;
            done += take;
            __syncwarp();
            if (nb == B) {
                process_batch<NQ, RO>(S, Rv, Q, nb, b, lane, A.cstride, A.use_tc != 0);
                nb = 0;
                __syncwarp();
            }
        }
    }
    if (nb > 0) process_batch<NQ, RO>(S, Rv, Q, nb, b, lane, A.cstride, A.use_tc != 0);
    __syncwarp();
}

__device__ __forceinline__ RuleView dict_rule(const DevSys &S, const QuartetArgs &A, int r, bool judge)
{
    const RuleDev &D = A.rules[r];
    RuleView R;
    R.T = A.rule_T + D.T_off;
    R.strideD = (long long)(S.ncap + 1) * D.nq;
    R.t = A.rule_t + D.node_off;
    R.wk = A.rule_wk + D.node_off;
    R.wg = judge ? A.rule_wg + D.node_off : nullptr;
    R.gmax = D.gmax;
    return R;
}

// The consumer of a finished block (J/K, stored ERIs, blocks, primitive table)
__device__ void consume(const DevSys &S, const QuartetArgs &A, const QCtx &Q, const WarpBuf &b, int it, int lane,
                        int want)
{
    const double *blk = b.blkK;
    const int nA = Q.nA, nB = Q.nB, nC = Q.nC, nD = Q.nD;
    if (A.mode == TCE_MODE_BLOCK || A.mode == TCE_MODE_NOSCREEN) {
        double *o = A.blk_out + A.blk_off[it];
        for (int c = lane; c < Q.ncq; c += 32) o[c] = blk[c];
        if (A.blk_out2) {
            double *o2 = A.blk_out2 + A.blk_off[it];
            for (int c = lane; c < Q.ncq; c += 32) o2[c] = b.blkG[c];
        }
    } else if (A.mode == TCE_MODE_PRIMTAB) {
        if (lane == 0) {
            double m = 0.0;
            for (int a = 0; a < nA; ++a)
                for (int c = 0; c < nB; ++c) {
                    double v = sqrt(fabs(blk[a + nA * (c + nB * (a + nA * c))]));
                    if (v > m) m = v;
                }
            A.pp_rw[Q.Ub.pp_off + want].ps = m;
        }
    } else {
        const int fI = S.sh_first[Q.SI], fJ = S.sh_first[Q.SJ], fK = S.sh_first[Q.SK], fL = S.sh_first[Q.SL];
        for (int cq = lane; cq < Q.ncq; cq += 32) {
            int ca = cq % nA, r1 = cq / nA;
            int cb = r1 % nB, r2 = r1 / nB;
            int cc = r2 % nC, cd = r2 / nC;
            int f[4] = {fI + ca, fJ + cb, fK + cc, fL + cd};
            if (S.Q[f[0] + (long long)S.nbas * f[1]] * S.Q[f[2] + (long long)S.nbas * f[3]] < S.thr) continue;
            const double val = blk[cq];
            if (A.mode == TCE_MODE_STORE) {
                const int perm[8][4] = {{0,1,2,3},{1,0,2,3},{0,1,3,2},{1,0,3,2},{2,3,0,1},{3,2,0,1},{2,3,1,0},{3,2,1,0}};
                for (int ip = 0; ip < 8; ++ip) {
                    int g[4];
#pragma unroll
                    for (int ii = 0; ii < 4; ++ii) g[ii] = f[perm[ip][ii]];
                    const int4 rc = __ldg(S.fn_cell + g[0]);
#pragma unroll
                    for (int ii = 0; ii < 4; ++ii) g[ii] = tce_shift_fn(S, g[ii], rc.x, rc.y, rc.z);
                    long long e;
                    if (A.physicist)
                        e = g[0] + (long long)A.eri_size * (g[2] + (long long)S.nbas * (g[1] + (long long)S.nbas * g[3]));
                    else
                        e = g[0] + (long long)A.eri_size * (g[1] + (long long)S.nbas * (g[2] + (long long)S.nbas * g[3]));
                    A.eri[e] = val;
                }
                continue;
            }
            tce_scatter_jk(S, A.P, A.J, A.K, f, val, fI, nA, fJ, nB, fK, nC, fL, nD);
        }
    }
}

// Error estimate of a block from its Kronrod (blkK) and Gauss (blkG) values,
// in the form of QUADPACK's QK rules (Piessens et al. 1983): with
// e = max |K - G| and the block scale M = max |K|,
// est = M min(1, (200 e / M)^1.5)  (est = e when M = 0).
__device__ __forceinline__ double block_judge(const double *K, const double *G, int ncq, int lane)
{
    double e = 0.0, M = 0.0;
    for (int c = lane; c < ncq; c += 32) {
        e = fmax(e, fabs(K[c] - G[c]));
        M = fmax(M, fabs(K[c]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
        M = fmax(M, __shfl_xor_sync(0xffffffffu, M, o));
    }
    if (M <= 0.0 || e <= 0.0) return e;
    const double r = 200.0 * e / M;
    return r >= 1.0 ? M : M * r * sqrt(r);
}

__device__ __forceinline__ int item_count(const QuartetArgs &A)
{
    return A.nitems_dev ? (int)*A.nitems_dev : A.nitems;
}

// method 0: one fixed rule for every item (the system's rule, or dictionary rule
// rule_override, judged when blk_out2 is set); method 1: the learned grid.
template <int NQ>
__global__ void __launch_bounds__(256) k_quartets(DevSys S, QuartetArgs A)
{
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const WarpBuf b = warp_buf(A, smem + (size_t)wib * A.warp_smem_doubles, 3 - S.ndp, (NQ < 32 ? NQ : 32) + 1);
    const bool lg = (A.method == TCE_METHOD_LEARNED);
    RuleView Rfix;
    if (A.rule_override >= 0) {
        Rfix = dict_rule(S, A, A.rule_override, A.blk_out2 != nullptr);
    } else {
        Rfix.T = S.Tt;
        Rfix.strideD = (long long)(S.ncap + 1) * S.nq;
        Rfix.t = S.tnode;
        Rfix.wk = S.tweight;
        Rfix.wg = nullptr;
        Rfix.gmax = A.fixed_gmax;
    }
    const int nitems = item_count(A);
    while (true) {
        int it = 0;
        if (lane == 0) it = (int)atomicAdd(A.next, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= nitems) break;
        QCtx Q;
        make_ctx(S, A.items[it], Q);
        int want = -1;
        if (A.mode == TCE_MODE_PRIMTAB) want = A.prim_sel[2 * it] * Q.Ub.np2 + A.prim_sel[2 * it + 1];
        if (lg) {
            const RuleView R = dict_rule(S, A, A.item_rule[it], true);
            eval_block<NQ, true>(S, A, R, Q, b, lane, want);
            const double e = block_judge(b.blkK, b.blkG, Q.ncq, lane);
            if (!(e <= A.judge_tol)) {      // the judge rejects the predicted rule
                if (lane == 0) {
                    unsigned int slot = atomicAdd(A.fb_count, 1u);
                    A.fb_items[slot] = A.items[it];
                    if (A.fb_index) A.fb_index[slot] = it;
                }
                __syncwarp();
                continue;
            }
        } else {
            eval_block<NQ, true>(S, A, Rfix, Q, b, lane, want);
        }
        consume(S, A, Q, b, it, lane, want);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// The plain method.  Per panel [a,b] of u the warp computes the Bessel columns
// c_n e^{-C} I_n(C), C = 2 t^2 / a^2, of the panel's 15 nodes (lane k: node k)
// into its HBM scratch:
//   C <= 125: Miller recurrence from nneed + 30 + sqrt(80 C), normalised by
//             e^{-C} I_0(C), as the system's t-tables (setup_t_tables,
//             clifford_tools.f90:620-709);
//   C >  125: the two top orders Ns+1, Ns (Ns >= 50, where I_n/I_0 has fallen
//             to about 1e-30 or at nneed + 1) from Debye's uniform asymptotic
//             expansion (Abramowitz & Stegun 9.7.7, terms u_0..u_13), then the
//             stable downward recurrence I_{n-1} = I_{n+1} + (2n/C) I_n.
// Either way the column is truncated 5 orders past the first entry below
// 1e-16 of I~_0, like the t-tables.  Then the warp evaluates the block and
// keeps splitting the panel with the largest error estimate (block_judge) at
// its middle until the summed estimates are below plain_tol or
// plain_max_panels panels are in use.
// ---------------------------------------------------------------------------
#define TCE_DEBYE_K 14
__constant__ double c_debye[TCE_DEBYE_K][TCE_DEBYE_K];   // u_k(p) = p^k sum_j c[k][j] p^{2j}

__device__ __forceinline__ double tce_ive_debye(double nu, double x)
{
    const double z = x / nu, w = sqrt(1.0 + z * z), p = 1.0 / w, p2 = p * p;
    double s = 0.0, pk = 1.0, ik = 1.0;
    const double inv = 1.0 / nu;
#pragma unroll
    for (int k = 0; k < TCE_DEBYE_K; ++k) {
        double P = c_debye[k][k];
        for (int j = k - 1; j >= 0; --j) P = fma(P, p2, c_debye[k][j]);
        s = fma(pk * ik, P, s);
        pk *= p;
        ik *= inv;
    }
    return exp(nu * (1.0 / (w + z) + log(z / (1.0 + w)))) / sqrt(2.0 * PI_D * nu * w) * s;
}

__device__ void plain_columns(const DevSys &S, const QuartetArgs &A, double *T, int nneed, double a, double bnd,
                              double *tn, double *wk, double *wg, int *gmax, int lane)
{
    double t = 0.0, w1 = 0.0, w2 = 0.0;
    if (lane < 15) {
        const double u = a + (bnd - a) * A.gk_u[lane];
        const double jac = (bnd - a) * A.plain_scale / ((1.0 - u) * (1.0 - u));
        t = A.plain_scale * u / (1.0 - u);
        w1 = A.gk_wk[lane] * jac;
        w2 = A.gk_wg[lane] * jac;
    }
    if (lane < 16) {
        tn[lane] = t;
        wk[lane] = w1;
        wg[lane] = w2;
    }
    for (int d = 0; d < S.ndp; ++d) {
        double *Td = T + (size_t)d * (nneed + 1) * 16;
        int tnm = -1;
        if (lane < 15) {
            const double C = 2.0 * t * t / (S.a[d] * S.a[d]);
            if (C < 1e-12) {
                for (int n = 0; n <= nneed; ++n) Td[(size_t)n * 16 + lane] = (n == 0) ? 1.0 : 0.0;
                tnm = 0;
            } else {
                double norm = 1.0;
                if (C <= 125.0) {
                    const long long n0 = (long long)nneed + 30 + (long long)sqrt(80.0 * C);
                    double ip1 = 0.0, ik = 1e-300, im1;
                    for (long long kk = n0; kk >= 1; --kk) {
                        im1 = ip1 + (2.0 * (double)kk / C) * ik;
                        ip1 = ik;
                        ik = im1;
                        if (kk - 1 <= nneed) Td[(size_t)(kk - 1) * 16 + lane] = ik;
                        if (fabs(ik) > 1e250) {
                            for (long long m = kk - 1; m <= nneed; ++m) Td[(size_t)m * 16 + lane] *= 1e-250;
                            ip1 *= 1e-250;
                            ik *= 1e-250;
                        }
                    }
                    norm = tce_iv0_scaled(C) / Td[lane];
                } else {
                    int Ns = (int)ceil(sqrt(140.0 * C)) + 10;
                    if (Ns > nneed + 1) Ns = nneed + 1;
                    if (Ns < 50) Ns = 50;
                    double ip1 = tce_ive_debye((double)(Ns + 1), C), ik = tce_ive_debye((double)Ns, C), im1;
                    for (int n = Ns + 1; n <= nneed; ++n) Td[(size_t)n * 16 + lane] = 0.0;
                    if (Ns <= nneed) Td[(size_t)Ns * 16 + lane] = ik;
                    for (int n = Ns; n >= 1; --n) {
                        im1 = ip1 + (2.0 * (double)n / C) * ik;
                        ip1 = ik;
                        ik = im1;
                        if (n - 1 <= nneed) Td[(size_t)(n - 1) * 16 + lane] = ik;
                    }
                }
                const double w0 = Td[lane];
                tnm = nneed;
                for (int n = 0; n <= nneed; ++n)
                    if (Td[(size_t)n * 16 + lane] < 1e-16 * w0) {
                        tnm = (n + 5 < nneed) ? n + 5 : nneed;
                        break;
                    }
                for (int n = 0; n <= nneed; ++n) {
                    const double v = Td[(size_t)n * 16 + lane] * norm;
                    Td[(size_t)n * 16 + lane] = (n == 0) ? v : (n <= tnm ? 2.0 * v : 0.0);
                }
            }
        } else if (lane == 15) {
            for (int n = 0; n <= nneed; ++n) Td[(size_t)n * 16 + lane] = 0.0;
        }
        int g0 = lane < 8 ? tnm : -1;
        int g1 = (lane >= 8 && lane < 16) ? tnm : -1;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            g0 = max(g0, __shfl_xor_sync(0xffffffffu, g0, o));
            g1 = max(g1, __shfl_xor_sync(0xffffffffu, g1, o));
        }
        if (lane == 0) {
            gmax[d * TCE_MAXG + 0] = g0;
            gmax[d * TCE_MAXG + 1] = g1;
        }
    }
    __syncwarp();
}

__global__ void __launch_bounds__(128) k_plain(DevSys S, QuartetArgs A)
{
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const WarpBuf b = warp_buf(A, smem + (size_t)wib * A.warp_smem_doubles, 3 - S.ndp, 17);
    // extra: panel bounds and errors, the panel's nodes and weights, gmax
    double *pa = b.extra, *pb = pa + PLAIN_PMAX, *perr = pb + PLAIN_PMAX;
    double *tn = perr + PLAIN_PMAX, *wk = tn + 16, *wg = wk + 16;
    int *gmax = reinterpret_cast<int *>(wg + 16);
    const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + wib;
    double *T = A.scratch + gw * A.scratch_per_warp;
    double *pblk = T + A.T_doubles;      // [PLAIN_PMAX][blkcap]
    const int plimit = A.plain_max_panels < PLAIN_PMAX ? A.plain_max_panels : PLAIN_PMAX;
    for (int g = lane; g < 3 * TCE_MAXG; g += 32) gmax[g] = -1;
    __syncwarp();
    const int nitems = item_count(A);
    while (true) {
        int it = 0;
        if (lane == 0) it = (int)atomicAdd(A.next, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= nitems) break;
        QCtx Q;
        make_ctx(S, A.items[it], Q);
        int nneed = 0;
        {   // largest truncation order among the bra's pair primitives (bounds min(N_bra, N_ket))
            int m = 0;
            for (int x = lane; x < Q.Ub.npp; x += 32)
                for (int d = 0; d < S.ndp; ++d) m = max(m, S.pp[Q.Ub.pp_off + x].N[d]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
            nneed = m;
        }
        unsigned long long evals = 0;
        RuleView R;
        R.T = T;
        R.strideD = (long long)(nneed + 1) * 16;
        R.t = tn;
        R.wk = wk;
        R.wg = wg;
        R.gmax = gmax;
        auto eval_panel = [&](int slot, double a, double bnd) {
            plain_columns(S, A, T, nneed, a, bnd, tn, wk, wg, gmax, lane);
            eval_block<16, false>(S, A, R, Q, b, lane, -1);
            const double e = block_judge(b.blkK, b.blkG, Q.ncq, lane);
            for (int c = lane; c < Q.ncq; c += 32) pblk[(size_t)slot * A.blkcap + c] = b.blkK[c];
            if (lane == 0) {
                pa[slot] = a;
                pb[slot] = bnd;
                perr[slot] = e;
            }
            evals += 15;
            __syncwarp();
        };
        eval_panel(0, 0.0, 1.0);
        int np = 1;
        while (np < plimit) {
            double tot = 0.0, worst = -1.0;
            int wi = 0;
            for (int p = 0; p < np; ++p) {
                tot += perr[p];
                if (perr[p] > worst) {
                    worst = perr[p];
                    wi = p;
                }
            }
            if (tot <= A.plain_tol) break;
            const double a = pa[wi], bnd = pb[wi], m = 0.5 * (a + bnd);
            __syncwarp();
            eval_panel(wi, a, m);
            eval_panel(np, m, bnd);
            ++np;
        }
        for (int c = lane; c < Q.ncq; c += 32) {
            double v = 0.0;
            for (int p = 0; p < np; ++p) v += pblk[(size_t)p * A.blkcap + c];
            b.blkK[c] = v;
        }
        __syncwarp();
        if (lane == 0 && A.node_evals) atomicAdd(A.node_evals, evals);
        consume(S, A, Q, b, it, lane, -1);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// launch
// ---------------------------------------------------------------------------
// Warps per block and blocks per SM of k_quartets<NQ> for a per-warp buffer of
// wbytes: the shape with the most warps resident on an SM (shared memory and
// registers decide), found once per (NQ, wbytes) with the occupancy calculator.
template <int NQ>
static int2 quartet_shape(size_t wbytes)
{
    static std::mutex mu;
    static std::map<size_t, int2> known;
    std::lock_guard<std::mutex> lock(mu);
    auto it = known.find(wbytes);
    if (it != known.end()) return it->second;
    int2 best = make_int2(0, 0);   // (warps, blocks per SM)
    for (int w = 8; w >= 1; --w) {
        const size_t smem = wbytes * (size_t)w;
        if (smem > 220 * 1024) continue;
        cudaFuncSetAttribute(k_quartets<NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int per = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_quartets<NQ>, 32 * w, smem) != cudaSuccess) per = 0;
        if (per * w > best.x * best.y) best = make_int2(w, per);
    }
    known[wbytes] = best;
    return best;
}

template <int NQ>
static cudaError_t launch_nq(const DevSys &S, const QuartetArgs &A, size_t wbytes, int nsm, cudaStream_t st)
{
    const int2 sh = quartet_shape<NQ>(wbytes);
    if (sh.x < 1 || sh.y < 1) return cudaErrorInvalidConfiguration;
    const size_t smem = wbytes * (size_t)sh.x;
    cudaFuncSetAttribute(k_quartets<NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_quartets<NQ><<<nsm * sh.y, 32 * sh.x, smem, st>>>(S, A);
    return cudaGetLastError();
}

// Debye polynomials u_k(t) (Abramowitz & Stegun 9.3.9-9.3.10):
//   u_0 = 1, u_{k+1}(t) = t^2 (1 - t^2) u_k'(t) / 2 + (1/8) int_0^t (1 - 5 s^2) u_k(s) ds,
// generated in long double; u_k(t) = t^k sum_j c[k][j] t^{2j}.  Uploaded once per device.
static int upload_debye()
{
    static std::mutex mu;
    static bool done[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return TCE_ERR_CUDA;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return TCE_OK;
    std::vector<std::vector<long double>> U(1, std::vector<long double>(1, 1.0L));
    for (int k = 0; k + 1 < TCE_DEBYE_K; ++k) {
        const std::vector<long double> &u = U.back();
        std::vector<long double> nx(u.size() + 3, 0.0L);
        for (size_t i = 1; i < u.size(); ++i) {         // t^2 (1 - t^2) u' / 2
            const long double du = (long double)i * u[i];
            nx[i + 1] += 0.5L * du;
            nx[i + 3] -= 0.5L * du;
        }
        for (size_t i = 0; i < u.size(); ++i) {         // (1/8) int_0^t (1 - 5 s^2) u
            nx[i + 1] += u[i] / (8.0L * (long double)(i + 1));
            nx[i + 3] -= 5.0L * u[i] / (8.0L * (long double)(i + 3));
        }
        U.push_back(nx);
    }
    double c[TCE_DEBYE_K][TCE_DEBYE_K] = {};
    for (int k = 0; k < TCE_DEBYE_K; ++k)
        for (int j = 0; j <= k; ++j) {
            const size_t e = (size_t)(k + 2 * j);
            c[k][j] = e < U[k].size() ? (double)U[k][e] : 0.0;
        }
    if (cudaMemcpyToSymbol(c_debye, c, sizeof c) != cudaSuccess) return TCE_ERR_CUDA;
    done[dev] = true;
    return TCE_OK;
}

long long tce_plain_scratch_per_warp(const DevSys &S, int max_ncq)
{
    const int blkcap = (max_ncq + 3) / 4 * 4;
    return (long long)S.ndp * (S.ncap + 1) * 16 + (long long)PLAIN_PMAX * blkcap;
}

int tce_launch_quartets(const DevSys &S, const QuartetHostArgs &h, cudaStream_t st)
{
    QuartetArgs A;
    A.items = h.items;
    A.prim_sel = h.prim_sel;
    A.nitems = h.nitems;
    A.nitems_dev = h.nitems_dev;
    A.mode = h.mode;
    A.method = h.method;
    A.prim_screen = h.prim_screen;
    A.next = h.next;
    A.blk_out = h.blk_out;
    A.blk_out2 = h.blk_out2;
    A.blk_off = h.blk_off;
    A.P = h.P;
    A.J = h.J;
    A.K = h.K;
    A.eri = h.eri;
    A.eri_size = h.eri_size;
    A.physicist = h.physicist;
    A.pp_rw = h.pp_rw;
    A.use_tc = h.use_tc;
    A.fixed_gmax = h.fixed_gmax;
    A.rules = h.rules;
    A.rule_T = h.rule_T;
    A.rule_t = h.rule_t;
    A.rule_wk = h.rule_wk;
    A.rule_wg = h.rule_wg;
    A.item_rule = h.item_rule;
    A.rule_override = h.rule_override;
    A.judge_tol = h.judge_tol;
    A.fb_items = h.fb_items;
    A.fb_index = h.fb_index;
    A.fb_count = h.fb_count;
    A.scratch = h.scratch;
    A.plain_tol = h.plain_tol;
    A.plain_scale = h.plain_scale;
    A.plain_max_panels = h.plain_max_panels;
    A.gk_u = h.gk_u;
    A.gk_wk = h.gk_wk;
    A.gk_wg = h.gk_wg;
    A.node_evals = h.node_evals;
    const bool plain = (h.method == TCE_METHOD_PLAIN);
    const bool dict = (h.method == TCE_METHOD_LEARNED) || h.rule_override >= 0;
    if (plain && (h.mode == TCE_MODE_PRIMTAB || !h.scratch || !h.gk_u)) return TCE_ERR_ARG;
    if (dict && (!h.rules || !h.rule_T)) return TCE_ERR_ARG;
    if (h.method == TCE_METHOD_LEARNED && (!h.item_rule || !h.fb_items || !h.fb_count)) return TCE_ERR_ARG;
    if (!plain && !dict && !h.fixed_gmax) return TCE_ERR_ARG;
    const int nq = plain ? 16 : (dict ? h.dict_nq : S.nq);
    const int R = h.max_ncomb * S.ndp;
    const int rowcap = R > 32 ? R : 32;
    const int RS = (nq < 32 ? nq : 32) + 1;   // rows of one chunk of at most 32 nodes
    const int nreal = 3 - S.ndp;
    const int blkcap = (h.max_ncq + 3) / 4 * 4;
    long long wdoubles = 2LL * rowcap + (long long)rowcap * RS + (long long)nreal * h.max_ncomb * RS + 2LL * blkcap + 8;
    if (plain) wdoubles += 3 * PLAIN_PMAX + 48 + 3 * TCE_MAXG;
    wdoubles = (wdoubles + 31) / 32 * 32;
    A.rowcap = rowcap;
    A.cstride = h.max_ncomb;
    A.blkcap = blkcap;
    A.warp_smem_doubles = (int)wdoubles;
    const size_t wbytes = (size_t)wdoubles * sizeof(double);
    int warps = 4;
    while (warps > 1 && wbytes * warps > 220 * 1024) --warps;
    if (wbytes > 220 * 1024) return TCE_ERR_UNSUPPORTED;
    const size_t smem = wbytes * warps;
    if (cudaMemsetAsync(h.next, 0, sizeof(unsigned int), st) != cudaSuccess) return TCE_ERR_CUDA;
    const int nsm = h.num_sms > 0 ? h.num_sms : 148;
    cudaError_t e;
    if (plain) {
        if (upload_debye() != TCE_OK) return TCE_ERR_CUDA;
        A.T_doubles = (long long)S.ndp * (S.ncap + 1) * 16;
        A.scratch_per_warp = tce_plain_scratch_per_warp(S, h.max_ncq);
        cudaFuncSetAttribute(k_plain, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int per = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_plain, 32 * warps, smem);
        if (per < 1) per = 1;
        long long grid = (long long)nsm * per;
        if (grid * warps > h.scratch_warps) grid = h.scratch_warps / warps;
        // a list of known length takes no more warps than it has quartets: the
        // plain list runs next to the learned-grid kernels, and its idle blocks
        // would hold the registers and shared memory they need
        if (!h.nitems_dev && h.nitems > 0) grid = std::min<long long>(grid, (h.nitems + warps - 1) / warps);
        if (grid < 1) return TCE_ERR_NOMEM;
        k_plain<<<(unsigned)grid, 32 * warps, smem, st>>>(S, A);
        e = cudaGetLastError();
    } else if (nq == 32) e = launch_nq<32>(S, A, wbytes, nsm, st);
    else if (nq == 40) e = launch_nq<40>(S, A, wbytes, nsm, st);
    else if (nq == 64) e = launch_nq<64>(S, A, wbytes, nsm, st);
    else if (nq == 128) e = launch_nq<128>(S, A, wbytes, nsm, st);
    else return TCE_ERR_UNSUPPORTED;
    return e == cudaSuccess ? TCE_OK : TCE_ERR_CUDA;
}

int tce_preload_quartets(int nq)
{
    cudaFuncAttributes fa;
    cudaError_t e;
    if (nq == 32) e = cudaFuncGetAttributes(&fa, k_quartets<32>);
    else if (nq == 40) e = cudaFuncGetAttributes(&fa, k_quartets<40>);
    else if (nq == 64) e = cudaFuncGetAttributes(&fa, k_quartets<64>);
    else if (nq == 128) e = cudaFuncGetAttributes(&fa, k_quartets<128>);
    else return TCE_ERR_UNSUPPORTED;
    return e == cudaSuccess ? TCE_OK : TCE_ERR_CUDA;
}
