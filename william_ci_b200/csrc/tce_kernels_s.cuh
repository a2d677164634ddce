// tce_kernels_s.cuh -- register-resident quartet kernels for the dominant
// classes (sm_100a), J/K mode:
//   k_quartets_s   all-s shell quartets, any number of periodic directions
//   k_quartets_r1  one periodic direction, s and p shells (compile-time class)
// Both evaluate ERI_shell_block_toroidal (ERI_shell_block_toroidal.f90:28-366)
// for one primitive quartet per lane and scatter into J/K like direct_JK
// (eri_direct.f90:331-357).  With LG = true each shell quartet carries its own
// learned-grid rule (T table read from global memory / L2): the kernel sums
// the Kronrod and the embedded Gauss estimates, and the judge (QUADPACK-style
// estimate, as block_judge of the generic kernel) either scatters the block or
// queues the quartet for the plain method.
// Instantiated in tce_kernels_s.cu (system rule) and tce_kernels_slg.cu
// (learned grid).  AT = float gives the FP32-panel variant: the node sums of
// the periodic direction (the F_n x T[n][k] accumulation) in FP32 with an FP32
// copy of the rule's T table; phases, Bessel vectors, the real directions,
// the weights and the J/K accumulation stay FP64.  It is used for quartets
// whose Schwarz bound is below the FP32 threshold.
#pragma once
#include <type_traits>

#include "tce_device.cuh"
#include "tce_kernels.h"

#define PI_D 3.14159265358979323846

// judge of a finished block on every lane: Kronrod values K, Gauss values G
__device__ __forceinline__ bool tce_judge_accepts(double e, double M, double tol)
{
    if (!(M > 0.0) || !(e > 0.0)) return e <= tol;
    const double r = 200.0 * e / M;
    const double est = r >= 1.0 ? M : M * r * sqrt(r);
    return est <= tol;
}

// ============================================================================
// all-s shell quartets (s shells on all four centres): the dominant class of
// the s-rich workloads.  One primitive quartet per lane from start to end:
//   periodic d: I_d(t_k) = sum_n G_n H_n cos(n phi) T_d[n][k]   (real vectors,
//               Chebyshev recurrence for cos(n phi), resynchronised every 32)
//   real d    : closed form for s functions, pi sqrt(D) exp(-w R^2) per direction
//   value     : sum_k w_k prod_d I_d(t_k), contracted over the primitives.
// The T table sits in shared memory (only rows n <= t_nmax of each 8-node
// group), kept primitive quartets are pooled and sorted by truncation order
// before they are cut into batches of 32, the block reduces over the warp,
// lane 0 scatters into J and K.
// ============================================================================
struct SArgs {
    const int4 *items;
    int nitems;
    int prim_screen;
    unsigned int *next;
    const double *P;
    double *J, *K;
    int tsoff[3][TCE_MAXG];   // doubles from the start of the T buffer
    int ts_doubles;           // size of the T buffer
    int t_smem;               // 1: T copied to shared memory, 0: read from global
    // learned grid (LG instantiations)
    const int *item_rule;
    const RuleDev *rules;
    const double *rule_T, *rule_t, *rule_wk, *rule_wg;
    const float *rule_T32;    // FP32 copy of rule_T (FP32-panel instantiations)
    double judge_tol;
    int4 *fb_items;
    unsigned int *fb_count;
};

// Per-warp pool of kept primitive quartets (shared memory): pair indices,
// factor and sort key (the Bessel truncation order min(N_bra, N_ket), summed
// over the periodic directions).  A full pool is sorted by key, largest
// first, before it is cut into batches of 32 lanes, so that the lanes of a
// batch run the n loop for about the same number of orders.
constexpr int TCE_POOL = 128;
constexpr int TCE_POOL_BYTES = 20 * TCE_POOL;   // int2 + double + int per entry
struct PrimPool {
    int2 *pq;
    double *fac;
    int *key;
};
__device__ __forceinline__ PrimPool tce_pool(void *base, int wib)
{
    char *p = reinterpret_cast<char *>(base) + (size_t)wib * TCE_POOL_BYTES;
    return {reinterpret_cast<int2 *>(p), reinterpret_cast<double *>(p + 8 * TCE_POOL),
            reinterpret_cast<int *>(p + 16 * TCE_POOL)};
}

// bitonic sort of entries [0, n) by key, descending (entries [n, m) padded
// with key -1, m the power of two >= n); every lane owns indices lane + 32 j
__device__ __forceinline__ void tce_pool_sort(const PrimPool &P, int n, int lane)
{
    int m = 64;
    while (m < n) m <<= 1;
    for (int i = n + lane; i < m; i += 32) P.key[i] = -1;
    __syncwarp();
    for (int k = 2; k <= m; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < m; i += 32) {
                const int x = i ^ j;
                if (x > i) {
                    const int a = P.key[i], b = P.key[x];
                    const bool down = (i & k) == 0;
                    if (down ? (a < b) : (a > b)) {
                        P.key[i] = b;
                        P.key[x] = a;
                        const int2 t = P.pq[i];
                        P.pq[i] = P.pq[x];
                        P.pq[x] = t;
                        const double f = P.fac[i];
                        P.fac[i] = P.fac[x];
                        P.fac[x] = f;
                    }
                }
            }
            __syncwarp();
        }
}

// move the entries [from, from + rest) of the pool to its front (rest < 32)
__device__ __forceinline__ void tce_pool_carry(const PrimPool &P, int from, int rest, int lane)
{
    int2 q = make_int2(0, 0);
    double f = 0.0;
    int k = 0;
    if (lane < rest) {
        q = P.pq[from + lane];
        f = P.fac[from + lane];
        k = P.key[from + lane];
    }
    __syncwarp();
    if (lane < rest) {
        P.pq[lane] = q;
        P.fac[lane] = f;
        P.key[lane] = k;
    }
    __syncwarp();
}

// queue a quartet the judge rejected (lane 0)
__device__ __forceinline__ void tce_queue_fallback(const SArgs &A, int4 q)
{
    const unsigned int slot = atomicAdd(A.fb_count, 1u);
    A.fb_items[slot] = q;
}

template <int NQ, int NDP, bool LG, typename AT>
__global__ void __launch_bounds__(256, NDP == 1 ? 2 : 1) k_quartets_s(DevSys S, SArgs A)
{
    constexpr int NG = NQ / 8;
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *Tsm = smem;
    const PrimPool Pool = tce_pool(smem + A.ts_doubles, wib);
    // T rows n <= gmax of each group, 8 nodes per row (compact, copied once per CTA)
    if (!LG && A.t_smem) {
        for (int d = 0; d < NDP; ++d)
            for (int g = 0; g < NG; ++g) {
                int rows = S.gmax[d][g] + 1;
                double *dst = Tsm + A.tsoff[d][g];
                const double *src = S.Tt + (size_t)d * (S.ncap + 1) * NQ + 8 * g;
                for (int x = threadIdx.x; x < rows * 8; x += blockDim.x)
                    dst[x] = src[(size_t)(x >> 3) * NQ + (x & 7)];
            }
        __syncthreads();
    }
    const double PI2 = PI_D * PI_D;

    while (true) {
        int it = 0;
        if (lane == 0) it = (int)atomicAdd(A.next, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.nitems) break;
        const int4 q = A.items[it];
        // the quadrature rule of this quartet
        const double *Tg = nullptr, *tn = S.tnode, *wk = S.tweight, *wg = nullptr;
        const float *Tg32 = nullptr;
        const int *gm = nullptr;
        if (LG) {
            const RuleDev *D = A.rules + A.item_rule[it];
            Tg = A.rule_T + D->T_off;
            if (std::is_same<AT, float>::value) Tg32 = A.rule_T32 + D->T_off;
            gm = D->gmax;
            tn = A.rule_t + D->node_off;
            wk = A.rule_wk + D->node_off;
            wg = A.rule_wg + D->node_off;
        }
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
        double blk = 0.0, blkG = 0.0;
        int np = 0;
        for (long long base = 0; base < total; base += 32) {
            long long idx = base + lane;
            bool keep = idx < total;
            int ipb = 0, ipk = 0, key = 0;
            double fac = 0.0;
            if (keep) {
                ipb = (int)(idx / nppk);
                ipk = (int)(idx - (long long)ipb * nppk);
                const PairPrim &Pb = S.pp[Ub.pp_off + ipb];
                const PairPrim &Pk = S.pp[Uk.pp_off + ipk];
                fac = S.fac_const * Pb.pfac * Pk.pfac;
                double bra = fabs(S.fac_const * Pb.pfac) * Pb.cmax12;
                if (bra * Uk.ket_max <= 2.22e-16) keep = false;
                else if (fabs(fac) * Pb.cmax12 * Pk.cmax12 <= 2.22e-16) keep = false;
                else if (A.prim_screen && Pb.ps * Pk.ps < S.prim_thr) keep = false;
                if (keep) {   // fold the four contraction coefficients into the factor
                    fac *= S.sh_coef[S.sh_coff[q.x] + ipb / Ub.np2] * S.sh_coef[S.sh_coff[q.y] + ipb % Ub.np2] *
                           S.sh_coef[S.sh_coff[q.z] + ipk / Uk.np2] * S.sh_coef[S.sh_coff[q.w] + ipk % Uk.np2];
#pragma unroll
                    for (int d = 0; d < NDP; ++d) key += Pb.N[d] < Pk.N[d] ? Pb.N[d] : Pk.N[d];
                }
            }
            const unsigned msk = __ballot_sync(0xffffffffu, keep);
            const int pos = __popc(msk & ((1u << lane) - 1u));
            if (keep) {
                Pool.pq[np + pos] = make_int2(ipb, ipk);
                Pool.fac[np + pos] = fac;
                Pool.key[np + pos] = key;
            }
            np += __popc(msk);
            __syncwarp();
            const bool last = base + 32 >= total;
            if (np > TCE_POOL - 32 || (last && np > 0)) {
                if (np > 32) tce_pool_sort(Pool, np, lane);
                const int nproc = last ? np : (np & ~31);
                for (int b0 = 0; b0 < nproc; b0 += 32) {
                    const int nb = nproc - b0 < 32 ? nproc - b0 : 32;
                    if (lane < nb) {
                        const int2 pq = Pool.pq[b0 + lane];
                        const double f = Pool.fac[b0 + lane];
                        const PairPrim &Pb = S.pp[Ub.pp_off + pq.x];
                        const PairPrim &Pk = S.pp[Uk.pp_off + pq.y];
                        double prod[NDP > 1 ? NQ : 1];
                        double val = 0.0, valG = 0.0;
#pragma unroll
                        for (int d = 0; d < NDP; ++d) {
                            const double *G = reinterpret_cast<const double *>(S.vec + Ub.vec_off + (long long)(2 * d + 0) * Ub.Nlen * nppb) + 2 * pq.x;
                            const double *H = reinterpret_cast<const double *>(S.vec + Uk.vec_off + (long long)(2 * d + 1) * Uk.Nlen * nppk) + 2 * pq.y;
                            const int nm = Pb.N[d] < Pk.N[d] ? Pb.N[d] : Pk.N[d];
                            const double phi = S.a[d] * (Pb.cen[d] - (Pk.cen[d] + Tsh[d]));
                            const double cphi = cos(phi), two_c = 2.0 * cphi;
                            double R2 = 0.0;   // NDP == 1: both real directions at once
                            if (NDP == 1) {
#pragma unroll
                                for (int dd = 1; dd < 3; ++dd) {
                                    double R = Pb.cen[dd] - (Pk.cen[dd] + Tsh[dd]);
                                    R2 += R * R;
                                }
                            }
                            // node passes of up to 32 nodes: 32 accumulators, folded at the end of each pass
#pragma unroll
                            for (int g0 = 0; g0 < NG; g0 += 4) {
                                AT acc[32];
#pragma unroll
                                for (int k = 0; k < 32; ++k) acc[k] = (AT)0;
                                double cn = 1.0, cprev = cphi;        // cos(n phi), cos((n-1) phi) at n = 0
                                double gN = __ldg(G), hN = __ldg(H);  // values of row n (prefetched)
                                int n = 0;
#pragma unroll
                                for (int sgm = 0; sgm < 4; ++sgm) {
                                    if (g0 + sgm >= NG) break;
                                    int nend = LG ? gm[d * TCE_MAXG + g0 + sgm] : S.gmax[d][g0 + sgm];
                                    nend = nend < nm ? nend : nm;
                                    for (; n <= nend; ++n) {
                                        const double gv = gN, hv = hN;
                                        if (n + 1 <= nm) {
                                            gN = __ldg(G + 2 * (size_t)(n + 1) * nppb);
                                            hN = __ldg(H + 2 * (size_t)(n + 1) * nppk);
                                        }
                                        const double F = gv * hv * cn;
                                        double cnext;
                                        if (((n + 1) & 31) == 0) cnext = cos((double)(n + 1) * phi);
                                        else cnext = two_c * cn - cprev;
                                        cprev = cn;
                                        cn = cnext;
#pragma unroll
                                        for (int g = 0; g < 4; ++g) {
                                            if (g >= sgm && g0 + g < NG) {
                                                if constexpr (std::is_same<AT, float>::value) {
                                                    const float4 *T4 = reinterpret_cast<const float4 *>(
                                                        Tg32 + ((size_t)d * (S.ncap + 1) + n) * NQ + 8 * (g0 + g));
                                                    const float Ff = (float)F;
#pragma unroll
                                                    for (int kk = 0; kk < 2; ++kk) {
                                                        const float4 t = T4[kk];
                                                        acc[8 * g + 4 * kk] = fmaf(Ff, t.x, acc[8 * g + 4 * kk]);
                                                        acc[8 * g + 4 * kk + 1] = fmaf(Ff, t.y, acc[8 * g + 4 * kk + 1]);
                                                        acc[8 * g + 4 * kk + 2] = fmaf(Ff, t.z, acc[8 * g + 4 * kk + 2]);
                                                        acc[8 * g + 4 * kk + 3] = fmaf(Ff, t.w, acc[8 * g + 4 * kk + 3]);
                                                    }
                                                } else {
                                                    const double *Tr =
                                                        LG ? Tg + ((size_t)d * (S.ncap + 1) + n) * NQ + 8 * (g0 + g)
                                                           : (A.t_smem ? Tsm + A.tsoff[d][g0 + g] + 8 * n
                                                                       : S.Tt + ((size_t)d * (S.ncap + 1) + n) * NQ + 8 * (g0 + g));
                                                    const double2 *T2 = reinterpret_cast<const double2 *>(Tr);
#pragma unroll
                                                    for (int kk = 0; kk < 4; ++kk) {
                                                        const double2 t = T2[kk];
                                                        acc[8 * g + 2 * kk] = fma(F, t.x, acc[8 * g + 2 * kk]);
                                                        acc[8 * g + 2 * kk + 1] = fma(F, t.y, acc[8 * g + 2 * kk + 1]);
                                                    }
                                                }
                                            }
                                        }
                                    }
                                }
                                // fold the pass's nodes k = 8 g0 + x
#pragma unroll
                                for (int x = 0; x < 32; ++x) {
                                    const int k = 8 * g0 + x;
                                    if (k >= NQ) break;
                                    if (NDP == 1) {
                                        const double p = Pb.esum, qq = Pk.esum, pq_ = p * qq, ps = p + qq;
                                        const double t2 = tn[k] * tn[k];
                                        const double D2 = 1.0 / (pq_ + ps * t2);
                                        const double e = (R2 == 0.0) ? 1.0 : exp(-(pq_ * t2 * D2) * R2);
                                        if (LG) {
                                            const double base = (double)acc[x] * (PI2 * D2 * e);
                                            val = fma(base, wk[k], val);
                                            valG = fma(base, wg[k], valG);
                                        } else {
                                            val = fma((double)acc[x], S.tweight[k] * PI2 * D2 * e, val);
                                        }
                                    } else if (d == 0) {
                                        prod[k < (NDP > 1 ? NQ : 1) ? k : 0] = LG ? (double)acc[x] : (double)acc[x] * S.tweight[k];
                                    } else {
                                        prod[k < (NDP > 1 ? NQ : 1) ? k : 0] *= (double)acc[x];
                                    }
                                }
                            }
                        }
                        if (NDP == 2) {
                            const double p = Pb.esum, qq = Pk.esum, pq_ = p * qq, ps = p + qq;
                            const double R = Pb.cen[2] - (Pk.cen[2] + Tsh[2]);
                            const double R2 = R * R;
#pragma unroll
                            for (int k = 0; k < NQ; ++k) {
                                const double t2 = tn[k] * tn[k];
                                const double D2 = 1.0 / (pq_ + ps * t2);
                                const double e = (R2 == 0.0) ? 1.0 : exp(-(pq_ * t2 * D2) * R2);
                                const double base = prod[k < (NDP > 1 ? NQ : 1) ? k : 0] * (PI_D * sqrt(D2) * e);
                                if (LG) {
                                    val = fma(base, wk[k], val);
                                    valG = fma(base, wg[k], valG);
                                } else {
                                    val = fma(prod[k < (NDP > 1 ? NQ : 1) ? k : 0], PI_D * sqrt(D2) * e, val);
                                }
                            }
                        } else if (NDP == 3) {
#pragma unroll
                            for (int k = 0; k < NQ; ++k) {
                                if (LG) {
                                    val = fma(prod[k < (NDP > 1 ? NQ : 1) ? k : 0], wk[k], val);
                                    valG = fma(prod[k < (NDP > 1 ? NQ : 1) ? k : 0], wg[k], valG);
                                } else {
                                    val += prod[k < (NDP > 1 ? NQ : 1) ? k : 0];
                                }
                            }
                        }
                        blk = fma(f, val, blk);
                        if (LG) blkG = fma(f, valG, blkG);
                    }
                }
                __syncwarp();
                if (np > nproc) tce_pool_carry(Pool, nproc, np - nproc, lane);
                np -= nproc;
            }
        }
        blk = tce_warp_sum(blk);
        if (LG) {
            blkG = tce_warp_sum(blkG);
            if (!tce_judge_accepts(fabs(blk - blkG), fabs(blk), A.judge_tol)) {
                if (lane == 0) tce_queue_fallback(A, q);
                __syncwarp();
                continue;
            }
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
// 1D (ndp = 1) classes with s and p shells, compile-time class (LA,LB|LC,LD):
// one primitive quartet per lane from start to end.  For each power
// combination of the periodic direction (x) the lane builds the row
// I_x(t_k) = sgn sum_n Re[G_n H_n e^{i n phi}] T[n][k] into 32 accumulators,
// then adds w_k I_x I_y I_z of every component quartet whose x powers match
// that combination; the real directions use the McMurchie-Davidson sums
// S_N = sum (-1)^tau E_tau E'_nu and g_N(t) (ERI_shell_block_toroidal.f90:302-335).
// Components follow the reference order (s; px, py, pz).
// ============================================================================
__host__ __device__ constexpr int tce_pw(int l, int comp, int dir) { return l == 0 ? 0 : (comp == dir ? 1 : 0); }
// compact index of E_t(i,j) for i <= LI, j <= LJ, t <= i + j (i-major)
__host__ __device__ constexpr int tce_eoff(int LJ, int i, int j)
{
    int o = 0;
    for (int a = 0; a <= i; ++a)
        for (int b = 0; b <= LJ; ++b) {
            if (a == i && b == j) return o;
            o += a + b + 1;
        }
    return o;
}
__host__ __device__ constexpr int tce_ecount(int LI, int LJ) { return tce_eoff(LJ, LI, LJ) + LI + LJ + 1; }

template <int NQ, int LA, int LB, int LC, int LD, bool LG, typename AT>
__global__ void __launch_bounds__(256, LG ? 2 : 1) k_quartets_r1(DevSys S, SArgs A)
{
    constexpr int NG = NQ / 8;
    constexpr int NA = LA == 0 ? 1 : 3, NB = LB == 0 ? 1 : 3, NC = LC == 0 ? 1 : 3, ND = LD == 0 ? 1 : 3;
    constexpr int NCQ = NA * NB * NC * ND;
    constexpr int NCOMB = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
    constexpr int NN = LA + LB + LC + LD;
    constexpr int EB = tce_ecount(LA, LB), EK = tce_ecount(LC, LD);
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *Tsm = smem;
    const PrimPool Pool = tce_pool(smem + A.ts_doubles, wib);
    if (!LG && A.t_smem) {
        for (int g = 0; g < NG; ++g) {
            int rows = S.gmax[0][g] + 1;
            double *dst = Tsm + A.tsoff[0][g];
            const double *src = S.Tt + 8 * g;
            for (int x = threadIdx.x; x < rows * 8; x += blockDim.x) dst[x] = src[(size_t)(x >> 3) * NQ + (x & 7)];
        }
        __syncthreads();
    }

    while (true) {
        int it = 0;
        if (lane == 0) it = (int)atomicAdd(A.next, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.nitems) break;
        const int4 q = A.items[it];
        const double *Tg = nullptr, *tn = S.tnode, *wk = S.tweight, *wg = nullptr;
        const float *Tg32 = nullptr;
        const int *gm = nullptr;
        if (LG) {
            const RuleDev *D = A.rules + A.item_rule[it];
            Tg = A.rule_T + D->T_off;
            if (std::is_same<AT, float>::value) Tg32 = A.rule_T32 + D->T_off;
            gm = D->gmax;
            tn = A.rule_t + D->node_off;
            wk = A.rule_wk + D->node_off;
            wg = A.rule_wg + D->node_off;
        }
        const int cK = q.z / S.nshuc;
        const int SK0 = q.z - cK * S.nshuc;
        const int SLp = tce_shift_to(q.w, cK, S.nshuc, S.ncl);
        const UnitPair Ub = S.up[(long long)q.x * S.nsh + q.y];
        const UnitPair Uk = S.up[(long long)SK0 * S.nsh + SLp];
        const double Tx = S.sh_r[3 * q.z] - S.sh_r[3 * SK0];
        const int nppb = Ub.npp, nppk = Uk.npp;
        const int npA = S.sh_np[q.x], npB = S.sh_np[q.y], npC = S.sh_np[q.z], npD = S.sh_np[q.w];
        const long long total = (long long)nppb * nppk;
        double blk[NCQ], blkG[LG ? NCQ : 1];
#pragma unroll
        for (int c = 0; c < NCQ; ++c) blk[c] = 0.0;
#pragma unroll
        for (int c = 0; c < (LG ? NCQ : 1); ++c) blkG[c] = 0.0;
        int np = 0;
        for (long long base = 0; base < total; base += 32) {
            long long idx = base + lane;
            bool keep = idx < total;
            int ipb = 0, ipk = 0, key = 0;
            double fac = 0.0;
            if (keep) {
                ipb = (int)(idx / nppk);
                ipk = (int)(idx - (long long)ipb * nppk);
                const PairPrim &Pb = S.pp[Ub.pp_off + ipb];
                const PairPrim &Pk = S.pp[Uk.pp_off + ipk];
                fac = S.fac_const * Pb.pfac * Pk.pfac;
                double bra = fabs(S.fac_const * Pb.pfac) * Pb.cmax12;
                if (bra * Uk.ket_max <= 2.22e-16) keep = false;
                else if (fabs(fac) * Pb.cmax12 * Pk.cmax12 <= 2.22e-16) keep = false;
                else if (A.prim_screen && Pb.ps * Pk.ps < S.prim_thr) keep = false;
                key = Pb.N[0] < Pk.N[0] ? Pb.N[0] : Pk.N[0];
            }
            const unsigned msk = __ballot_sync(0xffffffffu, keep);
            const int pos = __popc(msk & ((1u << lane) - 1u));
            if (keep) {
                Pool.pq[np + pos] = make_int2(ipb, ipk);
                Pool.fac[np + pos] = fac;
                Pool.key[np + pos] = key;
            }
            np += __popc(msk);
            __syncwarp();
            const bool last = base + 32 >= total;
            if (np > TCE_POOL - 32 || (last && np > 0)) {
                if (np > 32) tce_pool_sort(Pool, np, lane);
                const int nproc = last ? np : (np & ~31);
                for (int b0 = 0; b0 < nproc; b0 += 32) {
                    const int nb = nproc - b0 < 32 ? nproc - b0 : 32;
                    if (lane < nb) {
                        const int2 pq = Pool.pq[b0 + lane];
                        const PairPrim &Pb = S.pp[Ub.pp_off + pq.x];
                        const PairPrim &Pk = S.pp[Uk.pp_off + pq.y];
                        const int i = pq.x / Ub.np2, j = pq.x - i * Ub.np2;
                        const int kp = pq.y / Uk.np2, lp = pq.y - kp * Uk.np2;
                        // Hermite coefficients of the real directions y (dr=0), z (dr=1)
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
                        const int nm = Pb.N[0] < Pk.N[0] ? Pb.N[0] : Pk.N[0];
                        const double phi = S.a[0] * (Pb.cen[0] - (Pk.cen[0] + Tx));
                        double cphi, sphi;
                        sincos(phi, &sphi, &cphi);
                        double val[NCQ], valG[LG ? NCQ : 1];
#pragma unroll
                        for (int c = 0; c < NCQ; ++c) val[c] = 0.0;
#pragma unroll
                        for (int c = 0; c < (LG ? NCQ : 1); ++c) valG[c] = 0.0;
                        // node passes of up to 32 nodes (32 accumulators per power combination)
#pragma unroll
                        for (int g0 = 0; g0 < NG; g0 += 4) {
#pragma unroll
                        for (int cmb = 0; cmb < NCOMB; ++cmb) {
                            const int ia = cmb % (LA + 1), ib = (cmb / (LA + 1)) % (LB + 1);
                            const int ic = (cmb / ((LA + 1) * (LB + 1))) % (LC + 1);
                            const int id = cmb / ((LA + 1) * (LB + 1) * (LC + 1));
                            const bool cplx = (ia + ib + ic + id) > 0;
                            const double2 *G = S.vec + Ub.vec_off +
                                               ((((long long)0 * (LA + 1) + ia) * (LB + 1) + ib) * 2 + 0) * Ub.Nlen * nppb + pq.x;
                            const double2 *H = S.vec + Uk.vec_off +
                                               ((((long long)0 * (LC + 1) + ic) * (LD + 1) + id) * 2 + 1) * Uk.Nlen * nppk + pq.y;
                            AT acc[32];
#pragma unroll
                            for (int k = 0; k < 32; ++k) acc[k] = (AT)0;
                            double cn = 1.0, sn = 0.0;
                            double2 gN = __ldg(G), hN = __ldg(H);
                            int n = 0;
#pragma unroll
                            for (int sgm = 0; sgm < 4; ++sgm) {
                                if (g0 + sgm >= NG) break;
                                int nend = LG ? gm[g0 + sgm] : S.gmax[0][g0 + sgm];
                                nend = nend < nm ? nend : nm;
                                for (; n <= nend; ++n) {
                                    const double2 gv = gN, hv = hN;
                                    if (n + 1 <= nm) {
                                        gN = __ldg(G + (size_t)(n + 1) * nppb);
                                        hN = __ldg(H + (size_t)(n + 1) * nppk);
                                    }
                                    double F;
                                    if (cplx) {
                                        const double ar = gv.x * hv.x - gv.y * hv.y, ai = gv.x * hv.y + gv.y * hv.x;
                                        F = ar * cn - ai * sn;
                                    } else {
                                        F = gv.x * hv.x * cn;
                                    }
                                    if (((n + 1) & 31) == 0) {
                                        sincos((double)(n + 1) * phi, &sn, &cn);
                                    } else {
                                        const double t = cn * cphi - sn * sphi;
                                        sn = sn * cphi + cn * sphi;
                                        cn = t;
                                    }
#pragma unroll
                                    for (int g = 0; g < 4; ++g) {
                                        if (g >= sgm && g0 + g < NG) {
                                            if constexpr (std::is_same<AT, float>::value) {
                                                const float4 *T4 =
                                                    reinterpret_cast<const float4 *>(Tg32 + (size_t)n * NQ + 8 * (g0 + g));
                                                const float Ff = (float)F;
#pragma unroll
                                                for (int kk = 0; kk < 2; ++kk) {
                                                    const float4 t = T4[kk];
                                                    acc[8 * g + 4 * kk] = fmaf(Ff, t.x, acc[8 * g + 4 * kk]);
                                                    acc[8 * g + 4 * kk + 1] = fmaf(Ff, t.y, acc[8 * g + 4 * kk + 1]);
                                                    acc[8 * g + 4 * kk + 2] = fmaf(Ff, t.z, acc[8 * g + 4 * kk + 2]);
                                                    acc[8 * g + 4 * kk + 3] = fmaf(Ff, t.w, acc[8 * g + 4 * kk + 3]);
                                                }
                                            } else {
                                                const double2 *T2 = reinterpret_cast<const double2 *>(
                                                    LG ? Tg + (size_t)n * NQ + 8 * (g0 + g)
                                                       : (A.t_smem ? Tsm + A.tsoff[0][g0 + g] + 8 * n
                                                                   : S.Tt + (size_t)n * NQ + 8 * (g0 + g)));
#pragma unroll
                                                for (int kk = 0; kk < 4; ++kk) {
                                                    const double2 t = T2[kk];
                                                    acc[8 * g + 2 * kk] = fma(F, t.x, acc[8 * g + 2 * kk]);
                                                    acc[8 * g + 2 * kk + 1] = fma(F, t.y, acc[8 * g + 2 * kk + 1]);
                                                }
                                            }
                                        }
                                    }
                                }
                            }
                            const double sgn = (ia + ib + ic + id) == 0 ? 1.0 : pow(S.a[0], -(double)(ia + ib + ic + id));
                            // components whose x powers are this combination, nodes k = 8 g0 + x
#pragma unroll
                            for (int x = 0; x < 32; ++x) {
                                const int k = 8 * g0 + x;
                                if (k >= NQ) break;
                                const double t2 = tn[k] * tn[k];
                                // D2 = 1 / (pq + (p + q) t^2) and PI sqrt(D2) from one reciprocal square root
                                const double rr = rsqrt(pq_ + ps * t2), D2 = rr * rr;
                                const double w = pq_ * t2 * D2, rs = PI_D * rr;
                                double gy[NN + 1], gz[NN + 1];
                                gy[0] = (Ry == 0.0) ? rs : rs * exp(-w * Ry * Ry);
                                gz[0] = (Rz == 0.0) ? rs : rs * exp(-w * Rz * Rz);
#pragma unroll
                                for (int m = 0; m < NN; ++m) {
                                    gy[m + 1] = 2.0 * w * Ry * gy[m] - (m > 0 ? 2.0 * m * w * gy[m - 1] : 0.0);
                                    gz[m + 1] = 2.0 * w * Rz * gz[m] - (m > 0 ? 2.0 * m * w * gz[m - 1] : 0.0);
                                }
                                const double xk = (double)acc[x] * sgn * wk[k];
                                const double xkG = LG ? (double)acc[x] * sgn * wg[k] : 0.0;
#pragma unroll
                                for (int c = 0; c < NCQ; ++c) {
                                    const int ca = c % NA, cb = (c / NA) % NB, cc = (c / (NA * NB)) % NC, cd = c / (NA * NB * NC);
                                    const int cx = tce_pw(LA, ca, 0) + (LA + 1) * (tce_pw(LB, cb, 0) + (LB + 1) * (tce_pw(LC, cc, 0) + (LC + 1) * tce_pw(LD, cd, 0)));
                                    if (cx != cmb) continue;
                                    double I[2];
#pragma unroll
                                    for (int dr = 0; dr < 2; ++dr) {
                                        const int pa = tce_pw(LA, ca, dr + 1), pb = tce_pw(LB, cb, dr + 1);
                                        const int pc = tce_pw(LC, cc, dr + 1), pd = tce_pw(LD, cd, dr + 1);
                                        const double *gg = dr == 0 ? gy : gz;
                                        double sacc = 0.0;
#pragma unroll
                                        for (int nn = 0; nn <= pa + pb; ++nn)
#pragma unroll
                                            for (int kk = 0; kk <= pc + pd; ++kk) {
                                                const double e1 = eb[dr][tce_eoff(LB, pa, pb) + nn];
                                                const double e2 = ek[dr][tce_eoff(LD, pc, pd) + kk];
                                                sacc += ((nn & 1) ? -e1 : e1) * e2 * gg[nn + kk];
                                            }
                                        I[dr] = sacc;
                                    }
                                    val[c] = fma(xk, I[0] * I[1], val[c]);
                                    if (LG) valG[LG ? c : 0] = fma(xkG, I[0] * I[1], valG[LG ? c : 0]);
                                }
                            }
                        }
                        }
                        const double fac = Pool.fac[b0 + lane];
#pragma unroll
                        for (int c = 0; c < NCQ; ++c) {
                            const int ca = c % NA, cb = (c / NA) % NB, cc = (c / (NA * NB)) % NC, cd = c / (NA * NB * NC);
                            const double cf = S.sh_coef[S.sh_coff[q.x] + ca * npA + i] * S.sh_coef[S.sh_coff[q.y] + cb * npB + j] *
                                              S.sh_coef[S.sh_coff[q.z] + cc * npC + kp] * S.sh_coef[S.sh_coff[q.w] + cd * npD + lp];
                            blk[c] = fma(fac * cf, val[c], blk[c]);
                            if (LG) blkG[LG ? c : 0] = fma(fac * cf, valG[LG ? c : 0], blkG[LG ? c : 0]);
                        }
                    }
                }
                __syncwarp();
                if (np > nproc) tce_pool_carry(Pool, nproc, np - nproc, lane);
                np -= nproc;
            }
        }
        const int fI = S.sh_first[q.x], fJ = S.sh_first[q.y], fK = S.sh_first[q.z], fL = S.sh_first[q.w];
#pragma unroll
        for (int c = 0; c < NCQ; ++c) blk[c] = tce_warp_sum(blk[c]);
        if (LG) {
            double e = 0.0, M = 0.0;
#pragma unroll
            for (int c = 0; c < NCQ; ++c) {
                const double vg = tce_warp_sum(blkG[LG ? c : 0]);
                e = fmax(e, fabs(blk[c] - vg));
                M = fmax(M, fabs(blk[c]));
            }
            if (!tce_judge_accepts(e, M, A.judge_tol)) {
                if (lane == 0) tce_queue_fallback(A, q);
                __syncwarp();
                continue;
            }
        }
#pragma unroll
        for (int c = 0; c < NCQ; ++c) {
            const double v = blk[c];
            if (lane == (c & 31)) {
                const int ca = c % NA, cb = (c / NA) % NB, cc = (c / (NA * NB)) % NC, cd = c / (NA * NB * NC);
                const int f[4] = {fI + ca, fJ + cb, fK + cc, fL + cd};
                if (S.Q[f[0] + (long long)S.nbas * f[1]] * S.Q[f[2] + (long long)S.nbas * f[3]] >= S.thr)
                    tce_scatter_jk(S, A.P, A.J, A.K, f, v, fI, NA, fJ, NB, fK, NC, fL, ND);
            }
        }
        __syncwarp();
    }
}

