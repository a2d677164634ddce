// tce_kernels.h -- host-side launch interface of the engine's kernels.
#pragma once
#include <cuda_runtime.h>
#include "tce_device.cuh"
#include "../../include/tce.h"

// consumers of a shell-quartet block (k_quartets, k_plain)
#define TCE_MODE_BLOCK    0   // prefactor screens, block written out (Schwarz pass)
#define TCE_MODE_NOSCREEN 1   // no screens, block written out (ps_noscreen)
#define TCE_MODE_PRIMTAB  2   // single primitive pair, no screens -> PairPrim::ps
#define TCE_MODE_JK       3   // fused J/K scatter (direct_JK)
#define TCE_MODE_STORE    4   // stored-ERI scatter (ERI_integral_toroidal)

// t-quadrature of the generic path: TCE_METHOD_* of tce.h (FIXED: the system's
// rule or one dictionary rule, rule_override; LEARNED: per-item dictionary rule
// + Kronrod/Gauss judge, rejects queued; PLAIN: adaptive 15/7 bisection, k_plain)

struct QuartetHostArgs {
    const int4 *items = nullptr;
    const int *prim_sel = nullptr;
    int nitems = 0;
    const unsigned int *nitems_dev = nullptr;   // item count read on the device (fallback lists)
    int mode = TCE_MODE_BLOCK;
    int method = TCE_METHOD_FIXED;
    int prim_screen = 0;
    unsigned int *next = nullptr;
    double *blk_out = nullptr;
    double *blk_out2 = nullptr;      // judge estimate of each block (dictionary rule override)
    const long long *blk_off = nullptr;
    const double *P = nullptr;
    double *J = nullptr, *K = nullptr;
    double *eri = nullptr;
    int eri_size = 0, physicist = 0;
    PairPrim *pp_rw = nullptr;
    int max_ncomb = 1;   // largest (lA+1)(lB+1)(lC+1)(lD+1) among the items
    int max_ncq = 1296;  // largest block (components) among the items
    int num_sms = 148;
    int use_tc = 0;      // rows of one periodic direction on the FP64 tensor cores (32/64-node rules)
    const int *fixed_gmax = nullptr;   // [3*TCE_MAXG] of the system's rule
    // learned grid
    const RuleDev *rules = nullptr;
    const double *rule_T = nullptr, *rule_t = nullptr, *rule_wk = nullptr, *rule_wg = nullptr;
    const int *item_rule = nullptr;
    int rule_override = -1;
    int dict_nq = 32;                // padded node count of the dictionary rules in use (32 or 64)
    double judge_tol = 1e-10;
    int4 *fb_items = nullptr;        // capacity >= nitems
    int *fb_index = nullptr;
    unsigned int *fb_count = nullptr;
    // plain
    double *scratch = nullptr;       // scratch_warps x tce_plain_scratch_per_warp doubles
    long long scratch_warps = 0;
    double plain_tol = 1e-11, plain_scale = 0.6;
    int plain_max_panels = 24;
    const double *gk_u = nullptr, *gk_wk = nullptr, *gk_wg = nullptr;   // 15 nodes on [0,1]
    unsigned long long *node_evals = nullptr;
};

long long tce_plain_scratch_per_warp(const DevSys &S, int max_ncq);
int tce_launch_quartets(const DevSys &S, const QuartetHostArgs &h, cudaStream_t st);
// Load the generic quartet kernel for nq nodes on the current device now (with
// lazy module loading it is otherwise loaded by its first launch).
int tce_preload_quartets(int nq);

// all-s shell quartets, J/K mode (k_quartets_s)
struct SArgsHost {
    const int4 *items = nullptr;
    int nitems = 0;
    int prim_screen = 0;
    unsigned int *next = nullptr;
    const double *P = nullptr;
    double *J = nullptr, *K = nullptr;
    int num_sms = 148;
    // learned grid (the _lg launchers): per-item rules, judge, fallback queue
    const int *item_rule = nullptr;
    const RuleDev *rules = nullptr;
    const double *rule_T = nullptr, *rule_t = nullptr, *rule_wk = nullptr, *rule_wg = nullptr;
    const float *rule_T32 = nullptr;
    double judge_tol = 1e-10;
    int4 *fb_items = nullptr;
    unsigned int *fb_count = nullptr;
};
int tce_launch_quartets_s(const DevSys &S, const SArgsHost &h, cudaStream_t st);
// 1D s/p classes (k_quartets_r1); cls bit i = angular momentum (0/1) of shell i
int tce_launch_quartets_r1(const DevSys &S, int cls, const SArgsHost &h, cudaStream_t st);
// the same kernels with per-item learned-grid rules of nq = 32 or 64 padded
// nodes; fp32: FP32 node sums (one periodic direction only)
int tce_launch_quartets_s_lg(const DevSys &S, const SArgsHost &h, int nq, bool fp32, cudaStream_t st);
int tce_launch_quartets_r1_lg(const DevSys &S, int cls, const SArgsHost &h, int nq, bool fp32, cudaStream_t st);
// all-s quartets of one periodic direction, learned grid, node sums on the FP64
// tensor cores (k_quartets_s_tc, mma.sync m8n8k4)
int tce_launch_quartets_s_tc(const DevSys &S, const SArgsHost &h, int nq, int shape, cudaStream_t st);
// number of tile shapes of the all-s tensor-core kernel for nq-node rules (shapes 1..n)
int tce_tc_shapes_s(int nq);
// s/p classes with one or two p shells of one periodic direction, learned
// grid, tensor-core node sums (k_quartets_sp_tc) in tile shape
// 1..tce_tc_shapes_sp(nq); cls: bit i set when shell i of (A, B | C, D) is p
int tce_launch_quartets_sp_tc(const DevSys &S, int cls, const SArgsHost &h, int nq, int shape, cudaStream_t st);
int tce_tc_shapes_sp(int nq);
inline bool tce_r1_supported(int ndp, int nq, int cls)
{
    return ndp == 1 && nq == 32 && cls >= 0 && cls < 16 && __builtin_popcount(cls) == 1;
}
int tce_launch_t_tables(int nq, int ndp, int ncap, const double *tnode, const double *a, double *tb, int *tnmax,
                        double *Tt, cudaStream_t st);
int tce_launch_pair_scalars(const DevSys &S, long long npp_tot, const int *pp_unit, PairPrim *pp, UnitPair *up,
                            double *ecoef, cudaStream_t st);
int tce_launch_pair_vectors(const DevSys &S, long long npp_tot, const int *pp_unit, const PairPrim *pp, int stride,
                            double *scratch, double2 *vec, cudaStream_t st);
int tce_launch_enumerate(const DevSys &S, const double *Qsh, double Qmax, int4 *items, unsigned long long *count,
                         unsigned long long cap, unsigned long long *nfunc, cudaStream_t st);
int tce_launch_stored_jk(int n1, int nbas, int physicist, const double *P, const double *eri, double *J, double *K,
                         cudaStream_t st);
int tce_launch_sym_fill(int nf, int fpuc, const int *ncl, double *eri, cudaStream_t st);
// Unique quartets in work order (most expensive first, ties by the quartet),
// with their costs; *d_max_ncomb (device) raised to the largest power-combination
// count among them.
int tce_sort_items(const DevSys &S, const int4 *items, long long n, int4 *sorted, double *cost_sorted,
                   int *d_max_ncomb, cudaStream_t st);
// The integral stream of trexio_conv_integrals from the full nbas^4 stored
// integrals on the device: *count entries; the first min(count, cap) packed as
// 1-based (i, j, k, l) into d_index[4 e ..] and their values into d_value.
int tce_trexio_stream(const double *d_eri, long long n, long long cap, int32_t *d_index, double *d_value,
                      long long *count, cudaStream_t st);
int tce_launch_count_work(const DevSys &S, const int4 *items, int nitems, int prim_screen, const int *tnmax,
                          unsigned long long *nprim, double *flops, cudaStream_t st, const int *item_rule = nullptr,
                          const RuleDev *rules = nullptr, const int *rule_tnmax = nullptr);
int tce_launch_fp64_probe(int nsm, int iters, double *sink, cudaStream_t st, long long *flops);
