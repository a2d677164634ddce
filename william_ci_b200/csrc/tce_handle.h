// tce_handle.h -- host-side state of one libtce handle and the helpers the
// host translation units share (error reporting, device allocation).
#pragma once
#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "tce_kernels.h"

namespace tcehost {

constexpr double kPi = 3.14159265358979323846;

struct Handle {
    std::string err;
    // system scalars
    int ndp = 0, nq = 0, ncap = 0, nbas = 0, nfuc = 0, nsh = 0, nshuc = 0, ncell = 1;
    int ncl[3] = {1, 1, 1};
    double a[3] = {0, 0, 0}, L[3] = {0, 0, 0};
    int physicist = 0, sao = 1, prim_screen = 1;
    double thr = 1e-13, prim_thr = 1e-14;
    // host copies
    std::vector<double> ctr, exps, coefs, tnode, tweight;
    std::vector<int> lxyz, poff;
    std::vector<int> sh_first, sh_n, sh_l, sh_np, sh_eoff, sh_coff;
    std::vector<double> sh_r, sh_exp, sh_coef, sh_cmax;
    std::vector<UnitPair> up;
    std::vector<double> Q, Qsh;
    double Qmax = 0.0;
    std::vector<int> tnmax;
    // device
    int dev = 0;                         // CUDA device the handle was built on
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;   // ordering with a caller on the legacy stream
    int num_sms = 148;
    std::vector<void *> allocs;
    size_t bytes = 0;
    DevSys S{};
    PairPrim *d_pp = nullptr;
    double *d_Qsh = nullptr;
    int4 *d_items = nullptr;
    long long nitems = 0;
    int max_ncomb = 1, max_ncq = 1;
    int *d_gmax = nullptr;              // [3*TCE_MAXG] of the system's rule
    long long n_func_q = 0, n_unit_sig = 0, n_prim_q = 0;
    double jk_flops = 0.0;
    std::vector<int4> items_host;       // sorted, most expensive first
    std::vector<double> cost_host;
    int shard_rank = 0, shard_nranks = 1;
    // the J/K work of this shard, one list per kernel: kind 0 generic
    // (k_quartets), 1 all-s (k_quartets_s), 2 one-periodic-direction s/p class
    // `cls` (k_quartets_r1)
    // (generic lists: cls = shells above p, 0..4; max_ncomb / max_ncq of the list's quartets)
    struct WorkList { int kind, cls; int4 *d = nullptr; long long n = 0; int max_ncomb = 1, max_ncq = 1; };
    std::vector<WorkList> lists;
    long long nitems_shard = 0;
    int *d_tnmax = nullptr;
    unsigned int *d_next = nullptr;
    double *d_P = nullptr, *d_J = nullptr, *d_K = nullptr;
    double *d_eri = nullptr;
    long long eri_elems = 0;
    int eri_size = 0;
    double *d_blk = nullptr;
    long long *d_blkoff = nullptr;
    int4 *d_one = nullptr;
    float last_ms = 0.f;
    // this shard's items (indices into items_host) and their device copy
    std::vector<long long> shard_idx;
    int4 *d_shard_items = nullptr;
    // quadrature method of the J/K pass (TCE_METHOD_*)
    int method = TCE_METHOD_FIXED;
    // learned grid: rule dictionary, per-item rules, lists, fallback queue
    int lg_nrules = 0;
    std::vector<RuleDev> rules_host;
    RuleDev *d_rules = nullptr;
    double *d_rule_T = nullptr, *d_rule_t = nullptr, *d_rule_wk = nullptr, *d_rule_wg = nullptr;
    int *d_rule_tnmax = nullptr;         // [r][3][64] truncation order per rule node
    std::vector<int> item_rule;          // per items_host entry; lg_nrules = plain directly
    // learned-grid work, one list per kernel and rule size: kind 0 generic
    // (k_quartets), 1 all-s (k_quartets_s), 2 one-periodic-direction s/p class
    // `cls` (k_quartets_r1); nq = 32 or 64 padded rule nodes
    // tc: kernel form chosen by tce_lg_autotune (-1: the default rule of
    // lg_tc_default, 0: CUDA cores, 1: FP64 tensor cores); tc_choice keeps the
    // choices per list key across rebuilds
    // generic lists (kind 0): cls = shells above p (0..4), and the largest
    // combination count and block of the list's quartets size its buffers
    struct LgList {
        int kind, cls, nq, fp32, tc = -1;
        int4 *d = nullptr;
        int *rule = nullptr;
        long long n = 0;
        int max_ncomb = 1, max_ncq = 1;
        double cost = 0.0;               // summed cost estimate of its quartets (chain balance)
    };
    std::vector<LgList> lg_lists;
    std::map<int, int> tc_choice;
    long long n_lg = 0, n_fp32 = 0;
    double fp32_thr = 0.0;               // FP32 node sums below this Schwarz product (0: off)
    float *d_rule_T32 = nullptr;         // FP32 copy of the rule T tables
    int4 *d_plain_items = nullptr;
    long long n_plain_direct = 0;
    int4 *d_fb_items = nullptr;
    unsigned int *d_fb_count = nullptr;
    // The judge's rejects depend on the integrals only, so they repeat every
    // pass: after a pass their count and the first fb_cap of them are copied to
    // pinned host memory (event ev_fb); the next call moves them to the plain
    // list, which runs on the side stream st2 while the learned-grid kernels run.
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_fb = nullptr;
    unsigned int *h_fb = nullptr;        // pinned: [0] count, items from word 4
    int fb_cap = 4096;
    int fb_pending = 0;
    long long fb_version = -1;           // work_version of the pass the copy came from
    int route_rejects = 1;
    double judge_tol = 1e-10, plain_tol = 1e-11;
    int plain_max_panels = 24;
    double plain_scale = 0.6;
    double *d_gk = nullptr;              // 15-point Kronrod rule on [0,1]: u[16], wk[16], wg[16]
    double *d_plain_scratch = nullptr;
    long long plain_scratch_warps = 0;
    unsigned long long *d_node_evals = nullptr;
    unsigned int *d_next2 = nullptr;     // work counter of the second kernel of a pass
    unsigned int *d_next3 = nullptr;
    // The learned-grid lists of a pass run as list_streams chains (1 or 2): the
    // second chain on st3, forked from and joined to the pass's stream, so
    // that one list's tail overlaps the next list's start; every list has its
    // own work counter (d_list_next[list]).
    int list_streams = 2;
    cudaStream_t st3 = nullptr;
    cudaEvent_t ev_fork3 = nullptr, ev_join3 = nullptr;
    unsigned int *d_list_next = nullptr;
    int list_next_cap = 0;
    // CUDA graph of the J/K pass (tce_set_graph); rebuilt when any key changes
    int use_graph = 0;
    int use_tc = 1;                      // FP64 tensor-core node sums where a kernel has them
    int blocks_only = 0;                 // tce_create_blocks: no Schwarz, primitive table or quartet list
    long long work_version = 0;          // bumped whenever work lists are rebuilt
    cudaGraphExec_t jk_exec = nullptr;
    const double *g_P = nullptr;
    double *g_J = nullptr, *g_K = nullptr;
    cudaStream_t g_st = nullptr;
    int g_method = -1;
    long long g_version = -1;
};

extern thread_local std::string g_err;

int fail(Handle *h, int code, const std::string &msg);

#define CK(h, call)                                                                          \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail((h), TCE_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define CKS(h, call)                                                  \
    do {                                                              \
        int s_ = (call);                                              \
        if (s_ != TCE_OK) {                                           \
            cudaError_t e_ = cudaGetLastError();                      \
            return fail((h), s_, std::string(#call) + " failed" +     \
                                     (e_ != cudaSuccess ? std::string(": ") + cudaGetErrorString(e_) : "")); \
        }                                                             \
    } while (0)

template <class T>
int dalloc(Handle *h, T **p, size_t n)
{
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(h, TCE_ERR_NOMEM, "device allocation of " + std::to_string(n * sizeof(T)) + " bytes failed: " +
                                          cudaGetErrorString(e));
    }
    h->allocs.push_back(*p);
    h->bytes += n * sizeof(T);
    return TCE_OK;
}

template <class T>
int upload(Handle *h, T **p, const std::vector<T> &v)
{
    int s = dalloc(h, p, v.size());
    if (s) return s;
    if (!v.empty()) CK(h, cudaMemcpyAsync(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, h->st));
    return TCE_OK;
}

void dfree(Handle *h, void *p);


// helpers defined in tce_api.cu
int shift_to(const Handle *h, int idx, int refcell, int nblk);
int ncomb_of(const Handle *h, int SI, int SJ, int SK, int SL);
int make_lists(Handle *h, const std::vector<int4> &items);
int direct_jk_device(Handle *h, const double *dP, double *dJ, double *dK, cudaStream_t st);
int direct_jk_on(Handle *h, const double *dP, double *dJ, double *dK, cudaStream_t st);
void drop_graph(Handle *h);
// learned-grid / plain passes of direct_jk_device (tce_lg.cu)
int lg_jk_passes(Handle *h, const double *dP, double *dJ, double *dK, cudaStream_t st);
int lg_rebuild_lists(Handle *h);
int lg_read_rejects(Handle *h, cudaStream_t st);
int lg_absorb_rejects(Handle *h);
void release_streams(Handle *h);

}  // namespace tcehost
