// tce_kernels_slg.cu -- launchers of the register-resident quartet kernels
// (tce_kernels_s.cuh) with per-quartet learned-grid rules: each shell
// quartet's T table comes from the rule dictionary in global memory, the
// kernel judges its block and queues rejects for the plain method.
#include "tce_kernels_s.cuh"

static void lg_args(SArgs &A, const SArgsHost &h)
{
    A.items = h.items;
    A.nitems = h.nitems;
    A.prim_screen = h.prim_screen;
    A.next = h.next;
    A.P = h.P;
    A.J = h.J;
    A.K = h.K;
    A.t_smem = 0;
    A.ts_doubles = 0;
    A.item_rule = h.item_rule;
    A.rules = h.rules;
    A.rule_T = h.rule_T;
    A.rule_t = h.rule_t;
    A.rule_wk = h.rule_wk;
    A.rule_wg = h.rule_wg;
    A.rule_T32 = h.rule_T32;
    A.judge_tol = h.judge_tol;
    A.fb_items = h.fb_items;
    A.fb_count = h.fb_count;
}

template <class Kern>
static void launch(Kern k, const DevSys &S, const SArgs &A, int nsm, cudaStream_t st)
{
    const size_t smem = 8 * (size_t)TCE_POOL_BYTES;   // per-warp primitive pools
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, 256, smem);
    if (per < 1) per = 1;
    k<<<nsm * per, 256, smem, st>>>(S, A);
}

int tce_launch_quartets_s_lg(const DevSys &S, const SArgsHost &h, int nq, bool fp32, cudaStream_t st)
{
    if (!h.item_rule || !h.rules || !h.rule_T || !h.fb_items || !h.fb_count) return TCE_ERR_ARG;
    if (fp32 && (!h.rule_T32 || S.ndp != 1)) return TCE_ERR_UNSUPPORTED;
    SArgs A{};
    lg_args(A, h);
    cudaMemsetAsync(h.next, 0, sizeof(unsigned int), st);
    const int nsm = h.num_sms > 0 ? h.num_sms : 148;
    if (fp32) {
        if (nq == 32) launch(k_quartets_s<32, 1, true, float>, S, A, nsm, st);
        else if (nq == 64) launch(k_quartets_s<64, 1, true, float>, S, A, nsm, st);
        else return TCE_ERR_UNSUPPORTED;
    } else if (nq == 32) {
        if (S.ndp == 1) launch(k_quartets_s<32, 1, true, double>, S, A, nsm, st);
        else if (S.ndp == 2) launch(k_quartets_s<32, 2, true, double>, S, A, nsm, st);
        else launch(k_quartets_s<32, 3, true, double>, S, A, nsm, st);
    } else if (nq == 64) {
        if (S.ndp == 1) launch(k_quartets_s<64, 1, true, double>, S, A, nsm, st);
        else if (S.ndp == 2) launch(k_quartets_s<64, 2, true, double>, S, A, nsm, st);
        else launch(k_quartets_s<64, 3, true, double>, S, A, nsm, st);
    } else {
        return TCE_ERR_UNSUPPORTED;
    }
    return cudaGetLastError() == cudaSuccess ? TCE_OK : TCE_ERR_CUDA;
}

int tce_launch_quartets_r1_lg(const DevSys &S, int cls, const SArgsHost &h, int nq, bool fp32, cudaStream_t st)
{
    if (!h.item_rule || !h.rules || !h.rule_T || !h.fb_items || !h.fb_count) return TCE_ERR_ARG;
    if (S.ndp != 1 || (nq != 32 && nq != 64)) return TCE_ERR_UNSUPPORTED;
    if (fp32 && !h.rule_T32) return TCE_ERR_UNSUPPORTED;
    SArgs A{};
    lg_args(A, h);
    cudaMemsetAsync(h.next, 0, sizeof(unsigned int), st);
    const int nsm = h.num_sms > 0 ? h.num_sms : 148;
#define TCE_R1_LG(NQv, AT)                                                                          \
    switch (cls) {                                                                                  \
    case 1: launch(k_quartets_r1<NQv, 1, 0, 0, 0, true, AT>, S, A, nsm, st); break;                 \
    case 2: launch(k_quartets_r1<NQv, 0, 1, 0, 0, true, AT>, S, A, nsm, st); break;                 \
    case 4: launch(k_quartets_r1<NQv, 0, 0, 1, 0, true, AT>, S, A, nsm, st); break;                 \
    case 8: launch(k_quartets_r1<NQv, 0, 0, 0, 1, true, AT>, S, A, nsm, st); break;                 \
    default: return TCE_ERR_UNSUPPORTED;                                                            \
    }
    if (nq == 32) {
        if (fp32) {
            TCE_R1_LG(32, float)
        } else {
            TCE_R1_LG(32, double)
        }
    } else {
        if (fp32) {
            TCE_R1_LG(64, float)
        } else {
            TCE_R1_LG(64, double)
        }
    }
#undef TCE_R1_LG
    return cudaGetLastError() == cudaSuccess ? TCE_OK : TCE_ERR_CUDA;
}
