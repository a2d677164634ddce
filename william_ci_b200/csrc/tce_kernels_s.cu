// tce_kernels_s.cu -- launchers of the register-resident quartet kernels
// (tce_kernels_s.cuh) with the system's t-quadrature rule.
#include "tce_kernels_s.cuh"

// class key for k_quartets_r1: bit i = l of shell i (s or p); the classes with
// one p shell are instantiated (tce_r1_supported); the others use k_quartets
int tce_launch_quartets_r1(const DevSys &S, int cls, const SArgsHost &h, cudaStream_t st)
{
    SArgs A{};
    A.items = h.items;
    A.nitems = h.nitems;
    A.prim_screen = h.prim_screen;
    A.next = h.next;
    A.P = h.P;
    A.J = h.J;
    A.K = h.K;
    int NG = S.nq / 8, tot = 0;
    for (int d = 0; d < 3; ++d)
        for (int g = 0; g < TCE_MAXG; ++g) {
            A.tsoff[d][g] = 0;
            if (d == 0 && g < NG) {
                A.tsoff[d][g] = tot;
                tot += (S.gmax[d][g] + 1) * 8;
            }
        }
    size_t qbytes = 8 * (size_t)TCE_POOL_BYTES;     // per-warp primitive pools
    size_t tbytes = (size_t)tot * sizeof(double);
    A.t_smem = (tbytes + qbytes <= 100 * 1024) ? 1 : 0;
    A.ts_doubles = A.t_smem ? tot : 0;
    size_t smem = (A.t_smem ? tbytes : 0) + qbytes;
    cudaMemsetAsync(h.next, 0, sizeof(unsigned int), st);
    int nsm = h.num_sms > 0 ? h.num_sms : 148;
#define TCE_R1(NQv, a, b, c, d)                                                                                   \
    do {                                                                                                          \
        cudaFuncSetAttribute(k_quartets_r1<NQv, a, b, c, d, false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,      \
                             (int)smem);                                                                          \
        int per = 0;                                                                                              \
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_quartets_r1<NQv, a, b, c, d, false, double>, 256, smem);    \
        if (per < 1) per = 1;                                                                                     \
        k_quartets_r1<NQv, a, b, c, d, false, double><<<nsm * per, 256, smem, st>>>(S, A);                                \
    } while (0)
#define TCE_R1_CLS(NQv)                                                                                            \
    switch (cls) {                                                                                                 \
    case 1: TCE_R1(NQv, 1, 0, 0, 0); break;   case 2: TCE_R1(NQv, 0, 1, 0, 0); break;                              \
    case 4: TCE_R1(NQv, 0, 0, 1, 0); break;   case 8: TCE_R1(NQv, 0, 0, 0, 1); break;                              \
    default: return TCE_ERR_UNSUPPORTED;                                                                           \
    }
    if (S.ndp != 1 || S.nq != 32) return TCE_ERR_UNSUPPORTED;
    TCE_R1_CLS(32)
#undef TCE_R1
#undef TCE_R1_CLS
    return cudaGetLastError() == cudaSuccess ? TCE_OK : TCE_ERR_CUDA;
}

int tce_launch_quartets_s(const DevSys &S, const SArgsHost &h, cudaStream_t st)
{
    SArgs A{};
    A.items = h.items;
    A.nitems = h.nitems;
    A.prim_screen = h.prim_screen;
    A.next = h.next;
    A.P = h.P;
    A.J = h.J;
    A.K = h.K;
    int NG = S.nq / 8, tot = 0;
    for (int d = 0; d < 3; ++d)
        for (int g = 0; g < TCE_MAXG; ++g) {
            A.tsoff[d][g] = 0;
            if (d < S.ndp && g < NG) {
                A.tsoff[d][g] = tot;
                tot += (S.gmax[d][g] + 1) * 8;
            }
        }
    size_t qbytes = 8 * (size_t)TCE_POOL_BYTES;     // per-warp primitive pools
    size_t tbytes = (size_t)tot * sizeof(double);
    A.t_smem = (tbytes + qbytes <= 200 * 1024) ? 1 : 0;
    A.ts_doubles = A.t_smem ? tot : 0;
    size_t smem = (A.t_smem ? tbytes : 0) + qbytes;
    cudaMemsetAsync(h.next, 0, sizeof(unsigned int), st);
    int nsm = h.num_sms > 0 ? h.num_sms : 148;
#define TCE_LAUNCH_S(NQv, NDPv)                                                                             \
    do {                                                                                                    \
        cudaFuncSetAttribute(k_quartets_s<NQv, NDPv, false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                             (int)smem);                                                                    \
        int per = 0;                                                                                        \
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_quartets_s<NQv, NDPv, false, double>, 256, smem);     \
        if (per < 1) per = 1;                                                                               \
        k_quartets_s<NQv, NDPv, false, double><<<nsm * per, 256, smem, st>>>(S, A);                                 \
    } while (0)
    if (S.nq == 32) {
        if (S.ndp == 1) TCE_LAUNCH_S(32, 1);
        else if (S.ndp == 2) TCE_LAUNCH_S(32, 2);
        else TCE_LAUNCH_S(32, 3);
    } else if (S.nq == 40) {
        if (S.ndp == 1) TCE_LAUNCH_S(40, 1);
        else if (S.ndp == 2) TCE_LAUNCH_S(40, 2);
        else TCE_LAUNCH_S(40, 3);
    } else {
        return TCE_ERR_UNSUPPORTED;
    }
#undef TCE_LAUNCH_S
    return cudaGetLastError() == cudaSuccess ? TCE_OK : TCE_ERR_CUDA;
}

