// tce_kernels_sp2.cu -- the s/p tensor-core kernel (k_quartets_sp_tc,
// tce_kernels_tc.cuh) for the six classes with two p shells of one periodic
// direction, in its three tile shapes: 8 primitive quartets x 16, 32 or 64
// nodes per pass (four power combinations per step loop).
#include "tce_kernels_tc.cuh"

int tce_sp2_launch(const DevSys &S, int cls, const SArgs &A, int nq, int shape, int nsm, cudaStream_t st)
{
#define TCE_SP2(NQv, MTv, NTv)                                                     \
    switch (cls) {                                                                 \
    case 3: sp_tc_launch<NQv, 1, 1, 0, 0, MTv, NTv>(S, A, nsm, st); break;         \
    case 5: sp_tc_launch<NQv, 1, 0, 1, 0, MTv, NTv>(S, A, nsm, st); break;         \
    case 6: sp_tc_launch<NQv, 0, 1, 1, 0, MTv, NTv>(S, A, nsm, st); break;         \
    case 9: sp_tc_launch<NQv, 1, 0, 0, 1, MTv, NTv>(S, A, nsm, st); break;         \
    case 10: sp_tc_launch<NQv, 0, 1, 0, 1, MTv, NTv>(S, A, nsm, st); break;        \
    case 12: sp_tc_launch<NQv, 0, 0, 1, 1, MTv, NTv>(S, A, nsm, st); break;        \
    default: return TCE_ERR_UNSUPPORTED;                                           \
    }
    if (nq == 32) {
        if (shape == 1) { TCE_SP2(32, 1, 2) } else { TCE_SP2(32, 1, 4) }
    } else {
        if (shape == 1) { TCE_SP2(64, 1, 2) } else if (shape == 2) { TCE_SP2(64, 1, 4) } else { TCE_SP2(64, 1, 8) }
    }
#undef TCE_SP2
    return TCE_OK;
}
