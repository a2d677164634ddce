// tce_mp2.cu -- DF-MP2 on the device: the (ov|ov) contraction of df_kMO
// (df_toroidal.f90:1018-1035),
//   (i k1, a k2 | j k3, b k4) = 1/N sum_Q L^Q_ia(k1,k2) L^Q_jb(k3,k4),
//   k4 = k1 - k2 + k3 (cell coordinates modulo the lattice),
// and the k-MP2 energy of kMP2_calc (MP2_SAO.f90:6-151).
//
// The contraction runs either in FP64 on the CUDA cores or on the tensor
// cores in split-BF16 with FP32 accumulation: every real operand x is split
// into x_hi = bf16(x) and x_lo = bf16(x - x_hi), and X Y^T is formed as
// X_hi Y_hi^T + X_hi Y_lo^T + X_lo Y_hi^T (the X_lo Y_lo^T term is below the
// FP32 accumulation error).  A complex product is two real GEMMs over
// K = 2 nau: Re = [Xr | Xi] [Yr | -Yi]^T, Im = [Xr | Xi] [Yi | Yr]^T.
// The energy sums (direct and exchange parts, zero-gap terms left out and
// counted) stay FP64.
#include <cuda_bf16.h>
#include <mma.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/tce.h"

using namespace nvcuda;

namespace {

thread_local std::string g_mp2_err;

int mp2_fail(int code, const std::string &m)
{
    g_mp2_err = m;
    return code;
}

struct Mp2Dims {
    int N, no, nv, nau, ov;
    int ncl[3];
};

__device__ __forceinline__ int cell_of(const int *crd, int k, int d) { return crd[3 * k + d]; }

// cell index of c1 - c2 + c3 (x fastest)
__device__ __forceinline__ int k4_of(const Mp2Dims &D, const int *crd, int k1, int k2, int k3)
{
    int idx = 0, mul = 1;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int n = D.ncl[d];
        int c = (cell_of(crd, k1, d) - cell_of(crd, k2, d) + cell_of(crd, k3, d)) % n;
        if (c < 0) c += n;
        idx += mul * c;
        mul *= n;
    }
    return idx;
}

// L(p, q, Q, k1, k2) complex, column-major (p fastest), interleaved re/im
__device__ __forceinline__ size_t lidx(const Mp2Dims &D, int ia, int Q, int k1, int k2)
{
    return (size_t)ia + (size_t)D.ov * ((size_t)Q + (size_t)D.nau * ((size_t)k1 + (size_t)D.N * k2));
}

// G(p, q, r, s, k1, k2, k3) complex, column-major
__device__ __forceinline__ size_t gidx(const Mp2Dims &D, int ia, int jb, int k1, int k2, int k3)
{
    return (size_t)ia + (size_t)D.ov * ((size_t)jb + (size_t)D.ov * ((size_t)k1 + (size_t)D.N * ((size_t)k2 + (size_t)D.N * k3)));
}

// FP64 contraction: one thread per (ia, jb, k1, k2, k3) element
__global__ void k_ovov_fp64(Mp2Dims D, const int *crd, const double2 *L, double2 *G)
{
    const long long tot = (long long)D.ov * D.ov * D.N * D.N * D.N;
    const double invN = 1.0 / D.N;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < tot;
         id += (long long)gridDim.x * blockDim.x) {
        long long r = id;
        const int ia = (int)(r % D.ov); r /= D.ov;
        const int jb = (int)(r % D.ov); r /= D.ov;
        const int k1 = (int)(r % D.N); r /= D.N;
        const int k2 = (int)(r % D.N); r /= D.N;
        const int k3 = (int)r;
        const int k4 = k4_of(D, crd, k1, k2, k3);
        double re = 0.0, im = 0.0;
        for (int Q = 0; Q < D.nau; ++Q) {
            const double2 x = L[lidx(D, ia, Q, k1, k2)];
            const double2 y = L[lidx(D, jb, Q, k3, k4)];
            re = fma(x.x, y.x, fma(-x.y, y.y, re));
            im = fma(x.x, y.y, fma(x.y, y.x, im));
        }
        G[gidx(D, ia, jb, k1, k2, k3)] = make_double2(re * invN, im * invN);
    }
}

// Split-BF16 tensor-core contraction.  One CTA per (k1, k2, chunk of 16/ov
// k3 values); the A operand [Xr | Xi] of (k1,k2) and the B operands of the
// chunk are split into bf16 hi/lo parts in shared memory; warps take 16x16
// output tiles.  MP = ov rounded up to 16, KP = 2 nau rounded up to 16.
constexpr int MP2_WARPS = 4;

__global__ void __launch_bounds__(32 * MP2_WARPS) k_ovov_bf16(Mp2Dims D, const int *crd, const double2 *L, double2 *G,
                                                             int MP, int KP, int k3_per_cta)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int k1 = blockIdx.x % D.N, k2 = blockIdx.x / D.N;
    const int k3_0 = blockIdx.y * k3_per_cta;
    const int nk3 = min(k3_per_cta, D.N - k3_0);
    const int NC = k3_per_cta * D.ov;                      // B rows (k3, jb) of this CTA
    const int NP = (NC + 15) / 16 * 16;
    // shared: Ahi, Alo [MP][KP]; Bre_hi, Bre_lo, Bim_hi, Bim_lo [NP][KP]; C tiles [warps][2][16*16] float
    __nv_bfloat16 *Ahi = reinterpret_cast<__nv_bfloat16 *>(smem_raw);
    __nv_bfloat16 *Alo = Ahi + MP * KP;
    __nv_bfloat16 *Brh = Alo + MP * KP;
    __nv_bfloat16 *Brl = Brh + NP * KP;
    __nv_bfloat16 *Bih = Brl + NP * KP;
    __nv_bfloat16 *Bil = Bih + NP * KP;
    float *Cs = reinterpret_cast<float *>(Bil + NP * KP);
    const int tid = threadIdx.x, nth = blockDim.x;
    const int nau = D.nau;
    // A = [Xr | Xi] rows ia of L(., ., k1, k2)
    for (int e = tid; e < MP * KP; e += nth) {
        const int row = e / KP, col = e % KP;
        double v = 0.0;
        if (row < D.ov && col < 2 * nau) {
            const double2 x = L[lidx(D, row, col % nau, k1, k2)];
            v = col < nau ? x.x : x.y;
        }
        const __nv_bfloat16 hi = __double2bfloat16(v);
        Ahi[e] = hi;
        Alo[e] = __double2bfloat16(v - (double)__bfloat162float(hi));
    }
    // B rows (k3, jb): Re operand [Yr | -Yi], Im operand [Yi | Yr]
    for (int e = tid; e < NP * KP; e += nth) {
        const int row = e / KP, col = e % KP;
        double vr = 0.0, vi = 0.0;
        if (row < nk3 * D.ov && col < 2 * nau) {
            const int k3 = k3_0 + row / D.ov, jb = row % D.ov;
            const int k4 = k4_of(D, crd, k1, k2, k3);
            const double2 y = L[lidx(D, jb, col % nau, k3, k4)];
            vr = col < nau ? y.x : -y.y;
            vi = col < nau ? y.y : y.x;
        }
        __nv_bfloat16 h = __double2bfloat16(vr);
        Brh[e] = h;
        Brl[e] = __double2bfloat16(vr - (double)__bfloat162float(h));
        h = __double2bfloat16(vi);
        Bih[e] = h;
        Bil[e] = __double2bfloat16(vi - (double)__bfloat162float(h));
    }
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31;
    float *Cw = Cs + warp * 2 * 256;
    const int tiles_m = MP / 16, tiles_n = NP / 16;
    const double invN = 1.0 / D.N;
    for (int t = warp; t < tiles_m * tiles_n; t += MP2_WARPS) {
        const int tm = t % tiles_m, tn = t / tiles_m;
        wmma::fragment<wmma::accumulator, 16, 16, 16, float> cr, ci;
        wmma::fill_fragment(cr, 0.0f);
        wmma::fill_fragment(ci, 0.0f);
        for (int kk = 0; kk < KP; kk += 16) {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> ah, al;
            wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::col_major> bh, bl;
            wmma::load_matrix_sync(ah, Ahi + tm * 16 * KP + kk, KP);
            wmma::load_matrix_sync(al, Alo + tm * 16 * KP + kk, KP);
            wmma::load_matrix_sync(bh, Brh + tn * 16 * KP + kk, KP);
            wmma::load_matrix_sync(bl, Brl + tn * 16 * KP + kk, KP);
            wmma::mma_sync(cr, ah, bh, cr);
            wmma::mma_sync(cr, ah, bl, cr);
            wmma::mma_sync(cr, al, bh, cr);
            wmma::load_matrix_sync(bh, Bih + tn * 16 * KP + kk, KP);
            wmma::load_matrix_sync(bl, Bil + tn * 16 * KP + kk, KP);
            wmma::mma_sync(ci, ah, bh, ci);
            wmma::mma_sync(ci, ah, bl, ci);
            wmma::mma_sync(ci, al, bh, ci);
        }
        wmma::store_matrix_sync(Cw, cr, 16, wmma::mem_row_major);
        wmma::store_matrix_sync(Cw + 256, ci, 16, wmma::mem_row_major);
        __syncwarp();
        for (int e = lane; e < 256; e += 32) {
            const int r = tm * 16 + e / 16, c = tn * 16 + e % 16;
            if (r < D.ov && c < nk3 * D.ov) {
                const int k3 = k3_0 + c / D.ov, jb = c % D.ov;
                G[gidx(D, r, jb, k1, k2, k3)] = make_double2((double)Cw[e] * invN, (double)Cw[256 + e] * invN);
            }
        }
        __syncwarp();
    }
}

// kMP2_calc: one thread per (ki, kj, ka) triple; FP64 sums, block reduction,
// one atomic per block.
__global__ void k_mp2_energy(Mp2Dims D, const int *crd, const double2 *G, const double *eo, const int *oo,
                             const double *ev, const int *ov_, double *acc /* e2d, e2x, gzero */,
                             unsigned long long *nzero)
{
    __shared__ double sd[256], sx[256];
    __shared__ unsigned long long sz[256];
    __shared__ double sg[256];
    double e2d = 0.0, e2x = 0.0, gz = 0.0;
    unsigned long long nz = 0;
    const long long tot = (long long)D.N * D.N * D.N;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < tot;
         id += (long long)gridDim.x * blockDim.x) {
        const int ki = (int)(id % D.N), kj = (int)((id / D.N) % D.N), ka = (int)(id / ((long long)D.N * D.N));
        const int kb = k4_of(D, crd, ki, ka, kj);
        for (int i = 0; i < D.no; ++i) {
            if (oo[ki * D.no + i] != 2) continue;
            for (int j = 0; j < D.no; ++j) {
                if (oo[kj * D.no + j] != 2) continue;
                for (int a = 0; a < D.nv; ++a) {
                    if (ov_[ka * D.nv + a] != 0) continue;
                    for (int b = 0; b < D.nv; ++b) {
                        if (ov_[kb * D.nv + b] != 0) continue;
                        const double Dn = ev[ka * D.nv + a] + ev[kb * D.nv + b] - eo[ki * D.no + i] - eo[kj * D.no + j];
                        const double2 gd = G[gidx(D, i + D.no * a, j + D.no * b, ki, ka, kj)];
                        if (fabs(Dn) < 1e-8) {
                            ++nz;
                            gz = fmax(gz, sqrt(gd.x * gd.x + gd.y * gd.y));
                            continue;
                        }
                        const double2 gx = G[gidx(D, i + D.no * b, j + D.no * a, ki, kb, kj)];
                        e2d -= (gd.x * gd.x + gd.y * gd.y) / Dn;
                        e2x -= (gd.x * gx.x + gd.y * gx.y) / Dn;
                    }
                }
            }
        }
    }
    sd[threadIdx.x] = e2d;
    sx[threadIdx.x] = e2x;
    sz[threadIdx.x] = nz;
    sg[threadIdx.x] = gz;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sd[threadIdx.x] += sd[threadIdx.x + s];
            sx[threadIdx.x] += sx[threadIdx.x + s];
            sz[threadIdx.x] += sz[threadIdx.x + s];
            sg[threadIdx.x] = fmax(sg[threadIdx.x], sg[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicAdd(acc, sd[0]);
        atomicAdd(acc + 1, sx[0]);
        atomicAdd(nzero, sz[0]);
        // gzero >= 0: the bit pattern order of non-negative doubles is their order
        atomicMax(reinterpret_cast<unsigned long long *>(acc + 2), (unsigned long long)__double_as_longlong(sg[0]));
    }
}

template <class T>
int dmalloc(T **p, size_t n, std::vector<void *> &keep)
{
    *p = nullptr;
    if (cudaMalloc((void **)p, (n ? n : 1) * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return mp2_fail(TCE_ERR_NOMEM, "device allocation of " + std::to_string(n * sizeof(T)) + " bytes failed");
    }
    keep.push_back(*p);
    return TCE_OK;
}

}  // namespace

extern "C" {

const char *tce_mp2_last_error(void) { return g_mp2_err.c_str(); }

int tce_dfmp2_energy(int32_t ncell, const int32_t ncl[3], const int32_t *kcoord, int32_t no, int32_t nv,
                     int32_t nau, const double *L, const double *eps_o, const int32_t *occ_o, const double *eps_v,
                     const int32_t *occ_v, int32_t mode, double *e2d, double *e2x, int64_t *nzero, double *gzero,
                     double *ms)
{
    if (ncell < 1 || !ncl || !kcoord || no < 1 || nv < 1 || nau < 1 || !L || !eps_o || !occ_o || !eps_v ||
        !occ_v || !e2d || !e2x)
        return mp2_fail(TCE_ERR_ARG, "bad argument");
    if (mode != 0 && mode != 1) return mp2_fail(TCE_ERR_ARG, "mode must be 0 (FP64) or 1 (split-BF16)");
    if ((long long)ncl[0] * ncl[1] * ncl[2] != ncell) return mp2_fail(TCE_ERR_ARG, "ncl does not match ncell");
    const int ov = no * nv;
    if (ov > 64) return mp2_fail(TCE_ERR_UNSUPPORTED, "no*nv above 64");
    Mp2Dims D{ncell, no, nv, nau, ov, {ncl[0], ncl[1], ncl[2]}};
    const size_t nL = (size_t)ov * nau * ncell * ncell;
    const size_t nG = (size_t)ov * ov * ncell * ncell * ncell;
    std::vector<void *> keep;
    auto cleanup = [&]() {
        for (void *p : keep) cudaFree(p);
    };
    int *d_crd = nullptr, *d_oo = nullptr, *d_ov = nullptr;
    double2 *d_L = nullptr, *d_G = nullptr;
    double *d_eo = nullptr, *d_ev = nullptr, *d_acc = nullptr;
    unsigned long long *d_nz = nullptr;
    int s = 0;
    if (!s) s = dmalloc(&d_crd, 3 * (size_t)ncell, keep);
    if (!s) s = dmalloc(&d_oo, (size_t)ncell * no, keep);
    if (!s) s = dmalloc(&d_ov, (size_t)ncell * nv, keep);
    if (!s) s = dmalloc(&d_L, nL, keep);
    if (!s) s = dmalloc(&d_G, nG, keep);
    if (!s) s = dmalloc(&d_eo, (size_t)ncell * no, keep);
    if (!s) s = dmalloc(&d_ev, (size_t)ncell * nv, keep);
    if (!s) s = dmalloc(&d_acc, 3, keep);
    if (!s) s = dmalloc(&d_nz, 1, keep);
    if (s) {
        cleanup();
        return s;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaMemcpy(d_crd, kcoord, sizeof(int) * 3 * ncell, cudaMemcpyHostToDevice);
    cudaMemcpy(d_oo, occ_o, sizeof(int) * ncell * no, cudaMemcpyHostToDevice);
    cudaMemcpy(d_ov, occ_v, sizeof(int) * ncell * nv, cudaMemcpyHostToDevice);
    cudaMemcpy(d_L, L, sizeof(double2) * nL, cudaMemcpyHostToDevice);
    cudaMemcpy(d_eo, eps_o, sizeof(double) * ncell * no, cudaMemcpyHostToDevice);
    cudaMemcpy(d_ev, eps_v, sizeof(double) * ncell * nv, cudaMemcpyHostToDevice);
    cudaMemset(d_acc, 0, sizeof(double) * 3);
    cudaMemset(d_nz, 0, sizeof(unsigned long long));
    cudaEventRecord(e0);
    if (mode == 0) {
        k_ovov_fp64<<<148 * 16, 256>>>(D, d_crd, d_L, d_G);
    } else {
        const int MP = (ov + 15) / 16 * 16, KP = (2 * nau + 15) / 16 * 16;
        const int k3c = std::max(1, 96 / ov);
        const int NP = (k3c * ov + 15) / 16 * 16;
        const size_t smem = sizeof(__nv_bfloat16) * ((size_t)2 * MP * KP + (size_t)4 * NP * KP) +
                            sizeof(float) * MP2_WARPS * 2 * 256;
        if (smem > 200 * 1024) {
            cleanup();
            return mp2_fail(TCE_ERR_UNSUPPORTED, "nau too large for the tensor-core tile");
        }
        cudaFuncSetAttribute(k_ovov_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        dim3 grid(ncell * ncell, (ncell + k3c - 1) / k3c);
        k_ovov_bf16<<<grid, 32 * MP2_WARPS, smem>>>(D, d_crd, d_L, d_G, MP, KP, k3c);
    }
    const long long ntrip = (long long)ncell * ncell * ncell;
    const int eblocks = (int)std::min<long long>((ntrip + 255) / 256, 148 * 8);
    k_mp2_energy<<<eblocks, 256>>>(D, d_crd, d_G, d_eo, d_oo, d_ev, d_ov, d_acc, d_nz);
    cudaEventRecord(e1);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cleanup();
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return mp2_fail(TCE_ERR_CUDA, std::string("DF-MP2 kernels: ") + cudaGetErrorString(e));
    }
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    double acc[3];
    unsigned long long nz = 0;
    cudaMemcpy(acc, d_acc, sizeof acc, cudaMemcpyDeviceToHost);
    cudaMemcpy(&nz, d_nz, sizeof nz, cudaMemcpyDeviceToHost);
    *e2d = acc[0];
    *e2x = acc[1];
    if (nzero) *nzero = (int64_t)nz;
    if (gzero) *gzero = acc[2];
    if (ms) *ms = t;
    cleanup();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return TCE_OK;
}

}  // extern "C"
