// tce_dfjk.cu -- density-fitted J and K of the SCF on the device (df_JK,
// df_toroidal.f90:850-956).
//
// Inputs kept on the device by tce_dfjk_create: the real-space fitted
// coefficients B = df_B(nfuc, nBas, naux) (a (nfuc nBas) x naux matrix,
// column-major) and the k-space Bh(mu, Q, nu0; k1, kh) of df_init
// (:660-678), complex, for the half set of k (df_khalf :103-114).
//
//   J: Ps(i, r) = P(r-block rows, (rs + r)-block columns) packed; G = B^T Ps
//      (tiled GEMM); gamma(c, Q) = sum_r G(c - r, Q; r) (gather over cells);
//      J(1:nfuc, :) = B gamma (GEMV).
//   K: P(k) = sum_r P(1:nfuc, r-block) e^{i k R}, hermitised; per k-point kk
//      Kloc(kk) = sum_{k1} sum_Q B_Q P(k1) B_Q^H with B_Q = Bh(:, Q, :, k1, k2),
//      k2 = kk - k1 (or conj Bh(-k1, -k2) when k2 is not in the half set);
//      K(1:nfuc, r-block) = Re sum_kk Kloc(kk) e^{-i kk R} (-1/2) / N^2.
// The reference contracts with the eigenvectors of P(k) whose eigenvalues
// exceed 1e-10 in magnitude, sum_i w_i (B c_i)(B c_i)^H; without the filter
// that sum is B P(k) B^H, which is what is computed here (the dropped
// components weigh at most 1e-10 each).
#include <cmath>
#include <string>
#include <vector>

#include "../../include/tce.h"
#include <cuda_runtime.h>

namespace {

struct DfjkHandle {
    std::string err;
    int nf = 0, nbas = 0, nau = 0, N = 0, naux = 0, nb = 0, nkh = 0;
    int ncl[3] = {1, 1, 1};
    std::vector<int> khi, cadd, csub;   // host tables
    double *B = nullptr;                // nb x naux
    double2 *Bh = nullptr;              // nf x nau x nf x N x nkh
    double2 *ph = nullptr;              // N x N: e^{2 pi i k.R / n}
    int *d_khi = nullptr, *d_cadd = nullptr, *d_csub = nullptr;
    double *P = nullptr, *Ps = nullptr, *G = nullptr, *gam = nullptr, *Jp = nullptr, *Kr = nullptr;
    double2 *Pk = nullptr, *Kt = nullptr;
    cudaStream_t st = nullptr;
};

thread_local std::string g_dferr;

int dfail(DfjkHandle *h, int code, const std::string &m)
{
    (h ? h->err : g_dferr) = m;
    return code;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// Ps(i, r), i = (a + nf b) + nf^2 rs: P(r nf + a, cadd(rs, r) nf + b)
__global__ void k_pack_ps(int nf, int N, int nbas, const int *cadd, const double *P, double *Ps)
{
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nb = (long long)nf * nbas;
    if (id >= nb * N) return;
    const int r = (int)(id / nb);
    const long long i = id - (long long)r * nb;
    const int rs = (int)(i / (nf * nf)), ab = (int)(i % (nf * nf)), a = ab % nf, b = ab / nf;
    const int c = cadd[rs * N + r];
    Ps[id] = P[(size_t)(r * nf + a) + (size_t)nbas * (c * nf + b)];
}

// G = B^T Ps: (naux x N), 16 x 16 tiles through shared memory
__global__ void k_gemm_tn(int M, int Ncol, int Kd, const double *A /* Kd x M */, const double *Bm /* Kd x Ncol */,
                          double *C /* M x Ncol */)
{
    __shared__ double As[16][17], Bs[16][17];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int row = blockIdx.y * 16 + ty, col = blockIdx.x * 16 + tx;
    double acc = 0.0;
    for (int k0 = 0; k0 < Kd; k0 += 16) {
        const int ka = k0 + tx, kb = k0 + ty;
        const int arow = blockIdx.y * 16 + ty;
        As[ty][tx] = (arow < M && ka < Kd) ? A[(size_t)ka + (size_t)Kd * arow] : 0.0;
        Bs[ty][tx] = (col < Ncol && kb < Kd) ? Bm[(size_t)kb + (size_t)Kd * col] : 0.0;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k) acc = fma(As[ty][k], Bs[k][tx], acc);
        __syncthreads();
    }
    if (row < M && col < Ncol) C[(size_t)row + (size_t)M * col] = acc;
}

// gamma(c nau + q) = sum_r G(csub(c, r) nau + q, r)
__global__ void k_gamma(int nau, int N, const int *csub, const double *G, double *gam)
{
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nau * N) return;
    const int c = id / nau, q = id % nau;
    const int naux = nau * N;
    double s = 0.0;
    for (int r = 0; r < N; ++r) s += G[(size_t)(csub[c * N + r] * nau + q) + (size_t)naux * r];
    gam[id] = s;
}

// Jp = B gamma (nb)
__global__ void k_gemv(long long nb, int naux, const double *B, const double *gam, double *Jp)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    double s = 0.0;
    for (int q = 0; q < naux; ++q) s = fma(B[(size_t)i + (size_t)nb * q], gam[q], s);
    Jp[i] = s;
}

// P(k)(a, b) hermitised
__global__ void k_pk(int nf, int N, int nbas, const double *P, const double2 *ph, double2 *Pk)
{
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= N * nf * nf) return;
    const int k = id / (nf * nf), ab = id % (nf * nf), a = ab % nf, b = ab / nf;
    double2 s = make_double2(0.0, 0.0), t = make_double2(0.0, 0.0);
    for (int r = 0; r < N; ++r) {
        const double2 e = ph[k * N + r];
        const double pab = P[(size_t)a + (size_t)nbas * (r * nf + b)];
        const double pba = P[(size_t)b + (size_t)nbas * (r * nf + a)];
        s.x += pab * e.x;
        s.y += pab * e.y;
        t.x += pba * e.x;
        t.y += pba * e.y;
    }
    // 0.5 (pk + pk^H): (a, b) -> 0.5 (pk(a,b) + conj pk(b,a))
    Pk[(size_t)k * nf * nf + a + nf * b] = make_double2(0.5 * (s.x + t.x), 0.5 * (s.y - t.y));
}

// Kloc(kk) = sum_k1 sum_Q B_Q P(k1) B_Q^H, one block per kk
__global__ void k_kloc(int nf, int nau, int N, const int *csub, const int *khi, const double2 *Bh, const double2 *Pk,
                       double2 *Kt, double scale)
{
    extern __shared__ double2 sm[];
    const int kk = blockIdx.x;
    const int sz = nf * nau * nf;
    double2 *Bs = sm;             // B(mu, Q, nu)
    double2 *Ms = Bs + sz;        // M(mu, Q, nu') = sum_nu B(mu, Q, nu) P(nu, nu')
    double2 *Ps = Ms + sz;        // P(k1)
    double2 acc = make_double2(0.0, 0.0);
    const int t = threadIdx.x;
    const int mu = t % nf, mv = t / nf;   // output element for threads < nf^2
    for (int k1 = 0; k1 < N; ++k1) {
        const int k2 = csub[kk * N + k1];
        bool conj_;
        const double2 *src;
        if (khi[k2] >= 0) {
            conj_ = false;
            src = Bh + ((size_t)khi[k2] * N + k1) * sz;
        } else {
            conj_ = true;
            const int mk1 = csub[0 * N + k1], mk2 = csub[0 * N + k2];
            src = Bh + ((size_t)khi[mk2] * N + mk1) * sz;
        }
        __syncthreads();
        for (int x = t; x < sz; x += blockDim.x) Bs[x] = conj_ ? cconj(src[x]) : src[x];
        for (int x = t; x < nf * nf; x += blockDim.x) Ps[x] = Pk[(size_t)k1 * nf * nf + x];
        __syncthreads();
        for (int x = t; x < sz; x += blockDim.x) {   // x = mu + nf (Q + nau nv)
            const int m0 = x % nf, rest = x / nf, Q = rest % nau, nv = rest / nau;
            double2 s = make_double2(0.0, 0.0);
            for (int nu = 0; nu < nf; ++nu) {
                const double2 p = cmul(Bs[m0 + nf * (Q + nau * nu)], Ps[nu + nf * nv]);
                s.x += p.x;
                s.y += p.y;
            }
            Ms[x] = s;
        }
        __syncthreads();
        if (t < nf * nf) {
            for (int Q = 0; Q < nau; ++Q)
                for (int nv = 0; nv < nf; ++nv) {
                    const double2 p = cmul(Ms[mu + nf * (Q + nau * nv)], cconj(Bs[mv + nf * (Q + nau * nv)]));
                    acc.x += p.x;
                    acc.y += p.y;
                }
        }
    }
    if (t < nf * nf) Kt[(size_t)kk * nf * nf + mu + nf * mv] = make_double2(acc.x * scale, acc.y * scale);
}

// K(a, r nf + b) = Re sum_kk Kt(kk)(a, b) e^{-i kk R} / N
__global__ void k_kreal(int nf, int N, const double2 *Kt, const double2 *ph, double *Kr)
{
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= N * nf * nf) return;
    const int r = id / (nf * nf), ab = id % (nf * nf);
    double s = 0.0;
    for (int kk = 0; kk < N; ++kk) {
        const double2 v = Kt[(size_t)kk * nf * nf + ab], e = ph[kk * N + r];
        s += v.x * e.x + v.y * e.y;   // Re(v conj(e))
    }
    Kr[id] = s / (double)N;
}

template <class T>
int dal(DfjkHandle *h, T **p, size_t n)
{
    if (cudaMalloc((void **)p, (n ? n : 1) * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return dfail(h, TCE_ERR_NOMEM, "device allocation failed");
    }
    return TCE_OK;
}

void release(DfjkHandle *h)
{
    for (void *p : {(void *)h->B, (void *)h->Bh, (void *)h->ph, (void *)h->d_khi, (void *)h->d_cadd, (void *)h->d_csub,
                    (void *)h->P, (void *)h->Ps, (void *)h->G, (void *)h->gam, (void *)h->Jp, (void *)h->Kr, (void *)h->Pk,
                    (void *)h->Kt})
        if (p) cudaFree(p);
    if (h->st) cudaStreamDestroy(h->st);
}

}  // namespace

extern "C" {

const char *tce_dfjk_last_error(void *handle)
{
    return handle ? static_cast<DfjkHandle *>(handle)->err.c_str() : g_dferr.c_str();
}

int tce_dfjk_create(int32_t nfuc, int32_t nbas, int32_t nau, const int32_t ncl[3], const double *B, const double *Bh,
                    void **handle)
{
    if (!handle || !ncl || !B || !Bh || nfuc < 1 || nau < 1 || nbas < nfuc || nbas % nfuc)
        return dfail(nullptr, TCE_ERR_ARG, "bad argument");
    *handle = nullptr;
    auto *h = new DfjkHandle();
    h->nf = nfuc;
    h->nbas = nbas;
    h->nau = nau;
    for (int d = 0; d < 3; ++d) h->ncl[d] = ncl[d] > 0 ? ncl[d] : 1;
    h->N = h->ncl[0] * h->ncl[1] * h->ncl[2];
    if (h->N * nfuc != nbas) {
        delete h;
        return dfail(nullptr, TCE_ERR_ARG, "nbas != nfuc x cells");
    }
    const size_t smem = (size_t)(2 * nfuc * nau * nfuc + nfuc * nfuc) * sizeof(double2);
    if (smem > 96 * 1024 || nfuc * nfuc > 1024) {
        delete h;
        return dfail(nullptr, TCE_ERR_UNSUPPORTED, "nfuc x nau too large for the exchange kernel");
    }
    const int N = h->N;
    h->naux = nau * N;
    h->nb = nfuc * nbas;
    // cell tables (coordinates x fastest), half set of k
    auto cell = [&](int x, int y, int z) {
        x = ((x % h->ncl[0]) + h->ncl[0]) % h->ncl[0];
        y = ((y % h->ncl[1]) + h->ncl[1]) % h->ncl[1];
        z = ((z % h->ncl[2]) + h->ncl[2]) % h->ncl[2];
        return x + h->ncl[0] * (y + h->ncl[1] * z);
    };
    h->cadd.resize((size_t)N * N);
    h->csub.resize((size_t)N * N);
    std::vector<double2> ph((size_t)N * N);
    for (int a = 0; a < N; ++a) {
        const int ax = a % h->ncl[0], ay = (a / h->ncl[0]) % h->ncl[1], az = a / (h->ncl[0] * h->ncl[1]);
        for (int b = 0; b < N; ++b) {
            const int bx = b % h->ncl[0], by = (b / h->ncl[0]) % h->ncl[1], bz = b / (h->ncl[0] * h->ncl[1]);
            h->cadd[(size_t)a * N + b] = cell(ax + bx, ay + by, az + bz);
            h->csub[(size_t)a * N + b] = cell(ax - bx, ay - by, az - bz);
            const double th = 2.0 * 3.14159265358979323846 * ((double)ax * bx / h->ncl[0] + (double)ay * by / h->ncl[1] +
                                             (double)az * bz / h->ncl[2]);
            ph[(size_t)a * N + b] = make_double2(std::cos(th), std::sin(th));
        }
    }
    h->khi.assign(N, -1);
    for (int k = 0; k < N; ++k)
        if (h->csub[(size_t)0 * N + k] >= k) h->khi[k] = h->nkh++;
    int s;
    const size_t nbh = (size_t)nfuc * nau * nfuc * N * h->nkh;
    if ((s = dal(h, &h->B, (size_t)h->nb * h->naux)) || (s = dal(h, &h->Bh, nbh)) || (s = dal(h, &h->ph, (size_t)N * N)) ||
        (s = dal(h, &h->d_khi, (size_t)N)) || (s = dal(h, &h->d_cadd, (size_t)N * N)) ||
        (s = dal(h, &h->d_csub, (size_t)N * N)) || (s = dal(h, &h->P, (size_t)nbas * nbas)) ||
        (s = dal(h, &h->Ps, (size_t)h->nb * N)) || (s = dal(h, &h->G, (size_t)h->naux * N)) ||
        (s = dal(h, &h->gam, (size_t)h->naux)) || (s = dal(h, &h->Jp, (size_t)h->nb)) ||
        (s = dal(h, &h->Kr, (size_t)N * nfuc * nfuc)) || (s = dal(h, &h->Pk, (size_t)N * nfuc * nfuc)) ||
        (s = dal(h, &h->Kt, (size_t)N * nfuc * nfuc))) {
        g_dferr = h->err;
        release(h);
        delete h;
        return s;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemcpy(h->B, B, sizeof(double) * (size_t)h->nb * h->naux, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->Bh, Bh, sizeof(double2) * nbh, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->ph, ph.data(), sizeof(double2) * ph.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_khi, h->khi.data(), sizeof(int) * N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_cadd, h->cadd.data(), sizeof(int) * h->cadd.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_csub, h->csub.data(), sizeof(int) * h->csub.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        g_dferr = std::string("tce_dfjk_create: ") + cudaGetErrorString(e);
        release(h);
        delete h;
        return TCE_ERR_CUDA;
    }
    *handle = h;
    return TCE_OK;
}

int tce_dfjk(void *handle, const double *P, double *J, double *K)
{
    auto *h = static_cast<DfjkHandle *>(handle);
    if (!h || !P || !J || !K) return dfail(h, TCE_ERR_ARG, "NULL argument");
    const int nf = h->nf, N = h->N, nbas = h->nbas;
    cudaStream_t st = h->st;
    cudaMemcpyAsync(h->P, P, sizeof(double) * (size_t)nbas * nbas, cudaMemcpyHostToDevice, st);
    const long long nps = (long long)h->nb * N;
    k_pack_ps<<<(unsigned)((nps + 255) / 256), 256, 0, st>>>(nf, N, nbas, h->d_cadd, h->P, h->Ps);
    dim3 tb(16, 16), gb((N + 15) / 16, (h->naux + 15) / 16);
    k_gemm_tn<<<gb, tb, 0, st>>>(h->naux, N, h->nb, h->B, h->Ps, h->G);
    k_gamma<<<(h->naux + 255) / 256, 256, 0, st>>>(h->nau, N, h->d_csub, h->G, h->gam);
    k_gemv<<<(unsigned)((h->nb + 255) / 256), 256, 0, st>>>(h->nb, h->naux, h->B, h->gam, h->Jp);
    k_pk<<<(N * nf * nf + 255) / 256, 256, 0, st>>>(nf, N, nbas, h->P, h->ph, h->Pk);
    const size_t smem = (size_t)(2 * nf * h->nau * nf + nf * nf) * sizeof(double2);
    int thr = nf * nf < 128 ? 128 : ((nf * nf + 31) / 32) * 32;
    k_kloc<<<N, thr, smem, st>>>(nf, h->nau, N, h->d_csub, h->d_khi, h->Bh, h->Pk, h->Kt, -0.5 / (double)N);
    k_kreal<<<(N * nf * nf + 255) / 256, 256, 0, st>>>(nf, N, h->Kt, h->ph, h->Kr);
    std::vector<double> jp((size_t)h->nb), kr((size_t)N * nf * nf);
    cudaMemcpyAsync(jp.data(), h->Jp, sizeof(double) * jp.size(), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(kr.data(), h->Kr, sizeof(double) * kr.size(), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return dfail(h, TCE_ERR_CUDA, std::string("tce_dfjk: ") + cudaGetErrorString(e));
    for (size_t i = 0; i < (size_t)nbas * nbas; ++i) J[i] = K[i] = 0.0;
    for (int j = 0; j < nbas; ++j)
        for (int a = 0; a < nf; ++a) J[(size_t)a + (size_t)nbas * j] = jp[(size_t)a + (size_t)nf * j];
    for (int r = 0; r < N; ++r)
        for (int b = 0; b < nf; ++b)
            for (int a = 0; a < nf; ++a)
                K[(size_t)a + (size_t)nbas * (r * nf + b)] = kr[(size_t)r * nf * nf + a + nf * b];
    return TCE_OK;
}

int tce_dfjk_destroy(void *handle)
{
    auto *h = static_cast<DfjkHandle *>(handle);
    if (!h) return TCE_OK;
    cudaStreamSynchronize(h->st);
    release(h);
    delete h;
    return TCE_OK;
}

}  // extern "C"
