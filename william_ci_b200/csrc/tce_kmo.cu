// tce_kmo.cu -- k-space MO integrals from the stored SAO integrals on the
// device (transform_ERI_AO_to_kMO, AO_to_MO_SAO.f90:34-393):
//   ERI_out(p, q, r, s, k1, k2, k3) = (p k1, q k2 | r k3, s k4),
//   k4 = k1 - k2 + k3, p, r in p_lo..p_hi, q, s in q_lo..q_hi.
// The handle's stored integrals ERI(a, j2, j3, j4) (tce_eri_stored with
// eri_size = nfuc, chemist order) stay on the device; per k4:
//   k_kmo_x1: X1(a, j2, j3, d)    = sum_R4 ERI(a, j2, j3, d R4) e^{+i k4 R4}
//   k_kmo_x2: X2(a, j2, c, d, k3) = sum_R3 X1(a, j2, c R3, d) e^{-i k3 R3}
//   k_kmo_q : one block per (k1, k2), k3 = k4 - k1 + k2:
//             S(a, b, c, d) = 1/N sum_R2 X2(a, b R2, c, d, k3) e^{+i k2 R2}
//             and the four quarter transforms with the k-block coefficients
//             C_k(a, p) = coeff_SAO(k nfuc + a, k nfuc + p), in shared memory.
#include <vector>

#include "tce_handle.h"

namespace {

__device__ __forceinline__ double2 kmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 kconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ void kadd(double2 &s, double2 v)
{
    s.x += v.x;
    s.y += v.y;
}

__global__ void k_kmo_x1(int nf, int nbas, int N, int k4, const double *eri, const double2 *ph, double2 *X1)
{
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;   // a + nf (j2 + nbas (j3 + nbas d))
    const long long n = (long long)nf * nbas * nbas * nf;
    if (id >= n) return;
    const long long abc = id % ((long long)nf * nbas * nbas);
    const int d = (int)(id / ((long long)nf * nbas * nbas));
    const long long slab = (long long)nf * nbas * nbas;
    double2 s = make_double2(0.0, 0.0);
    for (int r = 0; r < N; ++r) {
        const double v = eri[(size_t)abc + (size_t)slab * (d + (size_t)r * nf)];
        const double2 e = ph[(size_t)k4 * N + r];
        s.x += v * e.x;
        s.y += v * e.y;
    }
    X1[id] = s;
}

__global__ void k_kmo_x2(int nf, int nbas, int N, const double2 *ph, const double2 *X1, double2 *X2)
{
    // X2 index: a + nf (j2 + nbas (c + nf (d + nf k3)))
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long aj = (long long)nf * nbas;
    const long long n = aj * nf * nf * N;
    if (id >= n) return;
    const long long a2 = id % aj;
    long long rest = id / aj;
    const int c = (int)(rest % nf);
    rest /= nf;
    const int d = (int)(rest % nf);
    const int k3 = (int)(rest / nf);
    double2 s = make_double2(0.0, 0.0);
    for (int r = 0; r < N; ++r) {
        const double2 x = X1[(size_t)a2 + (size_t)aj * ((c + (size_t)r * nf) + (size_t)nbas * d)];
        kadd(s, kmul(x, kconj(ph[(size_t)k3 * N + r])));
    }
    X2[id] = s;
}

struct KmoArgs {
    int nf, nbas, N, no, nv, p0, q0, k4;
    const int *k3of;        // [k1 N + k2]
    const double2 *ph, *X2, *C;   // C: coeff_SAO (nbas x nbas), column-major
    double2 *out;           // (no, nv, no, nv, N, N, N)
};

__global__ void k_kmo_q(KmoArgs A)
{
    extern __shared__ double2 sq[];
    const int nf = A.nf, N = A.N, no = A.no, nv = A.nv, nbas = A.nbas;
    const int k1 = blockIdx.x / N, k2 = blockIdx.x % N, k4 = A.k4;
    const int k3 = A.k3of[k1 * N + k2];
    const int f2 = nf * nf, f3 = f2 * nf, f4 = f3 * nf;
    double2 *S = sq;                    // (a, b, c, d)
    double2 *T4 = S + f4;               // (a, b, c, s)
    double2 *T3 = T4 + f3 * nv;         // (a, b, r, s)
    double2 *T2 = T3 + f2 * no * nv;    // (a, q, r, s)
    const int t = threadIdx.x, nt = blockDim.x;
    const double invN = 1.0 / (double)N;
    const long long aj = (long long)nf * nbas;
    auto C = [&](int k, int a, int p) { return A.C[(size_t)(k * nf + a) + (size_t)nbas * (k * nf + p)]; };
    for (int x = t; x < f4; x += nt) {   // x = a + nf (b + nf (c + nf d))
        const int a = x % nf, b = (x / nf) % nf, c = (x / f2) % nf, d = x / f3;
        double2 s = make_double2(0.0, 0.0);
        for (int r = 0; r < N; ++r) {
            const double2 v = A.X2[(size_t)(a + (long long)nf * (b + (long long)r * nf)) +
                                   (size_t)aj * (c + (size_t)nf * (d + (size_t)nf * k3))];
            kadd(s, kmul(v, A.ph[(size_t)k2 * N + r]));
        }
        S[x] = make_double2(s.x * invN, s.y * invN);
    }
    __syncthreads();
    for (int x = t; x < f3 * nv; x += nt) {   // 4th index d -> s
        const int abc = x % f3, s = x / f3;
        double2 v = make_double2(0.0, 0.0);
        for (int d = 0; d < nf; ++d) kadd(v, kmul(S[abc + f3 * d], C(k4, d, A.q0 + s)));
        T4[x] = v;
    }
    __syncthreads();
    for (int x = t; x < f2 * no * nv; x += nt) {   // 3rd index c -> r (conjugated)
        const int ab = x % f2, r = (x / f2) % no, s = x / (f2 * no);
        double2 v = make_double2(0.0, 0.0);
        for (int c = 0; c < nf; ++c) kadd(v, kmul(T4[ab + f2 * c + f3 * s], kconj(C(k3, c, A.p0 + r))));
        T3[x] = v;
    }
    __syncthreads();
    for (int x = t; x < nf * nv * no * nv; x += nt) {   // 2nd index b -> q
        const int a = x % nf, q = (x / nf) % nv, rs = x / (nf * nv);
        double2 v = make_double2(0.0, 0.0);
        for (int b = 0; b < nf; ++b) kadd(v, kmul(T3[a + nf * b + f2 * rs], C(k2, b, A.q0 + q)));
        T2[x] = v;
    }
    __syncthreads();
    const long long blk = (long long)no * nv * no * nv;
    double2 *o = A.out + (size_t)blk * (k1 + (size_t)N * (k2 + (size_t)N * k3));
    for (int x = t; x < blk; x += nt) {   // 1st index a -> p (conjugated)
        const int p = x % no, qrs = x / no;
        double2 v = make_double2(0.0, 0.0);
        for (int a = 0; a < nf; ++a) kadd(v, kmul(kconj(C(k1, a, A.p0 + p)), T2[a + nf * qrs]));
        o[x] = v;
    }
}

}  // namespace

using namespace tcehost;

extern "C" int tce_ao_to_kmo(void *handle, const double *coeff, int32_t p_lo, int32_t p_hi, int32_t q_lo, int32_t q_hi,
                             double *out)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !coeff || !out) return fail(h, TCE_ERR_ARG, "NULL argument");
    const int nf = h->nfuc, nbas = h->nbas, N = h->ncell;
    if (p_lo < 1 || p_hi < p_lo || p_hi > nf || q_lo < 1 || q_hi < q_lo || q_hi > nf)
        return fail(h, TCE_ERR_ARG, "band ranges must lie in 1..nfuc");
    if (!h->d_eri || h->eri_size != nf || h->physicist)
        return fail(h, TCE_ERR_STATE, "needs the stored SAO integrals in chemist order (tce_eri_stored, eri_size = nfuc)");
    const int no = p_hi - p_lo + 1, nv = q_hi - q_lo + 1;
    const size_t smem = sizeof(double2) * ((size_t)nf * nf * nf * nf + (size_t)nf * nf * nf * nv +
                                           (size_t)nf * nf * no * nv + (size_t)nf * nv * no * nv);
    if (smem > 200 * 1024) return fail(h, TCE_ERR_UNSUPPORTED, "nfuc too large for the quarter-transform kernel");
    // cell coordinates (x fastest), phases, k3 = k4 - k1 + k2 per k4
    std::vector<int> cx(N), cy(N), cz(N);
    for (int k = 0; k < N; ++k) {
        cx[k] = k % h->ncl[0];
        cy[k] = (k / h->ncl[0]) % h->ncl[1];
        cz[k] = k / (h->ncl[0] * h->ncl[1]);
    }
    std::vector<double2> ph((size_t)N * N);
    for (int k = 0; k < N; ++k)
        for (int r = 0; r < N; ++r) {
            const double th = 2.0 * kPi * ((double)cx[k] * cx[r] / h->ncl[0] + (double)cy[k] * cy[r] / h->ncl[1] +
                                          (double)cz[k] * cz[r] / h->ncl[2]);
            ph[(size_t)k * N + r] = make_double2(std::cos(th), std::sin(th));
        }
    auto cell = [&](int x, int y, int z) {
        x = ((x % h->ncl[0]) + h->ncl[0]) % h->ncl[0];
        y = ((y % h->ncl[1]) + h->ncl[1]) % h->ncl[1];
        z = ((z % h->ncl[2]) + h->ncl[2]) % h->ncl[2];
        return x + h->ncl[0] * (y + h->ncl[1] * z);
    };
    std::vector<double2> Ch((size_t)nbas * nbas);
    for (size_t i = 0; i < Ch.size(); ++i) Ch[i] = make_double2(coeff[2 * i], coeff[2 * i + 1]);
    const size_t n1 = (size_t)nf * nbas * nbas * nf, n2 = (size_t)nf * nbas * nf * nf * N;
    const size_t nout = (size_t)no * nv * no * nv * N * N * N;
    double2 *d_ph = nullptr, *d_C = nullptr, *d_X1 = nullptr, *d_X2 = nullptr, *d_out = nullptr;
    int *d_k3 = nullptr;
    int s;
    auto cleanup = [&]() {
        dfree(h, d_ph);
        dfree(h, d_C);
        dfree(h, d_X1);
        dfree(h, d_X2);
        dfree(h, d_out);
        dfree(h, d_k3);
    };
    if ((s = upload(h, &d_ph, ph)) || (s = upload(h, &d_C, Ch)) || (s = dalloc(h, &d_X1, n1)) ||
        (s = dalloc(h, &d_X2, n2)) || (s = dalloc(h, &d_out, nout)) || (s = dalloc(h, &d_k3, (size_t)N * N))) {
        cleanup();
        return s;
    }
    std::vector<int> k3of((size_t)N * N);
    cudaFuncSetAttribute(k_kmo_q, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaError_t e = cudaSuccess;
    for (int k4 = 0; k4 < N && e == cudaSuccess; ++k4) {
        for (int k1 = 0; k1 < N; ++k1)
            for (int k2 = 0; k2 < N; ++k2)
                k3of[(size_t)k1 * N + k2] = cell(cx[k4] - cx[k1] + cx[k2], cy[k4] - cy[k1] + cy[k2], cz[k4] - cz[k1] + cz[k2]);
        e = cudaMemcpyAsync(d_k3, k3of.data(), sizeof(int) * k3of.size(), cudaMemcpyHostToDevice, h->st);
        if (e != cudaSuccess) break;
        k_kmo_x1<<<(unsigned)((n1 + 255) / 256), 256, 0, h->st>>>(nf, nbas, N, k4, h->d_eri, d_ph, d_X1);
        k_kmo_x2<<<(unsigned)((n2 + 255) / 256), 256, 0, h->st>>>(nf, nbas, N, d_ph, d_X1, d_X2);
        KmoArgs A{nf, nbas, N, no, nv, p_lo - 1, q_lo - 1, k4, d_k3, d_ph, d_X2, d_C, d_out};
        k_kmo_q<<<(unsigned)(N * N), 256, smem, h->st>>>(A);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);   // k3of is reused
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, d_out, sizeof(double2) * nout, cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    cleanup();
    if (e != cudaSuccess) return fail(h, TCE_ERR_CUDA, std::string("tce_ao_to_kmo: ") + cudaGetErrorString(e));
    return TCE_OK;
}
