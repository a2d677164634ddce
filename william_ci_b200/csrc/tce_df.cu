// tce_df.cu -- density fitting and DF-MP2 on the device, behind the C ABI.
//
// Replaces df_init (df_toroidal.f90:352-701), chol_f (:1174-1216), df_L_kap
// (:1053-1104) and, with tce_dfmp2_energy, kMP2_calc (MP2_SAO.f90:6-151):
//
//   * the system of the fit holds per cell the orbital functions, the
//     auxiliary functions and one constant dummy (s, exponent 0, coefficient
//     1) per atom; (mu nu|P) = (mu nu|P 1) and (P|Q) = (P 1|Q 1) are ordinary
//     shell blocks of a blocks-only handle (df_toroidal.f90:837), written by
//     the quartet kernel to device memory and scattered into
//       Vm(P0, Q R)          nau x naux         (naux = nau N)
//       T3(mu0, nu, P R)     nf x nb x naux     (nb = nf N), column-major;
//   * V(k) = sum_R (P0|Q R) e^{i k.R} (phase 2 pi sum_d k_d R_d / n_d, the
//     convention of SAO_Transfer.f90:34-44), Hermitised, factorised per k by a
//     pivoted Cholesky with tolerance 1e-10 and inverted on the host (nau x nau
//     per k), f(k)(piv(i), j) = conj(L^-1(j, i)), f(-k) = conj f(k);
//   * B = Re 1/N sum_k [sum_R T3(R) e^{i k.R}] f(k) e^{-i k.R'} (df_B), and the
//     half-set k-space Bh of the density-fitted J/K (:660-678);
//   * L^Q_pq(k1, k2) = sum_ab conj C_k1(a, p) [sum_R sum_s B(a, b R, Q s)
//     e^{-i kap.s} e^{i k2.R}] C_k2(b, q), kap = k2 - k1 (df_L_kap), then the
//     (ov|ov) contraction and the energy of tce_dfmp2_energy.
//
// Each transform is a sum over cells run as one thread per output element
// against a table of the N x N phases; with N = 128 cells, nf = 6, nau = 16 it
// is about 1e9 complex multiply-adds per step, a few milliseconds.
#include <algorithm>
#include <cmath>
#include <complex>
#include <string>
#include <vector>

#include "tce_handle.h"

using namespace tcehost;

namespace {

struct DfHandle {
    std::string err;
    void *eng = nullptr;      // blocks-only handle of the fit's system
    int N = 1, ncl[3] = {1, 1, 1}, nf = 0, nau = 0, nat = 0, nfc = 0;
    int ndrop = 0;
    cudaStream_t st = nullptr;
    double2 *d_ph = nullptr;  // [k * N + R] = e^{i k.R}
    int *d_crd = nullptr;     // [3 k + d] cell coordinates
    double *d_Vm = nullptr, *d_T3 = nullptr, *d_B = nullptr;
    double2 *d_W = nullptr;   // W(k)(x, q) = [sum_R T3(R) e^{ikR}] f(k), x = mu + nf nu
    std::vector<void *> mem;
};

thread_local std::string g_df_err;

int df_fail(DfHandle *d, int code, const std::string &m)
{
    if (d) d->err = m;
    g_df_err = m;
    return code;
}

template <class T>
int df_alloc(DfHandle *d, T **p, size_t n)
{
    *p = nullptr;
    if (cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return df_fail(d, TCE_ERR_NOMEM, "device allocation of " + std::to_string(n * sizeof(T)) + " bytes failed");
    }
    d->mem.push_back(*p);
    return TCE_OK;
}

void df_free(DfHandle *d, void *p)
{
    if (!p) return;
    cudaFree(p);
    d->mem.erase(std::remove(d->mem.begin(), d->mem.end(), p), d->mem.end());
}

#define DCK(d, call)                                                                                   \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return df_fail((d), TCE_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
// block element -> fit array: one warp per item, lanes over the block's
// elements (n1 x n2 x n3, the dummy's dimension is 1); dst index
// g1 + e1 + s2 (g2 + e2) + s3 (g3 + e3)
__global__ void k_df_scatter(const double *__restrict__ blk, const long long *__restrict__ off,
                             const int4 *__restrict__ dims, const int4 *__restrict__ base, long long nitems,
                             long long s2, long long s3, double *dst)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= nitems) return;
    const int4 n = dims[w], g = base[w];
    const long long o = off[w];
    const int tot = n.x * n.y * n.z;
    for (int e = lane; e < tot; e += 32) {
        const int e1 = e % n.x, r = e / n.x, e2 = r % n.y, e3 = r / n.y;
        dst[(g.x + e1) + s2 * (g.y + e2) + s3 * (g.z + e3)] = blk[o + e];
    }
}

// M(k)(p, q) = sum_R Vm(p, R nau + q) e^{ikR}, Hermitised later on the host
__global__ void k_df_metric_k(const double *__restrict__ Vm, const double2 *__restrict__ ph, int N, int nau,
                              double2 *M)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)N * nau * nau) return;
    const int p = (int)(t % nau), q = (int)((t / nau) % nau), k = (int)(t / ((long long)nau * nau));
    double re = 0.0, im = 0.0;
    for (int R = 0; R < N; ++R) {
        const double v = Vm[p + (long long)nau * (R * nau + q)];
        const double2 e = ph[(long long)k * N + R];
        re = fma(v, e.x, re);
        im = fma(v, e.y, im);
    }
    M[t] = make_double2(re, im);
}

// W(k)(x, q) = sum_p [sum_R T3(x, R nau + p) e^{ikR}] f(k)(p, q), x < X = nf nb
__global__ void k_df_w(const double *__restrict__ T3, const double2 *__restrict__ ph, const double2 *__restrict__ f,
                       long long X, int N, int nau, double2 *W)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= X * N) return;
    const long long x = t % X;
    const int k = (int)(t / X);
    double zr[32], zi[32];
    for (int p = 0; p < nau; ++p) {
        double re = 0.0, im = 0.0;
        for (int R = 0; R < N; ++R) {
            const double v = T3[x + X * ((long long)R * nau + p)];
            const double2 e = ph[(long long)k * N + R];
            re = fma(v, e.x, re);
            im = fma(v, e.y, im);
        }
        zr[p] = re;
        zi[p] = im;
    }
    const double2 *fk = f + (long long)k * nau * nau;
    for (int q = 0; q < nau; ++q) {
        double re = 0.0, im = 0.0;
        for (int p = 0; p < nau; ++p) {
            const double2 c = fk[p + nau * q];
            re += zr[p] * c.x - zi[p] * c.y;
            im += zr[p] * c.y + zi[p] * c.x;
        }
        W[((long long)k * nau + q) * X + x] = make_double2(re, im);
    }
}

// B(x, R nau + q) = Re 1/N sum_k W(k)(x, q) e^{-ikR}
__global__ void k_df_b(const double2 *__restrict__ W, const double2 *__restrict__ ph, long long X, int N, int nau,
                       double *B)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= X * N * nau) return;
    const long long x = t % X;
    const long long c = t / X;              // R nau + q
    const int q = (int)(c % nau), R = (int)(c / nau);
    double s = 0.0;
    for (int k = 0; k < N; ++k) {
        const double2 w = W[((long long)k * nau + q) * X + x];
        const double2 e = ph[(long long)k * N + R];
        s += w.x * e.x + w.y * e.y;         // Re(w conj(e))
    }
    B[t] = s / (double)N;
}

// Bh(mu, Q, nu0; k1, kh) = sum_R1 W(k)(mu, nu0 R1, Q) e^{i k1 R1} for the k of the half set
__global__ void k_df_bh(const double2 *__restrict__ W, const double2 *__restrict__ ph, const int *__restrict__ kh_k,
                        int nkh, long long X, int N, int nf, int nau, double2 *Bh)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long tot = (long long)nf * nau * nf * N * nkh;
    if (t >= tot) return;
    long long r = t;
    const int mu = (int)(r % nf); r /= nf;
    const int Q = (int)(r % nau); r /= nau;
    const int nu0 = (int)(r % nf); r /= nf;
    const int k1 = (int)(r % N);
    const int kh = (int)(r / N);
    const int k = kh_k[kh];
    double re = 0.0, im = 0.0;
    for (int R1 = 0; R1 < N; ++R1) {
        const long long x = mu + (long long)nf * ((long long)R1 * nf + nu0);
        const double2 w = W[((long long)k * nau + Q) * X + x];
        const double2 e = ph[(long long)k1 * N + R1];
        re += w.x * e.x - w.y * e.y;
        im += w.x * e.y + w.y * e.x;
    }
    Bh[t] = make_double2(re, im);
}

// G1(kap)(x, q) = sum_s B(x, s nau + q) conj e^{i kap s}
__global__ void k_df_g1(const double *__restrict__ B, const double2 *__restrict__ ph, long long X, int N, int nau,
                        double2 *G1)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= X * nau * N) return;
    const long long x = t % X;
    const long long c = t / X;
    const int q = (int)(c % nau), kap = (int)(c / nau);
    double re = 0.0, im = 0.0;
    for (int s = 0; s < N; ++s) {
        const double b = B[x + X * ((long long)s * nau + q)];
        const double2 e = ph[(long long)kap * N + s];
        re = fma(b, e.x, re);
        im = fma(-b, e.y, im);
    }
    G1[t] = make_double2(re, im);
}

// F(a, b, q, kap, k2) = sum_R G1(kap)(a + nf (R nf + b), q) e^{i k2 R}
__global__ void k_df_f(const double2 *__restrict__ G1, const double2 *__restrict__ ph, long long X, int N, int nf,
                       int nau, double2 *F)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long tot = (long long)nf * nf * nau * N * N;
    if (t >= tot) return;
    long long r = t;
    const int a = (int)(r % nf); r /= nf;
    const int b = (int)(r % nf); r /= nf;
    const int q = (int)(r % nau); r /= nau;
    const int kap = (int)(r % N);
    const int k2 = (int)(r / N);
    double re = 0.0, im = 0.0;
    const double2 *g = G1 + ((long long)kap * nau + q) * X;
    for (int R = 0; R < N; ++R) {
        const double2 v = g[a + (long long)nf * ((long long)R * nf + b)];
        const double2 e = ph[(long long)k2 * N + R];
        re += v.x * e.x - v.y * e.y;
        im += v.x * e.y + v.y * e.x;
    }
    F[t] = make_double2(re, im);
}

// L(p, v, q, k1, k2) = sum_ab conj C_k1(a, p0 + p) F(a, b, q, kap, k2) C_k2(b, v0 + v),
// kap = k2 - k1; C_k(a, j) = coeff(k nf + a, k nf + j)
__global__ void k_df_l(const double2 *__restrict__ F, const double2 *__restrict__ coeff, const int *__restrict__ crd,
                       int n0, int n1, int n2, int N, int nf, int nau, int p0, int no, int v0, int nv, double2 *L)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long tot = (long long)no * nv * nau * N * N;
    if (t >= tot) return;
    long long r = t;
    const int p = (int)(r % no); r /= no;
    const int v = (int)(r % nv); r /= nv;
    const int q = (int)(r % nau); r /= nau;
    const int k1 = (int)(r % N);
    const int k2 = (int)(r / N);
    const int nn[3] = {n0, n1, n2};
    int kap = 0, mul = 1;
    for (int d = 0; d < 3; ++d) {
        int c = crd[3 * k2 + d] - crd[3 * k1 + d];
        c += c < 0 ? nn[d] : 0;
        kap += mul * c;
        mul *= nn[d];
    }
    const long long nbas = (long long)nf * N;
    const double2 *F0 = F + (((long long)k2 * N + kap) * nau + q) * nf * nf;
    double re = 0.0, im = 0.0;
    for (int b = 0; b < nf; ++b) {
        const double2 cb = coeff[((long long)k2 * nf + b) + nbas * ((long long)k2 * nf + v0 + v)];
        double tr = 0.0, ti = 0.0;          // sum_a conj C1(a, p) F(a, b)
        for (int a = 0; a < nf; ++a) {
            const double2 ca = coeff[((long long)k1 * nf + a) + nbas * ((long long)k1 * nf + p0 + p)];
            const double2 f = F0[a + (long long)nf * b];
            tr += ca.x * f.x + ca.y * f.y;
            ti += ca.x * f.y - ca.y * f.x;
        }
        re += tr * cb.x - ti * cb.y;
        im += tr * cb.y + ti * cb.x;
    }
    L[t] = make_double2(re, im);
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
using cplx = std::complex<double>;

// Pivoted Cholesky of a Hermitian positive semi-definite n x n matrix A
// (column-major) to the rank where the largest remaining diagonal falls to
// tol (at the first step: to zero), in the order of operations of LAPACK's
// unblocked zpstf2 (lower), which zpstrf runs for matrices of this size
// (chol_f, df_toroidal.f90:1174-1216): the remaining diagonal is A(i,i) minus
// the running sum of |L(i,c)|^2, the first maximum is the pivot, column j is
// A(j+1:n, j) - sum_c L(:,c) conj L(j,c) in order c = 1..j-1, scaled by
// 1 / L(j,j).  Then f(piv(i), j) = conj(L^-1(j, i)) for i, j < rank, zero
// elsewhere.  Returns the rank.  Where remaining diagonals tie exactly
// (symmetry-equivalent auxiliary functions), the pivot picked depends on the
// last bits of the running sums, in LAPACK as here; the fitted space, and so
// the fitted integrals, do not.
int chol_f(int n, std::vector<cplx> A, double tol, std::vector<cplx> &f)
{
    std::vector<int> piv(n);
    for (int i = 0; i < n; ++i) piv[i] = i;
    std::vector<double> d0(n), work(n, 0.0);
    for (int i = 0; i < n; ++i) d0[i] = A[i + (size_t)n * i].real();
    std::vector<cplx> L((size_t)n * n, 0.0);
    auto at = [&](int i, int j) -> cplx & { return A[i + (size_t)n * j]; };
    int m = n;
    int pvt = 0;
    for (int i = 1; i < n; ++i)
        if (d0[i] > d0[pvt]) pvt = i;
    double ajj = d0[pvt];
    if (!(ajj > 0.0)) m = 0;
    for (int j = 0; j < m; ++j) {
        if (j > 0) {
            for (int i = j; i < n; ++i) work[i] += std::norm(L[i + (size_t)n * (j - 1)]);
            pvt = j;
            for (int i = j + 1; i < n; ++i)
                if (d0[i] - work[i] > d0[pvt] - work[pvt]) pvt = i;
            ajj = d0[pvt] - work[pvt];
            if (ajj <= tol || std::isnan(ajj)) {
                m = j;
                break;
            }
        }
        if (pvt != j) {
            for (int c = 0; c < n; ++c) std::swap(at(j, c), at(pvt, c));
            for (int r = 0; r < n; ++r) std::swap(at(r, j), at(r, pvt));
            for (int c = 0; c < j; ++c) std::swap(L[j + (size_t)n * c], L[pvt + (size_t)n * c]);
            std::swap(d0[j], d0[pvt]);
            std::swap(work[j], work[pvt]);
            std::swap(piv[j], piv[pvt]);
        }
        const double ljj = std::sqrt(ajj), rj = 1.0 / ljj;
        L[j + (size_t)n * j] = ljj;
        for (int i = j + 1; i < n; ++i) {
            cplx s = at(i, j);
            for (int c = 0; c < j; ++c) s -= L[i + (size_t)n * c] * std::conj(L[j + (size_t)n * c]);
            L[i + (size_t)n * j] = s * rj;
        }
    }
    // inverse of the leading m x m lower triangle (forward substitution per column)
    std::vector<cplx> Li((size_t)m * m, 0.0);
    for (int c = 0; c < m; ++c) {
        Li[c + (size_t)m * c] = 1.0 / L[c + (size_t)n * c];
        for (int i = c + 1; i < m; ++i) {
            cplx s = 0.0;
            for (int k = c; k < i; ++k) s += L[i + (size_t)n * k] * Li[k + (size_t)m * c];
            Li[i + (size_t)m * c] = -s / L[i + (size_t)n * i];
        }
    }
    f.assign((size_t)n * n, 0.0);
    for (int i = 0; i < m; ++i)
        for (int jj = 0; jj < m; ++jj) f[piv[i] + (size_t)n * jj] = std::conj(Li[jj + (size_t)m * i]);
    return m;
}

void cell_coords(const int ncl[3], int k, int c[3])
{
    c[0] = k % ncl[0];
    c[1] = (k / ncl[0]) % ncl[1];
    c[2] = k / (ncl[0] * ncl[1]);
}

int neg_cell(const int ncl[3], int k)
{
    int c[3];
    cell_coords(ncl, k, c);
    for (int d = 0; d < 3; ++d) c[d] = (ncl[d] - c[d]) % ncl[d];
    return c[0] + ncl[0] * (c[1] + ncl[1] * c[2]);
}

// the blocks of host items on the device, concatenated (offsets returned)
int device_blocks(DfHandle *d, Handle *h, const std::vector<int4> &items, double **d_out,
                  std::vector<long long> &off)
{
    off.assign(items.size() + 1, 0);
    int mx = 1, mq = 1;
    for (size_t i = 0; i < items.size(); ++i) {
        const int4 &q = items[i];
        const long long n = (long long)h->sh_n[q.x] * h->sh_n[q.y] * h->sh_n[q.z] * h->sh_n[q.w];
        off[i + 1] = off[i] + n;
        mq = std::max<int>(mq, (int)n);
        mx = std::max(mx, ncomb_of(h, q.x, q.y, q.z, q.w));
    }
    int4 *d_it = nullptr;
    long long *d_off = nullptr;
    int s;
    if ((s = df_alloc(d, &d_it, items.size()))) return s;
    if ((s = df_alloc(d, &d_off, off.size()))) return s;
    if ((s = df_alloc(d, d_out, (size_t)off.back()))) return s;
    DCK(d, cudaMemcpyAsync(d_it, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice, d->st));
    DCK(d, cudaMemcpyAsync(d_off, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice, d->st));
    QuartetHostArgs a;
    a.items = d_it;
    a.nitems = (int)items.size();
    a.mode = TCE_MODE_BLOCK;           // prefactor screens, no primitive screen (as ps_on = .false.)
    a.prim_screen = 0;
    a.next = h->d_next;
    a.blk_out = *d_out;
    a.blk_off = d_off;
    a.pp_rw = h->d_pp;
    a.max_ncomb = mx;
    a.max_ncq = std::max(mq, 1);
    a.fixed_gmax = h->d_gmax;
    a.num_sms = h->num_sms;
    if (tce_launch_quartets(h->S, a, d->st) != TCE_OK)
        return df_fail(d, TCE_ERR_CUDA, std::string("fit integrals: ") + cudaGetErrorString(cudaGetLastError()));
    DCK(d, cudaStreamSynchronize(d->st));
    df_free(d, d_it);
    df_free(d, d_off);
    return TCE_OK;
}

int scatter(DfHandle *d, const double *blk, const std::vector<long long> &off, const std::vector<int4> &dims,
            const std::vector<int4> &base, long long s2, long long s3, double *dst)
{
    const long long n = (long long)dims.size();
    if (n == 0) return TCE_OK;
    long long *d_off = nullptr;
    int4 *d_dims = nullptr, *d_base = nullptr;
    int s;
    if ((s = df_alloc(d, &d_off, off.size()))) return s;
    if ((s = df_alloc(d, &d_dims, dims.size()))) return s;
    if ((s = df_alloc(d, &d_base, base.size()))) return s;
    DCK(d, cudaMemcpyAsync(d_off, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice, d->st));
    DCK(d, cudaMemcpyAsync(d_dims, dims.data(), sizeof(int4) * dims.size(), cudaMemcpyHostToDevice, d->st));
    DCK(d, cudaMemcpyAsync(d_base, base.data(), sizeof(int4) * base.size(), cudaMemcpyHostToDevice, d->st));
    k_df_scatter<<<nblk(32 * n, 256), 256, 0, d->st>>>(blk, d_off, d_dims, d_base, n, s2, s3, dst);
    DCK(d, cudaGetLastError());
    DCK(d, cudaStreamSynchronize(d->st));
    df_free(d, d_off);
    df_free(d, d_dims);
    df_free(d, d_base);
    return TCE_OK;
}

int df_build(DfHandle *d, const tce_system *ao, const tce_system *aux, int natoms, const double *geo)
{
    if (!ao || !aux || !geo || natoms < 1) return df_fail(d, TCE_ERR_ARG, "NULL argument");
    if (ao->ndp != aux->ndp) return df_fail(d, TCE_ERR_ARG, "orbital and auxiliary systems differ in ndp");
    for (int k = 0; k < 3; ++k)
        if (ao->ncell[k] != aux->ncell[k] || ao->L[k] != aux->L[k])
            return df_fail(d, TCE_ERR_ARG, "orbital and auxiliary systems differ in cells or torus lengths");
    for (int k = 0; k < 3; ++k) d->ncl[k] = std::max(1, ao->ncell[k]);
    d->N = d->ncl[0] * d->ncl[1] * d->ncl[2];
    const int N = d->N;
    if (natoms % N) return df_fail(d, TCE_ERR_ARG, "atom count not a multiple of the cell count");
    d->nf = ao->nfuc;
    d->nau = aux->nfuc;
    d->nat = natoms / N;
    if (d->nau > 32) return df_fail(d, TCE_ERR_UNSUPPORTED, "more than 32 auxiliary functions per cell");
    d->nfc = d->nf + d->nau + d->nat;
    const int nf = d->nf, nau = d->nau, nat = d->nat, nfc = d->nfc;
    // ---- the fit's system: per cell the orbital, auxiliary and dummy functions
    std::vector<double> ctr, exps, coefs;
    std::vector<int32_t> lxyz, poff{0};
    auto add = [&](const tce_system *s, int f) {
        for (int k = 0; k < 3; ++k) {
            ctr.push_back(s->ctr[3 * f + k]);
            lxyz.push_back(s->lxyz[3 * f + k]);
        }
        for (int p = s->prim_off[f]; p < s->prim_off[f + 1]; ++p) {
            exps.push_back(s->exps[p]);
            coefs.push_back(s->coefs[p]);
        }
        poff.push_back((int32_t)exps.size());
    };
    for (int c = 0; c < N; ++c) {
        for (int f = 0; f < nf; ++f) add(ao, c * nf + f);
        for (int f = 0; f < nau; ++f) add(aux, c * nau + f);
        for (int a = 0; a < nat; ++a) {
            for (int k = 0; k < 3; ++k) {
                ctr.push_back(geo[(size_t)(c * nat + a) + (size_t)natoms * k]);
                lxyz.push_back(0);
            }
            exps.push_back(0.0);
            coefs.push_back(1.0);
            poff.push_back((int32_t)exps.size());
        }
    }
    tce_system sys = *ao;
    sys.nfuc = nfc;
    sys.nbas = nfc * N;
    sys.ctr = ctr.data();
    sys.lxyz = lxyz.data();
    sys.prim_off = poff.data();
    sys.exps = exps.data();
    sys.coefs = coefs.data();
    sys.prim_screen = 0;
    int s = tce_create_blocks(&sys, &d->eng);
    if (s) return df_fail(d, s, std::string("fit system: ") + tce_last_error(nullptr));
    Handle *h = static_cast<Handle *>(d->eng);
    d->st = h->st;
    // ---- shells: kind (0 orbital, 1 auxiliary, 2 dummy), index of the first
    // function in its numbering (orbital nu = R nf + i, auxiliary R nau + P), and
    // the dummy at an auxiliary shell's centre
    const int nsh = h->nsh;
    std::vector<int> kind(nsh), gidx(nsh), dummy(nsh, -1);
    for (int S = 0; S < nsh; ++S) {
        const int f = h->sh_first[S], c = f / nfc, loc = f - c * nfc;
        kind[S] = loc < nf ? 0 : (loc < nf + nau ? 1 : 2);
        gidx[S] = kind[S] == 0 ? c * nf + loc : (kind[S] == 1 ? c * nau + (loc - nf) : -1);
    }
    for (int S = 0; S < nsh; ++S) {
        if (kind[S] != 1) continue;
        const int f = h->sh_first[S];
        for (int T = 0; T < nsh && dummy[S] < 0; ++T) {
            if (kind[T] != 2) continue;
            const int g = h->sh_first[T];
            double d2 = 0.0;
            for (int k = 0; k < 3; ++k) d2 += (ctr[3 * f + k] - ctr[3 * g + k]) * (ctr[3 * f + k] - ctr[3 * g + k]);
            if (d2 < 1e-16) dummy[S] = T;
        }
        if (dummy[S] < 0) return df_fail(d, TCE_ERR_ARG, "an auxiliary function has no atom at its centre");
    }
    std::vector<int> ao_uc, ao_all, aux_uc, aux_all;
    for (int S = 0; S < nsh; ++S) {
        if (kind[S] == 0) {
            ao_all.push_back(S);
            if (S < h->nshuc) ao_uc.push_back(S);
        } else if (kind[S] == 1) {
            aux_all.push_back(S);
            if (S < h->nshuc) aux_uc.push_back(S);
        }
    }
    const long long naux = (long long)nau * N, nb = (long long)nf * N, X = (long long)nf * nb;
    // ---- metric Vm(P0, Q R) = (P 1 | Q 1)
    if ((s = df_alloc(d, &d->d_Vm, (size_t)nau * naux))) return s;
    if ((s = df_alloc(d, &d->d_T3, (size_t)X * naux))) return s;
    DCK(d, cudaMemsetAsync(d->d_Vm, 0, sizeof(double) * nau * naux, d->st));
    DCK(d, cudaMemsetAsync(d->d_T3, 0, sizeof(double) * X * naux, d->st));
    {
        std::vector<int4> items, dims, base;
        for (int p : aux_uc)
            for (int q : aux_all) {
                items.push_back(make_int4(p, dummy[p], q, dummy[q]));
                dims.push_back(make_int4(h->sh_n[p], h->sh_n[q], 1, 0));
                base.push_back(make_int4(gidx[p], gidx[q], 0, 0));
            }
        double *blk = nullptr;
        std::vector<long long> off;
        if ((s = device_blocks(d, h, items, &blk, off))) return s;
        // blocks are (nP, 1, nQ, 1): element (e1, e2) -> Vm(g1 + e1, g2 + e2)
        if ((s = scatter(d, blk, off, dims, base, nau, 0, d->d_Vm))) return s;
        df_free(d, blk);
    }
    // ---- three-index T3(mu0, nu, P R) = (mu0 nu | P 1), in pieces of at most
    // 4M items (the unit-cell orbital shell times all orbital shells at a time)
    for (int a : ao_uc) {
        std::vector<int4> items, dims, base;
        for (int b : ao_all)
            for (int p : aux_all) {
                items.push_back(make_int4(a, b, p, dummy[p]));
                dims.push_back(make_int4(h->sh_n[a], h->sh_n[b], h->sh_n[p], 0));
                base.push_back(make_int4(gidx[a], gidx[b], gidx[p], 0));
            }
        double *blk = nullptr;
        std::vector<long long> off;
        if ((s = device_blocks(d, h, items, &blk, off))) return s;
        if ((s = scatter(d, blk, off, dims, base, nf, X, d->d_T3))) return s;
        df_free(d, blk);
    }
    // ---- phases e^{i k.R} and cell coordinates
    {
        std::vector<double2> ph((size_t)N * N);
        std::vector<int> crd(3 * (size_t)N);
        for (int k = 0; k < N; ++k) {
            int ck[3];
            cell_coords(d->ncl, k, ck);
            for (int dd = 0; dd < 3; ++dd) crd[3 * k + dd] = ck[dd];
            for (int R = 0; R < N; ++R) {
                int cr[3];
                cell_coords(d->ncl, R, cr);
                double th = 0.0;
                for (int dd = 0; dd < 3; ++dd) th += (double)((ck[dd] * cr[dd]) % d->ncl[dd]) / (double)d->ncl[dd];
                th *= 2.0 * kPi;
                ph[(size_t)k * N + R] = make_double2(std::cos(th), std::sin(th));
            }
        }
        if ((s = df_alloc(d, &d->d_ph, ph.size()))) return s;
        if ((s = df_alloc(d, &d->d_crd, crd.size()))) return s;
        DCK(d, cudaMemcpyAsync(d->d_ph, ph.data(), sizeof(double2) * ph.size(), cudaMemcpyHostToDevice, d->st));
        DCK(d, cudaMemcpyAsync(d->d_crd, crd.data(), sizeof(int) * crd.size(), cudaMemcpyHostToDevice, d->st));
    }
    // ---- V(k), its factor f(k) on the host
    std::vector<double2> f_all((size_t)N * nau * nau);
    {
        double2 *d_M = nullptr;
        if ((s = df_alloc(d, &d_M, (size_t)N * nau * nau))) return s;
        k_df_metric_k<<<nblk((long long)N * nau * nau, 256), 256, 0, d->st>>>(d->d_Vm, d->d_ph, N, nau, d_M);
        DCK(d, cudaGetLastError());
        std::vector<double2> M((size_t)N * nau * nau);
        DCK(d, cudaMemcpyAsync(M.data(), d_M, sizeof(double2) * M.size(), cudaMemcpyDeviceToHost, d->st));
        DCK(d, cudaStreamSynchronize(d->st));
        df_free(d, d_M);
        std::vector<std::vector<cplx>> fk(N);
        d->ndrop = 0;
        for (int k = 0; k < N; ++k) {
            const int mk = neg_cell(d->ncl, k);
            if (mk < k) continue;
            std::vector<cplx> A((size_t)nau * nau);
            for (int p = 0; p < nau; ++p)
                for (int q = 0; q < nau; ++q) {
                    const double2 a = M[(size_t)k * nau * nau + p + (size_t)nau * q];
                    const double2 b = M[(size_t)k * nau * nau + q + (size_t)nau * p];
                    A[p + (size_t)nau * q] = 0.5 * (cplx(a.x, a.y) + std::conj(cplx(b.x, b.y)));
                }
            const int m = chol_f(nau, A, 1e-10, fk[k]);
            d->ndrop = std::max(d->ndrop, nau - m);
        }
        for (int k = 0; k < N; ++k) {
            const int mk = neg_cell(d->ncl, k);
            const bool cj = mk < k;
            const std::vector<cplx> &src = cj ? fk[mk] : fk[k];
            for (size_t i = 0; i < (size_t)nau * nau; ++i) {
                const cplx v = cj ? std::conj(src[i]) : src[i];
                f_all[(size_t)k * nau * nau + i] = make_double2(v.real(), v.imag());
            }
        }
    }
    // ---- W(k) and B
    double2 *d_f = nullptr;
    if ((s = df_alloc(d, &d_f, f_all.size()))) return s;
    DCK(d, cudaMemcpyAsync(d_f, f_all.data(), sizeof(double2) * f_all.size(), cudaMemcpyHostToDevice, d->st));
    if ((s = df_alloc(d, &d->d_W, (size_t)X * nau * N))) return s;
    if ((s = df_alloc(d, &d->d_B, (size_t)X * naux))) return s;
    k_df_w<<<nblk(X * N, 128), 128, 0, d->st>>>(d->d_T3, d->d_ph, d_f, X, N, nau, d->d_W);
    DCK(d, cudaGetLastError());
    k_df_b<<<nblk(X * naux, 256), 256, 0, d->st>>>(d->d_W, d->d_ph, X, N, nau, d->d_B);
    DCK(d, cudaGetLastError());
    DCK(d, cudaStreamSynchronize(d->st));
    df_free(d, d_f);
    return TCE_OK;
}

void df_release(DfHandle *d)
{
    for (void *p : d->mem) cudaFree(p);
    d->mem.clear();
    if (d->eng) tce_destroy(d->eng);
    d->eng = nullptr;
}

}  // namespace

extern "C" {

const char *tce_df_last_error(void *df)
{
    if (df) return static_cast<DfHandle *>(df)->err.c_str();
    return g_df_err.c_str();
}

int tce_df_create(const tce_system *ao, const tce_system *aux, int32_t natoms, const double *geometry, void **df)
{
    if (!df) return df_fail(nullptr, TCE_ERR_ARG, "handle is NULL");
    *df = nullptr;
    DfHandle *d = new DfHandle();
    const int s = df_build(d, ao, aux, natoms, geometry);
    if (s) {
        g_df_err = d->err;
        df_release(d);
        delete d;
        return s;
    }
    *df = d;
    return TCE_OK;
}

int tce_df_destroy(void *df)
{
    DfHandle *d = static_cast<DfHandle *>(df);
    if (!d) return TCE_OK;
    df_release(d);
    delete d;
    return TCE_OK;
}

int tce_df_integrals(void *df, double *Vm, double *T3)
{
    DfHandle *d = static_cast<DfHandle *>(df);
    if (!d) return df_fail(d, TCE_ERR_ARG, "NULL handle");
    const size_t naux = (size_t)d->nau * d->N, X = (size_t)d->nf * d->nf * d->N;
    if (Vm) DCK(d, cudaMemcpy(Vm, d->d_Vm, sizeof(double) * d->nau * naux, cudaMemcpyDeviceToHost));
    if (T3) DCK(d, cudaMemcpy(T3, d->d_T3, sizeof(double) * X * naux, cudaMemcpyDeviceToHost));
    return TCE_OK;
}

int tce_df_fitted(void *df, double *B, double *Bh, int32_t *ndrop)
{
    DfHandle *d = static_cast<DfHandle *>(df);
    if (!d) return df_fail(d, TCE_ERR_ARG, "NULL handle");
    const int N = d->N, nf = d->nf, nau = d->nau;
    const long long X = (long long)nf * nf * N;
    if (ndrop) *ndrop = d->ndrop;
    if (B) DCK(d, cudaMemcpy(B, d->d_B, sizeof(double) * X * nau * N, cudaMemcpyDeviceToHost));
    if (Bh) {
        std::vector<int> kh;
        for (int k = 0; k < N; ++k)
            if (neg_cell(d->ncl, k) >= k) kh.push_back(k);
        const long long tot = (long long)nf * nau * nf * N * (long long)kh.size();
        int *d_kh = nullptr;
        double2 *d_Bh = nullptr;
        int s;
        if ((s = df_alloc(d, &d_kh, kh.size()))) return s;
        if ((s = df_alloc(d, &d_Bh, (size_t)tot))) return s;
        DCK(d, cudaMemcpyAsync(d_kh, kh.data(), sizeof(int) * kh.size(), cudaMemcpyHostToDevice, d->st));
        k_df_bh<<<nblk(tot, 256), 256, 0, d->st>>>(d->d_W, d->d_ph, d_kh, (int)kh.size(), X, N, nf, nau, d_Bh);
        DCK(d, cudaGetLastError());
        DCK(d, cudaMemcpyAsync(Bh, d_Bh, sizeof(double2) * tot, cudaMemcpyDeviceToHost, d->st));
        DCK(d, cudaStreamSynchronize(d->st));
        df_free(d, d_kh);
        df_free(d, d_Bh);
    }
    return TCE_OK;
}

int tce_dfmp2(void *df, const double *coeff, const double *eps, const int32_t *occ, int32_t mode, double *e_mp2,
              double *e2d, double *e2x)
{
    DfHandle *d = static_cast<DfHandle *>(df);
    if (!d || !coeff || !eps || !occ || !e_mp2) return df_fail(d, TCE_ERR_ARG, "NULL argument");
    const int N = d->N, nf = d->nf, nau = d->nau;
    const long long nbas = (long long)nf * N, X = (long long)nf * nbas;
    // band ranges of cc_dims: occupied 1..max_k nocc(k), virtual min_k nocc(k)+1..nfuc
    int ohi = 0, vlo = nf;
    for (int k = 0; k < N; ++k) {
        int no = 0;
        for (int j = 0; j < nf; ++j) no += occ[k * nf + j] == 2;
        ohi = std::max(ohi, no);
        vlo = std::min(vlo, no);
    }
    const int no = ohi, nv = nf - vlo;
    if (no < 1 || nv < 1) return df_fail(d, TCE_ERR_ARG, "no occupied or no virtual bands");
    int s;
    double2 *d_G1 = nullptr, *d_F = nullptr, *d_C = nullptr, *d_L = nullptr;
    if ((s = df_alloc(d, &d_G1, (size_t)X * nau * N))) return s;
    k_df_g1<<<nblk(X * nau * N, 256), 256, 0, d->st>>>(d->d_B, d->d_ph, X, N, nau, d_G1);
    DCK(d, cudaGetLastError());
    const long long nF = (long long)nf * nf * nau * N * N;
    if ((s = df_alloc(d, &d_F, (size_t)nF))) return s;
    k_df_f<<<nblk(nF, 256), 256, 0, d->st>>>(d_G1, d->d_ph, X, N, nf, nau, d_F);
    DCK(d, cudaGetLastError());
    DCK(d, cudaStreamSynchronize(d->st));
    df_free(d, d_G1);
    if ((s = df_alloc(d, &d_C, (size_t)nbas * nbas))) return s;
    DCK(d, cudaMemcpyAsync(d_C, coeff, sizeof(double2) * nbas * nbas, cudaMemcpyHostToDevice, d->st));
    const long long nL = (long long)no * nv * nau * N * N;
    if ((s = df_alloc(d, &d_L, (size_t)nL))) return s;
    k_df_l<<<nblk(nL, 256), 256, 0, d->st>>>(d_F, d_C, d->d_crd, d->ncl[0], d->ncl[1], d->ncl[2], N, nf, nau, 0, no,
                                             vlo, nv, d_L);
    DCK(d, cudaGetLastError());
    std::vector<double> L(2 * (size_t)nL);
    DCK(d, cudaMemcpyAsync(L.data(), d_L, sizeof(double2) * nL, cudaMemcpyDeviceToHost, d->st));
    DCK(d, cudaStreamSynchronize(d->st));
    df_free(d, d_F);
    df_free(d, d_C);
    df_free(d, d_L);
    std::vector<int32_t> crd(3 * (size_t)N), oo((size_t)N * no), ov((size_t)N * nv);
    std::vector<double> eo((size_t)N * no), ev((size_t)N * nv);
    for (int k = 0; k < N; ++k) {
        int c[3];
        cell_coords(d->ncl, k, c);
        for (int dd = 0; dd < 3; ++dd) crd[3 * k + dd] = c[dd];
        for (int i = 0; i < no; ++i) {
            eo[(size_t)k * no + i] = eps[k * nf + i];
            oo[(size_t)k * no + i] = occ[k * nf + i];
        }
        for (int a = 0; a < nv; ++a) {
            ev[(size_t)k * nv + a] = eps[k * nf + vlo + a];
            ov[(size_t)k * nv + a] = occ[k * nf + vlo + a];
        }
    }
    double a2d = 0.0, a2x = 0.0;
    int64_t nz = 0;
    double gz = 0.0, ms = 0.0;
    s = tce_dfmp2_energy(N, d->ncl, crd.data(), no, nv, nau, L.data(), eo.data(), oo.data(), ev.data(), ov.data(),
                         mode, &a2d, &a2x, &nz, &gz, &ms);
    if (s) return df_fail(d, s, std::string("contraction: ") + tce_mp2_last_error());
    *e_mp2 = 2.0 * a2d - a2x;
    if (e2d) *e2d = a2d;
    if (e2x) *e2x = a2x;
    return TCE_OK;
}

}  // extern "C"
