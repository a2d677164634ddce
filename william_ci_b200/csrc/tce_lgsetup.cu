// tce_lgsetup.cu -- the learned grid's set-up behind the C ABI: the rule
// dictionary (mapped Gauss-Kronrod rules) built in C++, training labels of a
// sample of quartets against the 128-node reference rule, the rule-picking
// network trained on the GPU and the rules predicted for every quartet, so
// that a caller without a Python interpreter (the Fortran host) can switch
// the learned grid on with one call.  No counterpart in the reference.
//
// Quadrature on [-1, 1] from the Legendre recurrence (monic: alpha_k = 0,
// beta_0 = 2, beta_k = k^2 / (4 k^2 - 1)):
//   * Gauss-Legendre by Golub and Welsch (1969): the nodes are the
//     eigenvalues of the n x n Jacobi matrix, the weights beta_0 times the
//     squared first components of its normalised eigenvectors;
//   * Gauss-Kronrod (2n+1 nodes) by Laurie's algorithm (Math. Comp. 66, 1997,
//     1133-1145): the recurrence coefficients of the Jacobi-Kronrod matrix
//     of order 2n+1 from the first floor(3n/2)+1 Legendre coefficients, then
//     the same eigenvalue problem.
// Both in long double with an implicit QL iteration that carries only the
// first row of the eigenvector matrix.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <random>
#include <string>
#include <vector>

#include "../../include/tce.h"

namespace {

using ld = long double;

// Eigenvalues of the symmetric tridiagonal matrix (diagonal d[0..n-1],
// off-diagonal e[i] between rows i and i+1) and the squared first components
// of its normalised eigenvectors; implicit QL with Wilkinson's shift.
bool tridiag_eig(int n, std::vector<ld> d, std::vector<ld> e, std::vector<ld> &x, std::vector<ld> &z2)
{
    e.resize(n, 0.0L);
    std::vector<ld> z(n, 0.0L);
    z[0] = 1.0L;
    for (int l = 0; l < n; ++l) {
        for (int iter = 0;; ++iter) {
            int m = l;
            for (; m < n - 1; ++m) {
                const ld dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= std::numeric_limits<ld>::epsilon() * 0.5L * dd) break;
            }
            if (m == l) break;
            if (iter > 200) return false;
            ld g = (d[l + 1] - d[l]) / (2.0L * e[l]);
            ld r = std::hypot(g, 1.0L);
            g = d[m] - d[l] + e[l] / (g + (g >= 0 ? std::fabs(r) : -std::fabs(r)));
            ld s = 1.0L, c = 1.0L, p = 0.0L;
            int i = m - 1;
            for (; i >= l; --i) {
                ld f = s * e[i], b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0L) {
                    d[i + 1] -= p;
                    e[m] = 0.0L;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0L * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                // the first row of the eigenvector matrix follows the rotation
                f = z[i + 1];
                z[i + 1] = s * z[i] + c * f;
                z[i] = c * z[i] - s * f;
            }
            if (r == 0.0L && i >= l) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0L;
        }
    }
    std::vector<int> ord(n);
    for (int i = 0; i < n; ++i) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return d[a] < d[b]; });
    x.resize(n);
    z2.resize(n);
    for (int i = 0; i < n; ++i) {
        x[i] = d[ord[i]];
        z2[i] = z[ord[i]] * z[ord[i]];
    }
    return true;
}

ld legendre_beta(int k) { return k == 0 ? 2.0L : (ld)k * k / (4.0L * k * k - 1.0L); }

bool gauss_legendre(int n, std::vector<ld> &x, std::vector<ld> &w)
{
    std::vector<ld> d(n, 0.0L), e(n, 0.0L);
    for (int k = 1; k < n; ++k) e[k - 1] = std::sqrt(legendre_beta(k));
    std::vector<ld> z2;
    if (!tridiag_eig(n, d, e, x, z2)) return false;
    w.resize(n);
    for (int i = 0; i < n; ++i) w[i] = legendre_beta(0) * z2[i];
    return true;
}

// Laurie's construction of the Jacobi-Kronrod matrix of order 2n+1: on entry
// a[i], b[i] (i <= floor(3n/2)) hold the recurrence coefficients, on exit
// a[0..2n], b[0..2n] those of the Kronrod matrix (b[0] the total weight).
void laurie(int n, std::vector<ld> &a, std::vector<ld> &b)
{
    const int h = n / 2 + 2;
    std::vector<ld> s(h, 0.0L), t(h, 0.0L);
    t[1] = b[n + 1];
    for (int m = 0; m <= n - 2; ++m) {
        ld u = 0.0L;
        for (int k = (m + 1) / 2; k >= 0; --k) {
            const int l = m - k;
            u += (a[k + n + 1] - a[l]) * t[k + 1] + b[k + n + 1] * s[k] - b[l] * s[k + 1];
            s[k + 1] = u;
        }
        std::swap(s, t);
    }
    for (int j = n / 2; j >= 0; --j) s[j + 1] = s[j];
    for (int m = n - 1; m <= 2 * n - 3; ++m) {
        ld u = 0.0L;
        int j = 0;
        for (int k = m + 1 - n; k <= (m - 1) / 2; ++k) {
            const int l = m - k;
            j = n - 1 - l;
            u += -(a[k + n + 1] - a[l]) * t[j + 1] - b[k + n + 1] * s[j + 1] + b[l] * s[j + 2];
            s[j + 1] = u;
        }
        if (m % 2 == 0) {
            const int k = m / 2;
            a[k + n + 1] = a[k] + (s[j + 1] - b[k + n + 1] * s[j + 2]) / t[j + 2];
        } else {
            const int k = (m + 1) / 2;
            b[k + n + 1] = s[j + 1] / s[j + 2];
        }
        std::swap(s, t);
    }
    a[2 * n] = a[n - 1] - b[2 * n] * s[1] / t[1];
}

// Gauss-Kronrod rule of 2n+1 nodes on [0, 1] (ascending) with the embedded
// n-point Gauss weights (zero off the Gauss nodes)
bool gauss_kronrod01(int n, std::vector<double> &u, std::vector<double> &wk, std::vector<double> &wg)
{
    if (n < 1) return false;
    const int N2 = 2 * n + 1;
    std::vector<ld> a(N2 + 1, 0.0L), b(N2 + 1, 0.0L);
    for (int i = 0; i <= N2; ++i) b[i] = legendre_beta(i);
    laurie(n, a, b);
    std::vector<ld> d(N2), e(N2, 0.0L);
    for (int i = 0; i < N2; ++i) d[i] = a[i];
    for (int i = 1; i < N2; ++i) {
        if (!(b[i] > 0.0L)) return false;      // no real Kronrod extension
        e[i - 1] = std::sqrt(b[i]);
    }
    std::vector<ld> x, z2;
    if (!tridiag_eig(N2, d, e, x, z2)) return false;
    std::vector<ld> xg, wgl;
    if (!gauss_legendre(n, xg, wgl)) return false;
    u.assign(N2, 0.0);
    wk.assign(N2, 0.0);
    wg.assign(N2, 0.0);
    for (int i = 0; i < N2; ++i) {
        u[i] = (double)((x[i] + 1.0L) / 2.0L);
        wk[i] = (double)(b[0] * z2[i] / 2.0L);
    }
    // the Gauss nodes are every other Kronrod node
    for (int g = 0; g < n; ++g) {
        const int i = 2 * g + 1;
        if (std::fabs(x[i] - xg[g]) > 1e-12L) return false;
        wg[i] = (double)(wgl[g] / 2.0L);
    }
    return true;
}

// The learned grid's rule dictionary: Kronrod orders K15, K21, K31, K41, K61
// (n = 7, 10, 15, 20, 30) times 21 map scales s = 0.6 2^(j/2), j = -18..2,
// order-major; each rule mapped by t = s u/(1-u), dt = s/(1-u)^2 du, padded to
// 64 entries.
constexpr int kOrders[5] = {7, 10, 15, 20, 30};
constexpr int kScales = 21;

bool dictionary(std::vector<int32_t> &nn, std::vector<double> &t, std::vector<double> &wk, std::vector<double> &wg)
{
    const int R = 5 * kScales;
    nn.assign(R, 0);
    t.assign((size_t)R * 64, 0.0);
    wk.assign((size_t)R * 64, 0.0);
    wg.assign((size_t)R * 64, 0.0);
    for (int o = 0; o < 5; ++o) {
        std::vector<double> u, a, b;
        if (!gauss_kronrod01(kOrders[o], u, a, b)) return false;
        for (int j = 0; j < kScales; ++j) {
            const int r = o * kScales + j;
            const double sc = 0.6 * std::pow(2.0, (double)(j - 18) / 2.0);
            nn[r] = (int32_t)u.size();
            for (size_t k = 0; k < u.size(); ++k) {
                const double jac = sc / ((1.0 - u[k]) * (1.0 - u[k]));
                t[(size_t)r * 64 + k] = sc * u[k] / (1.0 - u[k]);
                wk[(size_t)r * 64 + k] = a[k] * jac;
                wg[(size_t)r * 64 + k] = b[k] * jac;
            }
        }
    }
    return true;
}

// the judge's error estimate of a block (the form of QUADPACK's QK rules):
// M min(1, (200 e / M)^1.5), e = max |K - G|, M = max |K|
double judge_estimate(const double *K, const double *G, long long n)
{
    double e = 0.0, M = 0.0;
    for (long long i = 0; i < n; ++i) {
        e = std::max(e, std::fabs(K[i] - G[i]));
        M = std::max(M, std::fabs(K[i]));
    }
    if (M <= 0.0 || e <= 0.0) return e;
    const double r = 200.0 * e / M;
    return r >= 1.0 ? M : M * r * std::sqrt(r);
}

}  // namespace

extern "C" {

int tce_gk_rule(int32_t n, double *u, double *wk, double *wg)
{
    if (n < 1 || n > 64 || !u || !wk || !wg) return TCE_ERR_ARG;
    std::vector<double> a, b, c;
    if (!gauss_kronrod01(n, a, b, c)) return TCE_ERR_UNSUPPORTED;
    std::memcpy(u, a.data(), sizeof(double) * a.size());
    std::memcpy(wk, b.data(), sizeof(double) * b.size());
    std::memcpy(wg, c.data(), sizeof(double) * c.size());
    return TCE_OK;
}

int tce_lg_dictionary(int32_t *nrules, int32_t *nn, double *t, double *wk, double *wg)
{
    if (!nrules) return TCE_ERR_ARG;
    std::vector<int32_t> a;
    std::vector<double> b, c, d;
    if (!dictionary(a, b, c, d)) return TCE_ERR_UNSUPPORTED;
    *nrules = (int32_t)a.size();
    if (nn) std::memcpy(nn, a.data(), sizeof(int32_t) * a.size());
    if (t) std::memcpy(t, b.data(), sizeof(double) * b.size());
    if (wk) std::memcpy(wk, c.data(), sizeof(double) * c.size());
    if (wg) std::memcpy(wg, d.data(), sizeof(double) * d.size());
    return TCE_OK;
}

int tce_lg_setup(void *handle, int64_t n_train, uint64_t seed, int32_t epochs, double label_tol, void **net_out)
{
    if (net_out) *net_out = nullptr;
    if (!handle || n_train < 1 || epochs < 1 || !(label_tol > 0.0)) return TCE_ERR_ARG;
    int s;
    tce_info info;
    if ((s = tce_get_info(handle, &info))) return s;
    const long long nit = info.n_shell_quartets;
    if (nit < 1) return TCE_ERR_STATE;
    // ---- the dictionary and the plain method's panel rule (K15 on [0, 1], scale 0.6)
    std::vector<int32_t> nn;
    std::vector<double> t, wk, wg;
    if (!dictionary(nn, t, wk, wg)) return TCE_ERR_UNSUPPORTED;
    const int R = (int)nn.size();
    {
        std::vector<double> u, a, b;
        if (!gauss_kronrod01(7, u, a, b)) return TCE_ERR_UNSUPPORTED;
        if ((s = tce_set_plain_rule(handle, 15, u.data(), a.data(), b.data(), 0.6))) return s;
    }
    // ---- the training sample (seeded)
    std::vector<int32_t> all((size_t)nit * 4);
    if ((s = tce_items(handle, all.data()))) return s;
    const long long n = std::min<long long>(n_train, nit);
    std::vector<long long> pick((size_t)nit);
    for (long long i = 0; i < nit; ++i) pick[(size_t)i] = i;
    std::mt19937_64 rng(seed);
    for (long long i = 0; i < n; ++i) {
        std::uniform_int_distribution<long long> dist(i, nit - 1);
        std::swap(pick[(size_t)i], pick[(size_t)dist(rng)]);
    }
    std::vector<int32_t> items((size_t)n * 4);
    for (long long i = 0; i < n; ++i)
        for (int c = 0; c < 4; ++c) items[(size_t)i * 4 + c] = all[(size_t)pick[(size_t)i] * 4 + c];
    all.clear();
    all.shrink_to_fit();
    // block offsets
    std::vector<int32_t> first(info.nsh), cnt(info.nsh);
    if ((s = tce_shells(handle, first.data(), cnt.data()))) return s;
    std::vector<long long> off((size_t)n + 1, 0);
    for (long long i = 0; i < n; ++i) {
        const int32_t *q = &items[(size_t)i * 4];
        off[(size_t)i + 1] = off[(size_t)i] + (long long)cnt[q[0]] * cnt[q[1]] * cnt[q[2]] * cnt[q[3]];
    }
    const size_t nb = (size_t)off.back();
    // ---- reference blocks: the 128-node mapped Gauss-Legendre rule (scale 1)
    // as two 64-node rules on the engine itself
    std::vector<double> T(nb, 0.0);
    {
        std::vector<ld> x, w;
        if (!gauss_legendre(128, x, w)) return TCE_ERR_UNSUPPORTED;
        int32_t hn[2] = {64, 64};
        std::vector<double> ht(128), hw(128), hz(128, 0.0);
        for (int k = 0; k < 128; ++k) {
            const double u = (double)((x[k] + 1.0L) / 2.0L), wu = (double)(w[k] / 2.0L);
            ht[k] = u / (1.0 - u);
            hw[k] = wu / ((1.0 - u) * (1.0 - u));
        }
        if ((s = tce_lg_set_rules(handle, 2, hn, ht.data(), hw.data(), hz.data()))) return s;
        std::vector<double> K(nb);
        for (int half = 0; half < 2; ++half) {
            if ((s = tce_rule_blocks(handle, half, 1, n, items.data(), K.data(), nullptr))) return s;
            for (size_t i = 0; i < nb; ++i) T[i] += K[i];
        }
    }
    if ((s = tce_lg_set_rules(handle, R, nn.data(), t.data(), wk.data(), wg.data()))) return s;
    // ---- every rule's error against the reference and its judge estimate
    std::vector<unsigned char> good((size_t)n * R), ok((size_t)n * R);
    {
        std::vector<double> K(nb), G(nb);
        for (int r = 0; r < R; ++r) {
            if ((s = tce_rule_blocks(handle, r, 1, n, items.data(), K.data(), G.data()))) return s;
            for (long long i = 0; i < n; ++i) {
                const long long o0 = off[(size_t)i], o1 = off[(size_t)i + 1];
                double e = 0.0;
                for (long long k = o0; k < o1; ++k) e = std::max(e, std::fabs(K[(size_t)k] - T[(size_t)k]));
                const double je = judge_estimate(&K[(size_t)o0], &G[(size_t)o0], o1 - o0);
                good[(size_t)i * R + r] = e <= label_tol;
                ok[(size_t)i * R + r] = e <= label_tol && je <= 1e-10;
            }
        }
    }
    // a rule counts as correct only when the two next smaller scales of its
    // order are correct too (a margin against scales predicted too small)
    const int margin = 2;
    std::vector<float> Y((size_t)n * R, 0.f);
    for (long long i = 0; i < n; ++i)
        for (int o = 0; o < 5; ++o)
            for (int j = 0; j < kScales; ++j) {
                const int r = o * kScales + j;
                bool v = ok[(size_t)i * R + r];
                for (int k = 1; k <= margin && v; ++k) v = j - k >= 0 && good[(size_t)i * R + r - k];
                Y[(size_t)i * R + r] = v ? 1.f : 0.f;
            }
    // ---- features, network, training on the GPU, rules for every quartet
    std::vector<float> X((size_t)n * TCE_NFEAT);
    if ((s = tce_item_features(handle, n, items.data(), X.data()))) return s;
    void *net = nullptr;
    if ((s = tce_mlp_create(TCE_NFEAT, 64, R, seed, &net))) return s;
    float loss = 0.f;
    s = tce_mlp_train(net, n, X.data(), Y.data(), epochs, 256, 2e-3f, seed, &loss);
    if (!s) s = tce_lg_predict_rules(handle, net, 10.0);
    if (s || !net_out) tce_mlp_destroy(net);
    else *net_out = net;
    return s;
}

}  // extern "C"
