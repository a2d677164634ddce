// tce_api.cu -- host side of libtce: the C ABI declared in include/tce.h.
//
// tce_create mirrors the set-up the reference does before its quartet loops
// (direct_init eri_direct.f90:76-225; ERI_integral_toroidal
// ERI_toroidal.f90:93-337): t-tables, shells, Schwarz bounds, primitive-pair
// table, then the symmetry-unique quartet list, everything evaluated on the
// device.  Host code here only sizes buffers, orders the work list and moves
// data.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <mutex>
#include <queue>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "tce_handle.h"

namespace tcehost {

thread_local std::string g_err;

int fail(Handle *h, int code, const std::string &msg)
{
    if (h) h->err = msg;
    g_err = msg;
    return code;
}

void dfree(Handle *h, void *p)
{
    if (!p) return;
    cudaFree(p);
    auto it = std::find(h->allocs.begin(), h->allocs.end(), p);
    if (it != h->allocs.end()) h->allocs.erase(it);
}

// Gauss-Legendre nodes on [0,1] by Newton on P_n, mapped t = 0.6 u/(1-u)
// (fast_quad_points, precompute_t.f90:906-942).
void mapped_gauss_legendre(int n, std::vector<double> &t, std::vector<double> &w)
{
    const double scale = 0.6;
    t.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 1; i <= n; ++i) {
        double x = std::cos(kPi * (i - 0.25) / (n + 0.5));
        double p0 = 1, p1 = x, dp = 1;
        for (int it = 0; it < 100; ++it) {
            p0 = 1.0;
            p1 = x;
            for (int j = 2; j <= n; ++j) {
                double p2 = ((2.0 * j - 1.0) * x * p1 - (j - 1.0) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (x * p1 - p0) / (x * x - 1.0);
            double dx = p1 / dp;
            x -= dx;
            if (std::fabs(dx) < 1e-15) break;
        }
        p0 = 1.0;
        p1 = x;
        for (int j = 2; j <= n; ++j) {
            double p2 = ((2.0 * j - 1.0) * x * p1 - (j - 1.0) * p0) / j;
            p0 = p1;
            p1 = p2;
        }
        dp = n * (x * p1 - p0) / (x * x - 1.0);
        double u = 0.5 * (1.0 - x);
        double wu = 1.0 / ((1.0 - x * x) * dp * dp);
        t[i - 1] = scale * u / (1.0 - u);
        w[i - 1] = wu * scale / ((1.0 - u) * (1.0 - u));
    }
}

int mod_pos(int a, int m) { int r = a % m; return r < 0 ? r + m : r; }

// index shifted by -(cell of ref), cells x fastest (translate_to_unit_cell)
int shift_to(const Handle *h, int idx, int refcell, int nblk)
{
    const int *ncl = h->ncl;
    int tx = refcell % ncl[0], ty = (refcell / ncl[0]) % ncl[1], tz = refcell / (ncl[0] * ncl[1]);
    int c = idx / nblk, loc = idx % nblk;
    int cx = mod_pos(c % ncl[0] - tx, ncl[0]);
    int cy = mod_pos((c / ncl[0]) % ncl[1] - ty, ncl[1]);
    int cz = mod_pos(c / (ncl[0] * ncl[1]) - tz, ncl[2]);
    return (cx + ncl[0] * (cy + ncl[1] * cz)) * nblk + loc;
}

// index shifted by +(cell ct) (shift_cell, eri_direct.f90:228-236)
int shift_by(const Handle *h, int idx, int ct, int nblk)
{
    const int *ncl = h->ncl;
    int c = idx / nblk, loc = idx % nblk;
    int cx = mod_pos(c % ncl[0] + ct % ncl[0], ncl[0]);
    int cy = mod_pos((c / ncl[0]) % ncl[1] + (ct / ncl[0]) % ncl[1], ncl[1]);
    int cz = mod_pos(c / (ncl[0] * ncl[1]) + ct / (ncl[0] * ncl[1]), ncl[2]);
    return (cx + ncl[0] * (cy + ncl[1] * cz)) * nblk + loc;
}

// which kernel evaluates a quartet in J/K mode: key = kind * 16 + cls
int route(const Handle *h, const int4 &q)
{
    const int l[4] = {h->sh_l[q.x], h->sh_l[q.y], h->sh_l[q.z], h->sh_l[q.w]};
    int cls = 0;
    bool sp = true;
    for (int i = 0; i < 4; ++i) {
        if (l[i] > 1) sp = false;
        else cls |= l[i] << i;
    }
    if (sp) {
        for (int i = 0; i < 4; ++i) {   // r1 needs the reference component order px, py, pz
            int S = (&q.x)[i];
            if (l[i] == 1)
                for (int c = 0; c < 3; ++c)
                    for (int d = 0; d < 3; ++d)
                        if (h->lxyz[3 * (h->sh_first[S] + c) + d] != (c == d ? 1 : 0)) sp = false;
        }
    }
    if (cls == 0 && sp && (h->nq == 32 || h->nq == 40)) return 1 * 16;
    if (sp && tce_r1_supported(h->ndp, h->nq, cls)) return 2 * 16 + cls;
    // generic kernel: one list per number of shells above p, each launched with
    // its own largest block (buffers sized for the list, not for (dd|dd))
    return (l[0] > 1) + (l[1] > 1) + (l[2] > 1) + (l[3] > 1);
}

// split a list of quartets (most expensive first) into per-kernel device lists
int make_lists(Handle *h, const std::vector<int4> &items)
{
    ++h->work_version;
    for (auto &w : h->lists) dfree(h, w.d);
    h->lists.clear();
    std::vector<std::vector<int4>> by(3 * 16);
    for (const int4 &q : items) by[route(h, q)].push_back(q);
    h->nitems_shard = 0;
    for (int key = 0; key < 3 * 16; ++key) {
        if (by[key].empty()) continue;
        Handle::WorkList w;
        w.kind = key / 16;
        w.cls = key % 16;
        w.n = (long long)by[key].size();
        for (const int4 &q : by[key]) {
            w.max_ncomb = std::max(w.max_ncomb, ncomb_of(h, q.x, q.y, q.z, q.w));
            w.max_ncq = std::max(w.max_ncq, h->sh_n[q.x] * h->sh_n[q.y] * h->sh_n[q.z] * h->sh_n[q.w]);
        }
        int s = upload(h, &w.d, by[key]);
        if (s) return s;
        h->nitems_shard += w.n;
        h->lists.push_back(w);
    }
    return TCE_OK;
}

int ncomb_of(const Handle *h, int SI, int SJ, int SK, int SL)
{
    return (h->sh_l[SI] + 1) * (h->sh_l[SJ] + 1) * (h->sh_l[SK] + 1) * (h->sh_l[SL] + 1);
}

// run the quartet kernel on a host list of items in a block-output mode
int run_blocks(Handle *h, const std::vector<int4> &items, const std::vector<int> *prim_sel, int mode, int prim_screen,
               std::vector<double> *blocks, std::vector<long long> *offs)
{
    if (items.empty()) return TCE_OK;
    std::vector<long long> off(items.size() + 1, 0);
    int mx = 1;
    for (size_t i = 0; i < items.size(); ++i) {
        const int4 &q = items[i];
        off[i + 1] = off[i] + (long long)h->sh_n[q.x] * h->sh_n[q.y] * h->sh_n[q.z] * h->sh_n[q.w];
        mx = std::max(mx, ncomb_of(h, q.x, q.y, q.z, q.w));
    }
    int4 *d_it = nullptr;
    int *d_sel = nullptr;
    double *d_out = nullptr;
    long long *d_off = nullptr;
    int s;
    if ((s = upload(h, &d_it, items))) return s;
    if (prim_sel && (s = upload(h, &d_sel, *prim_sel))) return s;
    if (mode != TCE_MODE_PRIMTAB) {
        if ((s = dalloc(h, &d_out, (size_t)off.back()))) return s;
        if ((s = upload(h, &d_off, off))) return s;
    }
    QuartetHostArgs a;
    a.items = d_it;
    a.prim_sel = d_sel;
    a.nitems = (int)items.size();
    a.mode = mode;
    a.prim_screen = prim_screen;
    a.next = h->d_next;
    a.blk_out = d_out;
    a.blk_off = d_off;
    a.pp_rw = h->d_pp;
    a.max_ncomb = mx;
    a.max_ncq = h->max_ncq;
    a.fixed_gmax = h->d_gmax;
    a.num_sms = h->num_sms;
    CKS(h, tce_launch_quartets(h->S, a, h->st));
    if (blocks) {
        blocks->resize(off.back());
        CK(h, cudaMemcpyAsync(blocks->data(), d_out, off.back() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    }
    CK(h, cudaStreamSynchronize(h->st));
    if (offs) *offs = off;
    dfree(h, d_it);
    dfree(h, d_sel);
    dfree(h, d_out);
    dfree(h, d_off);
    return TCE_OK;
}

// Wall time of the phases of build() on stderr when TCE_TIMING is set (the
// device phases are synchronised where the phase ends anyway).
struct PhaseClock {
    bool on = std::getenv("TCE_TIMING") != nullptr;
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    void mark(const char *what)
    {
        if (!on) return;
        auto n = std::chrono::steady_clock::now();
        std::fprintf(stderr, "tce_create %-28s %8.3f s\n", what, std::chrono::duration<double>(n - t).count());
        t = n;
    }
};

int build(Handle *h, const tce_system *sys)
{
    PhaseClock clk;
    // ---------------- validate + copy ----------------
    if (!sys) return fail(h, TCE_ERR_ARG, "sys is NULL");
    if (sys->ndp < 1 || sys->ndp > 3) return fail(h, TCE_ERR_ARG, "ndp must be 1, 2 or 3");
    if (sys->nbas <= 0 || sys->nfuc <= 0) return fail(h, TCE_ERR_ARG, "nbas and nfuc must be positive");
    if (!sys->ctr || !sys->lxyz || !sys->prim_off || !sys->exps || !sys->coefs)
        return fail(h, TCE_ERR_ARG, "NULL basis array");
    h->ndp = sys->ndp;
    h->nbas = sys->nbas;
    h->nfuc = sys->nfuc;
    for (int d = 0; d < 3; ++d) h->ncl[d] = sys->ncell[d] > 1 ? sys->ncell[d] : 1;
    h->ncell = h->ncl[0] * h->ncl[1] * h->ncl[2];
    if (h->nbas != h->nfuc * h->ncell)
        return fail(h, TCE_ERR_UNSUPPORTED, "the shells must be the same in every cell (nbas != nfuc * ncell)");
    for (int d = 0; d < 3; ++d) {
        h->L[d] = sys->L[d];
        h->a[d] = sys->L[d] > 0 ? 2.0 * kPi / sys->L[d] : 0.0;
        if (d < h->ndp && !(sys->L[d] > 0)) return fail(h, TCE_ERR_ARG, "periodic length must be positive");
    }
    h->physicist = sys->physicist != 0;
    h->sao = sys->sao != 0;
    h->prim_screen = sys->prim_screen != 0;
    h->thr = sys->schwarz_thr > 0 ? sys->schwarz_thr : 1e-13;
    h->prim_thr = sys->prim_thr > 0 ? sys->prim_thr : 1e-14;
    const int nbas = h->nbas;
    h->ctr.assign(sys->ctr, sys->ctr + 3 * nbas);
    h->lxyz.assign(sys->lxyz, sys->lxyz + 3 * nbas);
    h->poff.assign(sys->prim_off, sys->prim_off + nbas + 1);
    if (h->poff[0] != 0) return fail(h, TCE_ERR_ARG, "prim_off[0] must be 0");
    for (int f = 0; f < nbas; ++f)
        if (h->poff[f + 1] <= h->poff[f]) return fail(h, TCE_ERR_ARG, "every function needs at least one primitive");
    int nprim = h->poff[nbas];
    h->exps.assign(sys->exps, sys->exps + nprim);
    h->coefs.assign(sys->coefs, sys->coefs + nprim);
    for (int f = 0; f < nbas; ++f) {
        int l = h->lxyz[3 * f] + h->lxyz[3 * f + 1] + h->lxyz[3 * f + 2];
        if (h->lxyz[3 * f] < 0 || h->lxyz[3 * f + 1] < 0 || h->lxyz[3 * f + 2] < 0)
            return fail(h, TCE_ERR_ARG, "negative Cartesian power");
        if (l > TCE_LMAX) return fail(h, TCE_ERR_UNSUPPORTED, "angular momentum above d is not supported");
    }
    // nodes
    if (sys->t_nodes) {
        if (!sys->t_weights) return fail(h, TCE_ERR_ARG, "t_weights is NULL");
        h->tnode.assign(sys->t_nodes, sys->t_nodes + sys->nquad);
        h->tweight.assign(sys->t_weights, sys->t_weights + sys->nquad);
    } else {
        mapped_gauss_legendre(sys->nquad, h->tnode, h->tweight);
    }
    h->nq = sys->nquad;
    if (h->nq != 32 && h->nq != 40 && h->nq != 64 && h->nq != 128)
        return fail(h, TCE_ERR_UNSUPPORTED, "nquad must be 32, 40, 64 or 128");

    // ---------------- shells (ERI_toroidal.f90:106-125) ----------------
    for (int i = 0; i < nbas;) {
        int lt = h->lxyz[3 * i] + h->lxyz[3 * i + 1] + h->lxyz[3 * i + 2];
        int ncomp = (lt + 1) * (lt + 2) / 2;
        bool same = (i + ncomp - 1 <= nbas - 1);
        if (same)
            for (int j = i + 1; j <= i + ncomp - 1 && same; ++j) {
                int lj = h->lxyz[3 * j] + h->lxyz[3 * j + 1] + h->lxyz[3 * j + 2];
                int npi = h->poff[i + 1] - h->poff[i], npj = h->poff[j + 1] - h->poff[j];
                same = lj == lt && h->ctr[3 * j] == h->ctr[3 * i] && h->ctr[3 * j + 1] == h->ctr[3 * i + 1] &&
                       h->ctr[3 * j + 2] == h->ctr[3 * i + 2] && npi == npj;
                for (int p = 0; same && p < npi; ++p) same = h->exps[h->poff[j] + p] == h->exps[h->poff[i] + p];
            }
        if (!same) ncomp = 1;
        h->sh_first.push_back(i);
        h->sh_n.push_back(ncomp);
        h->sh_l.push_back(lt);
        i += ncomp;
    }
    h->nsh = (int)h->sh_first.size();
    {
        int mxn = 1;
        for (int n : h->sh_n) mxn = std::max(mxn, n);
        h->max_ncq = mxn * mxn * mxn * mxn;
    }
    h->nshuc = 0;
    for (int S = 0; S < h->nsh; ++S)
        if (h->sh_first[S] < h->nfuc) ++h->nshuc;
    bool sym_ok = (h->nsh == h->nshuc * h->ncell);
    for (int S = 0; sym_ok && S < h->nsh - h->nshuc; ++S)
        if (h->sh_n[S + h->nshuc] != h->sh_n[S] || h->sh_first[S + h->nshuc] != h->sh_first[S] + h->nfuc) sym_ok = false;
    if (!sym_ok) return fail(h, TCE_ERR_UNSUPPORTED, "the shells must be the same in every cell");
    for (int S = 0; S < h->nsh; ++S) {
        int f = h->sh_first[S], np = h->poff[f + 1] - h->poff[f];
        h->sh_np.push_back(np);
        h->sh_eoff.push_back((int)h->sh_exp.size());
        h->sh_coff.push_back((int)h->sh_coef.size());
        for (int d = 0; d < 3; ++d) h->sh_r.push_back(h->ctr[3 * f + d]);
        for (int p = 0; p < np; ++p) h->sh_exp.push_back(h->exps[h->poff[f] + p]);
        for (int c = 0; c < h->sh_n[S]; ++c)
            for (int p = 0; p < np; ++p) h->sh_coef.push_back(h->coefs[h->poff[f + c] + p]);
        for (int p = 0; p < np; ++p) {
            double m = 0.0;
            for (int c = 0; c < h->sh_n[S]; ++c) m = std::max(m, std::fabs(h->coefs[h->poff[f + c] + p]));
            h->sh_cmax.push_back(m);
        }
    }

    // ---------------- t-table size (ERI_toroidal.f90:93-104) ----------------
    int lmax = 0;
    double emax = 0.0;
    for (int f = 0; f < nbas; ++f) {
        for (int d = 0; d < h->ndp; ++d) lmax = std::max(lmax, h->lxyz[3 * f + d]);
        for (int p = h->poff[f]; p < h->poff[f + 1]; ++p) emax = std::max(emax, h->exps[p]);
    }
    double amin = h->a[0];
    for (int d = 1; d < h->ndp; ++d) amin = std::min(amin, h->a[d]);
    double Acap = 4.0 * emax / (amin * amin);
    h->ncap = 20 + (int)std::ceil(9.0 * std::sqrt(Acap > 0 ? Acap : 0.0)) + 2 * lmax + 1;

    // ---------------- device ----------------
    int dev = 0;
    CK(h, cudaGetDevice(&dev));
    h->dev = dev;
    CK(h, cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, dev));
    CK(h, cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
    CK(h, cudaEventCreate(&h->ev0));
    CK(h, cudaEventCreate(&h->ev1));
    CK(h, cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming));
    CK(h, cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming));
    CK(h, cudaStreamCreateWithFlags(&h->st2, cudaStreamNonBlocking));
    CK(h, cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
    CK(h, cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    CK(h, cudaEventCreateWithFlags(&h->ev_fb, cudaEventDisableTiming));
    CK(h, cudaStreamCreateWithFlags(&h->st3, cudaStreamNonBlocking));
    CK(h, cudaEventCreateWithFlags(&h->ev_fork3, cudaEventDisableTiming));
    CK(h, cudaEventCreateWithFlags(&h->ev_join3, cudaEventDisableTiming));
    int s;
    DevSys &S = h->S;
    S.ndp = h->ndp; S.nq = h->nq; S.ncap = h->ncap; S.nbas = nbas; S.nfuc = h->nfuc;
    S.nsh = h->nsh; S.nshuc = h->nshuc; S.ncell = h->ncell;
    for (int d = 0; d < 3; ++d) { S.ncl[d] = h->ncl[d]; S.a[d] = h->a[d]; S.L[d] = h->L[d]; }
    S.fac_const = 2.0 / std::sqrt(kPi);
    for (int d = 0; d < h->ndp; ++d) S.fac_const *= h->L[d] * h->L[d];
    S.thr = h->thr;
    S.prim_thr = h->prim_thr;
    {
        int *p;
        double *q;
        if ((s = upload(h, &p, h->sh_first))) return s; S.sh_first = p;
        if ((s = upload(h, &p, h->sh_n))) return s; S.sh_n = p;
        if ((s = upload(h, &p, h->sh_l))) return s; S.sh_l = p;
        if ((s = upload(h, &p, h->sh_np))) return s; S.sh_np = p;
        if ((s = upload(h, &p, h->sh_eoff))) return s; S.sh_eoff = p;
        if ((s = upload(h, &p, h->sh_coff))) return s; S.sh_coff = p;
        if ((s = upload(h, &q, h->sh_r))) return s; S.sh_r = q;
        if ((s = upload(h, &q, h->sh_exp))) return s; S.sh_exp = q;
        if ((s = upload(h, &q, h->sh_coef))) return s; S.sh_coef = q;
        if ((s = upload(h, &q, h->sh_cmax))) return s; S.sh_cmax = q;
        if ((s = upload(h, &p, h->lxyz))) return s; S.fn_pw = p;
        {
            std::vector<int4> fc((size_t)nbas);
            for (int f = 0; f < nbas; ++f) {
                const int c = f / h->nfuc;
                fc[(size_t)f] = make_int4(c % h->ncl[0], (c / h->ncl[0]) % h->ncl[1], c / (h->ncl[0] * h->ncl[1]),
                                          f - c * h->nfuc);
            }
            int4 *d_fc = nullptr;
            if ((s = upload(h, &d_fc, fc))) return s;
            S.fn_cell = d_fc;
        }
        if ((s = upload(h, &q, h->tnode))) return s; S.tnode = q;
        if ((s = upload(h, &q, h->tweight))) return s; S.tweight = q;
    }
    if ((s = dalloc(h, &h->d_next, 1))) return s;

    clk.mark("setup (host shells, device)");
    // ---------------- t-tables (setup_t_tables) ----------------
    {
        double *tb, *Tt;
        int *tn;
        if ((s = dalloc(h, &tb, (size_t)(h->ncap + 1) * h->nq * h->ndp))) return s;
        if ((s = dalloc(h, &Tt, (size_t)(h->ncap + 1) * h->nq * h->ndp))) return s;
        if ((s = dalloc(h, &tn, (size_t)h->nq * h->ndp))) return s;
        CKS(h, tce_launch_t_tables(h->nq, h->ndp, h->ncap, S.tnode, h->a, tb, tn, Tt, h->st));
        h->tnmax.resize((size_t)h->nq * h->ndp);
        CK(h, cudaMemcpyAsync(h->tnmax.data(), tn, h->tnmax.size() * sizeof(int), cudaMemcpyDeviceToHost, h->st));
        CK(h, cudaStreamSynchronize(h->st));
        dfree(h, tb);
        h->d_tnmax = tn;
        S.Tt = Tt;
        for (int d = 0; d < 3; ++d)
            for (int g = 0; g < TCE_MAXG; ++g) S.gmax[d][g] = -1;
        for (int d = 0; d < h->ndp; ++d)
            for (int g = 0; g < h->nq / 8; ++g) {
                int m = 0;
                for (int k = 8 * g; k < 8 * g + 8; ++k) m = std::max(m, h->tnmax[(size_t)d * h->nq + k]);
                S.gmax[d][g] = m;
            }
        std::vector<int> gm(3 * TCE_MAXG);
        for (int d = 0; d < 3; ++d)
            for (int g = 0; g < TCE_MAXG; ++g) gm[d * TCE_MAXG + g] = S.gmax[d][g];
        if ((s = upload(h, &h->d_gmax, gm))) return s;
    }

    clk.mark("t-tables");
    // ---------------- unit pairs + primitive-pair scalars ----------------
    const int nreal = 3 - h->ndp;
    long long npp_tot = 0, e_tot = 0;
    std::vector<int> pp_unit;
    for (int S1 = 0; S1 < h->nshuc; ++S1)
        for (int S2 = 0; S2 < h->nsh; ++S2) {
            UnitPair U{};
            U.S1 = S1; U.S2 = S2; U.l1 = h->sh_l[S1]; U.l2 = h->sh_l[S2];
            U.np1 = h->sh_np[S1]; U.np2 = h->sh_np[S2]; U.npp = U.np1 * U.np2;
            U.pp_off = npp_tot;
            U.e_off = e_tot;
            npp_tot += U.npp;
            e_tot += (long long)U.npp * nreal * (U.l1 + 1) * (U.l2 + 1) * TCE_ECO;
            for (int p = 0; p < U.npp; ++p) pp_unit.push_back((int)h->up.size());
            h->up.push_back(U);
        }
    int *d_ppu = nullptr;
    UnitPair *d_up = nullptr;
    double *d_e = nullptr;
    if ((s = upload(h, &d_ppu, pp_unit))) return s;
    if ((s = upload(h, &d_up, h->up))) return s;
    if ((s = dalloc(h, &h->d_pp, (size_t)npp_tot))) return s;
    if ((s = dalloc(h, &d_e, (size_t)e_tot))) return s;
    S.up = d_up;
    S.pp = h->d_pp;
    S.ecoef = d_e;
    CKS(h, tce_launch_pair_scalars(S, npp_tot, d_ppu, h->d_pp, d_up, d_e, h->st));
    std::vector<PairPrim> hpp((size_t)npp_tot);
    CK(h, cudaMemcpyAsync(hpp.data(), h->d_pp, npp_tot * sizeof(PairPrim), cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    long long v_tot = 0;
    for (auto &U : h->up) {
        int nmax = 0;
        double km = 0.0;
        for (int p = 0; p < U.npp; ++p) {
            const PairPrim &P = hpp[U.pp_off + p];
            for (int d = 0; d < h->ndp; ++d) nmax = std::max(nmax, P.N[d]);
            km = std::max(km, std::fabs(P.pfac) * P.cmax12);
        }
        U.Nlen = nmax + 1;
        U.ket_max = km;
        U.vec_off = v_tot;
        v_tot += (long long)h->ndp * (U.l1 + 1) * (U.l2 + 1) * 2 * U.Nlen * U.npp;
    }
    CK(h, cudaMemcpyAsync(d_up, h->up.data(), h->up.size() * sizeof(UnitPair), cudaMemcpyHostToDevice, h->st));
    double2 *d_vec = nullptr;
    if ((s = dalloc(h, &d_vec, (size_t)v_tot))) return s;
    S.vec = d_vec;
    {
        int stride = h->ncap + 2 * TCE_LMAX + 2;
        double *scr = nullptr;
        if ((s = dalloc(h, &scr, (size_t)npp_tot * h->ndp * stride))) return s;
        CKS(h, tce_launch_pair_vectors(S, npp_tot, d_ppu, h->d_pp, stride, scr, d_vec, h->st));
        CK(h, cudaStreamSynchronize(h->st));
        dfree(h, scr);
    }

    // a handle for shell blocks only (tce_create_blocks): no Schwarz pass, no
    // primitive table, no quartet list; blocks are evaluated with the prefactor
    // screens of the kernel only
    if (h->blocks_only) {
        h->Q.assign((size_t)nbas * nbas, 1.0);
        h->Qsh.assign((size_t)h->nsh * h->nsh, 1.0);
        h->Qmax = 1.0;
        h->prim_screen = 0;
        double *dQ;
        if ((s = upload(h, &dQ, h->Q))) return s;
        S.Q = dQ;
        if ((s = upload(h, &h->d_Qsh, h->Qsh))) return s;
        if ((s = dalloc(h, &h->d_P, (size_t)nbas * nbas))) return s;
        if ((s = dalloc(h, &h->d_J, (size_t)h->nfuc * nbas))) return s;
        if ((s = dalloc(h, &h->d_K, (size_t)h->nfuc * nbas))) return s;
        h->shard_idx.clear();
        CK(h, cudaStreamSynchronize(h->st));
        return TCE_OK;
    }

    clk.mark("unit pairs");
    // ---------------- Schwarz: diagonal blocks, SI in the unit cell (ERI_toroidal.f90:200-236) ----------
    {
        std::vector<int4> items;
        for (int SI = 0; SI < h->nshuc; ++SI)
            for (int SJ = 0; SJ < h->nsh; ++SJ) items.push_back(make_int4(SI, SJ, SI, SJ));
        std::vector<double> blocks;
        std::vector<long long> off;
        if ((s = run_blocks(h, items, nullptr, TCE_MODE_BLOCK, 0, &blocks, &off))) return s;
        h->Q.assign((size_t)nbas * nbas, 0.0);
        for (size_t it = 0; it < items.size(); ++it) {
            int SI = items[it].x, SJ = items[it].y, ni = h->sh_n[SI], nj = h->sh_n[SJ];
            for (int a = 0; a < ni; ++a)
                for (int b = 0; b < nj; ++b) {
                    double qv = std::sqrt(std::fabs(blocks[off[it] + a + ni * (b + nj * (a + ni * b))]));
                    int i = h->sh_first[SI] + a, j = h->sh_first[SJ] + b;
                    for (int ct = 0; ct < h->ncell; ++ct) {
                        int ii = shift_by(h, i, ct, h->nfuc), jj = shift_by(h, j, ct, h->nfuc);
                        h->Q[ii + (size_t)nbas * jj] = qv;
                        h->Q[jj + (size_t)nbas * ii] = qv;
                    }
                }
        }
        h->Qsh.assign((size_t)h->nsh * h->nsh, 0.0);
        h->Qmax = 0.0;
        for (int SI = 0; SI < h->nsh; ++SI)
            for (int SJ = 0; SJ < h->nsh; ++SJ) {
                double m = 0.0;
                for (int a = 0; a < h->sh_n[SI]; ++a)
                    for (int b = 0; b < h->sh_n[SJ]; ++b)
                        m = std::max(m, h->Q[(h->sh_first[SI] + a) + (size_t)nbas * (h->sh_first[SJ] + b)]);
                h->Qsh[SI + (size_t)h->nsh * SJ] = m;
                h->Qmax = std::max(h->Qmax, m);
            }
        double *dQ;
        if ((s = upload(h, &dQ, h->Q))) return s;
        S.Q = dQ;
        if ((s = upload(h, &h->d_Qsh, h->Qsh))) return s;
        for (auto &U : h->up)
            if (h->Qsh[U.S1 + (size_t)h->nsh * U.S2] * h->Qmax >= h->thr) ++h->n_unit_sig;
    }

    clk.mark("Schwarz");
    // ---------------- primitive Schwarz table (ERI_toroidal.f90:296-337) ----------------
    if (h->prim_screen) {
        std::vector<int4> items;
        std::vector<int> sel;
        for (const auto &U : h->up)
            for (int p1 = 0; p1 < U.np1; ++p1)
                for (int p2 = 0; p2 < U.np2; ++p2) {
                    items.push_back(make_int4(U.S1, U.S2, U.S1, U.S2));
                    sel.push_back(p1);
                    sel.push_back(p2);
                }
        if ((s = run_blocks(h, items, &sel, TCE_MODE_PRIMTAB, 0, nullptr, nullptr))) return s;
    }

    clk.mark("primitive table");
    // ---------------- unique quartets (ERI_toroidal.f90:342-401) ----------------
    {
        unsigned long long *d_cnt = nullptr;
        if ((s = dalloc(h, &d_cnt, 2))) return s;
        CK(h, cudaMemsetAsync(d_cnt, 0, 2 * sizeof(unsigned long long), h->st));
        CKS(h, tce_launch_enumerate(S, h->d_Qsh, h->Qmax, nullptr, d_cnt, 0ull, d_cnt + 1, h->st));
        unsigned long long cnt[2];
        CK(h, cudaMemcpyAsync(cnt, d_cnt, sizeof cnt, cudaMemcpyDeviceToHost, h->st));
        CK(h, cudaStreamSynchronize(h->st));
        h->nitems = (long long)cnt[0];
        h->n_func_q = (long long)cnt[1];
        if (h->nitems > 0x7fffffffLL) return fail(h, TCE_ERR_UNSUPPORTED, "more than 2^31 unique shell quartets");
        int4 *d_raw = nullptr;
        if ((s = dalloc(h, &d_raw, (size_t)h->nitems))) return s;
        CK(h, cudaMemsetAsync(d_cnt, 0, 2 * sizeof(unsigned long long), h->st));
        CKS(h, tce_launch_enumerate(S, h->d_Qsh, h->Qmax, d_raw, d_cnt, (unsigned long long)h->nitems, d_cnt + 1, h->st));
    clk.mark("enumeration");
        // work order on the device (tce_sort_items): most expensive first, ties by
        // the quartet, so that the enumeration's arbitrary order never leaks
        // into the list every rank of a sharded run must share
        double *d_cost = nullptr;
        int *d_mnc = nullptr;
        if ((s = dalloc(h, &h->d_items, (size_t)h->nitems))) return s;
        if ((s = dalloc(h, &d_cost, (size_t)h->nitems))) return s;
        if ((s = dalloc(h, &d_mnc, 1))) return s;
        CK(h, cudaMemsetAsync(d_mnc, 0, sizeof(int), h->st));
        CKS(h, tce_sort_items(S, d_raw, h->nitems, h->d_items, d_cost, d_mnc, h->st));
        std::vector<int4> sorted((size_t)h->nitems);
        h->cost_host.resize((size_t)h->nitems);
        int mnc = 1;
        CK(h, cudaMemcpyAsync(sorted.data(), h->d_items, sorted.size() * sizeof(int4), cudaMemcpyDeviceToHost, h->st));
        CK(h, cudaMemcpyAsync(h->cost_host.data(), d_cost, h->cost_host.size() * sizeof(double),
                              cudaMemcpyDeviceToHost, h->st));
        CK(h, cudaMemcpyAsync(&mnc, d_mnc, sizeof(int), cudaMemcpyDeviceToHost, h->st));
        CK(h, cudaStreamSynchronize(h->st));
        h->max_ncomb = std::max(h->max_ncomb, mnc);
        dfree(h, d_raw);
        dfree(h, d_cnt);
        dfree(h, d_cost);
        dfree(h, d_mnc);
    clk.mark("cost + sort");
        h->items_host = std::move(sorted);
        h->shard_idx.resize(h->items_host.size());
        std::iota(h->shard_idx.begin(), h->shard_idx.end(), 0LL);
        if ((s = make_lists(h, h->items_host))) return s;
        if ((s = lg_rebuild_lists(h))) return s;
    clk.mark("work lists");
        // algorithmic work of one J/K pass
        unsigned long long *d_np = nullptr;
        double *d_fl = nullptr;
        if ((s = dalloc(h, &d_np, 1))) return s;
        if ((s = dalloc(h, &d_fl, 1))) return s;
        CK(h, cudaMemsetAsync(d_np, 0, sizeof(unsigned long long), h->st));
        CK(h, cudaMemsetAsync(d_fl, 0, sizeof(double), h->st));
        CKS(h, tce_launch_count_work(S, h->d_items, (int)h->nitems, h->prim_screen, h->d_tnmax, d_np, d_fl, h->st));
        unsigned long long np_ = 0;
        CK(h, cudaMemcpyAsync(&np_, d_np, sizeof np_, cudaMemcpyDeviceToHost, h->st));
        CK(h, cudaMemcpyAsync(&h->jk_flops, d_fl, sizeof(double), cudaMemcpyDeviceToHost, h->st));
        CK(h, cudaStreamSynchronize(h->st));
        h->n_prim_q = (long long)np_;
        dfree(h, d_np);
        dfree(h, d_fl);
    }
    clk.mark("work count");
    if ((s = dalloc(h, &h->d_P, (size_t)nbas * nbas))) return s;
    if ((s = dalloc(h, &h->d_J, (size_t)h->nfuc * nbas))) return s;
    if ((s = dalloc(h, &h->d_K, (size_t)h->nfuc * nbas))) return s;
    if ((s = dalloc(h, &h->d_one, 1))) return s;
    if ((s = dalloc(h, &h->d_blkoff, 2))) return s;
    {
        long long z[2] = {0, 0};
        CK(h, cudaMemcpyAsync(h->d_blkoff, z, sizeof z, cudaMemcpyHostToDevice, h->st));
    }
    if ((s = dalloc(h, &h->d_blk, (size_t)TCE_NCOMP_MAX * TCE_NCOMP_MAX * TCE_NCOMP_MAX * TCE_NCOMP_MAX))) return s;
    CK(h, cudaStreamSynchronize(h->st));
    return TCE_OK;
}

// the launches of one J/K pass (zeroing of J and K included)
static int jk_body(Handle *h, const double *dP, double *dJ, double *dK, cudaStream_t st)
{
    CK(h, cudaMemsetAsync(dJ, 0, sizeof(double) * h->nfuc * h->nbas, st));
    CK(h, cudaMemsetAsync(dK, 0, sizeof(double) * h->nfuc * h->nbas, st));
    if (h->method != TCE_METHOD_FIXED) return lg_jk_passes(h, dP, dJ, dK, st);
    for (const auto &w : h->lists) {
        if (w.n == 0) continue;
        if (w.kind == 0) {   // every other class: generic kernel
            QuartetHostArgs a;
            a.items = w.d;
            a.nitems = (int)w.n;
            a.mode = TCE_MODE_JK;
            a.prim_screen = h->prim_screen;
            a.next = h->d_next;
            a.P = dP;
            a.J = dJ;
            a.K = dK;
            a.max_ncomb = w.max_ncomb;
            a.max_ncq = w.max_ncq;
            a.fixed_gmax = h->d_gmax;
            a.num_sms = h->num_sms;
            a.use_tc = h->use_tc && h->nq == 64;   // tensor-core rows measured faster with 64 nodes only
            CKS(h, tce_launch_quartets(h->S, a, st));
        } else {             // register-resident kernels of the dominant classes
            SArgsHost b;
            b.items = w.d;
            b.nitems = (int)w.n;
            b.prim_screen = h->prim_screen;
            b.next = h->d_next;
            b.P = dP;
            b.J = dJ;
            b.K = dK;
            b.num_sms = h->num_sms;
            if (w.kind == 1) CKS(h, tce_launch_quartets_s(h->S, b, st));
            else CKS(h, tce_launch_quartets_r1(h->S, w.cls, b, st));
        }
    }
    return TCE_OK;
}

// streams, events and pinned host memory of a handle
void release_streams(Handle *h)
{
    if (h->st) cudaStreamDestroy(h->st);
    if (h->st2) cudaStreamDestroy(h->st2);
    if (h->st3) cudaStreamDestroy(h->st3);
    for (cudaEvent_t e : {h->ev0, h->ev1, h->ev_in, h->ev_out, h->ev_fork, h->ev_join, h->ev_fb, h->ev_fork3, h->ev_join3})
        if (e) cudaEventDestroy(e);
    if (h->h_fb) cudaFreeHost(h->h_fb);
    h->st = h->st2 = h->st3 = nullptr;
    h->ev0 = h->ev1 = h->ev_in = h->ev_out = h->ev_fork = h->ev_join = h->ev_fb = nullptr;
    h->ev_fork3 = h->ev_join3 = nullptr;
    h->h_fb = nullptr;
}

void drop_graph(Handle *h)
{
    if (h->jk_exec) cudaGraphExecDestroy(h->jk_exec);
    h->jk_exec = nullptr;
}

// One J/K pass.  With graphs on, the pass is captured once into a CUDA graph
// (per pointer triple, stream, method and work lists) and replayed as one
// graph launch per call; the events around it time the whole pass.  The
// legacy default stream cannot be captured: a caller on it is ordered with the
// handle's own stream by events, and the graph runs there.
int direct_jk_device(Handle *h, const double *dP, double *dJ, double *dK, cudaStream_t caller)
{
    cudaStream_t st = caller;
    const bool legacy =
        h->use_graph && (caller == nullptr || caller == cudaStreamLegacy || caller == cudaStreamPerThread);
    if (legacy) {
        st = h->st;
        CK(h, cudaEventRecord(h->ev_in, caller));
        CK(h, cudaStreamWaitEvent(st, h->ev_in, 0));
    }
    int s = direct_jk_on(h, dP, dJ, dK, st);
    if (s) return s;
    if (legacy) {
        CK(h, cudaEventRecord(h->ev_out, st));
        CK(h, cudaStreamWaitEvent(caller, h->ev_out, 0));
    }
    return TCE_OK;
}

int direct_jk_on(Handle *h, const double *dP, double *dJ, double *dK, cudaStream_t st)
{
    const bool lg = h->method == TCE_METHOD_LEARNED;
    if (lg) {   // the last pass's rejects join the plain list (the work lists change once)
        int s = lg_absorb_rejects(h);
        if (s) return s;
    }
    if (!h->use_graph) {
        CK(h, cudaEventRecord(h->ev0, st));
        int s = jk_body(h, dP, dJ, dK, st);
        if (s) return s;
        CK(h, cudaEventRecord(h->ev1, st));
        return lg ? lg_read_rejects(h, st) : TCE_OK;
    }
    const bool same = h->jk_exec && h->g_P == dP && h->g_J == dJ && h->g_K == dK && h->g_st == st &&
                      h->g_method == h->method && h->g_version == h->work_version;
    if (!same) {
        drop_graph(h);
        cudaGraph_t g = nullptr;
        CK(h, cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        int s = jk_body(h, dP, dJ, dK, st);
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (s) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (e != cudaSuccess) return fail(h, TCE_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&h->jk_exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            h->jk_exec = nullptr;
            return fail(h, TCE_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
        h->g_P = dP;
        h->g_J = dJ;
        h->g_K = dK;
        h->g_st = st;
        h->g_method = h->method;
        h->g_version = h->work_version;
    }
    CK(h, cudaEventRecord(h->ev0, st));
    CK(h, cudaGraphLaunch(h->jk_exec, st));
    CK(h, cudaEventRecord(h->ev1, st));
    return lg ? lg_read_rejects(h, st) : TCE_OK;
}

}  // namespace tcehost

using namespace tcehost;

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

const char *tce_version(void) { return "libtce 0.1 (sm_100a, FP64 toroidal ERI / J-K engine)"; }

const char *tce_last_error(void *handle)
{
    if (handle) return static_cast<Handle *>(handle)->err.c_str();
    return g_err.c_str();
}

static int noalloc_prepare(Handle *h);

static int create_impl(const tce_system *sys, void **handle, bool blocks_only)
{
    if (!handle) return fail(nullptr, TCE_ERR_ARG, "handle is NULL");
    *handle = nullptr;
    Handle *h = new Handle();
    h->blocks_only = blocks_only ? 1 : 0;
    int s = build(h, sys);
    if (s == TCE_OK) s = noalloc_prepare(h);
    if (s != TCE_OK) {
        g_err = h->err;
        for (void *p : h->allocs) cudaFree(p);
        release_streams(h);
        delete h;
        return s;
    }
    *handle = h;
    return TCE_OK;
}

int tce_create(const tce_system *sys, void **handle) { return create_impl(sys, handle, false); }

int tce_create_blocks(const tce_system *sys, void **handle) { return create_impl(sys, handle, true); }

int tce_destroy(void *handle)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h) return TCE_OK;
    if (h->st) cudaStreamSynchronize(h->st);
    drop_graph(h);
    if (h->st2) cudaStreamSynchronize(h->st2);
    if (h->st3) cudaStreamSynchronize(h->st3);
    for (void *p : h->allocs) cudaFree(p);
    release_streams(h);
    delete h;
    return TCE_OK;
}

int tce_pass_kernels(void *handle, int32_t *n)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !n) return fail(h, TCE_ERR_ARG, "NULL argument");
    int k = 0;
    if (h->method == TCE_METHOD_FIXED) {
        for (const auto &w : h->lists) k += w.n > 0 ? 1 : 0;
    } else if (h->method == TCE_METHOD_PLAIN) {
        k = h->shard_idx.empty() ? 0 : 1;
    } else {
        k = (int)h->lg_lists.size() + (h->n_plain_direct > 0 ? 1 : 0) + (h->n_lg > 0 ? 1 : 0);
    }
    *n = k;
    return TCE_OK;
}

int tce_get_info(void *handle, tce_info *info)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !info) return fail(h, TCE_ERR_ARG, "NULL argument");
    info->nsh = h->nsh;
    info->nshuc = h->nshuc;
    info->ncap = h->ncap;
    info->nquad = h->nq;
    info->n_shell_quartets = h->nitems;
    info->n_func_quartets = h->n_func_q;
    info->n_unit_pairs = h->n_unit_sig;
    info->device_bytes = (int64_t)h->bytes;
    info->n_prim_quartets = h->n_prim_q;
    info->jk_flops = h->jk_flops;
    info->shard_rank = h->shard_rank;
    info->shard_nranks = h->shard_nranks;
    info->shard_shell_quartets = h->nitems_shard;
    return TCE_OK;
}

int tce_shard_plan(const double *cost, int64_t n, int32_t nranks, int32_t *owner)
{
    if (nranks < 1 || n < 0 || (n > 0 && (!cost || !owner))) return fail(nullptr, TCE_ERR_ARG, "bad argument");
    // least-loaded owner first, ties to the lowest rank: a min-heap of
    // (load, rank), O(n log nranks) so that fine partitions stay cheap
    using Slot = std::pair<double, int32_t>;
    std::priority_queue<Slot, std::vector<Slot>, std::greater<Slot>> heap;
    for (int32_t r = 0; r < nranks; ++r) heap.push(Slot(0.0, r));
    for (int64_t i = 0; i < n; ++i) {
        Slot sl = heap.top();
        heap.pop();
        owner[i] = sl.second;
        sl.first += cost[i] > 0 ? cost[i] : 0.0;
        heap.push(sl);
    }
    return TCE_OK;
}

int tce_set_shard(void *handle, int32_t rank, int32_t nranks)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || nranks < 1 || rank < 0 || rank >= nranks) return fail(h, TCE_ERR_ARG, "bad shard");
    std::vector<int32_t> owner(h->items_host.size());
    int s = tce_shard_plan(h->cost_host.data(), (int64_t)owner.size(), nranks, owner.data());
    if (s) return fail(h, s, "shard plan failed");
    std::vector<int4> mine;
    h->shard_idx.clear();
    for (size_t i = 0; i < owner.size(); ++i)
        if (owner[i] == rank) {
            mine.push_back(h->items_host[i]);
            h->shard_idx.push_back((long long)i);
        }
    if ((s = make_lists(h, mine))) return s;
    if ((s = lg_rebuild_lists(h))) return s;
    h->shard_rank = rank;
    h->shard_nranks = nranks;
    CK(h, cudaStreamSynchronize(h->st));
    return TCE_OK;
}

int tce_shard_items(void *handle, int64_t *n, int32_t *items)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !n) return fail(h, TCE_ERR_ARG, "NULL argument");
    *n = (int64_t)h->shard_idx.size();
    if (items)
        for (size_t i = 0; i < h->shard_idx.size(); ++i) {
            const int4 &q = h->items_host[(size_t)h->shard_idx[i]];
            items[4 * i] = q.x;
            items[4 * i + 1] = q.y;
            items[4 * i + 2] = q.z;
            items[4 * i + 3] = q.w;
        }
    return TCE_OK;
}

int tce_set_graph(void *handle, int32_t on)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h) return fail(h, TCE_ERR_ARG, "NULL handle");
    h->use_graph = on ? 1 : 0;
    if (!on) drop_graph(h);
    return TCE_OK;
}

int tce_set_tensor_cores(void *handle, int32_t on)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h) return fail(h, TCE_ERR_ARG, "NULL handle");
    h->use_tc = on ? 1 : 0;
    ++h->work_version;   // a captured pass is re-captured
    return TCE_OK;
}

int tce_set_list_streams(void *handle, int32_t n)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h) return fail(h, TCE_ERR_ARG, "NULL handle");
    if (n != 1 && n != 2) return fail(h, TCE_ERR_ARG, "list streams: 1 or 2");
    h->list_streams = n;
    // a captured pass is re-captured; the lists are unchanged, so rejects
    // read from the last pass still apply
    const bool keep_fb = h->fb_version == h->work_version;
    ++h->work_version;
    if (keep_fb) h->fb_version = h->work_version;
    return TCE_OK;
}

int tce_fp64_peak(double *tflops)
{
    if (!tflops) return fail(nullptr, TCE_ERR_ARG, "NULL argument");
    Handle tmp;
    Handle *h = &tmp;
    int dev = 0, nsm = 148;
    CK(h, cudaGetDevice(&dev));
    CK(h, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t st;
    CK(h, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    double *sink = nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess) return fail(nullptr, TCE_ERR_NOMEM, "probe alloc");
    long long fl = 0;
    double best = 0.0;
    for (int rep = 0; rep < 6; ++rep) {
        cudaEventRecord(e0, st);
        tce_launch_fp64_probe(nsm, 20000, sink, st, &fl);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms > 0) best = std::max(best, fl / (ms * 1e-3) / 1e12);
    }
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(sink);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    if (e != cudaSuccess) return fail(nullptr, TCE_ERR_CUDA, cudaGetErrorString(e));
    *tflops = best;
    return TCE_OK;
}

int tce_shells(void *handle, int32_t *first, int32_t *n)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !first || !n) return fail(h, TCE_ERR_ARG, "NULL argument");
    for (int S = 0; S < h->nsh; ++S) {
        first[S] = h->sh_first[S];
        n[S] = h->sh_n[S];
    }
    return TCE_OK;
}

int tce_schwarz(void *handle, double *Q)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !Q) return fail(h, TCE_ERR_ARG, "NULL argument");
    std::memcpy(Q, h->Q.data(), h->Q.size() * sizeof(double));
    return TCE_OK;
}

// Start-up accuracy gate of the fixed rule (fast_quad_self_check,
// fast_quad_self_check.f90:30-233, ERI part): the on-site quartets
// (SI SI|SI SI) of the unit cell plus 50 pseudo-random quartets drawn with the
// reference's generator (seed 12345, x <- (1103515245 x + 12345) mod 2^31,
// value x/16), each evaluated with the prefactor screens only on `fast` (the
// 32/40-node rule) and on `full` (the 64/128-point table) of the same system.
int tce_quad_self_check(void *fast, void *full, double *dmax, int32_t *nsample)
{
    Handle *hf = static_cast<Handle *>(fast), *hF = static_cast<Handle *>(full);
    if (!hf || !hF || !dmax) return fail(hf, TCE_ERR_ARG, "NULL argument");
    if (hf->nsh != hF->nsh || hf->nshuc != hF->nshuc || hf->nbas != hF->nbas)
        return fail(hf, TCE_ERR_ARG, "the two handles describe different systems");
    const int nshuc = std::max(hf->nshuc, 1), nsh = hf->nsh, nrand = 50;
    long long seed = 12345;
    auto next = [&]() {
        seed = (seed * 1103515245LL + 12345LL) % 2147483648LL;
        return seed / 16;
    };
    std::vector<int4> items;
    for (int it = 0; it < nshuc + nrand; ++it) {
        if (it < nshuc) {
            items.push_back(make_int4(it, it, it, it));
        } else {
            const int a = (int)(next() % nshuc);
            const int b = (int)(next() % nsh);
            const int c = (int)(next() % nsh);
            const int d = (int)(next() % nsh);
            items.push_back(make_int4(a, b, c, d));
        }
    }
    std::vector<double> b1, b2;
    std::vector<long long> o1, o2;
    int s = run_blocks(hf, items, nullptr, TCE_MODE_BLOCK, 0, &b1, &o1);
    if (s) return s;
    s = run_blocks(hF, items, nullptr, TCE_MODE_BLOCK, 0, &b2, &o2);
    if (s) return fail(hf, s, "full-table blocks: " + hF->err);
    double m = 0.0;
    for (size_t i = 0; i < b1.size() && i < b2.size(); ++i) m = std::max(m, std::fabs(b1[i] - b2[i]));
    *dmax = m;
    if (nsample) *nsample = (int32_t)items.size();
    return TCE_OK;
}

int tce_shell_block(void *handle, const int32_t sh4[4], int32_t mode, double *blk)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !sh4 || !blk) return fail(h, TCE_ERR_ARG, "NULL argument");
    for (int i = 0; i < 4; ++i)
        if (sh4[i] < 0 || sh4[i] >= h->nsh) return fail(h, TCE_ERR_ARG, "shell index out of range");
    if (mode < 0 || mode > 2) return fail(h, TCE_ERR_ARG, "mode must be 0, 1 or 2");
    if (mode == 1 && !h->prim_screen) return fail(h, TCE_ERR_STATE, "mode 1 needs prim_screen");
    // translate the quartet so that S1 lies in the unit cell (values are translation invariant)
    int c1 = sh4[0] / h->nshuc;
    int4 q = make_int4(shift_to(h, sh4[0], c1, h->nshuc), shift_to(h, sh4[1], c1, h->nshuc),
                       shift_to(h, sh4[2], c1, h->nshuc), shift_to(h, sh4[3], c1, h->nshuc));
    std::vector<int4> items{q};
    std::vector<double> blocks;
    int s = run_blocks(h, items, nullptr, mode == 2 ? TCE_MODE_NOSCREEN : TCE_MODE_BLOCK, mode == 1, &blocks, nullptr);
    if (s) return s;
    std::memcpy(blk, blocks.data(), blocks.size() * sizeof(double));
    return TCE_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free shell-quartet block.  The scratch the quartet kernel needs
// for one block (its work counter, the work item, the block offsets and the
// block itself, at most 6^4 doubles for d shells) lives in this file-scope
// device array instead of buffers allocated per call, so the call makes no
// cudaMalloc/cudaFree.  Every GPU that loads the library holds the array
// (12 KiB) until the process exits.
// ---------------------------------------------------------------------------
#define TCE_STATIC_SCRATCH_BYTES (12 * 1024)
#define TCE_STATIC_MAX_BLOCK (TCE_NCOMP_MAX * TCE_NCOMP_MAX * TCE_NCOMP_MAX * TCE_NCOMP_MAX)
static __device__ __align__(256) unsigned char g_tce_static_scratch[TCE_STATIC_SCRATCH_BYTES];
// layout inside the array (byte offsets)
#define TCE_STATIC_OFF_NEXT 0      // unsigned int work counter
#define TCE_STATIC_OFF_ITEM 256    // int4 work item
#define TCE_STATIC_OFF_BOFF 512    // long long block offsets [2]
#define TCE_STATIC_OFF_BLK 1024    // double block[TCE_STATIC_MAX_BLOCK]
static_assert(TCE_STATIC_OFF_BLK + TCE_STATIC_MAX_BLOCK * sizeof(double) <= TCE_STATIC_SCRATCH_BYTES,
              "static scratch too small for a (dd|dd) block");

// Device address of the array in the current context.  The symbol name is only
// a host-side stand-in for the device storage, so host code must ask the
// runtime for the address; the lookup is repeated on every call (it is cheap)
// so that a context created anew after cudaDeviceReset is never handed an old
// address.
static int static_scratch(Handle *h, unsigned char **out)
{
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_tce_static_scratch);
    if (e != cudaSuccess)
        return fail(h, TCE_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    *out = static_cast<unsigned char *>(p);
    return TCE_OK;
}

// Run at handle creation, on the handle's device: resolve the array's address
// and load the quartet kernel of the handle's rule, so that with lazy module
// loading (the CUDA default) neither happens during a tce_shell_block_noalloc
// call, where loading a module could take device memory.
static int noalloc_prepare(Handle *h)
{
    unsigned char *p = nullptr;
    int s = static_scratch(h, &p);
    if (s) return s;
    if (tce_preload_quartets(h->S.nq) != TCE_OK) {
        cudaError_t e = cudaGetLastError();
        return fail(h, TCE_ERR_CUDA, std::string("loading the quartet kernel: ") + cudaGetErrorString(e));
    }
    return TCE_OK;
}

// Makes the handle's device current for the duration of a call and restores
// the caller's device afterwards.
struct DeviceScope {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceScope(int dev)
    {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != dev) err = cudaSetDevice(dev);
        else prev = -1;
    }
    ~DeviceScope()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int tce_shell_block_noalloc(void *handle, const int32_t sh4[4], int32_t mode, double *blk)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !sh4 || !blk) return fail(h, TCE_ERR_ARG, "NULL argument");
    for (int i = 0; i < 4; ++i)
        if (sh4[i] < 0 || sh4[i] >= h->nsh) return fail(h, TCE_ERR_ARG, "shell index out of range");
    if (mode < 0 || mode > 2) return fail(h, TCE_ERR_ARG, "mode must be 0, 1 or 2");
    if (mode == 1 && !h->prim_screen) return fail(h, TCE_ERR_STATE, "mode 1 needs prim_screen");
    long long nblk = (long long)h->sh_n[sh4[0]] * h->sh_n[sh4[1]] * h->sh_n[sh4[2]] * h->sh_n[sh4[3]];
    if (nblk > TCE_STATIC_MAX_BLOCK)
        return fail(h, TCE_ERR_UNSUPPORTED, "block of " + std::to_string(nblk) + " integrals exceeds the static scratch (" +
                                                 std::to_string(TCE_STATIC_MAX_BLOCK) + ")");
    // the array, the stream and the kernel all belong to the handle's device,
    // whichever device the calling thread has current
    DeviceScope dscope(h->dev);
    CK(h, dscope.err);
    unsigned char *base = nullptr;
    int s = static_scratch(h, &base);
    if (s) return s;
    int c1 = sh4[0] / h->nshuc;
    int4 q = make_int4(shift_to(h, sh4[0], c1, h->nshuc), shift_to(h, sh4[1], c1, h->nshuc),
                       shift_to(h, sh4[2], c1, h->nshuc), shift_to(h, sh4[3], c1, h->nshuc));
    long long off[2] = {0, nblk};
    // The item and offsets are rewritten every call; the launch below zeroes the
    // work counter itself.  Every element of the block is written by the kernel
    // (TCE_MODE_BLOCK / NOSCREEN copy the whole block), so the previous call's
    // contents of the array cannot reach this result.
    CK(h, cudaMemcpyAsync(base + TCE_STATIC_OFF_ITEM, &q, sizeof q, cudaMemcpyHostToDevice, h->st));
    CK(h, cudaMemcpyAsync(base + TCE_STATIC_OFF_BOFF, off, sizeof off, cudaMemcpyHostToDevice, h->st));
    QuartetHostArgs a;
    a.items = reinterpret_cast<const int4 *>(base + TCE_STATIC_OFF_ITEM);
    a.nitems = 1;
    a.mode = mode == 2 ? TCE_MODE_NOSCREEN : TCE_MODE_BLOCK;
    a.prim_screen = mode == 1;
    a.next = reinterpret_cast<unsigned int *>(base + TCE_STATIC_OFF_NEXT);
    a.blk_out = reinterpret_cast<double *>(base + TCE_STATIC_OFF_BLK);
    a.blk_off = reinterpret_cast<const long long *>(base + TCE_STATIC_OFF_BOFF);
    a.max_ncomb = ncomb_of(h, q.x, q.y, q.z, q.w);
    a.max_ncq = h->max_ncq;
    a.fixed_gmax = h->d_gmax;
    a.num_sms = h->num_sms;
    CKS(h, tce_launch_quartets(h->S, a, h->st));
    CK(h, cudaMemcpyAsync(blk, base + TCE_STATIC_OFF_BLK, sizeof(double) * nblk, cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return TCE_OK;
}

int tce_direct_jk_device(void *handle, const double *dP, double *dJ, double *dK, void *stream)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !dP || !dJ || !dK) return fail(h, TCE_ERR_ARG, "NULL argument");
    return direct_jk_device(h, dP, dJ, dK, static_cast<cudaStream_t>(stream));
}

int tce_direct_jk(void *handle, const double *P, double *J, double *K)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !P || !J || !K) return fail(h, TCE_ERR_ARG, "NULL argument");
    const int n = h->nbas, nf = h->nfuc;
    CK(h, cudaMemcpyAsync(h->d_P, P, sizeof(double) * n * n, cudaMemcpyHostToDevice, h->st));
    int s = direct_jk_device(h, h->d_P, h->d_J, h->d_K, h->st);
    if (s) return s;
    std::memset(J, 0, sizeof(double) * n * n);
    std::memset(K, 0, sizeof(double) * n * n);
    // rows < nfuc: device leading dimension nf -> host leading dimension n
    CK(h, cudaMemcpy2DAsync(J, sizeof(double) * n, h->d_J, sizeof(double) * nf, sizeof(double) * nf, n,
                            cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaMemcpy2DAsync(K, sizeof(double) * n, h->d_K, sizeof(double) * nf, sizeof(double) * nf, n,
                            cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return TCE_OK;
}

int tce_last_kernel_ms(void *handle, double *ms)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !ms) return fail(h, TCE_ERR_ARG, "NULL argument");
    float f = 0.f;
    CK(h, cudaEventSynchronize(h->ev1));
    CK(h, cudaEventElapsedTime(&f, h->ev0, h->ev1));
    *ms = f;
    return TCE_OK;
}

int tce_eri_stored(void *handle, int64_t eri_size, double *eri)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !eri) return fail(h, TCE_ERR_ARG, "NULL argument");
    int esz = h->sao ? h->nfuc : h->nbas;
    if (eri_size != esz) return fail(h, TCE_ERR_ARG, "eri_size must be nfuc (sao) or nbas");
    const long long n = h->nbas;
    long long elems = (long long)esz * n * n * n;
    if (!h->d_eri || h->eri_elems != elems) {
        if (h->d_eri) dfree(h, h->d_eri);
        h->d_eri = nullptr;
        int s = dalloc(h, &h->d_eri, (size_t)elems);
        if (s) return s;
        h->eri_elems = elems;
    }
    h->eri_size = esz;
    CK(h, cudaMemsetAsync(h->d_eri, 0, sizeof(double) * elems, h->st));
    if (h->nitems > 0) {
        QuartetHostArgs a;
        a.items = h->d_items;
        a.nitems = (int)h->nitems;
        a.mode = TCE_MODE_STORE;
        a.prim_screen = h->prim_screen;
        a.next = h->d_next;
        a.eri = h->d_eri;
        a.eri_size = esz;
        a.physicist = h->physicist;
        a.max_ncomb = h->max_ncomb;
        a.max_ncq = h->max_ncq;
        a.fixed_gmax = h->d_gmax;
        a.num_sms = h->num_sms;
        CKS(h, tce_launch_quartets(h->S, a, h->st));
    }
    if (!h->sao) CKS(h, tce_launch_sym_fill(h->nbas, h->nfuc, h->ncl, h->d_eri, h->st));
    CK(h, cudaMemcpyAsync(eri, h->d_eri, sizeof(double) * elems, cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return TCE_OK;
}

int tce_trexio_eri(void *handle, int64_t cap, int32_t *index, double *value, int64_t *count)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !count || cap < 0 || (cap > 0 && (!index || !value))) return fail(h, TCE_ERR_ARG, "bad argument");
    if (!h->d_eri || h->eri_size != h->nbas)
        return fail(h, TCE_ERR_STATE, "needs the full stored integrals: tce_eri_stored with sao = 0 first");
    int32_t *d_idx = nullptr;
    double *d_val = nullptr;
    int s;
    if (cap > 0) {
        if ((s = dalloc(h, &d_idx, (size_t)cap * 4))) return s;
        if ((s = dalloc(h, &d_val, (size_t)cap))) return s;
    }
    long long cnt = 0;
    if (tce_trexio_stream(h->d_eri, h->nbas, cap, d_idx, d_val, &cnt, h->st) != TCE_OK)
        return fail(h, TCE_ERR_CUDA, "integral stream kernels failed");
    *count = cnt;
    const long long m = std::min<long long>(cnt, cap);
    if (m > 0) {
        CK(h, cudaMemcpyAsync(index, d_idx, sizeof(int32_t) * 4 * (size_t)m, cudaMemcpyDeviceToHost, h->st));
        CK(h, cudaMemcpyAsync(value, d_val, sizeof(double) * (size_t)m, cudaMemcpyDeviceToHost, h->st));
        CK(h, cudaStreamSynchronize(h->st));
    }
    dfree(h, d_idx);
    dfree(h, d_val);
    return TCE_OK;
}

int tce_stored_jk(void *handle, const double *P, double *J, double *K)
{
    Handle *h = static_cast<Handle *>(handle);
    if (!h || !P || !J || !K) return fail(h, TCE_ERR_ARG, "NULL argument");
    if (!h->d_eri) return fail(h, TCE_ERR_STATE, "tce_eri_stored has not been called");
    const int n = h->nbas, n1 = h->eri_size;
    double *dJ = nullptr, *dK = nullptr;
    int s;
    if ((s = dalloc(h, &dJ, (size_t)n1 * n))) return s;
    if ((s = dalloc(h, &dK, (size_t)n1 * n))) return s;
    CK(h, cudaMemcpyAsync(h->d_P, P, sizeof(double) * n * n, cudaMemcpyHostToDevice, h->st));
    CK(h, cudaMemsetAsync(dJ, 0, sizeof(double) * n1 * n, h->st));
    CK(h, cudaMemsetAsync(dK, 0, sizeof(double) * n1 * n, h->st));
    CKS(h, tce_launch_stored_jk(n1, n, h->physicist, h->d_P, h->d_eri, dJ, dK, h->st));
    std::memset(J, 0, sizeof(double) * n * n);
    std::memset(K, 0, sizeof(double) * n * n);
    CK(h, cudaMemcpy2DAsync(J, sizeof(double) * n, dJ, sizeof(double) * n1, sizeof(double) * n1, n,
                            cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaMemcpy2DAsync(K, sizeof(double) * n, dK, sizeof(double) * n1, sizeof(double) * n1, n,
                            cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    dfree(h, dJ);
    dfree(h, dK);
    return TCE_OK;
}

int tce_hartree_exchange(int32_t n1, int32_t nbas, int32_t physicist, const double *P, const double *eri, double *J,
                         double *K)
{
    if (n1 <= 0 || nbas <= 0 || n1 > nbas || !P || !eri || !J || !K)
        return fail(nullptr, TCE_ERR_ARG, "bad argument");
    Handle tmp;
    Handle *h = &tmp;
    CK(h, cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
    long long elems = (long long)n1 * nbas * nbas * nbas;
    double *dE = nullptr, *dP = nullptr, *dJ = nullptr, *dK = nullptr;
    int s = TCE_OK;
    auto cleanup = [&]() {
        for (void *p : h->allocs) cudaFree(p);
        cudaStreamDestroy(h->st);
    };
    if ((s = dalloc(h, &dE, (size_t)elems)) || (s = dalloc(h, &dP, (size_t)nbas * nbas)) ||
        (s = dalloc(h, &dJ, (size_t)n1 * nbas)) || (s = dalloc(h, &dK, (size_t)n1 * nbas))) {
        cleanup();
        return s;
    }
    cudaMemcpyAsync(dE, eri, sizeof(double) * elems, cudaMemcpyHostToDevice, h->st);
    cudaMemcpyAsync(dP, P, sizeof(double) * nbas * nbas, cudaMemcpyHostToDevice, h->st);
    cudaMemsetAsync(dJ, 0, sizeof(double) * n1 * nbas, h->st);
    cudaMemsetAsync(dK, 0, sizeof(double) * n1 * nbas, h->st);
    s = tce_launch_stored_jk(n1, nbas, physicist, dP, dE, dJ, dK, h->st);
    std::memset(J, 0, sizeof(double) * nbas * nbas);
    std::memset(K, 0, sizeof(double) * nbas * nbas);
    cudaMemcpy2DAsync(J, sizeof(double) * nbas, dJ, sizeof(double) * n1, sizeof(double) * n1, nbas,
                      cudaMemcpyDeviceToHost, h->st);
    cudaMemcpy2DAsync(K, sizeof(double) * nbas, dK, sizeof(double) * n1, sizeof(double) * n1, nbas,
                      cudaMemcpyDeviceToHost, h->st);
    cudaError_t e = cudaStreamSynchronize(h->st);
    cleanup();
    if (s != TCE_OK) return fail(nullptr, s, "stored J/K launch failed");
    if (e != cudaSuccess) return fail(nullptr, TCE_ERR_CUDA, cudaGetErrorString(e));
    return TCE_OK;
}

}  // extern "C"
