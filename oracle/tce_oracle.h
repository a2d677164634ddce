/*
 * tce_oracle.h -- CPU oracle for the toroidal (Clifford-Gaussian) ERI path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (ALRAKIK/William_CI, Fortran) used as the checker of the CUDA
 * engine.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.  The product library (libtce) never links or calls it.
 *
 * Parity status: the reference cannot be compiled in this environment (no
 * Fortran compiler), so no reference-produced outputs exist.  The oracle is
 * pinned instead by (a) the reference's own quadrature tables (fixture read
 * from the reference source), (b) its runtime self-checks restated as
 * properties (fast vs full quadrature <= 1e-10, 8-fold symmetry, direct J/K ==
 * stored J/K, <phi|phi> = 1), (c) the L -> infinity limit against an
 * independently written Boys-function GTO ERI, and (d) brute-force real-space
 * quadrature of the periodic direction.
 *
 * Indices are 0-based here; the Fortran originals are 1-based.
 */
#ifndef TCE_ORACLE_H
#define TCE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Flat description of a supercell basis (same layout as include/tce.h). */
typedef struct {
    int32_t ndp;          /* periodic directions 1..ndp (1, 2, 3)            */
    int32_t ncell[3];     /* nx, ny, nz (cells x fastest)                    */
    int32_t nfuc;         /* functions per unit cell                         */
    int32_t nbas;         /* functions in the supercell                      */
    int32_t nquad;        /* t nodes                                          */
    double  L[3];         /* Lx, Ly, Lz (a_d = 2 pi / L_d)                   */
    const double  *ctr;   /* [3*nbas] centres                                */
    const int32_t *lxyz;  /* [3*nbas] Cartesian powers                       */
    const int32_t *prim_off; /* [nbas+1] CSR offsets into exps/coefs         */
    const double  *exps;  /* primitive exponents                             */
    const double  *coefs; /* normalised contraction coefficients             */
    const double  *t_nodes;   /* [nquad] t nodes, NULL: mapped GL (fast_quad) */
    const double  *t_weights; /* [nquad] t weights                           */
    int32_t physicist;    /* stored layout: 0 chemist (ij|kl), 1 physicist   */
    int32_t sao;          /* 1: ERI_size = nfuc, 0: ERI_size = nbas          */
    int32_t prim_screen;  /* primitive-pair Schwarz screening (default 1)    */
    double  schwarz_thr;  /* 1e-13                                           */
    double  prim_thr;     /* 1e-14                                           */
} orc_system;

/* ---- math primitives ---- */
double orc_iv_log(double v, double x);
double orc_iv_scaled(int n, double x);
void   orc_bessel_scaled_vector(int N, double A, double *Iv);
void   orc_bessel_scaled_vector_fast(int N, double A, double *Iv);
int    orc_bessel_nmax_estimate(double A);
void   orc_fourier_sin_product(int i, int l, double phA, double phB, double *d_re, double *d_im);
void   orc_pair_vector(int N, double A, int i, int l, double phA, double phB, int sgn,
                       double *v_re, double *v_im);
void   orc_fast_quad_points(int n, double *t, double *w);
void   orc_bary(double e1, double e2, double x1, double x2, double L, double a,
                double *pe, double *cen);
void   orc_hermite_E_1D(int i, int j, double p, double PA, double PB, double *E17);

/* ---- the engine state (direct_init / ERI driver preamble) ---- */
typedef struct orc_ctx orc_ctx;
orc_ctx *orc_create(const orc_system *sys);
void     orc_destroy(orc_ctx *c);
/* Blocks of n shell quartets, concatenated in item order (OpenMP over them). */
int64_t  orc_shell_blocks(orc_ctx *c, int64_t n, const int32_t *items4, int mode, double *out);
/* Release the pair-vector memo of the timing build (pair_cache_free,
 * clifford_tools.f90:555-561); a no-op in the parity build. */
void     orc_pair_cache_free(void);
int      orc_nshells(const orc_ctx *c, int *nshuc, int *ncap);
void     orc_shell_info(const orc_ctx *c, int s, int *first, int *n);
/* Schwarz matrix Q (nbas x nbas, col-major), shell maxima Qsh (nsh x nsh) */
const double *orc_schwarz(const orc_ctx *c);
const double *orc_schwarz_shell(const orc_ctx *c);
/* prim table ps_qp(mp,mp,nshuc,nsh), col-major; returns mp */
const double *orc_prim_table(const orc_ctx *c, int *mp);
/* t-tables: nodes, weights, t_bessel((ncap+1) x nq x ndp), t_nmax (nq x ndp) */
void orc_t_tables(const orc_ctx *c, const double **node, const double **weight,
                  const double **tbessel, const int **tnmax);

/* ERI_shell_block_toroidal for shells (S1,S2|S3,S4), 0-based shell ids.
 * mode 0: prefactor screens on, prim screen off (Schwarz pass)
 * mode 1: prefactor screens on, prim screen on (main loops)
 * mode 2: all screens off (primitive table pass)
 * blk is column-major (n1,n2,n3,n4). */
void orc_shell_block(orc_ctx *c, int S1, int S2, int S3, int S4, int mode, double *blk);

/* Stored ERIs: eri[ERI_size * nbas^3] column-major, ERI_size = nfuc (sao) or nbas.
 * Returns the number of computed shell quartets. */
int64_t orc_eri_stored(orc_ctx *c, double *eri);
/* Integral-direct J/K (rows < nfuc filled, others 0), col-major nbas x nbas. */
int64_t orc_direct_jk(orc_ctx *c, const double *P, double *J, double *K);
/* J/K from a stored array ERI(n1,nbas,nbas,nbas). */
void orc_hartree_exchange(int n1, int nbas, int physicist, const double *P,
                          const double *eri, double *J, double *K);
/* Rows i > nfuc by translation, in place (non-SAO). */
void orc_sym_fill_eri(int nbas, int nfuc, const int32_t ncell[3], double *eri);

/* Unique shell quartets in driver order (out4: 4 ints per quartet). */
int64_t orc_items(orc_ctx *c, int32_t *out4, int64_t cap);
/* direct_JK over an explicit quartet list; J/K accumulated; returns the
 * function quartets evaluated. */
int64_t orc_direct_jk_items(orc_ctx *c, const int32_t *items4, int64_t nitems, const double *P, double *J, double *K);

/* Counting helpers for the bench: unique shell quartets, function quartets
 * (after the function-level Schwarz screen) and primitive quartets evaluated. */
void orc_count(orc_ctx *c, int64_t *n_shell_q, int64_t *n_func_q, int64_t *n_prim_q);

/* ---- one-electron pieces needed to build normalised inputs ---- */
double orc_overlap_pair(int ndp, const double L[3], const int32_t l1[3], const int32_t l2[3],
                        const double r1[3], const double r2[3],
                        int n1, const double *e1, const double *c1,
                        int n2, const double *e2, const double *c2);
/* normalize_AO_toroidal_{1,2,3}D: coefs (CSR like orc_system) updated in place */
double orc_normalize(int ndp, const double L[3], int nbas, const double *ctr, const int32_t *lxyz,
                     const int32_t *prim_off, const double *exps, double *coefs);

/* ---- one-electron matrices and nuclear repulsion (RHF_SAO inputs) ---- */
double orc_kinetic_pair(int ndp, const double L[3], const int32_t l1[3], const int32_t l2[3],
                        const double r1[3], const double r2[3], int n1, const double *e1, const double *c1,
                        int n2, const double *e2, const double *c2);
/* S, T, V (nbas x nbas, col-major), geometry [3*natoms], charges [natoms] */
void orc_one_electron(orc_ctx *c, int natoms, const double *geo, const int32_t *Z, double *S, double *T, double *V);
double orc_nuclear_repulsion(int ndp, const double L[3], int natoms, const double *geo, const int32_t *Z);

#ifdef __cplusplus
}
#endif
#endif
