/*
 * tce.h -- C ABI of the B200 toroidal-ERI engine (libtce.so).
 *
 * Drop-in boundary for the integral and SCF path of ALRAKIK/William_CI.  The
 * reference has no FFI layer: the path sits behind Fortran subroutines and
 * module globals.  Each entry point below names the reference routine it
 * replaces (paths relative to the reference project root).  A Fortran
 * caller binds them with ISO_C_BINDING; a nonzero status maps to the
 * reference's `error stop`.
 *
 * Conventions
 *   - All matrices are column-major (Fortran order), double precision.
 *   - Indices in tce_system are 0-based; shells are found exactly as the
 *     reference finds them (consecutive Cartesian components with the same
 *     centre and exponents, ERI_toroidal.f90:106-125).
 *   - Calls on one handle come from a single host thread.  Device memory is
 *     owned by the handle.  There is no CPU fallback: without a usable B200
 *     every call returns TCE_ERR_CUDA.
 */
#ifndef TCE_H
#define TCE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TCE_OK              0
#define TCE_ERR_ARG         1   /* bad argument / inconsistent system        */
#define TCE_ERR_UNSUPPORTED 2   /* angular momentum or layout not supported  */
#define TCE_ERR_CUDA        3   /* CUDA error (no device, launch failure ...) */
#define TCE_ERR_STATE       4   /* call order (e.g. stored ERIs not built)    */
#define TCE_ERR_NOMEM       5   /* device allocation failed                   */

/* Flat, C-interoperable copy of the supercell basis.  Replaces the module
 * globals torus_init (Torus_init.f90:1-31), unitcell_module (unitcell.f90),
 * keywords c_physicist/c_SAO/c_prim_screen (keywords.f90), nquad_point /
 * t_val / w_val (precompute_t.f90:5-14) and the AO array of ERI_function
 * (ERI_mod.f90:5-12), which has allocatable components and is not
 * interoperable. */
typedef struct {
    int32_t ndp;              /* periodic directions 1..ndp (Tori1D/2D/3D)   */
    int32_t ncell[3];         /* nx, ny, nz; cells numbered x fastest        */
    int32_t nfuc;             /* functions per unit cell                     */
    int32_t nbas;             /* functions in the supercell                  */
    int32_t nquad;            /* t nodes: 32/40 mapped GL (fast_quad) or the
                                 number of entries of t_nodes                */
    double  L[3];             /* Lx, Ly, Lz; a_d = 2 pi / L_d                */
    const double  *ctr;       /* [3*nbas] centres (x,y,z per function)       */
    const int32_t *lxyz;      /* [3*nbas] Cartesian powers (class.f90 order) */
    const int32_t *prim_off;  /* [nbas+1] CSR offsets into exps/coefs        */
    const double  *exps;      /* primitive exponents                         */
    const double  *coefs;     /* NORMALISED contraction coefficients
                                 (normalize_AO_toroidal_*D already applied)  */
    const double  *t_nodes;   /* [nquad] or NULL: mapped Gauss-Legendre,
                                 t = 0.6 u/(1-u) (precompute_t.f90:906-942)  */
    const double  *t_weights; /* [nquad] or NULL                             */
    int32_t physicist;        /* stored layout: 0 chemist, 1 physicist       */
    int32_t sao;              /* 1: ERI_size = nfuc, 0: ERI_size = nbas      */
    int32_t prim_screen;      /* primitive-pair Schwarz screen (default 1)   */
    double  schwarz_thr;      /* 1e-13 (ERI_toroidal.f90:64)                 */
    double  prim_thr;         /* 1e-14 (clifford_tools.f90:74)               */
} tce_system;

/* Counters of the work set (translation- and 8-fold-unique quartets). */
typedef struct {
    int32_t nsh, nshuc, ncap, nquad;
    int64_t n_shell_quartets;     /* unique shell quartets after screening  */
    int64_t n_func_quartets;      /* function quartets after the Q screen   */
    int64_t n_unit_pairs;         /* significant unit-cell shell pairs       */
    int64_t device_bytes;         /* device memory held by the handle        */
    int64_t n_prim_quartets;      /* primitive quartets evaluated per J/K pass
                                     (after the prefactor and primitive screens) */
    double  jk_flops;             /* algorithmic FP64 operations of one J/K pass,
                                     counted from the reference's operation counts
                                     (see the work-count kernel)               */
    int32_t shard_rank, shard_nranks;  /* current shard (0, 1 when unsharded) */
    int64_t shard_shell_quartets; /* shell quartets this shard evaluates       */
} tce_info;

/* Build the engine for one supercell basis: t-tables, shells, Schwarz
 * bounds, primitive-pair table and the unique-quartet work list, all on the
 * device.  Replaces direct_init (eri_direct.f90:76-225) and the preamble of
 * ERI_integral_toroidal (ERI_toroidal.f90:93-337). */
int tce_create(const tce_system *sys, void **handle);
int tce_destroy(void *handle);
const char *tce_last_error(void *handle);   /* handle may be NULL */

/* A handle for shell blocks only (tce_shell_block, tce_rule_blocks): t-tables,
 * shells and pair data, but no Schwarz pass, primitive table or quartet
 * list, so J/K are not available.  Used for density fitting (df_init,
 * df_toroidal.f90:352-701): the system then holds the orbital functions, the
 * auxiliary functions and constant dummies (one s function of exponent 0 and
 * coefficient 1 next to the auxiliary functions of each atom), and
 * (mu nu|P) = (mu nu|P 1), (P|Q) = (P 1|Q 1) are ordinary blocks.  Pairs of two
 * exponent-0 functions have zero weight. */
int tce_create_blocks(const tce_system *sys, void **handle);
int tce_get_info(void *handle, tce_info *info);

/* One shell quartet block (S1 S2|S3 S4), blk column-major (n1,n2,n3,n4).
 * Parity hook for ERI_shell_block_toroidal (ERI_shell_block_toroidal.f90:28).
 * mode 0: prefactor screens (Schwarz pass); 1: + primitive screen (the main
 * loops; needs S1 in the unit cell); 2: no screens (primitive-table pass). */
int tce_shell_block(void *handle, const int32_t sh4[4], int32_t mode, double *blk);

/* Same block as tce_shell_block, for callers that cannot have the library
 * allocate device memory during the call: a host program whose device
 * memory is reserved up front by its own pool allocator, where a cudaMalloc
 * inside the library would fail or fragment the pool.  No counterpart in the
 * reference.  The call allocates nothing: its scratch (work counter, work
 * item, block) is one file-scope device array of 12 KiB that every GPU using
 * the library holds until exit.  The array's device address is resolved and
 * the quartet kernel loaded when the handle is created (tce_create /
 * tce_create_blocks), so that a call never loads a module lazily; the call
 * runs on the handle's device whichever device the calling thread has
 * current.  Blocks of more than 6^4 integrals are rejected
 * (TCE_ERR_UNSUPPORTED).  All calls share the array: calls that overlap on
 * the GPU race, so do not issue them concurrently from several threads or
 * handles. */
int tce_shell_block_noalloc(void *handle, const int32_t sh4[4], int32_t mode, double *blk);

/* Start-up accuracy gate of the fast rule (replaces the ERI part of
 * fast_quad_self_check, fast_quad_self_check.f90:30-233): `fast` and `full`
 * are handles of the same system built with the 32/40-node rule and with the
 * 64/128-point table.  The on-site quartets (SI SI|SI SI) of the unit cell and
 * 50 pseudo-random quartets (the reference's generator and seed) are
 * evaluated on both; dmax is the largest difference.  The reference keeps the
 * fast rule when dmax <= 1e-10, the caller does the same with its handles. */
int tce_quad_self_check(void *fast, void *full, double *dmax, int32_t *nsample);

/* The whole gate of fast_quad_self_check (fast_quad_self_check.f90:30-233):
 * the ERI sample of tce_quad_self_check (dmax, nq elements) and then, with
 * the same generator continuing, the nuclear-attraction sample of :135-172:
 * V(i,i) for the first function of every unit-cell shell, 20 random pairs in
 * the unit cell, 20 with j anywhere (nv elements), each computed with both
 * handles; dV is the largest difference.  The reference keeps the fast rule
 * when dmax <= 1e-10 and dV <= 1e-10.  geometry and Z as
 * tce_nuclear_attraction. */
int tce_quad_self_check_nuc(void *fast, void *full, int32_t natoms, const double *geometry, const int32_t *Z,
                            double *dmax, double *dV, int32_t *nq, int32_t *nv);

/* Shell list: first function and component count of each shell. */
int tce_shells(void *handle, int32_t *first, int32_t *n);

/* Schwarz matrix Q(i,j) = sqrt|(ij|ij)| (nbas x nbas), as built by the
 * driver (ERI_toroidal.f90:200-236). */
int tce_schwarz(void *handle, double *Q);

/* Stored ERIs ERI(eri_size, nbas, nbas, nbas), chemist or physicist order,
 * eri_size = nfuc (sao) or nbas (rows i > nfuc filled by translation,
 * symmetric_matrix.f90:62-131).  Replaces ERI_integral_toroidal
 * (ERI_toroidal.f90:36).  The array is also kept on the device for
 * tce_stored_jk. */
int tce_eri_stored(void *handle, int64_t eri_size, double *eri);

/* The two-electron part of the TREXIO export (trexio_conv_integrals,
 * trexio_conv.f90:267-359): from the full stored integrals on the device
 * (tce_eri_stored with sao = 0; the reference reads a full nbas^4 array, so
 * SAO mode has no export), the entries it writes, in its order: (i, j, k, l)
 * with i fastest, then j, k, l, kept when i >= j, (i == j => k >= l) and
 * ERI(i, k, j, l) != 0; index[4e..4e+3] = (i, j, k, l) 1-based, value[e] =
 * ERI(i, k, j, l).  *count = the stream's length; the first min(count, cap)
 * entries are written (cap 0: count only).  The caller passes them to
 * trexio_write_ao_2e_int_eri in chunks, as the reference does with BUFSIZE
 * 10000.  libtrexio itself is not part of this library. */
int tce_trexio_eri(void *handle, int64_t cap, int32_t *index, double *value, int64_t *count);

/* J and K from the device-resident stored ERIs (rows < ERI_size filled).
 * Replaces hartree_exchange_potential (hartree_exchange_potential.f90:30). */
int tce_stored_jk(void *handle, const double *P, double *J, double *K);

/* J and K from a caller-provided stored ERI array (uploaded per call); same
 * formulas as hartree_exchange_potential (hartree_exchange_potential.f90:30)
 * with n1 = ERI_size. */
int tce_hartree_exchange(int32_t n1, int32_t nbas, int32_t physicist, const double *P,
                         const double *eri, double *J, double *K);

/* Integral-direct J/K for one SCF iteration: rows < nfuc of J and K filled,
 * the others zero.  Host arrays, nbas x nbas.  Replaces direct_JK
 * (eri_direct.f90:262-374). */
int tce_direct_jk(void *handle, const double *P, double *J, double *K);

/* Same with device pointers on the caller's stream (cudaStream_t as void*):
 * dP nbas x nbas, dJ and dK nfuc x nbas (column-major, leading dim nfuc). */
int tce_direct_jk_device(void *handle, const double *dP, double *dJ, double *dK, void *stream);

/* Elapsed device time (ms) of the last tce_direct_jk[_device] call's quartet
 * kernel, measured with CUDA events on the launching stream. */
int tce_last_kernel_ms(void *handle, double *ms);

/* CUDA graphs: with on != 0, every J/K pass of this handle (all its kernel
 * launches and the zeroing of J and K) is captured once into a CUDA graph and
 * replayed as one graph launch per call, e.g. once per SCF iteration.  The
 * graph is re-captured when the pointers, the stream, the method or the work
 * lists change.  Default off. */
int tce_set_graph(void *handle, int32_t on);

/* Node sums of the learned-grid pass on the FP64 tensor cores (mma.sync
 * m8n8k4, FP64 in and out) where a kernel has that form: the all-s quartets
 * and the s/p classes with one or two p shells of one periodic direction
 * (32- and 64-node rules, tile shapes from tce_lg_autotune), and the rows
 * (primitive quartet x power combination) of the generic kernel.  Default
 * on; off gives the FP64 CUDA-core kernels.  Same arithmetic type, different
 * summation order.  No reference counterpart. */
int tce_set_tensor_cores(void *handle, int32_t on);

/* The learned-grid work lists of a pass as n chains (1 or 2; default 2): the
 * lists split by their summed cost estimates, longest first, each chain on
 * its own stream inside the pass (and its CUDA graph), so that the tail of
 * one list's persistent launch overlaps the start of the next.  Every list
 * has its own work counter.  No reference counterpart (execution option). */
int tce_set_list_streams(void *handle, int32_t n);

/* Kernel-form tuning of the learned-grid pass (after tce_lg_predict_rules /
 * tce_lg_set_item_rules): every work list that has both a CUDA-core and an
 * FP64 tensor-core kernel is timed in each of its forms (the CUDA-core
 * kernel, the tensor-core kernel, and for the all-s quartets each tile shape
 * of the tensor-core kernel: 16 primitive quartets x 32 nodes per pass, 32 x
 * 16, 16 x 16, 8 x 64) with reps launches each (CUDA events; the fastest
 * launch counts) and keeps the fastest, also when the lists are rebuilt later
 * (new rules, rejects moved to the plain list).
 * ntuned: lists timed; nswitched: lists whose choice differs from the built-in
 * default; ms_saved: estimated time per pass saved against the default.  Uses
 * the handle's host-entry J/K buffers as scratch; results of later passes are
 * the same up to the summation order.  No reference counterpart. */
int tce_lg_autotune(void *handle, int32_t reps, int32_t *ntuned, int32_t *nswitched, double *ms_saved);

/* Set the kernel form of learned-grid work list `list` (its index in
 * tce_lg_lists) by hand, as tce_lg_autotune would: 0 the CUDA-core kernel,
 * 1 the tensor-core kernel, for all-s lists 1..4 its tile shape.  The form is
 * kept for the list's key across rebuilds.  No reference counterpart. */
int tce_lg_set_list_form(void *handle, int32_t list, int32_t form);

/* The learned-grid work lists of the handle: *n lists; with info (6 int32
 * per list, *n on entry = its capacity in lists): kind (0 generic, 1 all-s,
 * 2 one-p), class bits, padded rule nodes (32/64), FP32 panels, kernel form in
 * use (0 CUDA cores, >= 1 FP64 tensor cores; for the all-s kernel 1..4 its
 * tile shape in the order of tce_lg_autotune), quartets.  No reference
 * counterpart. */
int tce_lg_lists(void *handle, int32_t *n, int32_t *info);

/* Per-list measurement of the learned-grid pass: each work list (in the order
 * and kernel form tce_lg_lists reports) launched alone reps times on the
 * handle's stream, ms[i] the fastest launch (CUDA events), flops[i] its
 * algorithmic FP64 operations (counted as tce_lg_work).  With ms or flops
 * NULL only *n (the number of lists) is set.  Uses the handle's host-entry
 * J/K buffers as scratch.  No reference counterpart. */
int tce_lg_list_profile(void *handle, int32_t reps, int32_t *n, double *ms, double *flops);

/* Nuclear attraction matrix of the handle's system (replaces
 * nuclear_attraction_matrix_toroidal_{1,2,3}D, 1D_Nuclear_attraction_toroidal.f90
 * :169-276 / 3D_Nuclear_attraction_toroidal.f90:113-196, with the per-pair
 * integral of :26-163 / :18-111): V (nbas x nbas, column-major) with the rows
 * of the unit cell computed on the device (|V| < 1e-14 set to zero) and the
 * other rows by translation, as the reference's fill_with_symmetry.  geometry
 * is the reference's geometry(natoms, 3), column-major (x of every atom, then
 * y, then z); Z the nuclear charges.  Uses the handle's t-rule and tables (one periodic direction: node sums on the FP64 tensor cores when
 * tce_set_tensor_cores is on). */
int tce_nuclear_attraction(void *handle, int32_t natoms, const double *geometry, const int32_t *Z, double *V);

/* k-space MO integrals from the stored SAO integrals (replaces
 * transform_ERI_AO_to_kMO, AO_to_MO_SAO.f90:34-393, and its integral-direct
 * twin transform_ERI_direct_kMO, AO_to_MO_SAO_direct.f90:26-176):
 * out(p,q,r,s,k1,k2,k3) = (p k1, q k2 | r k3, s k4), k4 = k1 - k2 + k3, complex
 * (interleaved re/im), shape (no, nv, no, nv, cells, cells, cells)
 * column-major, no = p_hi - p_lo + 1, nv = q_hi - q_lo + 1; band indices
 * 1-based inclusive within 1..nfuc as the reference.  coeff is coeff_SAO
 * (nbas x nbas complex, column-major, k blocks on the diagonal).  Needs the
 * stored integrals of tce_eri_stored (eri_size = nfuc, chemist order) on the
 * handle. */
int tce_ao_to_kmo(void *handle, const double *coeff, int32_t p_lo, int32_t p_hi, int32_t q_lo, int32_t q_hi,
                  double *out);

/* Density-fitted J and K of the SCF (replaces df_JK, df_toroidal.f90:850-956).
 * tce_dfjk_create keeps on the device the fitted coefficients B =
 * df_B(nfuc, nbas, naux) (column-major, naux = nau x cells) and the k-space
 * Bh = df_Bh(nfuc, nau, nfuc, cells, nkh) of df_init (:660-678, complex as
 * interleaved re/im, k2 over the half set of df_khalf :103-114).  tce_dfjk
 * takes P (nbas x nbas) and returns J and K with rows > nfuc zero, as the
 * reference.  K is contracted with the whole P(k) (the reference drops the
 * eigen-components of P(k) below 1e-10 in magnitude).  Own error string:
 * tce_dfjk_last_error. */
int tce_dfjk_create(int32_t nfuc, int32_t nbas, int32_t nau, const int32_t ncl[3], const double *B, const double *Bh,
                    void **handle);
int tce_dfjk(void *handle, const double *P, double *J, double *K);
int tce_dfjk_destroy(void *handle);
const char *tce_dfjk_last_error(void *handle);

/* Multi-GPU: restrict tce_direct_jk[_device] on this handle to shard `rank`
 * of `nranks` (cost-balanced partition of the unique shell quartets, the same
 * partition on every rank).  The partial J/K of the ranks sum to the full J/K;
 * the caller reduces them (one all-reduce of 2 nfuc nbas doubles per SCF
 * iteration).  The OpenMP task unit of the reference is the bra shell pair
 * (eri_direct.f90:298-317); here it is the shell quartet. */
int tce_set_shard(void *handle, int32_t rank, int32_t nranks);

/* The shell quartets of the handle's current shard (all of them when
 * unsharded), in the engine's order: *n of them; with items != NULL,
 * items[4*i .. 4*i+3].  Lets a caller see which quartets a rank evaluates, or
 * check one shard against another implementation.  No reference counterpart
 * (the reference splits the bra shell pairs among OpenMP threads,
 * eri_direct.f90:298-317). */
int tce_shard_items(void *handle, int64_t *n, int32_t *items);

/* Host-only planner used by tce_set_shard: greedy longest-first assignment
 * of n work items with the given costs to nranks owners (owner[i] in
 * [0,nranks)).  Items are taken in the order given. */
int tce_shard_plan(const double *cost, int64_t n, int32_t nranks, int32_t *owner);

/* Measured FP64 FMA throughput of the current device (TFLOP/s), from a
 * probe kernel of independent FMA chains on every SM. */
int tce_fp64_peak(double *tflops);

/* ------------------------------------------------------------------------
 * Learned-grid t-quadrature.  No counterpart in the reference, whose
 * t-integral uses one fixed rule per run (fast_quad or the 64/128-point
 * tables, precompute_t.f90:5-14, 906-942).  A dictionary of mapped
 * Gauss-Kronrod rules (t = s u/(1-u), each with its embedded Gauss rule) is
 * loaded once; a small network picks one rule per shell quartet from
 * TCE_NFEAT features; in the J/K pass the Kronrod and Gauss estimates of the
 * quartet's block are compared (the judge) and a quartet with
 * max |K - G| > judge_tol is re-evaluated by the plain method: adaptive
 * bisection in u with 15-point Kronrod / 7-point Gauss panels, the Bessel
 * columns of every panel computed on the fly.
 * ------------------------------------------------------------------------ */
#define TCE_METHOD_FIXED   0   /* the system's rule (reference behaviour)      */
#define TCE_METHOD_LEARNED 1   /* per-quartet rule + judge + plain fallback    */
#define TCE_METHOD_PLAIN   2   /* plain adaptive method for every quartet      */
#define TCE_NFEAT 12           /* features per shell quartet                   */

/* The engine's work items (unique shell quartets, most expensive first):
 * items[4*i .. 4*i+3], i < n_shell_quartets. */
int tce_items(void *handle, int32_t *items);

/* Features of n shell quartets (items 4*n ints, any cell; NULL: the engine's
 * own items in order, n = n_shell_quartets) into feat[n*TCE_NFEAT]. */
int tce_item_features(void *handle, int64_t n, const int32_t *items, float *feat);

/* Rule dictionary: rule r has nn[r] <= 64 nodes t[64r+k], Kronrod weights
 * wk[64r+k] and embedded Gauss weights wg[64r+k] (0 off the Gauss nodes).
 * Builds each rule's Bessel table on the device. */
int tce_lg_set_rules(void *handle, int32_t nrules, const int32_t *nn, const double *t, const double *wk,
                     const double *wg);

/* Per-rule truncation orders gmax[r*48 + d*16 + g] (node group g of 8 nodes,
 * direction d): the last Bessel order with a nonzero table entry. */
int tce_lg_rule_gmax(void *handle, int32_t *gmax);

/* The plain method's panel rule: the 15-point Kronrod rule on u in [0,1]
 * (n = 15) with the embedded 7-point Gauss weights, mapped t = scale u/(1-u). */
int tce_set_plain_rule(void *handle, int32_t n, const double *u, const double *wk, const double *wg, double scale);

/* Host-only: the (2n+1)-point Gauss-Kronrod rule on u in [0, 1] (ascending
 * nodes u, Kronrod weights wk, embedded n-point Gauss weights wg, zero off the
 * Gauss nodes), by Laurie's algorithm and the Golub-Welsch eigenvalue
 * problem in extended precision; 1 <= n <= 64.  The rules of the
 * learned-grid dictionary are these, mapped by t = s u/(1-u). */
int tce_gk_rule(int32_t n, double *u, double *wk, double *wg);

/* Host-only: the learned grid's rule dictionary as tce_lg_setup loads it:
 * *nrules rules (K15, K21, K31, K41, K61 times 21 map scales 0.6 2^(j/2),
 * j = -18..2, order-major), rule r with nn[r] nodes t[64r+k], Kronrod weights
 * wk[64r+k] and Gauss weights wg[64r+k]; any array may be NULL. */
int tce_lg_dictionary(int32_t *nrules, int32_t *nn, double *t, double *wk, double *wg);

/* The whole set-up of the learned grid in one call, for a caller without the
 * Python host side: load the dictionary and the plain method's panel rule,
 * draw n_train of the handle's quartets (seeded), label them against the
 * 128-node mapped Gauss-Legendre reference evaluated on the handle (a rule is
 * correct when its block is within label_tol of the reference, 3e-14 is the
 * tested value, the judge accepts it, and the two next smaller scales of its
 * order are correct too), train the rule-picking network on the GPU (epochs,
 * batches of 256, Adam at 2e-3) and set every quartet's rule
 * (tce_lg_predict_rules, plain factor 10).  Then tce_set_method(h,
 * TCE_METHOD_LEARNED).  With net_out the trained network is returned (free it
 * with tce_mlp_destroy), else it is freed.  No reference counterpart. */
int tce_lg_setup(void *handle, int64_t n_train, uint64_t seed, int32_t epochs, double label_tol, void **net_out);

/* Per-item rules (engine item order); value nrules sends the item straight to
 * the plain method. */
int tce_lg_set_item_rules(void *handle, const int32_t *rule);
int tce_lg_item_rules(void *handle, int32_t *rule);

/* FP32 panels: learned-grid quartets of the register kernels (one periodic
 * direction) whose shell-pair Schwarz product Q(ij)Q(kl) is below thr sum
 * their periodic-direction node sums in FP32 (FP32 copy of the rule tables);
 * phases, Bessel vectors, real directions, weights, the judge and the J/K
 * accumulation stay FP64.  thr = 0 (default) turns it off; at most 1e-3. */
int tce_set_fp32_threshold(void *handle, double thr);

/* Quadrature method of tce_direct_jk[_device] (TCE_METHOD_*).  With
 * TCE_METHOD_LEARNED the quartets the judge rejected in a pass (their count
 * is read back asynchronously after the pass) are sent straight to the plain
 * method from the next pass on (up to 4096 of them; the work lists change
 * once, and tce_lg_item_rules then reports them as plain); the plain list
 * runs on a second stream of the handle next to the learned-grid kernels.
 * No reference counterpart: the reference has one quadrature. */
int tce_set_method(void *handle, int32_t method);

/* Kernels one J/K pass launches with the current method and work lists
 * (memsets and copies not counted).  No reference counterpart. */
int tce_pass_kernels(void *handle, int32_t *n);

/* Judge tolerance on max |K - G| of a block (default 1e-10), plain-method
 * tolerance on the summed panel estimates (default 1e-11) and its panel
 * budget (1..24, default 24). */
int tce_set_tolerances(void *handle, double judge_tol, double plain_tol, int32_t plain_max_panels);

/* Counters of the last J/K pass: stats[0] quartets on the learned grid,
 * stats[1] of those rejected by the judge, stats[2] quartets sent straight to
 * the plain method, stats[3] t nodes the plain method evaluated, stats[4]
 * learned-grid quartets with FP32 node sums (array of 5). */
int tce_lg_stats(void *handle, int64_t *stats);

/* Algorithmic FP64 operations and primitive quartets of the learned-grid pass
 * with the current per-item rules (quartets sent to the plain method
 * excluded), counted like tce_info.jk_flops with each quartet's own rule. */
int tce_lg_work(void *handle, double *flops, int64_t *nprim);

/* Blocks of n shell quartets with one quadrature, concatenated in item order
 * (each column-major n1 n2 n3 n4): rule >= 0 a dictionary rule (Kronrod
 * estimate in K, Gauss estimate in G when G is not NULL), -1 the system's
 * rule, -2 the plain method.  mode as tce_shell_block. */
int tce_rule_blocks(void *handle, int32_t rule, int32_t mode, int64_t n, const int32_t *items, double *K, double *G);

/* The rule-picking network: TCE_NFEAT -> nh -> nh -> nc (ReLU), FP32 on the
 * device, parameters flat W1[nh][nf] b1 W2[nh][nh] b2 W3[nc][nh] b3; inputs
 * are standardised with per-feature mean mu and scale sig.  Output c is the
 * logit of the probability that dictionary rule c is accepted by the judge
 * and correct for the quartet (nc = number of rules). */
int tce_mlp_create(int32_t nf, int32_t nh, int32_t nc, uint64_t seed, void **mlp);
int tce_mlp_destroy(void *mlp);
const char *tce_mlp_last_error(void *mlp);
int tce_mlp_nparams(void *mlp, int64_t *np);
int tce_mlp_get_params(void *mlp, float *p, float *mu, float *sig);
int tce_mlp_set_params(void *mlp, const float *p, const float *mu, const float *sig);
/* Sigmoid cross-entropy of the outputs against targets Y[n][nc] in [0,1],
 * summed over outputs and averaged over rows, and its gradient (forward and
 * backward kernels on the device). */
int tce_mlp_loss_grad(void *mlp, int64_t n, const float *X, const float *Y, float *loss, float *grad);
/* Adam training on shuffled mini-batches (standardisation set from X). */
int tce_mlp_train(void *mlp, int64_t n, const float *X, const float *Y, int32_t epochs, int32_t batch, float lr,
                  uint64_t seed, float *final_loss);
/* Output probabilities prob[n][nc]. */
int tce_mlp_predict(void *mlp, int64_t n, const float *X, float *prob);
/* Features of every engine item, network forward and the rule of least
 * expected cost on the device: cost_r + (1 - p_r) C_plain, C_plain =
 * plain_factor x the dearest rule's cost (nrules, i.e. the plain method, when
 * that is cheaper).  Sets the per-item rules; nc must equal nrules. */
int tce_lg_predict_rules(void *handle, void *mlp, double plain_factor);

/* ------------------------------------------------------------------------
 * DF-MP2 contraction and energy.  Replaces the (ov|ov) loop of df_kMO
 * (df_toroidal.f90:1018-1035) and kMP2_calc (MP2_SAO.f90:6-151):
 *   G(i a, j b; k1, k2, k3) = 1/N sum_Q L(i a, Q, k1, k2) L(j b, Q, k3, k4),
 *   k4 = k1 - k2 + k3,
 *   E2d = -sum |G(ia,jb;ki,ka,kj)|^2 / D,  E2x = -sum Re G(ia,jb;ki,ka,kj)
 *          conj G(ib,ja;ki,kb,kj) / D,  D = e_a(ka) + e_b(kb) - e_i(ki) - e_j(kj),
 *   E_MP2 = 2 E2d - E2x; terms with |D| < 1e-8 are left out and counted
 *   (nzero, largest |G| in gzero).
 * L: complex (re,im interleaved) L(p,q,Q,k1,k2), column-major, p < no
 * (occupied band range 1..o_hi), q < nv (virtual band range v_lo..nfuc);
 * kcoord[3k..3k+2]: cell coordinates of k (x fastest), ncl the lattice;
 * eps_o[k*no+i], occ_o[k*no+i], eps_v[k*nv+a], occ_v[k*nv+a]: band energies
 * and occupations (2 occupied, 0 virtual) of those ranges.
 * mode 0: contraction in FP64; mode 1: tensor cores in split-BF16 with FP32
 * accumulation (energy sums FP64 in both).  ms: device time of the kernels. */
int tce_dfmp2_energy(int32_t ncell, const int32_t ncl[3], const int32_t *kcoord, int32_t no, int32_t nv,
                     int32_t nau, const double *L, const double *eps_o, const int32_t *occ_o, const double *eps_v,
                     const int32_t *occ_v, int32_t mode, double *e2d, double *e2x, int64_t *nzero, double *gzero,
                     double *ms);
const char *tce_mp2_last_error(void);

/* ------------------------------------------------------------------------
 * Density fitting and DF-MP2 from one handle (replaces df_init,
 * df_toroidal.f90:352-701 with chol_f :1174-1216, df_L_kap :1053-1104 and
 * kMP2_calc, MP2_SAO.f90:6-151).  tce_df_create takes the orbital system (as
 * tce_create) and the auxiliary basis on the same supercell (normalised, cells
 * numbered as the orbitals), and the atoms (geometry(natoms,3) column-major,
 * cells x fastest, atoms of a cell together): it builds the fit's system
 * (per cell the orbital functions, the auxiliary functions and one constant
 * dummy per atom), computes the metric (P0|Q R) and the three-index
 * (mu0 nu|P R) integrals on the device, factorises V(k) per k (pivoted
 * Cholesky, tolerance 1e-10) and keeps df_B on the device.  At most 32
 * auxiliary functions per cell.  Own error string: tce_df_last_error. */
int tce_df_create(const tce_system *ao, const tce_system *aux, int32_t natoms, const double *geometry, void **df);
int tce_df_destroy(void *df);
const char *tce_df_last_error(void *df);
/* Host copies of the metric Vm(nau, naux) and T3(nfuc, nbas, naux), naux = nau
 * cells, column-major (either may be NULL). */
int tce_df_integrals(void *df, double *Vm, double *T3);
/* Host copies of df_B(nfuc, nbas, naux) and of the k-space
 * df_Bh(nfuc, nau, nfuc, cells, nkh) (complex, interleaved), the inputs of
 * tce_dfjk_create; ndrop: the most metric pivots dropped at any k.  Any
 * pointer may be NULL. */
int tce_df_fitted(void *df, double *B, double *Bh, int32_t *ndrop);
/* E_MP2 = 2 E2d - E2x of an RHF solution: coeff is coeff_SAO (nbas x nbas
 * complex, interleaved, column-major, k blocks on the diagonal), eps and occ
 * the orbital energies and occupations (2 or 0) in the same order (k block by
 * k block).  The band ranges are cc_dims' (occupied 1..max_k nocc(k), virtual
 * min_k nocc(k)+1..nfuc); the L vectors are formed on the device and
 * contracted as tce_dfmp2_energy (mode 0 FP64, 1 split-BF16).  e2d, e2x may be
 * NULL. */
int tce_dfmp2(void *df, const double *coeff, const double *eps, const int32_t *occ, int32_t mode, double *e_mp2,
              double *e2d, double *e2x);

/* Library build identification (sm_100a, version). */
const char *tce_version(void);

#ifdef __cplusplus
}
#endif
#endif
