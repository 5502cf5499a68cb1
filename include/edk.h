/*
 * edk.h -- C-ABI of the B200-native Krylov engine for the ed_solver
 * exact-diagonalisation impurity solver.
 *
 * Every entry point returns an int status (EDK_OK = 0) and never exits the
 * process.  Handles are opaque; one handle is used by one host thread at a
 * time.  Vectors follow the reference layout: an (N_up, N_dn) sector vector
 * is a dim_up x dim_dn Fortran array, up index fastest
 * (rank = iup + ido*dim_up, 0-based here; the reference is 1-based,
 * quantum_fermion_sector_class.f90:256-264).  Basis states of one spin species
 * are the integers with the sector's popcount in increasing order
 * (quantum_fermion_hilbert_class.f90:385-404); bath site k is bit k and
 * impurity site c is bit nb+c (quantum_algebra_Anderson_Impurity_class.f90:73-87).
 *
 * Pointers named *_dev are device pointers on the context's device; *_host
 * are host pointers.  Nothing here takes or returns a torch type.
 */
#ifndef EDK_H
#define EDK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define EDK_OK                 0
#define EDK_ERR_INVALID        1   /* bad argument or inconsistent sizes (reference: STOP) */
#define EDK_ERR_CUDA           2   /* a CUDA runtime call failed */
#define EDK_ERR_NOMEM          3   /* device or host allocation failed */
#define EDK_KRYLOV_EXHAUSTED   4   /* |w| fell below cutoff_min_lanczos_vec: the
                                      tridiagonal was truncated (Lanczos_plain.h:85-91
                                      STOPs there; here it is a normal early end) */
#define EDK_ERR_ZERO_START     5   /* start vector of (near) zero norm */
#define EDK_ERR_CF_ZERO_DEN    6   /* zero denominator in the continued fraction
                                      (matrices_tridiag.f90:176-190) */
#define EDK_ERR_TIMEOUT        7   /* a bounded device-side wait gave up */
#define EDK_ERR_NOT_FINITE     8   /* NaN/Inf met in a Krylov coefficient or in the
                                      start vector */
#define EDK_ERR_UNSUPPORTED    9

/* ---- element types ----------------------------------------------------- */
#define EDK_F64 0   /* FP64 vectors and arithmetic (the reference's REAL(DBL) path) */
#define EDK_F32 1   /* FP32 vectors; H*v coefficients, accumulation, norms, alpha/beta in FP64 */

typedef struct edk_ctx edk_ctx;   /* device, stream, workspaces */
typedef struct edk_h edk_h;       /* one sector Hamiltonian on the device: (N_up, N_dn) or Nambu */

/* Anderson impurity model (replaces the AIM_type / JJmatrix globals read by
 * new_HAIMupdo, HAIMupdo.f90:53-121).  Matrices are row-major, spin-major:
 *   ec [2][nc][nc]  Ec_s(c,c')        eb [2][nb][nb]  Eb_s(k,k')
 *   vbc[2][nb][nc]  Vbc_s(k,c)        u  [nc][nc]     U(c,c')
 *   jj [nc][nc]     JJmatrix(c,c')    jhund           scalar gate |Jhund|>1e-5
 * cutoff_hamilt_param drops off-diagonal one-body terms with |t| <= cutoff
 * (HAIM_offdiag_arrays.f90:450,470,496). */
typedef struct edk_model {
    int32_t nc, nb;
    const double *ec, *eb, *vbc, *u, *jj;
    double jhund;
    double cutoff_hamilt_param;
} edk_model;

/* ---- context ----------------------------------------------------------- */
/* stream: a cudaStream_t (may be NULL for the legacy default stream). */
int edk_ctx_create(int device, void *stream, edk_ctx **out);
int edk_ctx_destroy(edk_ctx *ctx);
int edk_ctx_set_stream(edk_ctx *ctx, void *stream);
/* Human-readable text of the last error recorded on this context. */
const char *edk_ctx_last_error(const edk_ctx *ctx);
/* Number of kernels this library launched on the context since creation. */
int64_t edk_ctx_launch_count(const edk_ctx *ctx);
/* Per-kernel CUDA-event timing on the context's stream.  enable=1 starts
 * recording every row-kernel launch (H*v and Lanczos steps), 0 stops; the
 * report synchronises and returns, for kernel class `which` (0 = H*v,
 * 1 = first Lanczos step, 2 = fused Lanczos step, 3 = residual; add 4 for
 * FP32), the number of launches and their summed device time in ms. */
int edk_ctx_timing(edk_ctx *ctx, int enable);
/* Row-kernel selection: 0 = the fastest kernel whose preconditions hold
 * (default; the fast kernel's launch shape is timed once per sector shape
 * and element type, and the context keeps the choice for later Hamiltonians of
 * the same shape), 1 = always the generic kernel (for A/B checks), 2 or 3 = the
 * fast kernel where its preconditions hold with its default launch shape,
 * 16+i (i < 32) = the fast kernel with its i-th feasible launch shape (modulo
 * their number), for measurements. */
int edk_ctx_set_kernel_path(edk_ctx *ctx, int path);
/* 1 (default): Lanczos passes and Green chains replay pairs of fused steps as
 * one CUDA graph launch (captured once per run, from the third step on, on a
 * private stream, replayed on the context's stream); 0: plain launches.
 * Results are identical either way.  With per-launch timing on, a replay is
 * timed as a whole and counted as its two fused-step launches. */
int edk_ctx_set_graphs(edk_ctx *ctx, int enable);
int edk_ctx_timing_report(edk_ctx *ctx, int which, int64_t *launches, double *total_ms);
/* Sum over the timed launches of class `which` of the sector dimension each
 * processed (for algorithmic-byte accounting). */
int edk_ctx_timing_elements(edk_ctx *ctx, int which, double *elements);
/* Bytes the library copied host->device and device->host on this context. */
int edk_ctx_transfer_bytes(const edk_ctx *ctx, int64_t *h2d, int64_t *d2h);
/* Destroys the sector Hamiltonians edk_solve keeps on the context between
 * calls (they are reused when the same model and sector come back). */
int edk_ctx_clear_cache(edk_ctx *ctx);
/* Hands the device memory that the context's Krylov-basis pool keeps in
 * reserve (released bases, up to 5/8 of the device) back to the driver, so
 * that other allocators can use it.  The next pass that keeps its basis maps
 * memory again.  Nothing else is freed. */
int edk_ctx_trim(edk_ctx *ctx);
/* Caps the Krylov workspace (five vectors of the sector's size per element
 * type, shared by the context's passes): a pass that would need more than
 * `bytes` returns EDK_ERR_NOMEM before allocating; 0 removes the cap.  Where
 * the reference would die in an allocation, a caller with a memory budget
 * gets a status instead. */
int edk_ctx_set_workspace_limit(edk_ctx *ctx, int64_t bytes);
/* FP32 Krylov vectors of sectors with at least min_dim states: enable != 0
 * sums the up- and down-spin hop terms of H*v in FP32 (the diagonal and
 * density terms, the Lanczos recurrence and its norms stay FP64), which takes
 * most FP32 -> FP64 conversions out of the step.  Off by default; edk_solve
 * sets it for its FP32 passes from edk_solve_opts.fp32_sums. */
int edk_ctx_set_fp32_sums(edk_ctx *ctx, int enable, int64_t min_dim);

/* ---- basis (quantum_fermion_hilbert_class.f90:346-421) ----------------- */
int64_t edk_binom(int n, int k);
/* states[binom(ns,npart)] in increasing order */
int edk_basis(int ns, int npart, uint64_t *states_host);
/* rank_host[2^ns]: 0-based position of each state inside its popcount class */
int edk_rank_table(int ns, int32_t *rank_host);

/* The library's default 10001-entry start-vector table (stands in for the
 * reference's gfortran-seeded ran_tab, random.f90:684-704). Host-only. */
int edk_default_ran_tab(double *tab_host);

/* Host-only tab_HAIM2 (HAIM_offdiag_arrays.f90:210-606) for one spin species
 * and particle number: call once with NULL arrays to get *dim and *nnz, then
 * with ptr[dim+1], tgt[nnz], val[nnz], diag[dim] allocated.  Needs no GPU. */
int edk_build_table(const edk_model *m, int spin, int npart, int64_t *dim, int64_t *nnz,
                    int64_t *ptr_host, int32_t *tgt_host, double *val_host, double *diag_host);

/* ---- sector Hamiltonian: new_H / delete_H / dimen_H (H_class.f90:28-58,149-152) */
int edk_h_create(edk_ctx *ctx, const edk_model *m, int nup, int ndn, edk_h **out);
/* Destroy every Hamiltonian a caller created on a context before destroying
 * the context (the Hamiltonian synchronises on the context's stream). */
int edk_h_destroy(edk_h *h);
int edk_h_dims(const edk_h *h, int64_t *dim, int64_t *dim_up, int64_t *dim_dn);
/* The feasible launch shapes of the fast row kernels for this sector and
 * element type, in the order edk_ctx_set_kernel_path(ctx, 16 + i) selects
 * them; returns their number (or -1 on bad arguments) and writes the first
 * min(number, cap) as 5 ints each: rows per group, up-table bound, down-table
 * bound, block variant (0: 512 threads, 1: 256 x 2, 2: 128 x 4, 3: 768, 4: 640 per SM;
 * kinds 3 and 5: see below) and kernel kind (0: register-staged rows, 1 and 2:
 * rows staged by bulk copies, 3: two rows interleaved by column with packed
 * FP32x2 hop sums, FP32 hop sums only, variant 0: 256 x 2, 1: 512 x 1; 5: the
 * same arithmetic in two passes, the down-spin hops from L2-resident column
 * tiles, variant 0: two row pairs per up-pass block, 1: one, 2 to 5: four
 * rows interleaved in one buffer, 512, 640, 768 or 1024 threads; + 8: the
 * down pass on four columns per thread, 16-byte accesses).  FP32 shapes of
 * kinds 3 and 5 are listed while the context sums FP32 hops for this sector
 * (edk_ctx_set_fp32_sums). */
int edk_h_launch_shapes(const edk_h *h, int dtype, int32_t *desc, int32_t cap);
/* The launch shape the timing chose for this sector shape and element type
 * (with fp32_sums != 0: for FP32 hop sums): 1 and the 5 ints of
 * edk_h_launch_shapes in desc when one was chosen on this handle or on
 * another handle of the same sector shape in the context, 0 when none has
 * been, EDK_ERR_INVALID on bad arguments.  No counterpart in the reference
 * (a report of this library's own launch-shape tuning). */
int edk_h_launch_shape_chosen(const edk_h *h, int dtype, int fp32_sums, int32_t *desc);
/* Export one spin species' table (tab_HAIM2, HAIM_offdiag_arrays.f90:210-606)
 * as built for the device: CSR row pointer ptr[dim_s+1], 0-based target rank
 * tgt[nnz], value val[nnz], diagonal diag[dim_s].  Any pointer may be NULL;
 * *nnz receives the entry count. */
int edk_h_table(const edk_h *h, int spin, int64_t *nnz, int64_t *ptr_host,
                int32_t *tgt_host, double *val_host, double *diag_host);

/* Hmult__ (H_class.f90:69-136 -> HAIMupdo_multr, HAIMupdo.f90:677-1195):
 * y = H x on device buffers of n = dim elements.  In EDK_F64 the per-element
 * order of additions is the reference's, so results are bit-identical to a
 * sequential FP64 evaluation of HAIMupdo_multr. */
int edk_hmult(edk_h *h, int dtype, int64_t n, const void *x_dev, void *y_dev);
/* Same on host buffers: copies in, multiplies, copies out (synchronous). */
int edk_hmult_host(edk_h *h, int dtype, int64_t n, const void *x_host, void *y_host);
/* HAIMupdo_multr_split (HAIMupdo.f90:1221-1347, the matvec Hmultr calls under
 * USE_TRANSPOSE_TRICK_MPI, H_class.f90:115-119) on one GPU: the U(c,c) and
 * U(c1,c2) n1 n2 density terms (no -JJ terms, unlike edk_hmult), the
 * diagonal and the up hops; then x and the partial y are transposed, the down
 * hops are applied as up hops of the transposed arrays, and y is transposed
 * back.  Two of the context's Krylov workspace vectors hold the transposes
 * (x and y may be workspace vectors).  EDK_ERR_UNSUPPORTED where the reference
 * STOPs (|Jhund| > 1e-5) and for Nambu sectors.  FP64: bit-identical to a
 * sequential FP64 evaluation in the reference's order. */
int edk_hmult_split(edk_h *h, int dtype, int64_t n, const void *x_dev, void *y_dev);

/* ---- Lanczos (Lanczos_plain.f90:33-229, Lanczos_plain.h:66-173) --------- */
typedef struct edk_lanczos_opts {
    int32_t nitermax;            /* Nitermax; Niter = min(dim-1, nitermax) */
    int32_t neigen;              /* Neigen (<= 64) */
    double tolerance;            /* eigenvalue change for convergence */
    double demax;                /* keep eigenvalue k>1 if converged and <= E1+demax */
    double cutoff_min_lanczos_vec;  /* breakdown threshold (reference 1e-25) */
    int32_t dtype;               /* EDK_F64 or EDK_F32 */
    int32_t check_every;         /* host convergence check cadence (steps), >=1 */
    const double *ran_tab;       /* host, 10001 entries; NULL = the library's table */
    const void *start_dev;       /* optional start vector (dtype, dim); overrides ran_tab */
    int32_t use_target;          /* 1: follow the Ritz value nearest `target` instead of the
                                    lowest ones (refinement restart of an excited state) */
    double target;
    double residual_tol;         /* > 0: also require the Ritz residual beta_{k+1}|y_k| below
                                    this (an eigenvector criterion; the reference stops on the
                                    eigenvalue change alone) */
    int32_t keep_basis;          /* != 0 in pass 1: it writes its Krylov vectors into device memory
                                    kept on the Hamiltonian (as far as free memory allows, leaving
                                    1/16 of the device and at least 4 GB; pass 1 then runs without
                                    graph replay).  The memory comes from a pool owned by the
                                    context, which keeps released chunks (up to 5/8 of the device)
                                    for the next pass and returns them when the context is
                                    destroyed.  != 0 in pass 2 with the same start_dev and
                                    ran_tab pointers: psi is formed from the kept vectors in one
                                    pass instead of recomputing the recurrence (which it does when
                                    none are kept or too few); 1 releases them afterwards, 2 keeps
                                    them for another eigenvector of the same chain.  The next pass
                                    1 and edk_h_destroy release them too.  0: pass 2 recomputes
                                    (the reference's way).  edk_solve sets it unless
                                    edk_solve_opts.recompute_pass2 is set.  The start buffer (or
                                    the ran_tab array) must hold the same values in pass 2 as in
                                    pass 1: pass 2 compares the norm of start_dev and a sum of
                                    ran_tab with pass 1's and recomputes when they differ, which
                                    catches most but not all changes. */
} edk_lanczos_opts;

typedef struct edk_lanczos_result {
    int32_t nkept;               /* eigenvalues kept (>=1) */
    int32_t niter;               /* Lanczos iterations of pass 1 */
    int32_t status;              /* EDK_OK or EDK_KRYLOV_EXHAUSTED */
    double E[64];
    int32_t converged[64];
    double *diag;                /* host, capacity >= nitermax+1: alpha_k */
    double *subdiag;             /* host, capacity >= nitermax+1: subdiag[0]=|v0|, [k]=beta_{k+1} */
    double *vecp;                /* host, capacity >= neigen*(nitermax+1): column j = coefficients of E[j] */
} edk_lanczos_result;

/* Pass 1: eigenvalues and tridiagonal eigenvector coefficients. */
int edk_lanczos_e0(edk_h *h, const edk_lanczos_opts *o, edk_lanczos_result *r);
/* Pass 2 (Lanczos_get_GS_sector): psi = normalised sum_k coef[k] v_k, rebuilt
 * from the same start vector; psi_dev has dtype o->dtype and dim elements. */
int edk_lanczos_gs(edk_h *h, const edk_lanczos_opts *o, int32_t niter, const double *coef_host,
                   void *psi_dev);

/* ---- c / c+ (apply_Cupdo, apply_C.f90:497-653; Cup_sector/Cdo_sector :79-109)
 * src: the sector of in_dev; out_dev receives c[+]_{site,spin} in in the
 * target sector (N_spin +/- 1), fully overwritten.  site is the 0-based
 * impurity site, spin 0 = up, 1 = down.  with_site2 >= 0 adds
 * sign2 * c[+]_{site2,spin} (the symmetric combination of
 * green_class_compute_symmetric_combination.f90:39-138 with sign2 = +1). */
int edk_apply_c(edk_h *src, int dtype, int site, int spin, int dagger, int site2, int sign2,
                const void *in_dev, void *out_dev, int64_t *out_dim);

/* ---- dynamic correlation (compute_dynamic_cpu, green_class_compute_dynamic.f90:191-334)
 * target: Hamiltonian of the sector start_dev lives in.  Runs exactly
 * min(nitergreen, dim) steps from start/|start| (stops early only on
 * breakdown), then dyn(w) = |start|^2 <0|(i wn - ph*(T-e0))^-1|0> with ph=+1
 * (iph=1, particle) or -1 (iph=2, hole).  G_host is interleaved re/im,
 * length 2*nw.  diag/subdiag (host, capacity nitergreen+1) may be NULL. */
int edk_green_chain(edk_h *target, int dtype, const void *start_dev, int32_t nitergreen,
                    double e0, int iph, int32_t nw, const double *wn_host,
                    double cutoff_dynamic, double *G_host, double *diag_host,
                    double *subdiag_host, int32_t *niter_done);

/* invert_zmtridiag (matrices_tridiag.f90:163-198) for nchain tridiagonals of
 * n[c] levels each (diag/subdiag packed with stride ld) at nw frequencies,
 * scaled by scale[c] and the shift/sign of compute_dynamic:
 * G[c][w] = scale[c] * <0|(i wn[w] - ph[c]*(T_c - e[c]))^-1|0>.  Device-side. */
int edk_cf_eval(edk_ctx *ctx, int32_t nchain, int32_t ld, const int32_t *n_host,
                const double *diag_host, const double *subdiag_host, const double *e_host,
                const double *ph_host, const double *scale_host, int32_t nw,
                const double *wn_host, double *G_host);

/* The continued fractions of edk_cf_eval (same arguments, same results and
 * status codes) without any device allocation; it has no counterpart in the
 * reference.  For callers that cannot allocate device memory at that point:
 * code whose device memory is held by another allocator (a framework's caching
 * allocator, or Krylov workspaces sized to fill HBM), where cudaMalloc would
 * fail or cudaFree would stall the device.  Its device memory is one static
 * array of EDK_NOALLOC_SCRATCH_BYTES per device, cut per call into 256-byte
 * aligned regions (flag, n, diag, subdiag, e, ph, scale, wn, G); a call whose
 * regions exceed it returns EDK_ERR_INVALID with the byte counts in the error
 * text.  The first call on a device resolves the array's address
 * (cudaGetSymbolAddress, that device current); make it before any stream
 * capture.  All calls on a device share the array and clear its flag first:
 * calls whose GPU work overlaps race.  The call runs with the context's device
 * current and puts the caller's current device back before it returns. */
#define EDK_NOALLOC_SCRATCH_BYTES 4194304
int edk_cf_eval_noalloc(edk_ctx *ctx, int32_t nchain, int32_t ld, const int32_t *n_host,
                        const double *diag_host, const double *subdiag_host, const double *e_host,
                        const double *ph_host, const double *scale_host, int32_t nw,
                        const double *wn_host, double *G_host);

/* ---- observables --------------------------------------------------------
 * <psi| n_{site,up} n_{site,dn} |psi> (the double occupancy of
 * correlations_write.h:93-95) and |psi|^2 in one pass. */
int edk_double_occ(edk_h *h, int dtype, const void *psi_dev, int site, double *docc, double *norm2);
/* |H psi - e psi| and |psi| with the FP64 matvec (psi in FP64). */
int edk_residual(edk_h *h, const void *psi_dev, double e, double *res_norm, double *psi_norm);

/* ---- block Lanczos (Block_Lanczos_diagonalize, Block_Lanczos.f90:37-355) ----
 * The reference drives BLZPACK (not part of its sources) with H applied to a
 * block of NVOPU vectors (Block_Lanczos.f90:222-246).  This is a plain block
 * Lanczos of block size p: V_1 = QR of p periodic start vectors
 * (tab[(i + 977 c) % 10000 + 1] for column c), then
 *   W = H V_j - V_{j-1} B_j^T - V_j A_j  (A_j = V_j^T H V_j, orthogonalised twice),
 *   W = V_{j+1} B_{j+1} (modified Gram-Schmidt),
 * with the lowest eigenvalues of the block tridiagonal checked every
 * check_every block steps until each of the neigen lowest changes by less
 * than tolerance.  Eigenvectors, when vecs_dev is given (neigen x dim FP64,
 * vector e at e*dim), come from a second pass of the same recurrence.  FP64. */
typedef struct edk_block_opts {
    int32_t block;               /* block size p, 1..4 */
    int32_t nitermax;            /* block steps */
    int32_t neigen;              /* lowest eigenpairs (<= 64) */
    double tolerance;            /* eigenvalue change for convergence */
    int32_t check_every;         /* block steps between checks */
    const double *ran_tab;       /* 10001-entry start table (host), NULL = library table */
} edk_block_opts;
int edk_block_lanczos(edk_h *h, const edk_block_opts *opts, double *E_host, void *vecs_dev, int32_t *niter,
                      int32_t *converged);

/* ---- batched Green chains ------------------------------------------------
 * Many compute_dynamic chains (green_class_compute_dynamic.f90:191-334) at
 * once, as compute_greenAA issues them for every sector, particle/hole part,
 * eigenstate and orbital combination (green_class_computeAA.f90:105-126).
 * mode 0: one persistent launch over a work queue (largest chains first, one
 * thread block per chain, launch shape autotuned once per problem class and
 * cached on the context); mode 1: one grid per Lanczos step, chain after chain.
 * G_out[out][w] (interleaved re/im, nout x nw) accumulates weight * dyn. */
typedef struct edk_chain {
    edk_h *target;               /* Hamiltonian of the sector start_dev lives in */
    const void *start_dev;       /* start vector, batch dtype, target dimension */
    double e0;                   /* energy of the state the vector came from */
    int32_t iph;                 /* 1 = particle, 2 = hole */
    double weight;               /* e.g. the Boltzmann weight */
    int32_t out;                 /* output slot */
} edk_chain;

typedef struct edk_batch_stats {
    int64_t steps;               /* Lanczos steps run over all chains */
    int32_t chains;
    double kernel_ms;            /* device time of the persistent launch */
    int32_t block, rows, blocks_per_sm, tuned_shapes;
} edk_batch_stats;

int edk_green_batch(edk_ctx *ctx, int dtype, int32_t nchain, const edk_chain *chains, int32_t nitergreen,
                    int32_t nw, const double *wn_host, double cutoff_dynamic, int32_t nout, double *G_out,
                    int32_t mode, edk_batch_stats *stats);

/* Element-type conversion of a device vector (FP32 <-> FP64, or a copy). */
int edk_convert(edk_ctx *ctx, int from_dtype, int to_dtype, int64_t n, const void *in_dev, void *out_dev);

/* ---- adjoint: parameter gradients ------------------------------------------
 * The reference has no derivatives; these entry points differentiate its
 * quantities with respect to the model parameters of edk_model.  H is linear
 * in every parameter, so dH/dtheta is a fixed operator:
 *   EDK_PARAM_EC  (i,j): Ec(i,j) and Ec(j,i) together -- n_c (i=j) or the
 *                 impurity hop c+_i c_j + c+_j c_i (HAIM_offdiag_arrays.f90:419-464)
 *   EDK_PARAM_EB  (i,j): the same for Eb (bath levels and bath-bath hops, :469-486)
 *   EDK_PARAM_VBC (k,c): Vbc(k,c), both hop directions bath k <-> impurity c (:497-524)
 *   EDK_PARAM_U   (i,j): U(i,i): n_i,up n_i,dn; U(i,j), i<j: n_i n_j (HAIMupdo.f90:784-829)
 * spin: 0 = the up-spin entry only, 1 = down only, 2 = both spins' entries
 * (a spin-symmetric parameter); ignored for EDK_PARAM_U.  At most 64
 * parameters per call.  All vectors are FP64 device vectors of h's sector. */
#define EDK_PARAM_EC   0
#define EDK_PARAM_EB   1
#define EDK_PARAM_VBC  2
#define EDK_PARAM_U    3
typedef struct edk_param {
    int32_t kind, i, j, spin;
} edk_param;

/* out_host[q] = <a| dH/dtheta_q |b> for every parameter, one pass. */
int edk_dh_bilinear(edk_h *h, const void *a_dev, const void *b_dev, int32_t np, const edk_param *params,
                    double *out_host);
/* Hellmann-Feynman: dE/dtheta_q = <psi| dH/dtheta_q |psi> / <psi|psi>. */
int edk_grad_e0(edk_h *h, const void *psi_dev, int32_t np, const edk_param *params, double *grad_host);

/* One Green-function channel of an eigenstate: the compute_dynamic chain of
 * (c[+]_{site,spin} + sign2 c[+]_{site2,spin})|psi> (site2 < 0: single
 * operator), dagger = 1 particle part (iph = 1), 0 hole part (iph = 2). */
typedef struct edk_green_spec {
    int32_t site, spin, dagger, site2, sign2;
} edk_green_spec;
typedef struct edk_grad_stats {
    int64_t forward_steps, replay_steps, reverse_steps;
    int32_t cg_iterations;
    double cg_residual;
    int32_t stored_vectors;      /* FP64 vectors of the largest chain's checkpoints + segment */
} edk_grad_stats;
/* Vector-Jacobian product of the Green functions G_c(i wn) (the dyn of
 * edk_green_chain, nitergreen steps from |psi> normalised) and of E0 for the
 * eigenstate psi (FP64, energy e0) of h's sector:
 *   grad_q = sum_c sum_w Re(conj(gbar[c][w]) dG_c(i wn_w)/dtheta_q) + e0bar dE0/dtheta_q.
 * gbar_host: nchain x nw interleaved re/im (torch's complex-gradient
 * convention: dL/dRe G + i dL/dIm G).  The chain part is reverse mode through
 * the Lanczos recurrence with checkpointed replay; the eigenvector part solves
 * (H - E0) lambda = (1 - |psi><psi|) psibar by conjugate gradients to relative
 * residual cg_tol (psi must be a converged, non-degenerate ground state).
 * G_host (optional, nchain x nw interleaved) receives the forward G; stats may
 * be NULL.  Everything is FP64. */
int edk_grad_green(edk_h *h, const void *psi_dev, double e0, int32_t nchain, const edk_green_spec *chains,
                   int32_t nitergreen, int32_t nw, const double *wn_host, const double *gbar_host, double e0bar,
                   int32_t np, const edk_param *params, double cg_tol, double *grad_host, double *G_host,
                   edk_grad_stats *stats);

/* ---- solver driver -------------------------------------------------------
 * One solve of the impurity problem for the (N_up, N_dn) basis: the sector
 * scan and ground states of get_eigen_energies/get_GS (solver.h:11-237), the
 * Boltzmann window (eigen_class.f90:322-450), double occupancies
 * (correlations_write.h:93-95) and the (c, c+) Green functions of
 * compute_greenAA (green_class_computeAA.f90:40-185) for the requested
 * impurity orbital pairs and spins.  All inputs and outputs are host buffers;
 * vectors live on the device only.  dtype EDK_F32 = mixed precision: in
 * sectors of at least 2^20 states, FP32 Krylov vectors (H*v, alpha and beta
 * still computed in FP64), FP32 passes refined by one FP64 Lanczos restart per
 * state, FP64 residual check, FP64 continued fractions; smaller sectors, whose
 * kernels are latency-bound, run in FP64. */
typedef struct edk_solve_opts {
    int32_t dtype;
    int32_t nsectors;
    const int32_t *sectors;      /* 2*nsectors: (nup, ndn) scanned for eigenstates */
    int32_t neigen;              /* Neigen per sector */
    int32_t nitermax;            /* Nitermax */
    double tolerance;            /* eigenvalue tolerance (FP64 passes) */
    double tolerance_lowprec;    /* eigenvalue tolerance of the FP32 pass (mixed) */
    int32_t check_every;         /* Lanczos convergence check cadence */
    double beta;
    double demax0;               /* window dEmax = demax0/beta (dmft_ed_solver.f90:1468) */
    int32_t nitergreen;          /* Nitergreenmax */
    int32_t nw;                  /* fermionic Matsubara points i(2n-1)pi/beta */
    int32_t spin_mask;           /* bit 0: G of spin up, bit 1: spin down */
    int32_t npairs;
    const int32_t *pairs;        /* 2*npairs impurity orbital pairs (i,j) */
    double cutoff_dynamic;       /* skip |A psi|^2 below this (reference 1e-8) */
    const double *ran_tab;       /* start-vector table, NULL = library table */
    double residual_tol;         /* > 0: eigenvector criterion of the FP64 passes (see
                                    edk_lanczos_opts); mixed precision always refines to it */
    int32_t green_mode;          /* 0: the chains of target sectors below 2^20 states (FP64)
                                    run together in one persistent edk_green_batch launch per
                                    spin; 1: every chain on its own (edk_green_chain) */
    const char *gs_in;           /* NULL, or a GS.raw file (edk_gs_write): its eigenstates replace
                                    the sector scan, as solve_AIM does on its first call with an
                                    old GS (solver.f90:70-81, solver_init.h:163-182) */
    const char *gs_out;          /* NULL, or the path the eigenstates of the window are written to
                                    in GS.raw form (solver.f90:104-108) */
    const char *sector_bound_file;  /* NULL, or an ed.sector_bound_file: when it exists, only
                                    sectors with nup, ndn within the bounds +/- iwindow are scanned
                                    (solver.h:107-137), and the bounds of the states found are
                                    written back to it (get_new_bounds, solver.h:374-415) */
    int32_t iwindow;             /* window around the bounds (reference default 1) */
    int32_t recompute_pass2;     /* 0: each Lanczos pass 1 keeps its Krylov vectors on the device
                                    (edk_lanczos_opts.keep_basis) and pass 2 forms the eigenvector
                                    from them; 1: pass 2 reruns the recurrence (the reference's
                                    Lanczos_get_GS_sector) */
    int32_t reference_small_sectors;  /* 1: Green functions into target sectors of at most 40
                                    states (FULL_ED_SWITCH) take the reference's Lehmann branch
                                    (compute_dynamic_full_ed, green_class_compute_dynamic.f90:44-62,
                                    77-165): a sum over the eigenstates of that sector kept in the
                                    Boltzmann window, 0 when none is kept.  0: the continued
                                    fraction of min(nitergreen, dim) steps, exact for the sector */
    int64_t lowprec_min_dim;     /* mixed precision: sectors of at least this many states run
                                    FP32 Krylov vectors; 0 means 2^20 */
    int32_t fp32_sums;           /* mixed precision: 1 sums the hop terms of H*v in FP32 in the
                                    FP32 passes of sectors of at least 2^20 states
                                    (edk_ctx_set_fp32_sums); 0 keeps every sum in FP64 */
    int32_t batch_gs;            /* != 0: the ground states of the FP64 sectors of 41 to
                                    (batch_gs == 1 ? 2^14 : batch_gs) states (rows of at most
                                    12288 states; neigen <= 3; residual_tol 0) run batched: pass 1 of every such sector in one persistent
                                    launch over a work queue (one block per sector, the
                                    convergence test run on the device every check_every steps:
                                    the lowest neigen eigenvalues of T_n against those of T_{n-1},
                                    so a sector may take up to check_every-1 more steps than on
                                    its own), pass 2 of their kept states in a second one.
                                    0: every sector on its own (edk_lanczos_e0/gs) */
} edk_solve_opts;

typedef struct edk_solve_result {
    double e0, z;
    double e0_lowprec;           /* mixed: lowest FP32 eigenvalue before refinement */
    double residual;             /* |H psi0 - E0 psi0| / |psi0| with the FP64 matvec */
    int32_t nstates;             /* eigenstates in the Boltzmann window */
    int32_t lanczos_steps;       /* Lanczos steps of the eigen part as the reference counts them
                                    (pass 2 included, also when it is formed from kept vectors) */
    int32_t green_steps;         /* H*v applications of the Green part */
    double *G;                   /* host [2][npairs][nw][2] (spin, pair, w, re/im) or NULL */
    double *docc;                /* host [nc] or NULL */
    double *energies;            /* host [64] or NULL */
    int32_t *state_sectors;      /* host [128] or NULL */
} edk_solve_result;

int edk_solve(edk_ctx *ctx, const edk_model *m, const edk_solve_opts *o, edk_solve_result *r);

/* ---- eigenstate checkpoints: GS.raw (eigen_sector_class.f90:514-567) ------
 * The list-directed text file of write_raw_eigensectorlist: per sector a
 * T record, the sector ('updo' then norbs and npart of each spin species,
 * quantum_fermion_sector_class.f90:398-403; or 'sz' then norbs and npart,
 * quantum_fermion_hilbert_class.f90:190-195) and its eigenlist (per state:
 * T, the eigenvalue, the converged flag, the rank, the vector length and the
 * vector, eigen_class.f90:479-491, rcvector_class.f90:217-229, closed by F);
 * a final F.  The reader accepts any list-directed layout of those values
 * (line breaks inside the vector, commas, r*c repeat counts, .TRUE./.FALSE.,
 * quoted or bare sector names), as a Fortran READ(UNIT,*) does; each record
 * of the reference's starts on a new line.  Host-only. */
typedef struct edk_gs_entry {
    int32_t kind;                /* 0: (N_up, N_dn) sector, 1: Nambu (sz) sector */
    int32_t norbs;               /* orbitals per spin species (kind 0) or Nambu orbitals (kind 1) */
    int32_t nup, ndn;            /* kind 0: particle numbers; kind 1: nup = npart, ndn = -1 */
    double val;                  /* eigenvalue */
    int32_t converged;
    int32_t rank;
    int64_t n;                   /* vector length */
    int64_t offset;              /* first element of the vector in the vector pool */
} edk_gs_entry;
/* Entries of the same sector must be consecutive: each run is one eigensector. */
int edk_gs_write(const char *path, int32_t nentries, const edk_gs_entry *entries, const double *vec_pool_host);
/* Call with entries = NULL and vec_pool = NULL to get *nentries and
 * *vec_total, then with capacities at least those; offsets are assigned in
 * file order. */
int edk_gs_read(const char *path, int32_t cap, edk_gs_entry *entries, int32_t *nentries, int64_t vec_cap,
                double *vec_pool_host, int64_t *vec_total);
/* ed.sector_bound_file (solver.h:107-119, 396-402): bounds[6] = nupmin, nupmax,
 * ndnmin, ndnmax, szmin, szmax.  Reading a file without the third record
 * leaves szmin = 1000, szmax = -1000 and sets *has_sz = 0.  Host-only. */
int edk_sector_bounds_read(const char *path, int32_t *bounds, int32_t *has_sz);
int edk_sector_bounds_write(const char *path, const int32_t *bounds);

/* ---- Nambu (Sz) sectors: HAIMsz (HAIMsz.f90:51-1027) ----------------------
 * The superconducting basis of new_HAIMsz: one species of 2*ns orbitals, up
 * orbitals on bits 0..ns-1 (bath k -> bit k, impurity c -> bit nb+c) and the
 * particle-hole transformed down orbitals on bits ns..2ns-1 (a set bit is an
 * empty down orbital).  The sector of npart Nambu particles holds the states
 * of popcount npart (N_up + ns - N_dn = npart) in increasing order; vectors
 * have binom(2ns, npart) elements.  The Nambu matrices are those of
 * Nambu_Ec / Nambu_Eb / Nambu_Vbc (impurity_class.f90:1018-1037,
 * bath_class.f90:956-1022): [Ec_up, 0; 0, -Ec_dn^T], [Eb_up, Pb; Pb^T, -Eb_dn^T],
 * [Vbc_up, PVbc_2; PVbc_1, -Vbc_dn].  Physical energies are the Nambu
 * eigenvalues plus energy_shift = sum_c Ec_dn(c,c) + sum_k Eb_dn(k,k)
 * (eigen_sector_class.f90:329).  Requires ns <= 16, |jhund| <= 1e-5 (the
 * reference STOPs otherwise, HAIMsz.f90:470-473). */
typedef struct edk_model_sz {
    edk_model base;              /* normal part (jj unused) */
    const double *pb;            /* [nb][nb] bath pairing Pb(k,k'); NULL = none */
    const double *pvbc;          /* [2][nb][nc] impurity-to-bath pairing PVbc_s(k,c) of
                                    PAIRING_IMP_TO_BATH; NULL = off */
    int32_t on_fly;              /* 0: term order of the tabulated HAIMsz_multr (HAIMsz.f90:453-589),
                                    off-diagonal terms with |t| <= cutoff dropped; 1: order of
                                    HAIMsz_mult_fly_r (HAIMsz.f90:615-808), every non-zero term */
} edk_model_sz;

/* new_H for a Nambu sector.  The handle works with edk_hmult(_host),
 * edk_lanczos_e0/gs, edk_green_chain, edk_residual and edk_block_lanczos
 * like an (N_up, N_dn) one; edk_h_dims reports dim_up = dim, dim_dn = 1.
 * In EDK_F64, H*v adds per element in the reference's order of the selected
 * variant, bit-identical to a sequential FP64 evaluation. */
int edk_h_create_sz(edk_ctx *ctx, const edk_model_sz *m, int npart, edk_h **out);
/* npart (-1 for an (N_up, N_dn) sector) and energy_shift (0 there). */
int edk_h_sz_info(const edk_h *h, int32_t *npart, double *energy_shift);
/* apply_Csz_updo / apply_Csz_N_updo (apply_C.f90:344-483): physical
 * c[+]_{site,spin} on a Nambu vector.  Spin 0 creates (dagger = 1) or
 * destroys on the up orbital; spin 1 acts on the hole orbital with c and c+
 * exchanged (c+_dn empties the hole).  projected = 1 (apply_Csz_N_updo) keeps
 * only source states whose other spin on the site is occupied.  apply_Csz
 * (:273-333) on Nambu orbital iorb is site iorb, spin 0 for iorb < nc, and
 * site iorb-nc, spin 1, dagger flipped for iorb >= nc.  site2 >= 0 adds
 * sign2 * the same operator on site2.  out_dev (same dtype, fully
 * overwritten) lives in the sector npart +/- 1: binom(2ns, npart +/- 1)
 * elements, returned in out_dim; its Hamiltonian is edk_h_create_sz with
 * the returned *out_npart. */
/* The start vector of symmetric_combineAB (green_class_compute_symmetric_combination.f90:155-262)
 * for the A/B Green functions of the Nambu basis, e.g. GNF with A = the
 * projected c of apply_Csz_N_updo and B = c (correlations_dyn_stat.h:96):
 * out = A_site |in> + B_site2 |in>, with A and B each the operator of
 * edk_apply_csz on that site (same spin and dagger) and `proj`/`proj2`
 * selecting apply_Csz_N_updo for it; site2 may equal site.  The reference
 * reaches this channel only in the Nambu basis: its n c operator stops in
 * the (N_up, N_dn) basis (apply_C.f90:135-148). */
int edk_apply_csz_ab(edk_h *src, int dtype, int site, int proj, int site2, int proj2, int spin, int dagger,
                     const void *in_dev, void *out_dev, int64_t *out_dim, int32_t *out_npart);
int edk_apply_csz(edk_h *src, int dtype, int site, int spin, int dagger, int projected, int site2, int sign2,
                  const void *in_dev, void *out_dev, int64_t *out_dim, int32_t *out_npart);
/* apply_Csz (apply_C.f90:273-333) on Nambu impurity orbitals: b+_orb
 * (dagger = 1) or b_orb, orb in [0, 2nc) (orb < nc: the up orbital of site
 * orb; orb >= nc: the hole orbital of site orb - nc), plus sign2 times the
 * same operator on orb2 when orb2 >= 0 (the symmetric combinations of
 * green_class_compute_symmetric_combination.f90:39-138 in the Nambu basis,
 * e.g. b+_up + b+_hole for the anomalous part).  Target sector npart +/- 1. */
int edk_apply_cnambu(edk_h *src, int dtype, int orb, int dagger, int orb2, int sign2, const void *in_dev,
                     void *out_dev, int64_t *out_dim, int32_t *out_npart);

/* ED_diago (ED_ARPACK.f90:590-715): every eigenpair of a sector by dense
 * diagonalisation of the FP64 matrix that H*v gives on the unit vectors
 * (cyclic Jacobi on the host).  E_host[dim] ascending; V_host (may be NULL)
 * dim x dim row-major, column j = the eigenvector of E_host[j].  Sectors of
 * at most 4096 states, either basis. */
int edk_full_ed(edk_h *h, double *E_host, double *V_host);

/* ---- local two-particle vertex chi~_loc (Chiloc_Wenhu_version3.cpp:29-989) ----
 * chi_tilde_loc_ for many frequency triples at once: for each eigenstate i of
 * the sector (nup, ndn) (energies E[0]), the Lehmann sum over the eigenstates
 * j, k, l of its neighbour sectors of the Phi coefficients times four c+
 * matrix elements, weighted by exp(-beta (E_i - gs_e)) / Z.  Sector slots:
 *   0 i (nup,ndn)   1 pup (nup+1,ndn)   2 pdn (nup,ndn+1)   3 mup (nup-1,ndn)
 *   4 mdn (nup,ndn-1)   5 p2dn (nup,ndn+2)   6 m2dn (nup,ndn-2)
 *   7 puppdn (nup+1,ndn+1)   8 muppdn (nup-1,ndn+1)   9 pupmdn (nup+1,ndn-1)
 *   10 mupmdn (nup-1,ndn-1)
 * (dimension 0 for a sector outside the Hilbert space).  Matrix slots
 * (<target| c+ |source>, row-major target x source, the reference's cp_*
 * arrays):
 *   0 i_cdup (pup<-i)  1 i_cddn (pdn<-i)  2 pup_cddn (puppdn<-pup)
 *   3 pdn_cdup (puppdn<-pdn)  4 pdn_cddn (p2dn<-pdn)  5 mup_cdup (i<-mup)
 *   6 mup_cddn (muppdn<-mup)  7 mdn_cddn (i<-mdn)  8 mdn_cdup (pupmdn<-mdn)
 *   9 muppdn_cdup (pdn<-muppdn)  10 pupmdn_cddn (pup<-pupmdn)
 *   11 mupmdn_cdup (mdn<-mupmdn)  12 mupmdn_cddn (mup<-mupmdn)  13 m2dn_cddn (mdn<-m2dn)
 * w_host: nf x 6 doubles (re, im of w1, w2, w3).  op_mask bit 0: DNDN into
 * pdndn_host, bit 1: UPDN into pupdn_host (nf x 2 doubles each).  phi_eps is
 * the PHI_EPS threshold of the vanishing-denominator branches.  All arrays
 * are host arrays. */
typedef struct edk_chiloc_sectors {
    int32_t dim[11];
    const double *E[11];
    const double *C[14];
} edk_chiloc_sectors;
int edk_chiloc(edk_ctx *ctx, int32_t op_mask, double beta, double Z, double gs_e, double phi_eps, int32_t sites,
               int32_t nup, int32_t ndn, const edk_chiloc_sectors *s, int32_t nf, const double *w_host,
               double *pdndn_host, double *pupdn_host);
/* Process-wide kernel choice of edk_chiloc: 0 (default) = the kernel that
 * computes the one-index parts of the Phi coefficients once per block (when
 * they fit in 96 KB of shared memory), 1 = the per-element kernel, for A/B
 * checks. */
int edk_chiloc_set_kernel(int plain);

#ifdef __cplusplus
}
#endif
#endif /* EDK_H */
