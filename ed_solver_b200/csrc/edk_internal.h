// Internal structures shared by the host orchestration (edk_host.cpp) and the
// device kernels (edk_kernels.cu).  Not part of the public C-ABI.
#pragma once

#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/edk.h"

namespace edk {

constexpr int kMaxNc = 6;        // impurity sites per spin species
constexpr int kMaxNs = 30;       // orbitals per spin species
constexpr int kMaxSmemBytes = 220 * 1024;

// One spin species' table on the device (tab_HAIM2 output, HAIM_offdiag_arrays.f90:210-606).
struct SpinTabDev {
    const int32_t *ptr = nullptr;    // dim+1 CSR offsets
    const int32_t *tgt = nullptr;    // nnz, 0-based target rank
    const double *val = nullptr;     // nnz
    const double *diag = nullptr;    // dim
    const uint8_t *imp = nullptr;    // dim: occupation bits of the impurity sites
    const int32_t *move = nullptr;   // dim * nmove: (rank+1)*sign of moving one
                                     // electron between impurity sites, 0 if none
    // Column-major padded copy of the same table (entry k of state c at
    // k*dim + c), used for the up-spin gathers: packed = 24-bit target rank |
    // 8-bit palette index, or plain int32 target + value when the table has
    // more than 256 distinct values.  Padding entries point at the state
    // itself with value 0 (palette slot 0 holds +0.0).
    int ell_k = 0;
    int packed = 0;
    int npal = 0;
    const uint32_t *ell = nullptr;
    const double *ell_val = nullptr;
    const double *pal = nullptr;      // npal <= 256
    // Copy for the lean FP32 kernel (kind 3): the lean_ks entries of
    // column c contiguous at c*lean_ks + k (lean_ks = ell_k rounded up to an
    // even count), each (target << 14) | (palette index << 3) (padding: the
    // column itself, palette slot 0); lean_kw[j] = the largest hop count of
    // columns [64j, 64j + 64).  Null when the table is not packed, dim is odd
    // or at least 2^18.
    int lean_ks = 0;
    const uint32_t *lean = nullptr;
    const uint8_t *lean_kw = nullptr;
    // The same entries blocked by 64 columns, entry-major inside a block:
    // entry k of column c at (c/64)*64*lean_ks + k*64 + c%64, so entry k of a
    // warp's 64 columns is one contiguous 256-byte load (the two-pass step).
    const uint32_t *lean_b = nullptr;
};

// Everything a row kernel needs to evaluate (H x) for an element.
struct HamDev {
    int64_t dup = 0, ddn = 0;
    int nc = 0, nmove = 0;
    int hund = 0;                      // spin flip / pair hopping active
    int ncfg = 0;                      // 1 << nc
    int dn_kmax = 0;                   // longest down-table row
    SpinTabDev up, dn;
    const int32_t *int_off = nullptr;  // ncfg*ncfg+1 offsets into the coefficient lists
    const double *int_coef = nullptr;  // per (cfg_up, cfg_dn): the ordered density terms
    const double *jj = nullptr;        // nc*nc (device)
    const uint8_t *umask = nullptr;    // nc*nc
    const int32_t *row_order = nullptr;  // ddn: schedule of rows for L2 reuse
};

enum RowMode : int {
    kModeHv = 0,       // y = H x
    kModeFirst = 1,    // Lanczos step 1: w = H v1, sums for alpha_1, beta_2
    kModeStep = 2,     // Lanczos step k+1 from s_{k+1} = w_k (see edk_kernels.cu)
    kModeResid = 3,    // sums |Hx - e x|^2, |x|^2
};

// Arguments of the fused row kernel (raw pointers, element type erased).
struct RowArgs {
    int mode = kModeHv;
    const void *x = nullptr;       // gather source (x / v1 / s_{k+1})
    void *y = nullptr;             // H x, w, or s_{k+2}
    const void *vk = nullptr;      // v_k (step)
    const void *vkm1 = nullptr;    // v_{k-1} (step; may be null)
    void *vout = nullptr;          // v_{k+1} (step; may alias vkm1)
    void *psi = nullptr;           // pass-2 accumulator (may be null)
    const double *psi_coef = nullptr;  // device, coefficient of v_{k+1} at psi_coef[k]
    double *tri_diag = nullptr;    // device alpha array (Dagotto layout, 0-based alpha_{k+1} at [k])
    double *tri_sub = nullptr;     // device beta array (tri_sub[k] = beta_{k+1})
    int k = 0;                     // 1-based step index of v_k
    int *kdev = nullptr;           // when set (step mode), the index is read from here and the
                                   // last block advances it: consecutive steps replayable as a graph
    double gamma1 = 0.0;           // shift of the first stored vector s_2 = H v_1 - gamma1 v_1
    double eshift = 0.0;           // residual mode: e
    double cutoff = 1e-25;
    double *partials = nullptr;    // gridDim*4 doubles
    unsigned *counter = nullptr;   // last-block counter
    double *sums_out = nullptr;    // 4 doubles: final sums (deterministic order)
    int *flags = nullptr;          // [0] breakdown step (0 = none), [1] non-finite (1) or timeout (2)
    int sum32 = 0;                 // FP32 vectors: hop terms summed in FP32 (bulk-copy kernels)
    void *scratch = nullptr;       // kind 5: an FP32 vector of the sector's dimension (partial sums)
};

// Launch shape of the fast row kernel: rows per group, up/down table-width
// bounds, and block shape (variant 0: 512 threads, one block per SM;
// variant 1: 256 threads, two blocks per SM; variant 2: 128 threads, four
// blocks per SM, offered for rows of at most 4096 states; two columns per
// thread in all).
// One column per thread (24 resident warps instead of 16) was measured at
// ns=16 and never beat these two, so it is not instantiated.
// kind 0: the fast row kernel (edk_rows_fast.cuh); kinds 1 and 2: the same
// mathematics with rows staged by bulk copies (edk_rows_tma.cuh): 1 = one
// column per thread with the next column's loads in flight (any alignment,
// odd rows), 2 = two columns per thread.  Kinds 0 and 2 read column pairs and
// need vectors aligned to twice the element size and even rows.  Block
// variants: 0 = 512 threads x 1 block per SM, 1 = 256 x 2, 2 = 128 x 4,
// 3 = 768 x 1 and 4 = 640 x 1 (kind 2).
// kind 3: the lean FP32 kernel (edk_rows_lean.cuh), FP32 vectors with FP32
// hop sums only; kmu is its table width lean_ks; variants 0 = 256 x 2
// and 1 = 512 x 1; kind 5: the same arithmetic in two passes, the down-spin
// hops from L2-resident column tiles (edk_rows_tiled.cuh), with an FP32
// scratch vector (RowArgs::scratch); variant 0 stages two row pairs per
// up-pass block, 1 one pair.  Both need aligned column pairs.
inline bool shape_needs_pairs(int kind) { return kind == 0 || kind == 2 || kind == 3 || kind == 5; }
struct FastShape {
    int r = 0, kmu = 0, kmd = 0, variant = 0, kind = 0;
};

struct LaunchCfg {
    int grid = 0, block = 0, rows = 1, km = 0, num_sms = 1;
    int64_t groups = 0;
    size_t smem = 0;
    bool stage = true;
    bool fast = false;       // use row_fast_kernel (edk_rows_fast.cuh)
    FastShape fast_shape;    // its launch shape
};


// One Green chain of a batch (edk_batch.cu).
struct BatchItem {
    int32_t ham;             // index into the HamDev array
    int32_t niter;           // min(nitergreen, dim)
    int64_t dim;
    const void *start;       // start vector (batch element type)
    double gamma1;           // shift of the first stored vector (the state energy)
    double cutoff_dynamic;
    double *alpha;           // niter
    double *beta;            // niter + 1: beta[0] = |start|, beta[k] couples k-1,k
    int32_t *done;           // steps completed (0 if |start|^2 < cutoff_dynamic)
};
cudaError_t launch_batch(int dtype, int R, const HamDev *hams, const BatchItem *items, int nitems, int *queue,
                         void *work, int64_t maxdim, int64_t maxdup, double cutoff, int grid, int block,
                         cudaStream_t st);
int batch_max_blocks_per_sm(int dtype, int R, int block, int64_t maxdup);

// The ground state of one small FP64 sector in a batched launch (edk_batch.cu).
// Pass 1: up to niter_max Lanczos steps from the table start vector with the
// per-sector driver's convergence test on the lowest ne eigenvalues every
// `every` steps; writes alpha[0..n), beta[0..n] and result = {n, status}
// (status 1: Krylov space exhausted, 2: zero start).  Pass 2: niter_max = n
// steps again, forming the ne normalised states psi + j*dim from the
// tridiagonal eigenvector coefficients coef[j*niter_max + q].
constexpr int kGsMaxNe = 3;
struct GsItem {
    int32_t ham;
    int32_t niter_max;
    int64_t dim;
    int32_t ne;
    int32_t pad = 0;
    double tolerance;
    double *alpha;
    double *beta;
    int32_t *result;
    void *const *psi;      // pass 2: device array of ne state pointers
    const double *coef;
};
// One sector's outcome of the batched ground states (gs_batch, edk_host.cpp).
struct GsBatchSector {
    int niter = 0, status = 0, nkept = 0;
    double E[kGsMaxNe] = {0, 0, 0};
    int converged[kGsMaxNe] = {0, 0, 0};
    void *psi[kGsMaxNe] = {nullptr, nullptr, nullptr};   // cudaMalloc'd FP64 states, owned by the caller
};
// Ground states of nsec small FP64 sectors: pass 1 of all of them in one
// persistent launch, the host's eigenpairs of each tridiagonal (the window
// and kept states of edk_lanczos_e0), pass 2 in a second launch.
int gs_batch(edk_ctx *c, int nsec, edk_h *const *hs, int nitermax, int neigen, double tolerance, double demax,
             const double *ran_tab, int every, GsBatchSector *out);
cudaError_t launch_gs_batch(int R, const HamDev *hams, const GsItem *items, int nitems, int *queue, void *work,
                            int64_t maxdim, int64_t maxdup, int nmax, const double *tab, double cutoff, int every,
                            int pass, int grid, cudaStream_t st);

// ---- Nambu (Sz) sectors (edk_sz.cpp, edk_sz.cu) ----------------------------
// A Nambu state is 2*ns bits: low half l = up orbitals, high half h = down
// holes.  The states of popcount npart in increasing order group into rows
// of equal h (ascending); inside a row the low halves of popcount
// npart - |h| run in increasing order, so rank = off_h[h] + rank_low[l].
constexpr int kMaxSzNs = 16;
constexpr int kMaxSzTerms = 4096;

// One off-diagonal term c+_tgt c_src in the reference's visiting order.
struct SzTerm {
    uint32_t src, tgt;     // single-bit masks
    uint32_t btw;          // orbitals strictly between: their parity is the Jordan-Wigner sign
    uint32_t pad;
    double h;
};

// A maximal run of consecutive terms of one kind: 0 = both orbitals in the
// low half (up-up), 1 = both in the high half (hole-hole), 2 = one in each
// (pairing).  Up-up runs carry a table over the low halves: for low-half
// position p (low_states order) entry k at ell[ell_off + k*2^ns + p] is the
// k-th active term's target rank_low (16 bits) | sign (bit 16) | index in the
// run (bits 17..31), or 0xFFFFFFFF after the last.
struct SzRun {
    int32_t kind, first, count, kell;
    int64_t ell_off;
};

struct SzSectorDev {
    int npart = 0, nrows = 0, maxlen = 0;
    int64_t dim = 0;
    const uint32_t *row_h = nullptr;   // nrows high halves present in the sector, ascending
    const uint32_t *off_h = nullptr;   // 2^ns: rank of the first state of high half h
};

struct SzDev {
    int ns = 0, nb = 0, nc = 0;
    int order = 0;                          // 0: HAIMsz_multr, 1: HAIMsz_mult_fly_r
    SzSectorDev sec;
    const uint16_t *rank_low = nullptr;     // 2^ns: rank of l among the low halves of its popcount
    const uint16_t *low_states = nullptr;   // 2^ns low halves grouped by popcount, ascending
    const int32_t *class_start = nullptr;   // ns+2: start of popcount class k in low_states
    int nterm = 0;
    const SzTerm *terms = nullptr;
    int ndiag = 0;                          // Nambu orbitals in the order of the diagonal sum
    const uint32_t *diag_bit = nullptr;
    const double *diag_e = nullptr;
    const double *quart = nullptr;          // 4^nc: QUART_INT_SZ by impurity configuration
                                            // (up bits | hole bits << nc)
    int nrun = 0;
    const SzRun *runs = nullptr;
    const int32_t *term_run = nullptr;      // nterm: run of each term
    const uint32_t *ell = nullptr;          // the up-up runs' tables
};

struct SzHost;   // host tables and device copies of one Nambu sector (edk_sz.cpp)
int sz_create(const edk_model_sz *m, int npart, cudaStream_t st, SzHost **out, std::string *err);
void sz_destroy(SzHost *z);
const SzDev &sz_dev(const SzHost *z);
double sz_shift(const SzHost *z);
int64_t sz_upload_bytes(const SzHost *z);
// Row tables of the sector npart (another sector of the same model), cached
// on z; used for the targets of c and c+.
int sz_sector(SzHost *z, int npart, cudaStream_t st, const SzSectorDev **out, std::string *err);

// simple = 1: every state walks the whole term list (for A/B checks); 0: the
// per-row compacted lists with the own row staged where it fits.
cudaError_t launch_sz_rows(const SzDev &S, int dtype, const RowArgs &a, int num_sms, int simple, cudaStream_t st);
// out[t] over the target sector = sum over the (one or two) operators of
// sign * in[source(t)]; operator o: bit[o] toggled, create[o] (the target has
// the bit), source states with (s & pmask[o]) == pwant[o] only, sgn[o] = +-1.
struct SzOp {
    uint32_t bit = 0, pmask = 0, pwant = 0;
    int create = 0, sgn = 1;
};
cudaError_t launch_sz_apply_c(int dtype, const SzDev &src, const SzSectorDev &tgt, int nop, const SzOp *ops,
                              const void *in, void *out, int num_sms, cudaStream_t st);

// HAIMupdo_multr_split (edk_split.cu): y = H x through two transposes; xt, yt
// are scratch vectors of the sector's dimension; soff/scoef the split form's
// density terms per impurity-configuration pair (no -JJ terms).
cudaError_t launch_split_hv(const HamDev &H, int dtype, const int32_t *soff, const double *scoef, const void *x,
                            void *y, void *xt, void *yt, int num_sms, cudaStream_t st);

// ---- kernel launchers (edk_kernels.cu) ------------------------------------
LaunchCfg plan_rows(const HamDev &H, int elem_bytes, int num_sms);
cudaError_t launch_rows(const HamDev &H, int dtype, const RowArgs &a, const LaunchCfg &cfg,
                        cudaStream_t st);
bool fast_rows_ok(const HamDev &H, int elem_bytes);
// The feasible launch shapes of the fast kernel for H (the first is the default).
// sum32: FP32 vectors with FP32 hop sums, which adds the lean kernel's shapes.
int fast_shapes(const HamDev &H, int elem_bytes, int num_sms, FastShape *out, int cap, int sum32 = 0);
cudaError_t launch_rows_fast(const HamDev &H, int dtype, const RowArgs &a, int num_sms, const FastShape &s,
                             cudaStream_t st);
cudaError_t launch_set_int(int *p, int v, cudaStream_t st);
cudaError_t launch_start_vector(int dtype, int64_t n, const double *ran_tab_dev,
                                const void *user_start, void *v, double *partials,
                                unsigned *counter, double *sums_out, int grid, cudaStream_t st);
cudaError_t launch_scale(int dtype, int64_t n, void *v, const double *sums, int which,
                         void *psi, const double *psi_coef, double *tri_sub0, int grid,
                         cudaStream_t st);
cudaError_t launch_norm2(int dtype, int64_t n, const void *v, double *partials, unsigned *counter,
                         double *sums_out, int grid, cudaStream_t st);
// psi = sum_q coef[q] v_q over nv stored vectors (vecs_dev: device array of pointers)
cudaError_t launch_combine(int dtype, int64_t n, const void *const *vecs_dev, const double *coef_dev, int nv,
                           void *psi, int grid, cudaStream_t st);
cudaError_t launch_convert(int from_dtype, int to_dtype, int64_t n, const void *in, void *out,
                           cudaStream_t st);
cudaError_t launch_apply_c(int dtype, int spin, int64_t dother, int64_t dup_src, int64_t dup_tgt,
                           int64_t dim_sigma_tgt, const int32_t *src1, const int8_t *sg1,
                           const int32_t *src2, const int8_t *sg2, int sign2, const void *in, void *out,
                           cudaStream_t st);
cudaError_t launch_cf(int nchain, int ld, const int32_t *n, const double *diag,
                      const double *sub, const double *e, const double *ph,
                      const double *scale, int nw, const double *wn, double *G, int *flag,
                      cudaStream_t st);
cudaError_t launch_double_occ(int dtype, const HamDev &H, int site_bit_mask_up, int site_bit_mask_dn,
                              const void *psi, double *partials, unsigned *counter,
                              double *sums_out, int grid, cudaStream_t st);

}  // namespace edk
