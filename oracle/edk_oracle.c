/*
 * edk_oracle.c -- CPU restatement of the ed_solver Krylov hot path (FP64).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of bench.py call it.  Nothing in the
 * product library links or calls it.
 *
 * Parity status: the reference is Fortran 90 and cannot be compiled in this
 * environment (no Fortran compiler), so this restatement is pinned by
 *   (1) the reference's own golden output test/2b/bm/g_bm (two-orbital AIM,
 *       beta=50), reproduced through the Python drivers in oracle.py;
 *   (2) analytic limits (U=0 resolvent, V=0 atomic limit) and dense
 *       numpy eigh / Lehmann sums on small sectors.
 * The gfortran random_number table that seeds the reference's Lanczos start
 * vector is not reproducible here, so the exact (alpha_k, beta_k) sequence of
 * the reference is not pinned; converged quantities are.
 *
 * Every routine cites the reference file:line it follows (paths relative to
 * the reference project root).  Floating point: compiled with
 * -ffp-contract=off so that every "a = a + h*x" is a separate multiply and add,
 * the same rounding sequence the reference's Fortran performs per element.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <complex.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAXNC 8

/* ------------------------------------------------------------------------- */
/* combinatorics and basis (quantum_fermion_hilbert_class.f90:346-421)        */
/* ------------------------------------------------------------------------- */

int64_t orc_binom(int n, int k)
{
    if (k < 0 || k > n) return 0;
    int64_t r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

/* States of `ns` orbitals with popcount `np`, in increasing integer order:
 * the order in which new_fermion_Hilbert_space (quantum_fermion_hilbert_class.f90:385-404)
 * fills sector(npart)%state while scanning state = 0 .. 2**norbs-1. */
int64_t orc_basis(int ns, int np, uint64_t *states)
{
    int64_t n = 0;
    uint64_t top = 1ull << ns;
    for (uint64_t s = 0; s < top; ++s)
        if (__builtin_popcountll(s) == np) states[n++] = s;
    return n;
}

/* rank[s] = position (0-based) of s inside its popcount class; the reference
 * stores the same number 1-based in Hilbert%rank (quantum_fermion_hilbert_class.f90:402). */
void orc_rank_table(int ns, int32_t *rank)
{
    int32_t cnt[65];
    memset(cnt, 0, sizeof cnt);
    uint64_t top = 1ull << ns;
    for (uint64_t s = 0; s < top; ++s) rank[s] = cnt[__builtin_popcountll(s)]++;
}

/* ------------------------------------------------------------------------- */
/* ket algebra (quantum_fermion_ket_class.f90:483-618)                        */
/* ------------------------------------------------------------------------- */

/* Fermion_sign (:605-618): multiply by (-1) for every occupied orbital above
 * the 0-based bit `b`, evaluated on the ket AFTER the operator acted. */
static inline int above_parity(uint64_t s, int b)
{
    return (__builtin_popcountll(s >> (b + 1)) & 1) ? -1 : 1;
}

/* destroy (:573-594); returns 0 when the result is nil */
static inline int ket_destroy(uint64_t s, int b, uint64_t *out, int *sign)
{
    if (!((s >> b) & 1ull)) return 0;
    s &= ~(1ull << b);
    *sign *= above_parity(s, b);
    *out = s;
    return 1;
}

/* create (:545-563) */
static inline int ket_create(uint64_t s, int b, uint64_t *out, int *sign)
{
    if ((s >> b) & 1ull) return 0;
    s |= (1ull << b);
    *sign *= above_parity(s, b);
    *out = s;
    return 1;
}

/* hop(ket_out, tgt, src, ket_in) (:483-492): destroy src, then create tgt */
static inline int ket_hop(uint64_t s, int tgt, int src, uint64_t *out, int *sign)
{
    uint64_t t;
    *sign = 1;
    if (!ket_destroy(s, src, &t, sign)) return 0;
    return ket_create(t, tgt, out, sign);
}

/* ------------------------------------------------------------------------- */
/* model                                                                     */
/* ------------------------------------------------------------------------- */

/* Anderson impurity model, one (N_up,N_dn) basis.  Bit layout per spin species
 * (quantum_algebra_Anderson_Impurity_class.f90:73-87): bath site k -> bit k,
 * impurity site c -> bit nb+c.  Matrices are row-major, spin-major:
 *   ec [s][c][c'] = Ec_s(c,c')        (impurity quadratic)
 *   eb [s][k][k'] = Eb_s(k,k')        (bath quadratic)
 *   vbc[s][k][c]  = Vbc_s(k,c)        (bath-impurity hybridisation)
 *   u  [c][c']    = U(c,c')           (density-density, HAIMupdo.f90:784-829)
 *   jj [c][c']    = JJmatrix(c,c')    (Hund, HAIMupdo.f90:813-818,1017-1129)
 * jhund is the scalar gate |Jhund|>1e-5 of HAIMupdo.f90:1017,1087. */
typedef struct {
    int32_t nc, nb;
    const double *ec, *eb, *vbc, *u, *jj;
    double jhund;
    double cutoff;   /* cutoff_hamilt_param: drops |off-diagonal| <= cutoff */
} orc_model;

/* ------------------------------------------------------------------------- */
/* hopping tables: tab_HAIM2 (HAIM_offdiag_arrays.f90:210-606)                */
/* ------------------------------------------------------------------------- */

/* Visit the off-diagonal targets of one basis state in the reference's order:
 * impurity-impurity (:448-464), bath-bath (:469-486), hybridisation with
 * impurity->bath then bath->impurity for each (bath,imp) pair (:490-526).
 * Returns the number of entries; fills tgt_state/val when non-NULL. */
static int visit_offdiag(const orc_model *m, int spin, uint64_t s,
                         uint64_t *tgt_state, double *val)
{
    const int nc = m->nc, nb = m->nb;
    const double *ec = m->ec + (size_t)spin * nc * nc;
    const double *eb = m->eb + (size_t)spin * nb * nb;
    const double *vb = m->vbc + (size_t)spin * nb * nc;
    int n = 0;
    uint64_t out;
    int sg;
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
            double h = ec[i * nc + j];
            if (i == j || h == 0.0 || !(fabs(h) > m->cutoff)) continue;
            if (ket_hop(s, nb + i, nb + j, &out, &sg)) {
                if (tgt_state) { tgt_state[n] = out; val[n] = h * (double)sg; }
                ++n;
            }
        }
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) {
            double h = eb[i * nb + j];
            if (i == j || h == 0.0 || !(fabs(h) > m->cutoff)) continue;
            if (ket_hop(s, i, j, &out, &sg)) {
                if (tgt_state) { tgt_state[n] = out; val[n] = h * (double)sg; }
                ++n;
            }
        }
    for (int k = 0; k < nb; ++k)
        for (int c = 0; c < nc; ++c) {
            double h = vb[k * nc + c];
            if (h == 0.0 || !(fabs(h) > m->cutoff)) continue;
            if (ket_hop(s, k, nb + c, &out, &sg)) {          /* impurity -> bath */
                if (tgt_state) { tgt_state[n] = out; val[n] = h * (double)sg; }
                ++n;
            }
            if (ket_hop(s, nb + c, k, &out, &sg)) {          /* bath -> impurity */
                if (tgt_state) { tgt_state[n] = out; val[n] = h * (double)sg; }
                ++n;
            }
        }
    return n;
}

/* diag(istate) = sum of occupied impurity Ec(c,c) then occupied bath Eb(k,k)
 * (HAIM_offdiag_arrays.f90:419-427), accumulated in that order. */
static double diag_energy(const orc_model *m, int spin, uint64_t s)
{
    const int nc = m->nc, nb = m->nb;
    const double *ec = m->ec + (size_t)spin * nc * nc;
    const double *eb = m->eb + (size_t)spin * nb * nb;
    double d = 0.0;
    for (int c = 0; c < nc; ++c)
        if ((s >> (nb + c)) & 1ull) d = d + ec[c * nc + c];
    for (int k = 0; k < nb; ++k)
        if ((s >> k) & 1ull) d = d + eb[k * nb + k];
    return d;
}

/* Count pass (new_HAIM2 with NO_STORAGE, HAIM_offdiag_arrays.f90:89-148). */
int64_t orc_table_count(const orc_model *m, int spin, int np, int32_t *noff)
{
    int ns = m->nc + m->nb;
    int64_t dim = orc_binom(ns, np);
    uint64_t *st = (uint64_t *)malloc(sizeof(uint64_t) * (dim > 0 ? dim : 1));
    orc_basis(ns, np, st);
    int64_t tot = 0;
    for (int64_t i = 0; i < dim; ++i) {
        noff[i] = visit_offdiag(m, spin, st[i], NULL, NULL);
        tot += noff[i];
    }
    free(st);
    return tot;
}

/* Fill pass: CSR row pointer ptr[dim+1], 0-based target rank, value, diag. */
void orc_table_fill(const orc_model *m, int spin, int np, int64_t *ptr,
                    int32_t *tgt, double *val, double *diag)
{
    int ns = m->nc + m->nb;
    int64_t dim = orc_binom(ns, np);
    uint64_t *st = (uint64_t *)malloc(sizeof(uint64_t) * (dim > 0 ? dim : 1));
    int32_t *rank = (int32_t *)malloc(sizeof(int32_t) * ((size_t)1 << ns));
    orc_basis(ns, np, st);
    orc_rank_table(ns, rank);
    uint64_t ts[4 * 64 * ORC_MAXNC + 64 * 64];
    double tv[4 * 64 * ORC_MAXNC + 64 * 64];
    ptr[0] = 0;
    for (int64_t i = 0; i < dim; ++i) {
        int n = visit_offdiag(m, spin, st[i], ts, tv);
        for (int e = 0; e < n; ++e) {
            tgt[ptr[i] + e] = rank[ts[e]];
            val[ptr[i] + e] = tv[e];
        }
        ptr[i + 1] = ptr[i] + n;
        diag[i] = diag_energy(m, spin, st[i]);
    }
    free(rank);
    free(st);
}

/* ------------------------------------------------------------------------- */
/* sector Hamiltonian: new_HAIMupdo (HAIMupdo.f90:53-121)                     */
/* ------------------------------------------------------------------------- */

typedef struct {
    int64_t dim;
    uint64_t *st;
    int64_t *ptr;
    int32_t *tgt;
    double *val, *diag;
} orc_spin_table;

typedef struct orc_h {
    int nc, nb, ns, nup, ndn;
    int64_t dup, ddn, dim;
    orc_spin_table t[2];
    int32_t *rank;                 /* 2**ns */
    double u[ORC_MAXNC * ORC_MAXNC], jj[ORC_MAXNC * ORC_MAXNC];
    int umask[ORC_MAXNC * ORC_MAXNC];
    int offdiag_coulomb, hund;
    double jhund;
    struct orc_sz *sz;             /* Nambu sector (HAIMsz) when non-NULL */
} orc_h;

static void build_spin(const orc_model *m, int spin, int np, orc_spin_table *t)
{
    int ns = m->nc + m->nb;
    t->dim = orc_binom(ns, np);
    size_t d = (size_t)(t->dim > 0 ? t->dim : 1);
    int32_t *noff = (int32_t *)malloc(sizeof(int32_t) * d);
    int64_t nnz = orc_table_count(m, spin, np, noff);
    free(noff);
    t->st = (uint64_t *)malloc(sizeof(uint64_t) * d);
    orc_basis(ns, np, t->st);
    t->ptr = (int64_t *)malloc(sizeof(int64_t) * (d + 1));
    t->tgt = (int32_t *)malloc(sizeof(int32_t) * (nnz > 0 ? nnz : 1));
    t->val = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    t->diag = (double *)malloc(sizeof(double) * d);
    orc_table_fill(m, spin, np, t->ptr, t->tgt, t->val, t->diag);
}

orc_h *orc_h_new(const orc_model *m, int nup, int ndn)
{
    if (m->nc < 1 || m->nc > ORC_MAXNC || m->nb < 0 || m->nc + m->nb > 30) return NULL;
    orc_h *h = (orc_h *)calloc(1, sizeof(orc_h));
    h->nc = m->nc; h->nb = m->nb; h->ns = m->nc + m->nb;
    h->nup = nup; h->ndn = ndn;
    build_spin(m, 0, nup, &h->t[0]);
    build_spin(m, 1, ndn, &h->t[1]);
    h->dup = h->t[0].dim; h->ddn = h->t[1].dim; h->dim = h->dup * h->ddn;
    h->rank = (int32_t *)malloc(sizeof(int32_t) * ((size_t)1 << h->ns));
    orc_rank_table(h->ns, h->rank);
    int nc = m->nc;
    h->offdiag_coulomb = 0;
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
            h->u[i * nc + j] = m->u[i * nc + j];
            h->jj[i * nc + j] = m->jj[i * nc + j];
            h->umask[i * nc + j] = (m->u[i * nc + j] != 0.0);
            if (i != j && h->umask[i * nc + j]) h->offdiag_coulomb = 1;   /* :119 */
        }
    h->jhund = m->jhund;
    h->hund = (fabs(m->jhund) > 1e-5) && h->offdiag_coulomb;
    return h;
}

static void orc_sz_free(struct orc_sz *z);

void orc_h_free(orc_h *h)
{
    if (!h) return;
    if (h->sz) orc_sz_free(h->sz);
    for (int s = 0; s < 2; ++s) {
        free(h->t[s].st); free(h->t[s].ptr); free(h->t[s].tgt);
        free(h->t[s].val); free(h->t[s].diag);
    }
    free(h->rank);
    free(h);
}

int64_t orc_h_dim(const orc_h *h) { return h->dim; }
int64_t orc_h_dup(const orc_h *h) { return h->dup; }
int64_t orc_h_ddn(const orc_h *h) { return h->ddn; }

/* Export one spin table (for bit-exact comparison with the device builder). */
int64_t orc_h_table(const orc_h *h, int spin, uint64_t *st, int64_t *ptr,
                    int32_t *tgt, double *val, double *diag)
{
    const orc_spin_table *t = &h->t[spin];
    int64_t nnz = t->ptr[t->dim];
    if (st) memcpy(st, t->st, sizeof(uint64_t) * t->dim);
    if (ptr) memcpy(ptr, t->ptr, sizeof(int64_t) * (t->dim + 1));
    if (tgt) memcpy(tgt, t->tgt, sizeof(int32_t) * nnz);
    if (val) memcpy(val, t->val, sizeof(double) * nnz);
    if (diag) memcpy(diag, t->diag, sizeof(double) * t->dim);
    return nnz;
}

/* ------------------------------------------------------------------------- */
/* H*v: HAIMupdo_multr (HAIMupdo.f90:677-1195), real FP64, USE_CC gather      */
/* ------------------------------------------------------------------------- */

static inline int bt(uint64_t s, int b) { return (int)((s >> b) & 1ull); }

/* parity of occupied bits strictly between bits a and b (exclusive) */
static inline int between_sign(uint64_t s, int a, int b)
{
    int lo = a < b ? a : b, hi = a < b ? b : a;
    if (hi - lo <= 1) return 1;
    uint64_t mask = ((1ull << hi) - 1ull) & ~((1ull << (lo + 1)) - 1ull);
    return (__builtin_popcountll(s & mask) & 1) ? -1 : 1;
}

static void orc_sz_hmult(const struct orc_sz *z, const double *x, double *y);

void orc_hmult(const orc_h *h, const double *x, double *y)
{
    if (h->sz) { orc_sz_hmult(h->sz, x, y); return; }
    const int nc = h->nc, nb = h->nb;
    const int64_t sec = h->dup, ddn = h->ddn;
    const orc_spin_table *tu = &h->t[0], *td = &h->t[1];
    memset(y, 0, sizeof(double) * (size_t)h->dim);

    /* U(c,c) n_c,up n_c,dn  (:784-796) */
#pragma omp parallel for schedule(static)
    for (int64_t iup = 0; iup < sec; ++iup)
        for (int c = 0; c < nc; ++c) {
            if (!(h->umask[c * nc + c] && bt(tu->st[iup], nb + c))) continue;
            for (int64_t ido = 0; ido < ddn; ++ido)
                if (bt(td->st[ido], nb + c)) {
                    int64_t i = iup + ido * sec;
                    y[i] = y[i] + h->u[c * nc + c] * x[i];
                }
        }

    /* U(c1,c2) n_c1 n_c2 and -JJ for same-spin pairs (:798-829, Jhund_Slater_type) */
    if (h->offdiag_coulomb) {
#pragma omp parallel for schedule(static)
        for (int64_t iup = 0; iup < sec; ++iup)
            for (int64_t ido = 0; ido < ddn; ++ido)
                for (int s1 = 0; s1 < nc - 1; ++s1) {
                    int b1u = bt(tu->st[iup], nb + s1), b1d = bt(td->st[ido], nb + s1);
                    int n1 = b1u + b1d;
                    if (n1 == 0) continue;
                    for (int s2 = s1 + 1; s2 < nc; ++s2) {
                        if (!h->umask[s1 * nc + s2]) continue;
                        int b2u = bt(tu->st[iup], nb + s2), b2d = bt(td->st[ido], nb + s2);
                        int n2 = b2u + b2d;
                        if (n2 == 0) continue;
                        int64_t i = iup + ido * sec;
                        y[i] = y[i] + h->u[s1 * nc + s2] * (double)n1 * (double)n2 * x[i];
                        if (b1u && b2u) y[i] = y[i] - h->jj[s1 * nc + s2] * x[i];
                        if (b1d && b2d) y[i] = y[i] - h->jj[s1 * nc + s2] * x[i];
                    }
                }
    }

    /* (diagup + diagdo) * x  (:841-848) */
#pragma omp parallel for schedule(static)
    for (int64_t iup = 0; iup < sec; ++iup)
        for (int64_t ido = 0; ido < ddn; ++ido) {
            int64_t i = iup + ido * sec;
            y[i] = y[i] + (tu->diag[iup] + td->diag[ido]) * x[i];
        }

    /* up hopping, stride dim_up over ido (:865-881) */
#pragma omp parallel for schedule(static)
    for (int64_t iup = 0; iup < sec; ++iup)
        for (int64_t e = tu->ptr[iup]; e < tu->ptr[iup + 1]; ++e) {
            double hv = tu->val[e];
            int64_t jup = tu->tgt[e];
            for (int64_t ido = 0; ido < ddn; ++ido) {
                int64_t i = iup + ido * sec;
                y[i] = y[i] + hv * x[jup + ido * sec];
            }
        }

    /* down hopping, contiguous over iup (:883-900) */
#pragma omp parallel for schedule(static)
    for (int64_t ido = 0; ido < ddn; ++ido)
        for (int64_t e = td->ptr[ido]; e < td->ptr[ido + 1]; ++e) {
            double hv = td->val[e];
            int64_t jdo = td->tgt[e];
            for (int64_t iup = 0; iup < sec; ++iup) {
                int64_t i = iup + ido * sec;
                y[i] = y[i] + hv * x[iup + jdo * sec];
            }
        }

    if (!h->hund) return;

    /* Hund spin flip (:1017-1085) */
#pragma omp parallel for schedule(static)
    for (int64_t iup = 0; iup < sec; ++iup)
        for (int64_t ido = 0; ido < ddn; ++ido) {
            uint64_t su = tu->st[iup], sd = td->st[ido];
            int64_t i = iup + ido * sec;
            for (int s1 = 0; s1 < nc; ++s1) {
                int b1u = bt(su, nb + s1), b1d = bt(sd, nb + s1);
                if (b1u + b1d != 1) continue;
                for (int s2 = s1 + 1; s2 < nc; ++s2) {
                    if (!h->umask[s1 * nc + s2]) continue;
                    int b2u = bt(su, nb + s2), b2d = bt(sd, nb + s2);
                    if (b2u + b2d != 1) continue;
                    int p1 = nb + s1, p2 = nb + s2;
                    if (b1u && b2d) {
                        uint64_t uo = (su & ~(1ull << p1)) | (1ull << p2);
                        uint64_t dq = (sd & ~(1ull << p2)) | (1ull << p1);
                        int sg = between_sign(uo, p1, p2) * between_sign(dq, p2, p1);
                        int64_t j = h->rank[uo] + (int64_t)h->rank[dq] * sec;
                        y[i] = y[i] + x[j] * h->jj[s1 * nc + s2] * (double)sg;
                    }
                    if (b1d && b2u) {
                        uint64_t uo = (su & ~(1ull << p2)) | (1ull << p1);
                        uint64_t dq = (sd & ~(1ull << p1)) | (1ull << p2);
                        int sg = between_sign(uo, p2, p1) * between_sign(dq, p1, p2);
                        int64_t j = h->rank[uo] + (int64_t)h->rank[dq] * sec;
                        y[i] = y[i] + x[j] * h->jj[s1 * nc + s2] * (double)sg;
                    }
                }
            }
        }

    /* Hund pair hopping (:1087-1129) */
#pragma omp parallel for schedule(static)
    for (int64_t iup = 0; iup < sec; ++iup)
        for (int64_t ido = 0; ido < ddn; ++ido) {
            uint64_t su = tu->st[iup], sd = td->st[ido];
            int64_t i = iup + ido * sec;
            for (int s1 = 0; s1 < nc; ++s1) {
                if (!(bt(su, nb + s1) && bt(sd, nb + s1))) continue;
                for (int s2 = 0; s2 < nc; ++s2) {
                    if (s2 == s1 || !h->umask[s1 * nc + s2]) continue;
                    if (bt(su, nb + s2) || bt(sd, nb + s2)) continue;
                    int p1 = nb + s1, p2 = nb + s2;
                    uint64_t uo = (su & ~(1ull << p1)) | (1ull << p2);
                    uint64_t dq = (sd & ~(1ull << p1)) | (1ull << p2);
                    int sg = between_sign(uo, p1, p2) * between_sign(dq, p1, p2);
                    int64_t j = h->rank[uo] + (int64_t)h->rank[dq] * sec;
                    y[i] = y[i] + x[j] * h->jj[s1 * nc + s2] * (double)sg;
                }
            }
        }
}

/* Out-of-place transpose of an nrow x ncol array stored with the column index
 * fastest (a[c + r*ncol]) into b[r + c*nrow] (distributed_memory_transpose_mat
 * of one process, HAIMupdo.f90:1305-1306). */
static void transpose_mat(const double *a, double *b, int64_t ncol, int64_t nrow)
{
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < nrow; ++r)
        for (int64_t c = 0; c < ncol; ++c) b[r + c * nrow] = a[c + r * ncol];
}

/* HAIMupdo_multr_split (HAIMupdo.f90:1221-1347) on one process: U(c,c) terms,
 * U(c1,c2) n1 n2 terms (no -JJ terms, unlike HAIMupdo_multr), the diagonal,
 * the up hops; then both vectors transposed, the down hops applied as up hops
 * of the transposed array, and both transposed back.  Returns -1 where the
 * reference STOPs (|Jhund| > 1e-5, :1243-1246), 0 otherwise. */
int orc_hmult_split(const orc_h *h, const double *x, double *y)
{
    if (h->sz || fabs(h->jhund) > 1e-5) return -1;
    const int nc = h->nc, nb = h->nb;
    const int64_t sec = h->dup, ddn = h->ddn, n = h->dim;
    const orc_spin_table *tu = &h->t[0], *td = &h->t[1];
    memset(y, 0, sizeof(double) * (size_t)n);
    /* :1250-1261 */
#pragma omp parallel for schedule(static)
    for (int64_t iup = 0; iup < sec; ++iup)
        for (int c = 0; c < nc; ++c) {
            if (!(h->umask[c * nc + c] && bt(tu->st[iup], nb + c))) continue;
            for (int64_t ido = 0; ido < ddn; ++ido)
                if (bt(td->st[ido], nb + c)) {
                    int64_t i = iup + ido * sec;
                    y[i] = y[i] + h->u[c * nc + c] * x[i];
                }
        }
    /* :1263-1284 */
    if (h->offdiag_coulomb) {
#pragma omp parallel for schedule(static)
        for (int64_t iup = 0; iup < sec; ++iup)
            for (int64_t ido = 0; ido < ddn; ++ido)
                for (int s1 = 0; s1 < nc - 1; ++s1) {
                    int n1 = bt(tu->st[iup], nb + s1) + bt(td->st[ido], nb + s1);
                    if (n1 == 0) continue;
                    for (int s2 = s1 + 1; s2 < nc; ++s2) {
                        if (!h->umask[s1 * nc + s2]) continue;
                        int n2 = bt(tu->st[iup], nb + s2) + bt(td->st[ido], nb + s2);
                        if (n2 == 0) continue;
                        int64_t i = iup + ido * sec;
                        y[i] = y[i] + h->u[s1 * nc + s2] * (double)n1 * (double)n2 * x[i];
                    }
                }
    }
    /* :1286-1292 */
#pragma omp parallel for schedule(static)
    for (int64_t iup = 0; iup < sec; ++iup)
        for (int64_t ido = 0; ido < ddn; ++ido) {
            int64_t i = iup + ido * sec;
            y[i] = y[i] + (tu->diag[iup] + td->diag[ido]) * x[i];
        }
    /* :1294-1311 */
#pragma omp parallel for schedule(static)
    for (int64_t iup = 0; iup < sec; ++iup)
        for (int64_t e = tu->ptr[iup]; e < tu->ptr[iup + 1]; ++e) {
            double hv = tu->val[e];
            int64_t jup = tu->tgt[e];
            for (int64_t ido = 0; ido < ddn; ++ido) y[iup + ido * sec] = y[iup + ido * sec] + hv * x[jup + ido * sec];
        }
    /* :1313-1314, then the down hops of the transposed arrays (:1316-1334) */
    double *xt = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double *yt = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    transpose_mat(x, xt, sec, ddn);
    transpose_mat(y, yt, sec, ddn);
#pragma omp parallel for schedule(static)
    for (int64_t ido = 0; ido < ddn; ++ido)
        for (int64_t e = td->ptr[ido]; e < td->ptr[ido + 1]; ++e) {
            double hv = td->val[e];
            int64_t jdo = td->tgt[e];
            for (int64_t iup = 0; iup < sec; ++iup) yt[ido + iup * ddn] = yt[ido + iup * ddn] + hv * xt[jdo + iup * ddn];
        }
    /* :1336-1337 */
    transpose_mat(yt, y, ddn, sec);
    free(xt);
    free(yt);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* symmetric tridiagonal eigensolver (stands in for LAPACK DSTEDC,            */
/* matrices_tridiag.f90:210-259): implicit QL with Wilkinson shifts.          */
/* d[n] diagonal, e[n-1] off-diagonal; w[n] ascending eigenvalues; z (n*n,    */
/* column-major, column j = eigenvector j) when non-NULL.                     */
/* ------------------------------------------------------------------------- */

int orc_tridiag_eig(int n, const double *d_in, const double *e_in, double *w, double *z)
{
    if (n <= 0) return 0;
    double *d = (double *)malloc(sizeof(double) * n);
    double *e = (double *)calloc((size_t)n, sizeof(double));
    memcpy(d, d_in, sizeof(double) * n);
    for (int i = 0; i + 1 < n; ++i) e[i] = e_in[i];
    if (z) {
        memset(z, 0, sizeof(double) * (size_t)n * n);
        for (int i = 0; i < n; ++i) z[(size_t)i * n + i] = 1.0;
    }
    int status = 0;
    for (int l = 0; l < n; ++l) {
        int iter = 0, m;
        for (;;) {
            for (m = l; m < n - 1; ++m) {
                double dd = fabs(d[m]) + fabs(d[m + 1]);
                if (fabs(e[m]) <= 2.2e-16 * dd) break;
            }
            if (m == l) break;
            if (++iter > 60) { status = 1; break; }
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = hypot(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
            double s = 1.0, c = 1.0, p = 0.0;
            int i;
            for (i = m - 1; i >= l; --i) {
                double f = s * e[i], b = c * e[i];
                r = hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) { d[i + 1] -= p; e[m] = 0.0; break; }
                s = f / r; c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                if (z)
                    for (int k = 0; k < n; ++k) {
                        double t = z[(size_t)(i + 1) * n + k];
                        z[(size_t)(i + 1) * n + k] = s * z[(size_t)i * n + k] + c * t;
                        z[(size_t)i * n + k] = c * z[(size_t)i * n + k] - s * t;
                    }
            }
            if (r == 0.0 && i >= l) continue;
            d[l] -= p; e[l] = g; e[m] = 0.0;
        }
    }
    /* sort ascending (selection sort, moves eigenvectors along) */
    for (int i = 0; i < n - 1; ++i) {
        int k = i;
        for (int j = i + 1; j < n; ++j) if (d[j] < d[k]) k = j;
        if (k != i) {
            double t = d[i]; d[i] = d[k]; d[k] = t;
            if (z)
                for (int r2 = 0; r2 < n; ++r2) {
                    double tz = z[(size_t)i * n + r2];
                    z[(size_t)i * n + r2] = z[(size_t)k * n + r2];
                    z[(size_t)k * n + r2] = tz;
                }
        }
    }
    memcpy(w, d, sizeof(double) * n);
    free(d); free(e);
    return status;
}

/* ------------------------------------------------------------------------- */
/* Lanczos                                                                   */
/* ------------------------------------------------------------------------- */

/* create_fix_initial_vector (rcvector_class.f90:43-60): v(i) = ran_tab(modi(i,10000)),
 * i 1-based, modi (random.f90:71-76) maps to 1..10000.  ran_tab has 10001 entries. */
void orc_fix_initial_vector(int64_t n, const double *ran_tab, double *v)
{
    for (int64_t i = 1; i <= n; ++i) {
        int64_t k = i % 10000;
        if (k == 0) k = 10000;
        v[i - 1] = ran_tab[k];
    }
}

typedef struct {
    double normv_in, normv_out;
} orc_lanc_state;

/* one_step_Lanczos_fast + lanc_opt (Lanczos_plain.f90:247-302, Lanczos_plain.h:66-173).
 * diag/subdiag follow the Dagotto layout: subdiag[0] = |v0|, subdiag[k] couples k-1,k.
 * Returns 1 when the recurrence broke down (|w| < cutoff), 0 otherwise. */
static int lanczos_step(const orc_h *h, int iter, int ntri, double *vin, double *tmp,
                        double *vout, double *diag, double *subdiag, orc_lanc_state *st,
                        double cutoff_min)
{
    const int64_t n = h->dim;
    if (iter == 1) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) s += vin[i] * vin[i];
        st->normv_in = sqrt(fabs(s));
        st->normv_out = 0.0;
        for (int k = 0; k < ntri; ++k) { diag[k] = 0.0; subdiag[k] = 0.0; }
        subdiag[0] = st->normv_in;
        if (fabs(st->normv_in) < cutoff_min) return 2;
        double aa = 1.0 / st->normv_in;
        for (int64_t i = 0; i < n; ++i) vin[i] = vin[i] * aa;
    } else {
        if (fabs(st->normv_out) < cutoff_min) return 1;
        double aa = 1.0 / st->normv_out;
        for (int64_t i = 0; i < n; ++i) vin[i] = vin[i] * aa;
    }
    orc_hmult(h, vin, vout);
    double dd = 0.0;
    if (iter > 1) {
        double b = subdiag[iter - 1];
        for (int64_t i = 0; i < n; ++i) {
            vout[i] = vout[i] - b * tmp[i];
            dd += vout[i] * vin[i];
        }
    } else {
        for (int64_t i = 0; i < n; ++i) dd += vout[i] * vin[i];
    }
    diag[iter - 1] = dd;
    double nrm = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        vout[i] = vout[i] - dd * vin[i];
        nrm += vout[i] * vout[i];
    }
    st->normv_out = sqrt(nrm);
    if (iter < ntri) subdiag[iter] = st->normv_out;
    for (int64_t i = 0; i < n; ++i) { tmp[i] = vin[i]; vin[i] = vout[i]; }
    return 0;
}

/* Lanczos_fast_diagonalize (Lanczos_plain.f90:33-134), pass 1.
 * v0: start vector (length dim).  Outputs: E[neigen_kept], niter, the
 * tridiagonal (diag[niter], subdiag[niter]) and vecp[niter*nkept] (column j =
 * the tridiagonal eigenvector coefficients of kept eigenvalue j), conv[nkept].
 * Returns the number of kept eigenvalues (>=1) or <0 on error. */
int orc_lanczos_e0(const orc_h *h, const double *v0, int nitermax, int neigen,
                   double tolerance, double demax, double cutoff_min,
                   double *E, int *niter_out, double *diag, double *subdiag,
                   double *vecp, int *conv)
{
    const int64_t n = h->dim;
    int Niter = (int)((n - 1) < nitermax ? (n - 1) : nitermax);
    if (Niter < 1) return -1;
    int ne = neigen < n ? neigen : (int)n;
    ne = ne < Niter ? ne : Niter;
    double *vin = (double *)malloc(sizeof(double) * n);
    double *tmp = (double *)calloc((size_t)n, sizeof(double));
    double *vout = (double *)malloc(sizeof(double) * n);
    memcpy(vin, v0, sizeof(double) * n);
    double *valp = (double *)malloc(sizeof(double) * Niter);
    double *vp = (double *)malloc(sizeof(double) * (size_t)Niter * Niter);
    double last[64], rdist[64];
    int cv[64];
    for (int k = 0; k < 64; ++k) { last[k] = 1e300; rdist[k] = 1e300; cv[k] = 0; }
    orc_lanc_state st = {0, 0};
    int kept = 0;
    for (int iter = 1; iter <= Niter; ++iter) {
        int brk = lanczos_step(h, iter, Niter, vin, tmp, vout, diag, subdiag, &st, cutoff_min);
        if (brk == 2) { kept = -2; break; }
        int conv_one = (fabs(st.normv_out) < 1e-24 && iter == 1);
        orc_tridiag_eig(iter, diag, subdiag + 1, valp, NULL);
        int m = ne < iter ? ne : iter;
        int all = 1;
        for (int k = 0; k < m; ++k) {
            rdist[k] = valp[k] - last[k];
            cv[k] = (fabs(rdist[k]) < tolerance) && iter > 2;
        }
        for (int k = 0; k < ne; ++k) if (!(k < m && cv[k])) all = 0;
        int exhausted = (st.normv_out < cutoff_min);
        if (all || iter == Niter || conv_one || exhausted) {
            orc_tridiag_eig(iter, diag, subdiag + 1, valp, vp);
            for (int j = 0; j < ne; ++j) {
                int inwin = valp[j] >= valp[0] && valp[j] <= valp[0] + demax;
                if (j == 0 || (cv[j] && inwin)) {
                    E[kept] = valp[j];
                    conv[kept] = cv[j];
                    for (int k = 0; k < iter; ++k) vecp[(size_t)kept * iter + k] = vp[(size_t)j * iter + k];
                    ++kept;
                }
            }
            *niter_out = iter;
            break;
        }
        for (int k = 0; k < m; ++k) last[k] = valp[k];
    }
    free(vin); free(tmp); free(vout); free(valp); free(vp);
    return kept;
}

/* Lanczos_get_GS_sector (Lanczos_plain.f90:156-229), pass 2: rebuild the
 * eigenvector from the same start vector and the stored coefficients. */
int orc_lanczos_gs(const orc_h *h, const double *v0, int iter, const double *coef,
                   double cutoff_min, double *psi)
{
    const int64_t n = h->dim;
    const double rerror = 1e-13;
    double *vin = (double *)malloc(sizeof(double) * n);
    double *tmp = (double *)calloc((size_t)n, sizeof(double));
    double *vout = (double *)malloc(sizeof(double) * n);
    double *dg = (double *)calloc((size_t)iter + 1, sizeof(double));
    double *sd = (double *)calloc((size_t)iter + 1, sizeof(double));
    memcpy(vin, v0, sizeof(double) * n);
    orc_lanc_state st = {0, 0};
    double aa = 0.0;
    for (int64_t i = 0; i < n; ++i) aa += vin[i] * vin[i];
    aa = sqrt(aa);
    if (fabs(aa) < rerror) aa = rerror;
    aa = 1.0 / aa;
    for (int64_t i = 0; i < n; ++i) psi[i] = coef[0] * vin[i] * aa;
    lanczos_step(h, 1, iter + 1, vin, tmp, vout, dg, sd, &st, cutoff_min);
    if (!(fabs(st.normv_out) < 1e-24)) {
        for (int it = 2; it <= iter - 1; ++it) {
            double a2 = 0.0;
            for (int64_t i = 0; i < n; ++i) a2 += vout[i] * vout[i];
            a2 = sqrt(a2);
            if (fabs(a2) < rerror) a2 = rerror;
            a2 = 1.0 / a2;
            for (int64_t i = 0; i < n; ++i) { vout[i] *= a2; psi[i] = psi[i] + coef[it - 1] * vout[i]; }
            /* vec_in still holds the unnormalised w (copied at the end of the
             * previous step); lanc_opt rescales it by 1/normv_out itself */
            lanczos_step(h, it, iter + 1, vin, tmp, vout, dg, sd, &st, cutoff_min);
        }
        if (iter >= 2) {
            double a2 = 0.0;
            for (int64_t i = 0; i < n; ++i) a2 += vout[i] * vout[i];
            a2 = sqrt(a2);
            if (fabs(a2) < rerror) a2 = rerror;
            a2 = 1.0 / a2;
            for (int64_t i = 0; i < n; ++i) { vout[i] *= a2; psi[i] = psi[i] + coef[iter - 1] * vout[i]; }
        }
        double a3 = 0.0;
        for (int64_t i = 0; i < n; ++i) a3 += psi[i] * psi[i];
        a3 = sqrt(a3);
        if (fabs(a3) < rerror) a3 = rerror;
        a3 = 1.0 / a3;
        for (int64_t i = 0; i < n; ++i) psi[i] *= a3;
    }
    free(vin); free(tmp); free(vout); free(dg); free(sd);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* c / c^dagger on an (N_up,N_dn) vector: apply_Cupdo (apply_C.f90:497-653)   */
/* ------------------------------------------------------------------------- */

/* spin 0 = up (contiguous index), 1 = down.  `site` is the 0-based impurity
 * site; its bit is nb+site in either spin species (apply_C.f90:37-40).  The
 * output vector lives in the target sector (N_sigma +/- 1) and is overwritten. */
int orc_apply_c(int ns, int nb, int nup, int ndn, int site, int spin, int dagger,
                const double *in, double *out)
{
    int np = spin == 0 ? nup : ndn;
    int npt = np + (dagger ? 1 : -1);
    if (npt < 0 || npt > ns) return -1;
    int64_t dsrc = orc_binom(ns, np), dtgt = orc_binom(ns, npt);
    int64_t dother = orc_binom(ns, spin == 0 ? ndn : nup);
    uint64_t *st = (uint64_t *)malloc(sizeof(uint64_t) * (dsrc > 0 ? dsrc : 1));
    int32_t *rank = (int32_t *)malloc(sizeof(int32_t) * ((size_t)1 << ns));
    orc_basis(ns, np, st);
    orc_rank_table(ns, rank);
    int64_t dup_t = spin == 0 ? dtgt : dother;
    int64_t dup_s = spin == 0 ? dsrc : dother;
    memset(out, 0, sizeof(double) * (size_t)(dtgt * dother));
    int bit = nb + site;
    for (int64_t i = 0; i < dsrc; ++i) {
        uint64_t o;
        int sg = 1;
        int ok = dagger ? ket_create(st[i], bit, &o, &sg) : ket_destroy(st[i], bit, &o, &sg);
        if (!ok) continue;
        int64_t j = rank[o];
        if (spin == 0) {
            for (int64_t r = 0; r < dother; ++r)
                out[j + r * dup_t] = out[j + r * dup_t] + (double)sg * in[i + r * dup_s];
        } else {
            for (int64_t c = 0; c < dother; ++c)
                out[c + j * dup_t] = out[c + j * dup_t] + (double)sg * in[c + i * dup_s];
        }
    }
    free(st); free(rank);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* continued fraction: invert_zmtridiag (matrices_tridiag.f90:163-198)        */
/* ------------------------------------------------------------------------- */

/* <0|(z-T)^-1|0> for T = tridiag(diag[0..n-1], subdiag[1..n-1]).  Returns
 * 1 on a zero denominator (the reference STOPs there). */
int orc_cf(int n, const double *diag, const double *subdiag, double zr, double zi,
           double *outr, double *outi)
{
    double complex z = zr + I * zi;
    double complex aa = z - diag[n - 1];
    if (cabs(aa) < 2.220446049250313e-16) return 1;
    double complex r = 1.0 / aa;
    for (int it = n - 2; it >= 0; --it) {
        aa = z - diag[it] - r * subdiag[it + 1] * subdiag[it + 1];
        if (cabs(aa) < 2.220446049250313e-16) return 1;
        r = 1.0 / aa;
    }
    *outr = creal(r);
    *outi = cimag(r);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* compute_dynamic_cpu (green_class_compute_dynamic.f90:191-334), fermionic   */
/* ------------------------------------------------------------------------- */

/* Runs exactly min(nitergreen, dim) Lanczos steps from opm/|opm| (stops early
 * only on breakdown), then dyn(iw) = |opm|^2 * <0|(z - ph*(T-E))^-1|0> with
 * z = i*wn[iw] (fermion_sign=-1 so -fermion_sign = +1).  iph=1 particle
 * (ph=+1), iph=2 hole (ph=-1).  G is interleaved re/im, length 2*nw.
 * Returns the number of steps run, 0 when |opm|^2 < cutoff_dynamic. */
int orc_green_chain(const orc_h *h, const double *opm, int nitergreen, double e0,
                    int iph, int nw, const double *wn, double cutoff_dynamic,
                    double cutoff_min, double *G, double *diag_out, double *subdiag_out)
{
    const int64_t n = h->dim;
    int Niter = (int)(nitergreen < n ? nitergreen : n);
    double norm2 = 0.0;
    for (int64_t i = 0; i < n; ++i) norm2 += opm[i] * opm[i];
    for (int w = 0; w < 2 * nw; ++w) G[w] = 0.0;
    if (norm2 < cutoff_dynamic) return 0;
    double *vin = (double *)malloc(sizeof(double) * n);
    double *tmp = (double *)calloc((size_t)n, sizeof(double));
    double *vout = (double *)malloc(sizeof(double) * n);
    double *dg = (double *)calloc((size_t)Niter, sizeof(double));
    double *sd = (double *)calloc((size_t)Niter, sizeof(double));
    double nrm = sqrt(norm2);
    for (int64_t i = 0; i < n; ++i) vin[i] = opm[i] / nrm;
    orc_lanc_state st = {0, 0};
    int done = 0;
    for (int it = 1; it <= Niter; ++it) {
        int brk = lanczos_step(h, it, Niter, vin, tmp, vout, dg, sd, &st, cutoff_min);
        if (brk) break;
        done = it;
        if (st.normv_out < cutoff_min) break;
    }
    double ph = (iph == 1) ? 1.0 : -1.0;
    double *tdg = (double *)malloc(sizeof(double) * (done > 0 ? done : 1));
    for (int k = 0; k < done; ++k) tdg[k] = ph * (dg[k] - e0);
    for (int w = 0; w < nw; ++w) {
        double re = 0, im = 0;
        orc_cf(done, tdg, sd, 0.0, wn[w], &re, &im);
        G[2 * w] = re * norm2;
        G[2 * w + 1] = im * norm2;
    }
    if (diag_out) memcpy(diag_out, dg, sizeof(double) * done);
    if (subdiag_out) memcpy(subdiag_out, sd, sizeof(double) * done);
    free(vin); free(tmp); free(vout); free(dg); free(sd); free(tdg);
    return done;
}

/* <psi| n_c,up n_c,dn |psi> for impurity site c (double occupancy, the
 * quantity correlations_write.h:93-95 reports). */
double orc_double_occ(const orc_h *h, const double *psi, int site)
{
    double s = 0.0;
    int b = h->nb + site;
    for (int64_t ido = 0; ido < h->ddn; ++ido) {
        if (!bt(h->t[1].st[ido], b)) continue;
        for (int64_t iup = 0; iup < h->dup; ++iup)
            if (bt(h->t[0].st[iup], b)) {
                double v = psi[iup + ido * h->dup];
                s += v * v;
            }
    }
    return s;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* CPU-baseline sample: runs `nsteps` iterations of lanc_opt (Lanczos_plain.h:66-173)
 * from v0 on sector h; returns the number of iterations completed. */
int orc_lanczos_steps(const orc_h *h, const double *v0, int nsteps, double *diag, double *subdiag)
{
    const int64_t n = h->dim;
    double *vin = (double *)malloc(sizeof(double) * n);
    double *tmp = (double *)calloc((size_t)n, sizeof(double));
    double *vout = (double *)malloc(sizeof(double) * n);
    memcpy(vin, v0, sizeof(double) * n);
    orc_lanc_state st = {0, 0};
    int done = 0;
    for (int it = 1; it <= nsteps; ++it) {
        if (lanczos_step(h, it, nsteps + 1, vin, tmp, vout, diag, subdiag, &st, 1e-25)) break;
        done = it;
    }
    free(vin); free(tmp); free(vout);
    return done;
}

/* ------------------------------------------------------------------------- */
/* Nambu (Sz) sectors: HAIMsz (HAIMsz.f90:51-1027)                            */
/* ------------------------------------------------------------------------- */

/* Superconducting bath on top of orc_model (bath_class.f90:956-1022):
 * pb[k][k'] = Pb(k,k') (NULL = no pairing), pvbc[s][k][c] = PVbc_s(k,c)
 * (NULL unless PAIRING_IMP_TO_BATH).  on_fly = 1 follows HAIMsz_mult_fly_r's
 * order (HAIMsz.f90:615-808), 0 the tabulated HAIMsz_multr (:453-589). */
typedef struct {
    orc_model base;
    const double *pb, *pvbc;
    int32_t on_fly;
} orc_model_sz;

#define ORC_SZ_MAXNB 16

typedef struct orc_sz {
    int nc, nb, ns, npart, on_fly, nimp, nbath;   /* nimp = 2nc, nbath = 2nb Nambu orbitals */
    int imp_bit[2 * ORC_MAXNC], bath_bit[2 * ORC_SZ_MAXNB];
    double *ecn, *ebn, *vbcn;                     /* Nambu matrices, row-major */
    double u[ORC_MAXNC * ORC_MAXNC];
    int umask[ORC_MAXNC * ORC_MAXNC], offdiag_coulomb;
    double cutoff, shift1, shift2;
    int64_t dim;
    uint64_t *st;                                 /* sector states, ascending */
    double *quart;                                /* QUART_INT_SZ */
    double *diag;                                 /* diagsz (tabulated order) */
    int64_t *ptr, *tgt;                           /* offdiagsz CSR (tabulated order) */
    double *val;
} orc_sz;

/* Position of s among the states of its popcount in increasing order
 * (Hilbert%rank of new_fermion_Hilbert_space, quantum_fermion_hilbert_class.f90:385-404),
 * through the combinatorial number system: sum over the i-th lowest set bit p_i of C(p_i, i+1). */
int64_t orc_colex_rank(uint64_t s)
{
    int64_t r = 0;
    int i = 0;
    while (s) {
        int p = __builtin_ctzll(s);
        r += orc_binom(p, i + 1);
        ++i;
        s &= s - 1;
    }
    return r;
}

/* Nambu_Ec (impurity_class.f90:1018-1037), Nambu_Eb (bath_class.f90:956-986),
 * Nambu_Vbc (bath_class.f90:998-1022); Nambu orbital order of new_AIM2
 * (quantum_algebra_Anderson_Impurity_class2.f90:88-100): impurity up sites then
 * impurity down sites (bits nb+c and ns+nb+c), bath up then bath down (bits k, ns+k). */
static void sz_nambu(const orc_model_sz *m, orc_sz *z)
{
    const int nc = m->base.nc, nb = m->base.nb, ns = nc + nb, NI = 2 * nc, NB = 2 * nb;
    const double *ec = m->base.ec, *eb = m->base.eb, *vb = m->base.vbc;
    z->ecn = (double *)calloc((size_t)NI * NI, sizeof(double));
    z->ebn = (double *)calloc((size_t)(NB > 0 ? NB * NB : 1), sizeof(double));
    z->vbcn = (double *)calloc((size_t)(NB > 0 ? NB * NI : 1), sizeof(double));
    for (int i = 0; i < nc; ++i) {
        z->imp_bit[i] = nb + i;
        z->imp_bit[nc + i] = ns + nb + i;
        for (int j = 0; j < nc; ++j) {
            z->ecn[i * NI + j] = ec[i * nc + j];
            z->ecn[(nc + i) * NI + nc + j] = -ec[nc * nc + j * nc + i];
        }
    }
    for (int k = 0; k < nb; ++k) {
        z->bath_bit[k] = k;
        z->bath_bit[nb + k] = ns + k;
        for (int l = 0; l < nb; ++l) {
            z->ebn[k * NB + l] = eb[k * nb + l];
            z->ebn[(nb + k) * NB + nb + l] = -eb[nb * nb + l * nb + k];
            if (m->pb) {
                z->ebn[k * NB + nb + l] = m->pb[k * nb + l];
                z->ebn[(nb + k) * NB + l] = m->pb[l * nb + k];
            }
        }
        for (int c = 0; c < nc; ++c) {
            z->vbcn[k * NI + c] = vb[k * nc + c];
            z->vbcn[(nb + k) * NI + nc + c] = -vb[nb * nc + k * nc + c];
            if (m->pvbc) {
                z->vbcn[(nb + k) * NI + c] = m->pvbc[k * nc + c];
                z->vbcn[k * NI + nc + c] = m->pvbc[nb * nc + k * nc + c];
            }
        }
    }
    /* energy_global_shift = sum(diag(Ec(2))), energy_global_shift2 =
     * -sum(diag(lower block of EbNambu)); eigenvalues get + shift + shift2
     * (eigen_sector_class.f90:329) */
    double s1 = 0.0, s2 = 0.0;
    for (int c = 0; c < nc; ++c) s1 = s1 + ec[nc * nc + c * nc + c];
    for (int k = 0; k < nb; ++k) s2 = s2 + z->ebn[(nb + k) * NB + nb + k];
    z->shift1 = s1;
    z->shift2 = -s2;
}

static inline int sz_between_sign(uint64_t s, int a, int b) { return between_sign(s, a, b); }

/* hop tgt <- src on s: 0 when nil; else target state and the Jordan-Wigner sign
 * (hop, quantum_fermion_ket_class.f90:483-492: destroy then create) */
static inline int sz_hop(uint64_t s, int tgt, int src, uint64_t *out, int *sign)
{
    return ket_hop(s, tgt, src, out, sign);
}

/* tab_HAIM2 for the Nambu AIM2 (HAIM_offdiag_arrays.f90:419-526): visits the
 * off-diagonal targets of s in the tabulated order. */
static int sz_visit(const orc_sz *z, uint64_t s, uint64_t *ts, double *tv)
{
    const int NI = z->nimp, NB = z->nbath;
    int n = 0, sg;
    uint64_t out;
    for (int i = 0; i < NI; ++i)
        for (int j = 0; j < NI; ++j) {
            double h = z->ecn[i * NI + j];
            if (i == j || h == 0.0 || !(fabs(h) > z->cutoff)) continue;
            if (sz_hop(s, z->imp_bit[i], z->imp_bit[j], &out, &sg)) {
                if (ts) { ts[n] = out; tv[n] = h * (double)sg; }
                ++n;
            }
        }
    for (int i = 0; i < NB; ++i)
        for (int j = 0; j < NB; ++j) {
            double h = z->ebn[i * NB + j];
            if (i == j || h == 0.0 || !(fabs(h) > z->cutoff)) continue;
            if (sz_hop(s, z->bath_bit[i], z->bath_bit[j], &out, &sg)) {
                if (ts) { ts[n] = out; tv[n] = h * (double)sg; }
                ++n;
            }
        }
    for (int k = 0; k < NB; ++k)
        for (int c = 0; c < NI; ++c) {
            double h = z->vbcn[k * NI + c];
            if (h == 0.0 || !(fabs(h) > z->cutoff)) continue;
            if (sz_hop(s, z->bath_bit[k], z->imp_bit[c], &out, &sg)) {     /* impurity -> bath */
                if (ts) { ts[n] = out; tv[n] = h * (double)sg; }
                ++n;
            }
            if (sz_hop(s, z->imp_bit[c], z->bath_bit[k], &out, &sg)) {     /* bath -> impurity */
                if (ts) { ts[n] = out; tv[n] = h * (double)sg; }
                ++n;
            }
        }
    return n;
}

/* QUART_INT_SZ of one state (tab_HAIMsz, HAIMsz.f90:106-177): the down
 * occupation is the complement of the hole orbital's.  The Slater-type Hund
 * term is not reached: HAIMsz_mult* stop when |Jhund| > 1e-5. */
static double sz_quart(const orc_sz *z, uint64_t s)
{
    const int nc = z->nc;
    double q = 0.0;
    for (int s1 = 0; s1 < nc; ++s1) {
        const int b1u = bt(s, z->imp_bit[s1]), b1d = !bt(s, z->imp_bit[nc + s1]);
        const int n1 = b1u + b1d;
        if (n1 == 2 && z->umask[s1 * nc + s1]) q = q + z->u[s1 * nc + s1];
        if (z->offdiag_coulomb && n1 != 0)
            for (int s2 = s1 + 1; s2 < nc; ++s2) {
                if (!z->umask[s1 * nc + s2]) continue;
                const int n2 = bt(s, z->imp_bit[s2]) + !bt(s, z->imp_bit[nc + s2]);
                q = q + z->u[s1 * nc + s2] * (double)n1 * (double)n2;
            }
    }
    return q;
}

static void orc_sz_free(orc_sz *z)
{
    if (!z) return;
    free(z->ecn); free(z->ebn); free(z->vbcn); free(z->st); free(z->quart);
    free(z->diag); free(z->ptr); free(z->tgt); free(z->val);
    free(z);
}

/* new_HAIMsz (HAIMsz.f90:51-82) on the sector of `npart` Nambu particles in
 * 2*ns orbitals (new_fermion_sector with norbs = 2*ns).  offdiag_coulomb is the
 * intended "U has a non-zero off-diagonal element" (:68; the reference evaluates
 * it before filling its is_diag mask). */
orc_h *orc_h_new_sz(const orc_model_sz *m, int npart)
{
    const int nc = m->base.nc, nb = m->base.nb, ns = nc + nb;
    if (nc < 1 || nc > ORC_MAXNC || nb < 0 || nb > ORC_SZ_MAXNB || 2 * ns > 32) return NULL;
    if (npart < 0 || npart > 2 * ns) return NULL;
    if (fabs(m->base.jhund) > 1e-5) return NULL;   /* HAIMsz.f90:470-473 */
    orc_sz *z = (orc_sz *)calloc(1, sizeof(orc_sz));
    z->nc = nc; z->nb = nb; z->ns = ns; z->npart = npart; z->on_fly = m->on_fly;
    z->nimp = 2 * nc; z->nbath = 2 * nb;
    z->cutoff = m->base.cutoff;
    sz_nambu(m, z);
    for (int i = 0; i < nc * nc; ++i) {
        z->u[i] = m->base.u[i];
        z->umask[i] = m->base.u[i] != 0.0;
    }
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j)
            if (i != j && z->umask[i * nc + j]) z->offdiag_coulomb = 1;
    z->dim = orc_binom(2 * ns, npart);
    const int64_t d = z->dim;
    z->st = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(d > 0 ? d : 1));
    {
        /* increasing order: next state of the same popcount (Gosper) */
        uint64_t s = npart == 0 ? 0 : ((1ull << npart) - 1ull);
        for (int64_t i = 0; i < d; ++i) {
            z->st[i] = s;
            if (s == 0) break;
            uint64_t c = s & (~s + 1ull), r = s + c;
            s = (((r ^ s) >> 2) / c) | r;
        }
    }
    z->quart = (double *)malloc(sizeof(double) * (size_t)(d > 0 ? d : 1));
    z->diag = (double *)malloc(sizeof(double) * (size_t)(d > 0 ? d : 1));
    z->ptr = (int64_t *)malloc(sizeof(int64_t) * (size_t)(d + 1));
    int64_t nnz = 0;
    /* the on-the-fly variant tabulates nothing but QUART_INT_SZ (HAIMsz.f90:124) */
    if (!z->on_fly)
        for (int64_t i = 0; i < d; ++i) nnz += sz_visit(z, z->st[i], NULL, NULL);
    z->tgt = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nnz > 0 ? nnz : 1));
    z->val = (double *)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
    const int cap = z->nimp * z->nimp + z->nbath * z->nbath + 2 * z->nimp * z->nbath + 1;
    uint64_t *ts = (uint64_t *)malloc(sizeof(uint64_t) * cap);
    double *tv = (double *)malloc(sizeof(double) * cap);
    z->ptr[0] = 0;
    for (int64_t i = 0; i < d; ++i) {
        const uint64_t s = z->st[i];
        z->quart[i] = sz_quart(z, s);
        double dg = 0.0;                                  /* HAIM_offdiag_arrays.f90:419-427 */
        for (int o = 0; o < z->nimp; ++o)
            if (bt(s, z->imp_bit[o])) dg = dg + z->ecn[o * z->nimp + o];
        for (int o = 0; o < z->nbath; ++o)
            if (bt(s, z->bath_bit[o])) dg = dg + z->ebn[o * z->nbath + o];
        z->diag[i] = dg;
        int n = z->on_fly ? 0 : sz_visit(z, s, ts, tv);
        for (int e = 0; e < n; ++e) {
            z->tgt[z->ptr[i] + e] = orc_colex_rank(ts[e]);
            z->val[z->ptr[i] + e] = tv[e];
        }
        z->ptr[i + 1] = z->ptr[i] + n;
    }
    free(ts); free(tv);
    orc_h *h = (orc_h *)calloc(1, sizeof(orc_h));
    h->nc = nc; h->nb = nb; h->ns = ns;
    h->dim = d; h->dup = d; h->ddn = 1;
    h->sz = z;
    return h;
}

double orc_sz_shift(const orc_h *h) { return h->sz ? h->sz->shift1 + h->sz->shift2 : 0.0; }

/* Export per-state QUART_INT_SZ, diagsz and the CSR; any pointer may be NULL.
 * Returns the entry count. */
int64_t orc_sz_table(const orc_h *h, uint64_t *st, double *quart, double *diag, int64_t *ptr,
                     int64_t *tgt, double *val)
{
    const orc_sz *z = h->sz;
    if (!z) return -1;
    const int64_t d = z->dim, nnz = z->ptr[d];
    if (st) memcpy(st, z->st, sizeof(uint64_t) * d);
    if (quart) memcpy(quart, z->quart, sizeof(double) * d);
    if (diag) memcpy(diag, z->diag, sizeof(double) * d);
    if (ptr) memcpy(ptr, z->ptr, sizeof(int64_t) * (d + 1));
    if (tgt) memcpy(tgt, z->tgt, sizeof(int64_t) * nnz);
    if (val) memcpy(val, z->val, sizeof(double) * nnz);
    return nnz;
}

/* HAIMsz_multr with USE_CC (HAIMsz.f90:453-589) or HAIMsz_mult_fly_r
 * (HAIMsz.f90:615-808), real FP64, sequential per element. */
static void orc_sz_hmult(const orc_sz *z, const double *x, double *y)
{
    const int64_t d = z->dim;
    const int NI = z->nimp, NB = z->nbath;
    if (!z->on_fly) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < d; ++i) {
            double v = z->quart[i] * x[i];
            v = v + z->diag[i] * x[i];
            for (int64_t e = z->ptr[i]; e < z->ptr[i + 1]; ++e) v = v + z->val[e] * x[z->tgt[e]];
            y[i] = v;
        }
        return;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < d; ++i) {
        const uint64_t s = z->st[i];
        double v = z->quart[i] * x[i];
        for (int o = 0; o < NI; ++o)
            if (bt(s, z->imp_bit[o])) v = v + z->ecn[o * NI + o] * x[i];
        for (int o = 0; o < NB; ++o)
            if (bt(s, z->bath_bit[o])) v = v + z->ebn[o * NB + o] * x[i];
        /* one hop: source orbital a occupied, target b empty; sign from the
         * occupied orbitals strictly between (:686-694) */
#define SZ_FLY_HOP(a, b, hval)                                                     \
        do {                                                                       \
            const uint64_t o_ = (s & ~(1ull << (a)));                              \
            if (!bt(o_, (b))) {                                                    \
                const uint64_t t_ = o_ | (1ull << (b));                            \
                const double hh_ = (hval) * (double)sz_between_sign(t_, (a), (b)); \
                v = v + hh_ * x[orc_colex_rank(t_)];                               \
            }                                                                      \
        } while (0)
        for (int j = 0; j < NI; ++j) {
            if (!bt(s, z->imp_bit[j])) continue;
            for (int o = 0; o < NI; ++o)
                if (o != j && z->ecn[o * NI + j] != 0.0) SZ_FLY_HOP(z->imp_bit[j], z->imp_bit[o], z->ecn[o * NI + j]);
        }
        for (int j = 0; j < NB; ++j) {
            if (!bt(s, z->bath_bit[j])) continue;
            for (int o = 0; o < NB; ++o)
                if (o != j && z->ebn[o * NB + j] != 0.0) SZ_FLY_HOP(z->bath_bit[j], z->bath_bit[o], z->ebn[o * NB + j]);
        }
        for (int j = 0; j < NI; ++j) {                  /* impurity -> bath (:733-760) */
            if (!bt(s, z->imp_bit[j])) continue;
            for (int o = 0; o < NB; ++o)
                if (z->vbcn[o * NI + j] != 0.0) SZ_FLY_HOP(z->imp_bit[j], z->bath_bit[o], z->vbcn[o * NI + j]);
        }
        for (int o = 0; o < NB; ++o) {                  /* bath -> impurity (:762-790) */
            if (!bt(s, z->bath_bit[o])) continue;
            for (int j = 0; j < NI; ++j)
                if (z->vbcn[o * NI + j] != 0.0) SZ_FLY_HOP(z->bath_bit[o], z->imp_bit[j], z->vbcn[o * NI + j]);
        }
#undef SZ_FLY_HOP
        y[i] = v;
    }
}

/* apply_Csz_updo / apply_Csz_N_updo (apply_C.f90:344-483) on a Nambu vector:
 * physical c[+]_{site,spin}.  Spin up acts on the up orbital as written; spin
 * down acts on the hole orbital with the roles of c and c+ exchanged (CASE(2)
 * of :373-379).  projected = 1 is apply_Csz_N_updo: up only where the down
 * orbital of the site is occupied (its hole empty), down only where the up
 * orbital is occupied.  apply_Csz (:273-333) on Nambu orbital iorb is the
 * spin-up case for iorb < nc and the spin-down case with dagger flipped for
 * iorb >= nc.  out has binom(2ns, npart +/- 1) elements and is overwritten.
 * Returns the target npart, or -1. */
int orc_apply_csz(const orc_h *h, int site, int spin, int dagger, int projected, const double *in,
                  double *out)
{
    const orc_sz *z = h->sz;
    if (!z || site < 0 || site >= z->nc) return -1;
    const int bit = spin == 0 ? z->imp_bit[site] : z->imp_bit[z->nc + site];
    const int create = spin == 0 ? dagger : !dagger;
    const int npt = z->npart + (create ? 1 : -1);
    if (npt < 0 || npt > 2 * z->ns) return -1;
    const int64_t dt = orc_binom(2 * z->ns, npt);
    memset(out, 0, sizeof(double) * (size_t)dt);
    for (int64_t i = 0; i < z->dim; ++i) {
        if (in[i] == 0.0) continue;
        const uint64_t s = z->st[i];
        if (projected) {
            const int nup = bt(s, z->imp_bit[site]), ndn = bt(s, z->imp_bit[z->nc + site]);
            if (spin == 0 ? (ndn != 0) : (nup != 1)) continue;
        }
        uint64_t o;
        int sg = 1;
        const int ok = create ? ket_create(s, bit, &o, &sg) : ket_destroy(s, bit, &o, &sg);
        if (!ok) continue;
        const int64_t j = orc_colex_rank(o);
        out[j] = out[j] + (double)sg * in[i];
    }
    return npt;
}
