// edk_solve: the impurity-solver driver above the Krylov entry points.
//
// Restates, for the (N_up, N_dn) basis, the chain the reference runs for one
// DMFT iteration of the solver:
//   get_eigen_energies / get_GS (solver.h:11-237): sector scan, Lanczos pass 1
//     and pass 2 (dense diagonalisation below FULL_ED_SWITCH, ED_ARPACK.f90:590-715),
//     then the global window [E0, E0 + dEmax] and Boltzmann weights
//     (eigen_class.f90:322-450, eigen_sector_class.f90:431-446);
//   compute_greenAA (green_class_computeAA.f90:40-185) for the (c, c+)
//     channel of the requested impurity orbital pairs and spins: particle and
//     hole chains from (c+_i [+ c+_j])|psi> and (c_i [+ c_j])|psi>
//     (green_class_compute_symmetric_combination.f90:39-138), continued
//     fractions on the Matsubara axis, and the off-diagonal reshuffle
//     G_ij = (G_{i+j} - G_ii - G_jj)/2 (green_class_compute_symmetric_combination_AA.h:10-60);
//   the double occupancy of each impurity orbital (correlations_write.h:93-95).
// Mixed precision (dtype EDK_F32): in every sector of at least kLowprecMinDim
// states both Lanczos passes and the Green chains run on FP32 vectors (FP64
// coefficients and accumulation); every such ground state is refined once by
// an FP64 Lanczos restart from the FP32 vector and checked with the FP64
// matvec.  Smaller sectors stay in FP64: their kernels are bound by launch
// latency, so FP32 storage would add rounding without saving time.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "edk_internal.h"
#include "edk_tridiag.h"

namespace {

struct DBuf {
    void *p = nullptr;
    DBuf() = default;
    explicit DBuf(size_t bytes) { if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) p = nullptr; }
    // takes ownership of a cudaMalloc'd pointer
    static DBuf adopt(void *q) { DBuf b; b.p = q; return b; }
    DBuf(DBuf &&o) noexcept : p(o.p) { o.p = nullptr; }
    DBuf &operator=(DBuf &&o) noexcept { std::swap(p, o.p); return *this; }
    DBuf(const DBuf &) = delete;
    ~DBuf() { if (p) cudaFree(p); }
};

// Sectors with fewer states than this run in FP64 even in mixed precision,
// and their Green chains run batched (one persistent launch for all of them).
constexpr int64_t kLowprecMinDim = (int64_t)1 << 20;
// With edk_solve_opts.fp32_sums, FP32 passes of sectors of at least this many
// states sum their hop terms in FP32.  Smaller sectors keep FP64 sums even when
// lowprec_min_dim lets them run FP32 vectors: a chain with a pole close to the
// Fermi level in a sector of a few thousand states loses a factor of about 4
// in G with FP32 sums, while at 1.2e7 states the error stays at the level of
// the FP32 storage of the vectors.
constexpr int64_t kFp32SumsMinDim = (int64_t)1 << 20;
// Longest row the batched kernel stages in shared memory (FP64 elements).
constexpr int64_t kBatchMaxDup = 96 * 1024 / 8;
// With edk_solve_opts.batch_gs = 1, FP64 sectors of more than kFullEdSwitch
// and at most this many states run their ground states batched (gs_batch);
// a larger value of batch_gs is the bound itself.
constexpr int64_t kBatchGsMaxDim = (int64_t)1 << 14;
// Sectors of at most this many states are diagonalised densely (ED_diago),
// and with edk_solve_opts.reference_small_sectors their Green functions are
// Lehmann sums (FULL_ED_SWITCH, Global_Variables.f90:23).
constexpr int64_t kFullEdSwitch = 40;

struct State {
    int nup, ndn;
    double E;
    double E_pass1;            // energy of the first (possibly FP32) pass
    int dtype;                 // element type of psi
    DBuf psi;
    double boltz = 0.0;
    int converged = 1;
};

}  // namespace

#include <string>

extern "C" {

edk_h *edk_internal_cache_get(edk_ctx *ctx, const char *key, size_t len);
void edk_internal_cache_put(edk_ctx *ctx, const char *key, size_t len, edk_h *h);
cudaStream_t edk_internal_stream(edk_ctx *ctx);
int edk_internal_fail(edk_ctx *ctx, int code, const char *msg);
void edk_internal_count(edk_ctx *ctx, int64_t h2d, int64_t d2h);
edk_ctx *edk_internal_h_ctx(edk_h *h);
void edk_internal_fp32_sums(edk_ctx *ctx, int *enable, int64_t *min_dim);

int edk_convert(edk_ctx *ctx, int from_dtype, int to_dtype, int64_t n, const void *in_dev, void *out_dev)
{
    if (!ctx || !in_dev || !out_dev || n < 0) return EDK_ERR_INVALID;
    cudaError_t e = edk::launch_convert(from_dtype, to_dtype, n, in_dev, out_dev, edk_internal_stream(ctx));
    if (e != cudaSuccess) return edk_internal_fail(ctx, EDK_ERR_CUDA, cudaGetErrorString(e));
    return EDK_OK;
}

int edk_full_ed(edk_h *h, double *E_host, double *V_host)
{
    if (!h || !E_host) return EDK_ERR_INVALID;
    edk_ctx *ctx = edk_internal_h_ctx(h);
    int64_t dim = 0;
    edk_h_dims(h, &dim, nullptr, nullptr);
    if (dim < 1 || dim > 4096) return edk_internal_fail(ctx, EDK_ERR_INVALID, "full ED: dimension outside [1, 4096]");
    cudaStream_t st = edk_internal_stream(ctx);
    // the FP64 matrix from H*v on the unit vectors
    DBuf ein((size_t)dim * 8), hout((size_t)dim * 8), all((size_t)dim * dim * 8);
    if (!ein.p || !hout.p || !all.p) return edk_internal_fail(ctx, EDK_ERR_NOMEM, "full ED");
    std::vector<double> unit((size_t)dim, 0.0);
    int rc;
    for (int64_t i = 0; i < dim; ++i) {
        unit.assign((size_t)dim, 0.0);
        unit[(size_t)i] = 1.0;
        if (cudaMemcpyAsync(ein.p, unit.data(), (size_t)dim * 8, cudaMemcpyHostToDevice, st) != cudaSuccess)
            return edk_internal_fail(ctx, EDK_ERR_CUDA, "full ED upload");
        if ((rc = edk_hmult(h, EDK_F64, dim, ein.p, (char *)all.p + (size_t)i * dim * 8))) return rc;
        if (cudaStreamSynchronize(st) != cudaSuccess) return edk_internal_fail(ctx, EDK_ERR_CUDA, "full ED");
    }
    edk_internal_count(ctx, dim * dim * 8, dim * dim * 8);
    std::vector<double> Hd((size_t)dim * dim), w, V;
    if (cudaMemcpy(Hd.data(), all.p, (size_t)dim * dim * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        return edk_internal_fail(ctx, EDK_ERR_CUDA, "full ED download");
    // column i of the buffer is H e_i; H is symmetric, so the row-major reading is H
    edk::dense_eigh((int)dim, Hd, w, V);
    for (int64_t i = 0; i < dim; ++i) E_host[i] = w[(size_t)i];
    if (V_host) std::memcpy(V_host, V.data(), sizeof(double) * (size_t)dim * dim);
    return EDK_OK;
}

int edk_solve(edk_ctx *ctx, const edk_model *m, const edk_solve_opts *o, edk_solve_result *r)
{
    if (!ctx || !m || !o || !r || !o->sectors || o->nsectors < 1 || o->nw < 0 || o->beta <= 0)
        return EDK_ERR_INVALID;
    if (o->dtype != EDK_F64 && o->dtype != EDK_F32) return edk_internal_fail(ctx, EDK_ERR_INVALID, "dtype");
    if (o->npairs > 0 && !o->pairs) return edk_internal_fail(ctx, EDK_ERR_INVALID, "pairs");
    const int ns = m->nc + m->nb;
    cudaStream_t st = edk_internal_stream(ctx);
    const double demax = o->demax0 / o->beta;
    int rc;
    const int64_t lowprec_min = o->lowprec_min_dim > 0 ? o->lowprec_min_dim : kLowprecMinDim;
    // the context's FP32-sum setting for the duration of the solve
    struct SumsGuard {
        edk_ctx *c;
        int en = 0;
        int64_t md = 0;
        ~SumsGuard() { edk_ctx_set_fp32_sums(c, en, md); }
    } sums_guard{ctx};
    edk_internal_fp32_sums(ctx, &sums_guard.en, &sums_guard.md);
    edk_ctx_set_fp32_sums(ctx, o->dtype == EDK_F32 && o->fp32_sums ? 1 : 0, kFp32SumsMinDim);
    auto sector_dtype = [&](int64_t dim) {
        return (o->dtype == EDK_F32 && dim >= lowprec_min) ? EDK_F32 : EDK_F64;
    };

    // sector Hamiltonians are kept on the context, keyed by the model's bytes and the sector
    std::string mkey;
    {
        auto put = [&](const void *p, size_t n) { mkey.append(static_cast<const char *>(p), n); };
        put(&m->nc, 4); put(&m->nb, 4);
        put(m->ec, sizeof(double) * 2 * m->nc * m->nc);
        if (m->nb > 0) { put(m->eb, sizeof(double) * 2 * m->nb * m->nb); put(m->vbc, sizeof(double) * 2 * m->nb * m->nc); }
        put(m->u, sizeof(double) * m->nc * m->nc);
        put(m->jj, sizeof(double) * m->nc * m->nc);
        put(&m->jhund, 8); put(&m->cutoff_hamilt_param, 8);
    }
    auto getH = [&](int nu, int nd, edk_h **out) -> int {
        std::string key = mkey;
        key.append(reinterpret_cast<const char *>(&nu), 4);
        key.append(reinterpret_cast<const char *>(&nd), 4);
        if (edk_h *h = edk_internal_cache_get(ctx, key.data(), key.size())) { *out = h; return EDK_OK; }
        edk_h *h = nullptr;
        int rc2 = edk_h_create(ctx, m, nu, nd, &h);
        if (rc2) return rc2;
        edk_internal_cache_put(ctx, key.data(), key.size(), h);
        *out = h;
        return EDK_OK;
    };

    // ---------------- eigenstates ----------------
    std::vector<std::unique_ptr<State>> states;
    int64_t lanczos_steps = 0;
    double e0_low = 1e300;
    const int cap = std::max(4, o->nitermax + 4);
    std::vector<double> diag(cap), sub(cap), vecp((size_t)cap * std::max(1, o->neigen));
    // ed.sector_bound_file: when present only the window around its bounds is scanned
    int32_t bounds[6] = {0, 0, 0, 0, 1000, -1000};
    bool bounds_present = false;
    if (o->sector_bound_file) {
        if (FILE *bf = std::fopen(o->sector_bound_file, "r")) {
            std::fclose(bf);
            if (edk_sector_bounds_read(o->sector_bound_file, bounds, nullptr) != EDK_OK)
                return edk_internal_fail(ctx, EDK_ERR_INVALID, "unreadable sector bound file");
            bounds_present = true;
        }
    }
    if (o->gs_in) {
        // the eigenstates of a GS.raw file replace the scan (solver.f90:70-81)
        int32_t ne = 0;
        int64_t tot = 0;
        if (edk_gs_read(o->gs_in, 0, nullptr, &ne, 0, nullptr, &tot) != EDK_OK)
            return edk_internal_fail(ctx, EDK_ERR_INVALID, "unreadable GS file");
        std::vector<edk_gs_entry> ent((size_t)std::max(ne, 1));
        std::vector<double> pool((size_t)std::max<int64_t>(tot, 1));
        if (edk_gs_read(o->gs_in, ne, ent.data(), &ne, tot, pool.data(), &tot) != EDK_OK)
            return edk_internal_fail(ctx, EDK_ERR_INVALID, "unreadable GS file");
        for (int k = 0; k < ne; ++k) {
            const edk_gs_entry &e = ent[k];
            // INCONSISTENT INPUT SECTOR of init_solver (solver_init.h:174-178)
            if (e.kind != 0 || e.norbs != ns) return edk_internal_fail(ctx, EDK_ERR_INVALID, "GS file: sector of another model");
            edk_h *h = nullptr;
            if ((rc = getH(e.nup, e.ndn, &h))) return rc;
            int64_t dim = 0;
            edk_h_dims(h, &dim, nullptr, nullptr);
            if (e.n != dim) return edk_internal_fail(ctx, EDK_ERR_INVALID, "GS file: vector length");
            auto stt = std::make_unique<State>();
            stt->nup = e.nup; stt->ndn = e.ndn; stt->E = e.val; stt->E_pass1 = e.val;
            stt->converged = e.converged;
            stt->dtype = sector_dtype(dim);
            DBuf p64((size_t)dim * 8);
            if (!p64.p) return edk_internal_fail(ctx, EDK_ERR_NOMEM, "state vector");
            cudaMemcpyAsync(p64.p, pool.data() + e.offset, (size_t)dim * 8, cudaMemcpyHostToDevice, st);
            edk_internal_count(ctx, dim * 8, 0);
            if (stt->dtype == EDK_F64) {
                stt->psi = std::move(p64);
            } else {
                stt->psi = DBuf((size_t)dim * 4);
                if ((rc = edk_convert(ctx, EDK_F64, EDK_F32, dim, p64.p, stt->psi.p))) return rc;
            }
            if (cudaStreamSynchronize(st) != cudaSuccess) return edk_internal_fail(ctx, EDK_ERR_CUDA, "upload");
            states.push_back(std::move(stt));
        }
    }
    auto in_bounds = [&](int nu, int nd) {
        // goforit of get_eigen_energies (solver.h:134-137)
        const int w = o->iwindow;
        return !bounds_present ||
               (nu <= bounds[1] + w && nd <= bounds[3] + w && nu >= bounds[0] - w && nd >= bounds[2] - w);
    };
    // batched ground states of the small FP64 sectors (edk_solve_opts.batch_gs)
    std::map<int, edk::GsBatchSector> batched;
    struct BatchedGuard {   // states formed but not taken over (an error on the way) are freed
        std::map<int, edk::GsBatchSector> &m;
        ~BatchedGuard()
        {
            for (auto &kv : m)
                for (int k = 0; k < kv.second.nkept; ++k) cudaFree(kv.second.psi[k]);
        }
    } batched_guard{batched};
    if (o->batch_gs && !o->gs_in && o->neigen <= edk::kGsMaxNe && !(o->residual_tol > 0.0)) {
        std::vector<int> idx;
        std::vector<edk_h *> hs;
        for (int s = 0; s < o->nsectors; ++s) {
            const int nu = o->sectors[2 * s], nd = o->sectors[2 * s + 1];
            if (nu < 0 || nu > ns || nd < 0 || nd > ns || !in_bounds(nu, nd)) continue;
            edk_h *h = nullptr;
            if ((rc = getH(nu, nd, &h))) return rc;
            int64_t dim = 0, dup = 0;
            edk_h_dims(h, &dim, &dup, nullptr);
            const int64_t maxdim = o->batch_gs > 1 ? (int64_t)o->batch_gs : kBatchGsMaxDim;
            if (dim <= kFullEdSwitch || dim > maxdim || dup > kBatchMaxDup || sector_dtype(dim) != EDK_F64) continue;
            idx.push_back(s);
            hs.push_back(h);
        }
        std::vector<edk::GsBatchSector> res(hs.size());
        const int every = o->check_every > 0 ? o->check_every : 8;
        rc = edk::gs_batch(ctx, (int)hs.size(), hs.data(), o->nitermax, std::max(1, o->neigen), o->tolerance, demax,
                           o->ran_tab, every, res.data());
        for (size_t q = 0; q < res.size(); ++q) {
            if (rc) {
                for (void *p : res[q].psi) if (p) cudaFree(p);
            } else {
                batched[idx[q]] = res[q];
            }
        }
        if (rc) return rc;
    }
    for (int s = 0; s < (o->gs_in ? 0 : o->nsectors); ++s) {
        const int nu = o->sectors[2 * s], nd = o->sectors[2 * s + 1];
        if (nu < 0 || nu > ns || nd < 0 || nd > ns) return edk_internal_fail(ctx, EDK_ERR_INVALID, "sector");
        if (!in_bounds(nu, nd)) continue;
        edk_h *h = nullptr;
        if ((rc = getH(nu, nd, &h))) return rc;
        int64_t dim = 0;
        edk_h_dims(h, &dim, nullptr, nullptr);
        if (dim == 0) continue;
        std::vector<std::unique_ptr<State>> found;
        auto bt = batched.find(s);
        if (bt != batched.end()) {
            // the states the batched passes formed (FP64)
            const edk::GsBatchSector &g = bt->second;
            lanczos_steps += (int64_t)g.niter * (1 + g.nkept);
            for (int k = 0; k < g.nkept; ++k) {
                auto stt = std::make_unique<State>();
                stt->nup = nu; stt->ndn = nd; stt->E = g.E[k]; stt->E_pass1 = g.E[k]; stt->dtype = EDK_F64;
                stt->converged = g.converged[k];
                stt->psi = DBuf::adopt(g.psi[k]);
                found.push_back(std::move(stt));
            }
            batched.erase(bt);
        } else if (dim <= kFullEdSwitch) {
            // dense H from Hmult__ on unit vectors, FP64
            DBuf ecol((size_t)dim * 8), hcol((size_t)dim * dim * 8);
            std::vector<double> unit(dim, 0.0), Hd((size_t)dim * dim);
            for (int64_t i = 0; i < dim; ++i) {
                unit.assign(dim, 0.0);
                unit[i] = 1.0;
                cudaMemcpyAsync(ecol.p, unit.data(), dim * 8, cudaMemcpyHostToDevice, st);
                edk_internal_count(ctx, dim * 8, 0);
                if ((rc = edk_hmult(h, EDK_F64, dim, ecol.p, (char *)hcol.p + (size_t)i * dim * 8))) return rc;
                cudaStreamSynchronize(st);
            }
            cudaMemcpy(Hd.data(), hcol.p, (size_t)dim * dim * 8, cudaMemcpyDeviceToHost);
            lanczos_steps += dim;
            // Hd holds columns; H is symmetric so the row-major reading is the same matrix
            std::vector<double> w, V;
            edk::dense_eigh((int)dim, Hd, w, V);
            const int j = (int)std::min<int64_t>(dim, o->neigen);
            for (int k = 0; k < j; ++k) {
                if (k > 0 && !(w[k] <= w[0] + demax)) break;
                auto stt = std::make_unique<State>();
                stt->nup = nu; stt->ndn = nd; stt->E = w[k]; stt->E_pass1 = w[k]; stt->dtype = EDK_F64;
                stt->psi = DBuf((size_t)dim * 8);
                std::vector<double> col(dim);
                for (int64_t q = 0; q < dim; ++q) col[q] = V[(size_t)q * dim + k];
                cudaMemcpy(stt->psi.p, col.data(), dim * 8, cudaMemcpyHostToDevice);
                found.push_back(std::move(stt));
            }
        } else {
            const int sdt = sector_dtype(dim);
            const size_t ebytes = sdt == EDK_F64 ? 8 : 4;
            edk_lanczos_opts lo{};
            lo.nitermax = o->nitermax;
            lo.neigen = std::max(1, o->neigen);
            lo.tolerance = sdt == EDK_F32 ? std::max(o->tolerance, o->tolerance_lowprec) : o->tolerance;
            lo.demax = demax;
            lo.cutoff_min_lanczos_vec = 1e-25;
            lo.dtype = sdt;
            lo.check_every = o->check_every > 0 ? o->check_every : 8;
            lo.ran_tab = o->ran_tab;
            lo.residual_tol = sdt == EDK_F64 ? o->residual_tol : 0.0;
            lo.keep_basis = o->recompute_pass2 ? 0 : 1;   // pass 2 from pass 1's vectors
            edk_lanczos_result lr{};
            lr.diag = diag.data();
            lr.subdiag = sub.data();
            lr.vecp = vecp.data();
            if ((rc = edk_lanczos_e0(h, &lo, &lr))) return rc;
            lanczos_steps += lr.niter;
            // every state of the sector is formed from pass 1's kept vectors
            // before any FP64 refinement runs: a refinement is a Lanczos run of
            // its own, which would release that basis and reuse the pass-1
            // coefficient buffers
            for (int k = 0; k < lr.nkept; ++k) {
                auto stt = std::make_unique<State>();
                stt->nup = nu; stt->ndn = nd; stt->E = lr.E[k]; stt->E_pass1 = lr.E[k]; stt->dtype = sdt;
                stt->converged = lr.converged[k];
                stt->psi = DBuf((size_t)dim * ebytes);
                if (!stt->psi.p) return edk_internal_fail(ctx, EDK_ERR_NOMEM, "state vector");
                if (lo.keep_basis) lo.keep_basis = k + 1 < lr.nkept ? 2 : 1;
                if ((rc = edk_lanczos_gs(h, &lo, lr.niter, lr.vecp + (size_t)k * lr.niter, stt->psi.p))) return rc;
                lanczos_steps += lr.niter;      // the reference's count: pass 2 reruns the recurrence
                found.push_back(std::move(stt));
            }
            if (sdt == EDK_F32) {
                // FP64 refinement restart from each FP32 eigenvector, with its
                // own tridiagonal and coefficient buffers
                std::vector<double> rdiag(cap), rsub(cap), rvecp(cap);
                for (auto &stt : found) {
                    DBuf p64((size_t)dim * 8);
                    if (!p64.p) return edk_internal_fail(ctx, EDK_ERR_NOMEM, "refinement vector");
                    if ((rc = edk_convert(ctx, EDK_F32, EDK_F64, dim, stt->psi.p, p64.p))) return rc;
                    edk_lanczos_opts ro = lo;
                    ro.dtype = EDK_F64;
                    ro.tolerance = o->tolerance;
                    ro.neigen = 1;
                    ro.start_dev = p64.p;
                    ro.ran_tab = nullptr;
                    ro.use_target = 1;
                    ro.target = stt->E;
                    ro.check_every = 4;
                    ro.keep_basis = o->recompute_pass2 ? 0 : 1;
                    ro.residual_tol = o->residual_tol > 0.0 ? o->residual_tol : 1e-9 * std::max(1.0, std::fabs(stt->E));
                    edk_lanczos_result rr{};
                    rr.diag = rdiag.data();
                    rr.subdiag = rsub.data();
                    rr.vecp = rvecp.data();
                    if ((rc = edk_lanczos_e0(h, &ro, &rr))) return rc;
                    lanczos_steps += rr.niter;
                    DBuf q64((size_t)dim * 8);
                    if (!q64.p) return edk_internal_fail(ctx, EDK_ERR_NOMEM, "refinement vector");
                    if ((rc = edk_lanczos_gs(h, &ro, rr.niter, rr.vecp, q64.p))) return rc;
                    lanczos_steps += rr.niter;
                    stt->E = rr.E[0];
                    // the Green chains run on FP32 vectors: keep the refined state as FP32
                    if ((rc = edk_convert(ctx, EDK_F64, EDK_F32, dim, q64.p, stt->psi.p))) return rc;
                    stt->dtype = EDK_F32;
                }
            }
        }
        if (!found.empty()) {
            double es = 1e300;
            for (auto &f : found) es = std::min(es, f->E);
            for (auto &f : found)
                if (f->E <= es + demax) states.push_back(std::move(f));
        }
    }
    if (states.empty()) return edk_internal_fail(ctx, EDK_ERR_INVALID, "no eigenstate found");
    double e0 = 1e300;
    for (auto &s : states) e0 = std::min(e0, s->E);
    for (auto &s : states) e0_low = std::min(e0_low, s->E_pass1);
    std::vector<std::unique_ptr<State>> gs;
    for (auto &s : states)
        if (s->E <= e0 + demax) gs.push_back(std::move(s));
    double z = 0.0;
    for (auto &s : gs) z += std::exp(-o->beta * (s->E - e0));
    for (auto &s : gs) s->boltz = std::exp(-o->beta * (s->E - e0)) / z;
    if (o->gs_out) {
        // write_raw_eigensectorlist of the states in the window (solver.f90:104-108)
        std::vector<edk_gs_entry> ent;
        std::vector<double> pool;
        for (size_t k = 0; k < gs.size(); ++k) {
            edk_h *h = nullptr;
            if ((rc = getH(gs[k]->nup, gs[k]->ndn, &h))) return rc;
            int64_t dim = 0;
            edk_h_dims(h, &dim, nullptr, nullptr);
            edk_gs_entry e{};
            e.kind = 0;
            e.norbs = ns;
            e.nup = gs[k]->nup;
            e.ndn = gs[k]->ndn;
            e.val = gs[k]->E;
            e.converged = gs[k]->converged;
            e.rank = (k > 0 && gs[k - 1]->nup == e.nup && gs[k - 1]->ndn == e.ndn) ? ent.back().rank + 1 : 1;
            e.n = dim;
            e.offset = (int64_t)pool.size();
            pool.resize(pool.size() + (size_t)dim);
            DBuf p64;
            const void *p = gs[k]->psi.p;
            if (gs[k]->dtype != EDK_F64) {
                p64 = DBuf((size_t)dim * 8);
                if ((rc = edk_convert(ctx, gs[k]->dtype, EDK_F64, dim, gs[k]->psi.p, p64.p))) return rc;
                p = p64.p;
            }
            if (cudaMemcpyAsync(pool.data() + e.offset, p, (size_t)dim * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                return edk_internal_fail(ctx, EDK_ERR_CUDA, "state download");
            edk_internal_count(ctx, 0, dim * 8);
            ent.push_back(e);
        }
        if (edk_gs_write(o->gs_out, (int32_t)ent.size(), ent.data(), pool.data()) != EDK_OK)
            return edk_internal_fail(ctx, EDK_ERR_INVALID, "cannot write the GS file");
    }
    if (bounds_present) {
        // get_new_bounds (solver.h:374-415): the particle numbers of the kept states
        int32_t nb6[6] = {1000, -1000, 1000, -1000, 1000, -1000};
        for (auto &s : gs) {
            nb6[0] = std::min(nb6[0], s->nup); nb6[1] = std::max(nb6[1], s->nup);
            nb6[2] = std::min(nb6[2], s->ndn); nb6[3] = std::max(nb6[3], s->ndn);
        }
        if (edk_sector_bounds_write(o->sector_bound_file, nb6) != EDK_OK)
            return edk_internal_fail(ctx, EDK_ERR_INVALID, "cannot write the sector bound file");
    }
    r->e0 = e0;
    r->z = z;
    r->e0_lowprec = e0_low;
    r->nstates = (int)gs.size();
    for (size_t k = 0; k < gs.size() && k < 64; ++k) {
        if (r->energies) r->energies[k] = gs[k]->E;
        if (r->state_sectors) { r->state_sectors[2 * k] = gs[k]->nup; r->state_sectors[2 * k + 1] = gs[k]->ndn; }
    }
    // FP64 residual |H psi0 - E0 psi0| of the ground state
    for (auto &s : gs)
        if (s->E == e0) {
            edk_h *h = nullptr;
            if ((rc = getH(s->nup, s->ndn, &h))) return rc;
            int64_t dim = 0;
            edk_h_dims(h, &dim, nullptr, nullptr);
            DBuf p64;
            const void *p = s->psi.p;
            if (s->dtype != EDK_F64) {
                p64 = DBuf((size_t)dim * 8);
                if ((rc = edk_convert(ctx, s->dtype, EDK_F64, dim, s->psi.p, p64.p))) return rc;
                p = p64.p;
            }
            double res = 0, nrm = 0;
            if ((rc = edk_residual(h, p, s->E, &res, &nrm))) return rc;
            r->residual = res / (nrm > 0 ? nrm : 1.0);
            break;
        }
    // ---------------- double occupancy ----------------
    if (r->docc)
        for (int c = 0; c < m->nc; ++c) {
            double acc = 0.0;
            for (auto &s : gs) {
                edk_h *h = nullptr;
                if ((rc = getH(s->nup, s->ndn, &h))) return rc;
                double d = 0, n2 = 0;
                if ((rc = edk_double_occ(h, s->dtype, s->psi.p, c, &d, &n2))) return rc;
                acc += s->boltz * d / n2;
            }
            r->docc[c] = acc;
        }
    // ---------------- Green functions ----------------
    int64_t green_steps = 0;
    const int nw = o->nw;
    if (nw > 0 && o->npairs > 0 && r->G) {
        std::vector<double> wn(nw);
        for (int n = 0; n < nw; ++n) wn[n] = (2.0 * M_PI / o->beta) * (n + 1) - M_PI / o->beta;
        std::memset(r->G, 0, sizeof(double) * 2 * (size_t)o->npairs * nw * 2);
        // combinations needed: (i,i) for every orbital in a pair, (min,max) for off-diagonal pairs
        std::vector<std::pair<int, int>> combos;
        auto add = [&](int i, int j) {
            if (std::find(combos.begin(), combos.end(), std::make_pair(i, j)) == combos.end()) combos.push_back({i, j});
        };
        for (int p = 0; p < o->npairs; ++p) {
            const int i = o->pairs[2 * p], j = o->pairs[2 * p + 1];
            if (i < 0 || j < 0 || i >= m->nc || j >= m->nc) return edk_internal_fail(ctx, EDK_ERR_INVALID, "pair");
            add(i, i);
            add(j, j);
            if (i != j) add(std::min(i, j), std::max(i, j));
        }
        std::vector<double> raw((size_t)combos.size() * nw * 2);
        std::vector<double> Gc((size_t)2 * nw);
        // host copies of the window's states in sectors of at most kFullEdSwitch
        // states (FP64: those sectors are diagonalised densely), for the Lehmann branch
        std::map<const State *, std::vector<double>> small_psi;
        auto host_psi = [&](const State *s, int64_t dim, const std::vector<double> **out) -> int {
            auto it = small_psi.find(s);
            if (it == small_psi.end()) {
                std::vector<double> v((size_t)dim);
                if (s->dtype != EDK_F64) return edk_internal_fail(ctx, EDK_ERR_INVALID, "small sector state not FP64");
                if (cudaMemcpyAsync(v.data(), s->psi.p, (size_t)dim * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                    cudaStreamSynchronize(st) != cudaSuccess)
                    return edk_internal_fail(ctx, EDK_ERR_CUDA, "state download");
                edk_internal_count(ctx, 0, dim * 8);
                it = small_psi.emplace(s, std::move(v)).first;
            }
            *out = &it->second;
            return EDK_OK;
        };
        for (int spin = 0; spin < 2; ++spin) {
            if (!((o->spin_mask >> spin) & 1)) continue;
            std::fill(raw.begin(), raw.end(), 0.0);
            // chains of small target sectors, run together after the state loop
            std::vector<edk_chain> batch;
            std::vector<DBuf> batch_phi;
            for (auto &s : gs) {
                edk_h *hs_src = nullptr;
                if ((rc = getH(s->nup, s->ndn, &hs_src))) return rc;
                int64_t sdim = 0;
                edk_h_dims(hs_src, &sdim, nullptr, nullptr);
                // the state in the precision of each target sector's chains
                DBuf conv[2];
                auto psi_in = [&](int dt, const void **out) -> int {
                    if (s->dtype == dt) { *out = s->psi.p; return EDK_OK; }
                    if (!conv[dt].p) {
                        conv[dt] = DBuf((size_t)sdim * (dt == EDK_F64 ? 8 : 4));
                        if (!conv[dt].p) return edk_internal_fail(ctx, EDK_ERR_NOMEM, "state copy");
                        int rc2 = edk_convert(ctx, s->dtype, dt, sdim, s->psi.p, conv[dt].p);
                        if (rc2) return rc2;
                    }
                    *out = conv[dt].p;
                    return EDK_OK;
                };
                for (int iph = 1; iph <= 2; ++iph) {
                    const int d = iph == 1 ? 1 : -1;
                    const int tnu = s->nup + (spin == 0 ? d : 0), tnd = s->ndn + (spin == 1 ? d : 0);
                    if (tnu < 0 || tnu > ns || tnd < 0 || tnd > ns) continue;
                    edk_h *ht = nullptr;
                    if ((rc = getH(tnu, tnd, &ht))) return rc;
                    int64_t tdim = 0;
                    edk_h_dims(ht, &tdim, nullptr, nullptr);
                    if (tdim == 0) continue;
                    const int gdt = sector_dtype(tdim);
                    const void *psi = nullptr;
                    if ((rc = psi_in(gdt, &psi))) return rc;
                    int64_t tdup = 0;
                    edk_h_dims(ht, nullptr, &tdup, nullptr);
                    if (o->reference_small_sectors && tdim <= kFullEdSwitch) {
                        // compute_dynamic_full_ed (green_class_compute_dynamic.f90:77-165): with
                        // phi = A|psi> unnormalised, dyn(iw) = sum over the window's states |n>
                        // of the target sector of |<n|phi>|^2 / (iw - ph (E_n - E_psi)), and 0
                        // when |phi|^2 < cutoff_dynamic or no state of that sector is kept
                        const void *psi64 = nullptr;
                        if ((rc = psi_in(EDK_F64, &psi64))) return rc;
                        DBuf phi((size_t)tdim * 8);
                        std::vector<double> ph((size_t)tdim);
                        for (size_t q = 0; q < combos.size(); ++q) {
                            const int i = combos[q].first, j = combos[q].second;
                            int64_t od = 0;
                            if ((rc = edk_apply_c(hs_src, EDK_F64, i, spin, iph == 1, i == j ? -1 : j, 1, psi64,
                                                  phi.p, &od)))
                                return rc;
                            if (cudaMemcpyAsync(ph.data(), phi.p, (size_t)tdim * 8, cudaMemcpyDeviceToHost, st) !=
                                    cudaSuccess ||
                                cudaStreamSynchronize(st) != cudaSuccess)
                                return edk_internal_fail(ctx, EDK_ERR_CUDA, "Lehmann branch download");
                            edk_internal_count(ctx, 0, tdim * 8);
                            double n2 = 0.0;
                            for (int64_t t = 0; t < tdim; ++t) n2 += ph[t] * ph[t];
                            if (n2 < o->cutoff_dynamic) continue;
                            const double sgn = iph == 1 ? 1.0 : -1.0;
                            for (auto &n : gs) {
                                if (n->nup != tnu || n->ndn != tnd) continue;
                                const std::vector<double> *vn = nullptr;
                                if ((rc = host_psi(n.get(), tdim, &vn))) return rc;
                                double ov = 0.0;
                                for (int64_t t = 0; t < tdim; ++t) ov += (*vn)[t] * ph[t];
                                const double amp = ov * ov, de = sgn * (n->E - s->E);
                                for (int w = 0; w < nw; ++w) {
                                    // amp / (i wn - de)
                                    const double den = wn[w] * wn[w] + de * de;
                                    raw[q * 2 * nw + 2 * w] += s->boltz * amp * (-de) / den;
                                    raw[q * 2 * nw + 2 * w + 1] += s->boltz * amp * (-wn[w]) / den;
                                }
                            }
                        }
                        continue;
                    }
                    if (o->green_mode == 0 && gdt == EDK_F64 && tdim < kLowprecMinDim && tdup <= kBatchMaxDup) {
                        for (size_t q = 0; q < combos.size(); ++q) {
                            const int i = combos[q].first, j = combos[q].second;
                            batch_phi.emplace_back((size_t)tdim * 8);
                            if (!batch_phi.back().p) return edk_internal_fail(ctx, EDK_ERR_NOMEM, "chain start");
                            int64_t od = 0;
                            if ((rc = edk_apply_c(hs_src, gdt, i, spin, iph == 1, i == j ? -1 : j, 1, psi,
                                                  batch_phi.back().p, &od)))
                                return rc;
                            batch.push_back(edk_chain{ht, batch_phi.back().p, s->E, iph, s->boltz, (int32_t)q});
                        }
                        continue;
                    }
                    DBuf phi((size_t)tdim * (gdt == EDK_F64 ? 8 : 4));
                    for (size_t q = 0; q < combos.size(); ++q) {
                        const int i = combos[q].first, j = combos[q].second;
                        int64_t od = 0;
                        if ((rc = edk_apply_c(hs_src, gdt, i, spin, iph == 1, i == j ? -1 : j, 1, psi, phi.p, &od)))
                            return rc;
                        int32_t nd = 0;
                        if ((rc = edk_green_chain(ht, gdt, phi.p, o->nitergreen, s->E, iph, nw, wn.data(),
                                                  o->cutoff_dynamic, Gc.data(), nullptr, nullptr, &nd)))
                            return rc;
                        green_steps += nd;
                        for (int w = 0; w < 2 * nw; ++w) raw[q * 2 * nw + w] += s->boltz * Gc[w];
                    }
                }
            }
            if (!batch.empty()) {
                std::vector<double> Gb((size_t)combos.size() * 2 * nw);
                edk_batch_stats bst{};
                if ((rc = edk_green_batch(ctx, EDK_F64, (int32_t)batch.size(), batch.data(), o->nitergreen, nw,
                                          wn.data(), o->cutoff_dynamic, (int32_t)combos.size(), Gb.data(), 0, &bst)))
                    return rc;
                green_steps += bst.steps;
                for (size_t t = 0; t < Gb.size(); ++t) raw[t] += Gb[t];
            }
            auto idx = [&](int i, int j) {
                return (size_t)(std::find(combos.begin(), combos.end(), std::make_pair(i, j)) - combos.begin());
            };
            for (int p = 0; p < o->npairs; ++p) {
                const int i = o->pairs[2 * p], j = o->pairs[2 * p + 1];
                double *out = r->G + ((size_t)spin * o->npairs + p) * 2 * nw;
                if (i == j) {
                    std::memcpy(out, &raw[idx(i, i) * 2 * nw], sizeof(double) * 2 * nw);
                } else {
                    const size_t a = idx(std::min(i, j), std::max(i, j)), b = idx(i, i), cc = idx(j, j);
                    for (int w = 0; w < 2 * nw; ++w)
                        out[w] = 0.5 * (raw[a * 2 * nw + w] - raw[b * 2 * nw + w] - raw[cc * 2 * nw + w]);
                }
            }
        }
    }
    edk_internal_count(ctx, 0, (int64_t)sizeof(double) * 2 * o->npairs * nw * 2);
    r->lanczos_steps = (int32_t)lanczos_steps;
    r->green_steps = (int32_t)green_steps;
    return cudaStreamSynchronize(st) == cudaSuccess ? EDK_OK : edk_internal_fail(ctx, EDK_ERR_CUDA, "sync");
}

}  // extern "C"
