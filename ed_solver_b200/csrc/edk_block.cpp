// edk_block_lanczos: block Lanczos for the lowest eigenpairs of one sector
// (the role of Block_Lanczos_diagonalize, Block_Lanczos.f90:37-355, whose
// BLZPACK engine is not part of the reference's sources).
//
// Recurrence (block size p, FP64 device vectors, H applied column by column):
//   W = H V_j - V_{j-1} B_j^T,  A_j = V_j^T W,  W -= V_j A_j  (twice),
//   W = V_{j+1} B_{j+1}  (modified Gram-Schmidt, B upper triangular),
// so H V_j = V_{j-1} B_j^T + V_j A_j + V_{j+1} B_{j+1} and the block
// tridiagonal T has diagonal blocks A_j and sub-diagonal blocks B_{j+1}.
// Ritz values come from T on the host (Householder + Sturm bisection); the
// eigenvectors from a second pass that replays the recurrence (the kernels are
// deterministic, so the same V_j come back) and accumulates V_j Y_j.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "edk_grad.h"
#include "edk_internal.h"
#include "edk_tridiag.h"

extern "C" {
cudaStream_t edk_internal_stream(edk_ctx *ctx);
int edk_internal_fail(edk_ctx *ctx, int code, const char *msg);
edk_ctx *edk_internal_h_ctx(edk_h *h);
void edk_internal_add_launches(edk_ctx *ctx, int64_t n);
}

using namespace edk;

namespace {

struct DBuf {
    void *p = nullptr;
    DBuf() = default;
    explicit DBuf(size_t bytes) { if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) p = nullptr; }
    DBuf(DBuf &&o) noexcept : p(o.p) { o.p = nullptr; }
    DBuf &operator=(DBuf &&o) noexcept { std::swap(p, o.p); return *this; }
    DBuf(const DBuf &) = delete;
    ~DBuf() { if (p) cudaFree(p); }
    double *d() const { return static_cast<double *>(p); }
};

constexpr int kMaxBlock = 4;

struct Block {
    edk_h *h;
    edk_ctx *ctx;
    cudaStream_t st;
    int64_t n;
    int p;
    int grid;
    DBuf scratch;
    double *partials, *out;
    unsigned *counter;
    int fail(int code, const char *msg) { return edk_internal_fail(ctx, code, msg); }
    int cuda(cudaError_t e, const char *where)
    {
        if (e == cudaSuccess) return EDK_OK;
        char buf[256];
        snprintf(buf, sizeof buf, "block lanczos %s: %s", where, cudaGetErrorString(e));
        return fail(e == cudaErrorMemoryAllocation ? EDK_ERR_NOMEM : EDK_ERR_CUDA, buf);
    }
    int lincomb(double *o, bool acc, const double *x0, double c0, const double *x1 = nullptr, double c1 = 0,
                const double *x2 = nullptr, double c2 = 0, const double *x3 = nullptr, double c3 = 0)
    {
        edk_internal_add_launches(ctx, 1);
        return cuda(launch_lincomb(n, o, acc, x0, c0, x1, c1, x2, c2, x3, c3, grid, st), "lincomb");
    }
    int dot(const double *x, const double *y, double *r)
    {
        edk_internal_add_launches(ctx, 1);
        int rc = cuda(launch_dots(n, x, y, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, partials, counter, out,
                                  grid, st),
                      "dots");
        if (rc) return rc;
        if ((rc = cuda(cudaMemcpyAsync(r, out, sizeof(double), cudaMemcpyDeviceToHost, st), "d2h"))) return rc;
        return cuda(cudaStreamSynchronize(st), "sync");
    }
    // out = sum_l c[l] x[l] over the p block columns (accumulate when acc)
    int combo(double *o, bool acc, double *const *x, const double *c)
    {
        if (p == 1) return lincomb(o, acc, x[0], c[0]);
        if (p == 2) return lincomb(o, acc, x[0], c[0], x[1], c[1]);
        if (p == 3) return lincomb(o, acc, x[0], c[0], x[1], c[1], x[2], c[2]);
        return lincomb(o, acc, x[0], c[0], x[1], c[1], x[2], c[2], x[3], c[3]);
    }
};

// One block step j: from (Vm, Vj, Bj) to (A_j, B_{j+1}, Vn).  Returns
// EDK_KRYLOV_EXHAUSTED when the new block loses rank.
int block_step(Block &b, double *const *Vm, double *const *Vj, double *const *Vn, const double *Bj, bool first,
               double *Aj, double *Bn)
{
    const int p = b.p;
    int rc;
    for (int i = 0; i < p; ++i)
        if ((rc = edk_hmult(b.h, EDK_F64, b.n, Vj[i], Vn[i]))) return rc;
    if (!first)
        for (int i = 0; i < p; ++i) {
            double c[kMaxBlock];
            for (int l = 0; l < p; ++l) c[l] = -Bj[i * p + l];      // (V_{j-1} B_j^T)_i = sum_l V_{j-1,l} B_j[i][l]
            if ((rc = b.combo(Vn[i], true, Vm, c))) return rc;
        }
    std::fill(Aj, Aj + p * p, 0.0);
    for (int pass = 0; pass < 2; ++pass) {
        double a[kMaxBlock * kMaxBlock];
        for (int l = 0; l < p; ++l)
            for (int i = 0; i < p; ++i)
                if ((rc = b.dot(Vj[l], Vn[i], &a[l * p + i]))) return rc;
        for (int i = 0; i < p; ++i) {
            double c[kMaxBlock];
            for (int l = 0; l < p; ++l) c[l] = -a[l * p + i];
            if ((rc = b.combo(Vn[i], true, Vj, c))) return rc;
        }
        for (int k = 0; k < p * p; ++k) Aj[k] += a[k];
    }
    for (int l = 0; l < p; ++l)            // symmetric part
        for (int i = l + 1; i < p; ++i) {
            const double s = 0.5 * (Aj[l * p + i] + Aj[i * p + l]);
            Aj[l * p + i] = Aj[i * p + l] = s;
        }
    // modified Gram-Schmidt: W = V_{j+1} B_{j+1}
    std::fill(Bn, Bn + p * p, 0.0);
    double scale = 0.0;
    for (int k = 0; k < p * p; ++k) scale = std::max(scale, std::fabs(Aj[k]));
    for (int i = 0; i < p; ++i) {
        double r2 = 0.0;
        if ((rc = b.dot(Vn[i], Vn[i], &r2))) return rc;
        const double r = std::sqrt(std::max(r2, 0.0));
        if (!(r > 1e-13 * std::max(1.0, scale))) return EDK_KRYLOV_EXHAUSTED;
        Bn[i * p + i] = r;
        if ((rc = b.lincomb(Vn[i], false, Vn[i], 1.0 / r))) return rc;
        for (int l = i + 1; l < p; ++l) {
            double t = 0.0;
            if ((rc = b.dot(Vn[i], Vn[l], &t))) return rc;
            Bn[i * p + l] = t;
            if ((rc = b.lincomb(Vn[l], true, Vn[i], -t))) return rc;
        }
    }
    return EDK_OK;
}

// V_1: QR of the p periodic start vectors.
int block_start(Block &b, const double *tab_dev, double *const *V)
{
    int rc;
    for (int c = 0; c < b.p; ++c) {
        edk_internal_add_launches(b.ctx, 1);
        if ((rc = b.cuda(launch_fill_periodic(b.n, tab_dev, 977 * (int64_t)c, V[c], b.grid, b.st), "start"))) return rc;
    }
    for (int i = 0; i < b.p; ++i) {
        for (int l = 0; l < i; ++l) {
            double t = 0.0;
            if ((rc = b.dot(V[l], V[i], &t))) return rc;
            if ((rc = b.lincomb(V[i], true, V[l], -t))) return rc;
        }
        double r2 = 0.0;
        if ((rc = b.dot(V[i], V[i], &r2))) return rc;
        if (!(r2 > 1e-300)) return b.fail(EDK_ERR_ZERO_START, "block lanczos: dependent start vectors");
        if ((rc = b.lincomb(V[i], false, V[i], 1.0 / std::sqrt(r2)))) return rc;
    }
    return EDK_OK;
}

}  // namespace

extern "C" int edk_block_lanczos(edk_h *h, const edk_block_opts *o, double *E_host, void *vecs_dev, int32_t *niter,
                                 int32_t *converged)
{
    if (!h || !o || !E_host || !niter || !converged) return EDK_ERR_INVALID;
    Block b;
    b.h = h;
    b.ctx = edk_internal_h_ctx(h);
    b.st = edk_internal_stream(b.ctx);
    if (o->block < 1 || o->block > kMaxBlock || o->neigen < 1 || o->neigen > 64 || o->nitermax < 1)
        return b.fail(EDK_ERR_INVALID, "block lanczos: block 1..4, neigen 1..64, nitermax >= 1");
    int64_t dim = 0;
    edk_h_dims(h, &dim, nullptr, nullptr);
    b.n = dim;
    b.p = (int)std::min<int64_t>(o->block, dim);
    const int p = b.p;
    const int ne = (int)std::min<int64_t>(o->neigen, dim);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    b.grid = sms * 4;
    b.scratch = DBuf(sizeof(double) * ((size_t)b.grid * 4 + 8) + 64);
    if (!b.scratch.p) return b.fail(EDK_ERR_NOMEM, "block lanczos scratch");
    b.partials = b.scratch.d();
    b.out = b.partials + (size_t)b.grid * 4;
    b.counter = reinterpret_cast<unsigned *>(b.out + 6);
    int rc;
    if ((rc = b.cuda(cudaMemset(b.counter, 0, 16), "memset"))) return rc;
    std::vector<double> tab(10001);
    if (o->ran_tab) std::memcpy(tab.data(), o->ran_tab, sizeof(double) * 10001);
    else edk_default_ran_tab(tab.data());
    DBuf tab_d(sizeof(double) * 10001);
    if (!tab_d.p) return b.fail(EDK_ERR_NOMEM, "block lanczos table");
    if ((rc = b.cuda(cudaMemcpy(tab_d.p, tab.data(), sizeof(double) * 10001, cudaMemcpyHostToDevice), "h2d"))) return rc;
    const size_t vb = sizeof(double) * (size_t)dim;
    std::vector<DBuf> bufs(3 * p);
    for (auto &x : bufs) {
        x = DBuf(vb);
        if (!x.p) return b.fail(EDK_ERR_NOMEM, "block lanczos vectors");
    }
    double *V[3][kMaxBlock];
    for (int s = 0; s < 3; ++s)
        for (int i = 0; i < p; ++i) V[s][i] = bufs[s * p + i].d();
    const int K = (int)std::min<int64_t>(o->nitermax, std::max<int64_t>(1, dim / p));
    const int check = std::max(1, o->check_every);
    std::vector<double> A((size_t)K * p * p), B((size_t)(K + 1) * p * p, 0.0);
    std::vector<double> w, Y, wprev;
    int jdone = 0, conv = 0;
    auto ritz = [&](int j, std::vector<double> &wo, std::vector<double> &Yo) {
        const int m = j * p;
        std::vector<double> T((size_t)m * m, 0.0);
        for (int s = 0; s < j; ++s)
            for (int r = 0; r < p; ++r)
                for (int c = 0; c < p; ++c) {
                    T[(size_t)(s * p + r) * m + s * p + c] = A[(size_t)s * p * p + r * p + c];
                    if (s + 1 < j) {
                        // block (s+1, s) = B_{s+2}[r][c] (1-based): row (s+1)p+r, column s p+c
                        const double v = B[(size_t)(s + 1) * p * p + r * p + c];
                        T[(size_t)((s + 1) * p + r) * m + s * p + c] = v;
                        T[(size_t)(s * p + c) * m + (s + 1) * p + r] = v;
                    }
                }
        dense_lowest(m, T, std::min(ne, m), wo, Yo);
    };
    // ---- pass 1 ----
    if ((rc = block_start(b, tab_d.d(), V[1]))) return rc;
    int cur = 1, prev = 0, next = 2;
    bool exhausted = false;
    for (int j = 0; j < K; ++j) {
        // B[j] holds B_{j+1} (1-based) of the block feeding step j; B[0] unused
        rc = block_step(b, V[prev], V[cur], V[next], &B[(size_t)j * p * p], j == 0, &A[(size_t)j * p * p],
                        &B[(size_t)(j + 1) * p * p]);
        jdone = j + 1;
        if (rc == EDK_KRYLOV_EXHAUSTED) { exhausted = true; break; }
        if (rc) return rc;
        if ((j + 1) % check == 0 || j + 1 == K) {
            ritz(j + 1, w, Y);
            if ((int)wprev.size() == (int)w.size() && (j + 1) * p >= ne) {
                bool ok = true;
                for (size_t e = 0; e < w.size(); ++e) ok = ok && std::fabs(w[e] - wprev[e]) < o->tolerance;
                if (ok) { conv = 1; break; }
            }
            wprev = w;
        }
        const int t = prev;
        prev = cur;
        cur = next;
        next = t;
    }
    if (w.empty() || (int)(w.size()) != std::min(ne, jdone * p) || exhausted || !conv) ritz(jdone, w, Y);
    const int nk = (int)w.size();
    for (int e = 0; e < nk; ++e) E_host[e] = w[e];
    *niter = jdone;
    *converged = conv || exhausted;
    if (!vecs_dev) return EDK_OK;
    // ---- pass 2: replay and accumulate psi_e = sum_j V_j Y_j[:, e] ----
    const int m = jdone * p;
    double *vecs = static_cast<double *>(vecs_dev);
    if ((rc = b.cuda(cudaMemsetAsync(vecs, 0, vb * nk, b.st), "memset"))) return rc;
    if ((rc = block_start(b, tab_d.d(), V[1]))) return rc;
    cur = 1; prev = 0; next = 2;
    std::vector<double> Aj(p * p), Bn(p * p);
    for (int j = 0; j < jdone; ++j) {
        for (int e = 0; e < nk; ++e) {
            double c[kMaxBlock];
            for (int l = 0; l < p; ++l) c[l] = Y[(size_t)(j * p + l) * nk + e];
            if ((rc = b.combo(vecs + (size_t)e * dim, true, V[cur], c))) return rc;
        }
        if (j + 1 == jdone) break;
        rc = block_step(b, V[prev], V[cur], V[next], &B[(size_t)j * p * p], j == 0, Aj.data(), Bn.data());
        if (rc) return rc;
        const int t = prev;
        prev = cur;
        cur = next;
        next = t;
    }
    (void)m;
    // normalise
    for (int e = 0; e < nk; ++e) {
        double r2 = 0.0;
        if ((rc = b.dot(vecs + (size_t)e * dim, vecs + (size_t)e * dim, &r2))) return rc;
        if (r2 > 0.0 && (rc = b.lincomb(vecs + (size_t)e * dim, false, vecs + (size_t)e * dim, 1.0 / std::sqrt(r2))))
            return rc;
    }
    return EDK_OK;
}
