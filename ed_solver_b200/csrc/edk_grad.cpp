// Adjoint entry points: parameter gradients of E0 and of the Green functions.
//
// E0: Hellmann-Feynman, dE0/dtheta = <psi|dH/dtheta|psi>.
// G:  G_c(z) = b1^2 [ (z - ph (T - E0))^-1 ]_11 with T the Lanczos tridiagonal
//     of the start vector phi = C|psi> (compute_dynamic_cpu,
//     green_class_compute_dynamic.f90:191-334; b1 = |phi|).  The gradient is
//     taken exactly for the K-step recurrence (one_step_Lanczos_fast,
//     Lanczos_plain.f90:247-302):
//       w_k = H v_k - b_k v_{k-1},  a_k = <w_k, v_k>,  r_k = w_k - a_k v_k,
//       b_{k+1} = |r_k|,  v_{k+1} = r_k / b_{k+1}.
//     The continued fraction's vector-Jacobian product gives abar_k, bbar_k
//     and E0bar on the host; the recurrence is then reversed step by step
//     (one H*w product and one bilinear <wbar_k|dH|v_k> per step), with the
//     Lanczos vectors recomputed from checkpoints every m steps (m ~ sqrt(2K)).
//     The start-vector cotangent goes back through C^T (the same c/c+ map with
//     dagger flipped) to psibar.
// psi: psi is the normalised lowest eigenvector; its cotangent psibar adds
//     -<lambda|dH/dtheta|psi> with (H - E0) lambda = (1 - |psi><psi|) psibar,
//     solved by conjugate gradients on the complement of psi.
// All vectors and arithmetic are FP64.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "edk_grad.h"
#include "edk_internal.h"

extern "C" {
cudaStream_t edk_internal_stream(edk_ctx *ctx);
int edk_internal_fail(edk_ctx *ctx, int code, const char *msg);
void edk_internal_count(edk_ctx *ctx, int64_t h2d, int64_t d2h);
edk_ctx *edk_internal_h_ctx(edk_h *h);
void edk_internal_h_info(const edk_h *h, int *nc, int *nb, int *nup, int *ndn);
void edk_internal_add_launches(edk_ctx *ctx, int64_t n);
int edk_internal_h_sibling(edk_h *h, int nup, int ndn, edk_h **out);
const uint64_t *edk_internal_h_states(const edk_h *h, int spin);
int edk_internal_h_is_sz(const edk_h *h);
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

struct HDel {
    void operator()(edk_h *h) const { if (h) edk_h_destroy(h); }
};
using HPtr = std::unique_ptr<edk_h, HDel>;

// Jordan-Wigner sign of moving one electron between orbitals a and b of the
// same spin: parity of the occupied orbitals strictly between them.
int hop_sign(uint64_t s, int a, int b)
{
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    if (hi - lo < 2) return 1;
    const uint64_t mask = ((1ull << hi) - 1ull) & ~((1ull << (lo + 1)) - 1ull);
    return (__builtin_popcountll(s & mask) & 1) ? -1 : 1;
}

// Per-sector device data of the parameter operators and the reduction scratch.
struct Ops {
    edk_ctx *ctx = nullptr;
    cudaStream_t st = nullptr;
    int64_t dup = 0, ddn = 0, dim = 0;
    int np = 0, grid = 0;
    DBuf st_up, st_dn, params, scratch;
    std::vector<DBuf> maps;
    double *partials = nullptr, *out = nullptr;
    unsigned *counter = nullptr;
    int fail(int code, const char *msg) { return edk_internal_fail(ctx, code, msg); }
    int cuda(cudaError_t e, const char *where)
    {
        if (e == cudaSuccess) return EDK_OK;
        char buf[256];
        snprintf(buf, sizeof buf, "%s: %s", where, cudaGetErrorString(e));
        return fail(e == cudaErrorMemoryAllocation ? EDK_ERR_NOMEM : EDK_ERR_CUDA, buf);
    }
};

// Map of the symmetric hop c+_p c_q + c+_q c_p on one spin's basis:
// (rank of the target + 1) * sign, 0 where the hop does not apply.
int hop_map(const uint64_t *states, int64_t n, int p, int q, std::vector<int32_t> &map)
{
    map.assign(n, 0);
    const uint64_t bp = 1ull << p, bq = 1ull << q;
    for (int64_t i = 0; i < n; ++i) {
        const uint64_t s = states[i];
        const bool hp = (s & bp) != 0, hq = (s & bq) != 0;
        if (hp == hq) continue;
        const uint64_t t = s ^ bp ^ bq;
        const uint64_t *it = std::lower_bound(states, states + n, t);
        if (it == states + n || *it != t) return EDK_ERR_INVALID;
        map[i] = (int32_t)((it - states) + 1) * hop_sign(s, p, q);
    }
    return EDK_OK;
}

int ops_setup(edk_h *h, int np, const edk_param *prm, Ops &o)
{
    o.ctx = edk_internal_h_ctx(h);
    o.st = edk_internal_stream(o.ctx);
    if (np < 1 || np > kMaxGradParams || !prm) return o.fail(EDK_ERR_INVALID, "1..64 parameters");
    if (edk_internal_h_is_sz(h)) return o.fail(EDK_ERR_UNSUPPORTED, "parameter gradients of a Nambu sector");
    int nc, nb, nup, ndn;
    edk_internal_h_info(h, &nc, &nb, &nup, &ndn);
    edk_h_dims(h, &o.dim, &o.dup, &o.ddn);
    o.np = np;
    const int ns = nc + nb;
    if (ns > 32) return o.fail(EDK_ERR_UNSUPPORTED, "gradients need at most 32 orbitals per spin");
    const uint64_t *su = edk_internal_h_states(h, 0), *sd = edk_internal_h_states(h, 1);
    std::vector<uint32_t> u32(su, su + o.dup), d32(sd, sd + o.ddn);
    int rc;
    o.st_up = DBuf(sizeof(uint32_t) * std::max<int64_t>(o.dup, 1));
    o.st_dn = DBuf(sizeof(uint32_t) * std::max<int64_t>(o.ddn, 1));
    if (!o.st_up.p || !o.st_dn.p) return o.fail(EDK_ERR_NOMEM, "gradient tables");
    if ((rc = o.cuda(cudaMemcpy(o.st_up.p, u32.data(), sizeof(uint32_t) * o.dup, cudaMemcpyHostToDevice), "h2d")))
        return rc;
    if ((rc = o.cuda(cudaMemcpy(o.st_dn.p, d32.data(), sizeof(uint32_t) * o.ddn, cudaMemcpyHostToDevice), "h2d")))
        return rc;
    std::vector<ParamDev> pd(np);
    std::vector<int32_t> map;
    for (int q = 0; q < np; ++q) {
        const edk_param &p = prm[q];
        ParamDev &d = pd[q];
        d.mapu = d.mapd = nullptr;
        d.bq = 0;
        int a = -1, b = -1;
        if (p.kind == EDK_PARAM_EC) {
            if (p.i < 0 || p.i >= nc || p.j < 0 || p.j >= nc) return o.fail(EDK_ERR_INVALID, "Ec index");
            a = nb + p.i; b = nb + p.j;
        } else if (p.kind == EDK_PARAM_EB) {
            if (p.i < 0 || p.i >= nb || p.j < 0 || p.j >= nb) return o.fail(EDK_ERR_INVALID, "Eb index");
            a = p.i; b = p.j;
        } else if (p.kind == EDK_PARAM_VBC) {
            if (p.i < 0 || p.i >= nb || p.j < 0 || p.j >= nc) return o.fail(EDK_ERR_INVALID, "Vbc index");
            a = p.i; b = nb + p.j;
        } else if (p.kind == EDK_PARAM_U) {
            if (p.i < 0 || p.i >= nc || p.j < 0 || p.j >= nc) return o.fail(EDK_ERR_INVALID, "U index");
            a = nb + std::min(p.i, p.j); b = nb + std::max(p.i, p.j);
        } else {
            return o.fail(EDK_ERR_INVALID, "parameter kind");
        }
        if (p.kind != EDK_PARAM_U && (p.spin < 0 || p.spin > 2)) return o.fail(EDK_ERR_INVALID, "parameter spin");
        d.spin_mask = p.kind == EDK_PARAM_U ? 3 : (p.spin == 2 ? 3 : 1 << p.spin);
        d.bp = 1u << a;
        d.bq = 1u << b;
        if (p.kind == EDK_PARAM_U) {
            d.kind = a == b ? kParamDouble : kParamPair;
        } else if (a == b) {
            d.kind = kParamNumber;
        } else {
            d.kind = kParamHop;
            for (int s = 0; s < 2; ++s) {
                if (!((d.spin_mask >> s) & 1)) continue;
                const int64_t n = s == 0 ? o.dup : o.ddn;
                if (hop_map(s == 0 ? su : sd, n, a, b, map)) return o.fail(EDK_ERR_INVALID, "hop map");
                o.maps.emplace_back(sizeof(int32_t) * std::max<int64_t>(n, 1));
                if (!o.maps.back().p) return o.fail(EDK_ERR_NOMEM, "gradient maps");
                if ((rc = o.cuda(cudaMemcpy(o.maps.back().p, map.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice),
                                 "h2d")))
                    return rc;
                (s == 0 ? d.mapu : d.mapd) = static_cast<const int32_t *>(o.maps.back().p);
            }
        }
    }
    o.params = DBuf(sizeof(ParamDev) * np);
    if (!o.params.p) return o.fail(EDK_ERR_NOMEM, "gradient params");
    if ((rc = o.cuda(cudaMemcpy(o.params.p, pd.data(), sizeof(ParamDev) * np, cudaMemcpyHostToDevice), "h2d")))
        return rc;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    o.grid = sms * 4;
    const size_t nq = std::max(np, 4);
    o.scratch = DBuf(sizeof(double) * ((size_t)o.grid * nq + nq + 4) + 64);
    if (!o.scratch.p) return o.fail(EDK_ERR_NOMEM, "gradient scratch");
    o.partials = o.scratch.d();
    o.out = o.partials + (size_t)o.grid * nq;
    o.counter = reinterpret_cast<unsigned *>(o.out + nq + 2);
    if ((rc = o.cuda(cudaMemset(o.counter, 0, 16), "memset"))) return rc;
    edk_internal_count(o.ctx, (int64_t)(sizeof(uint32_t) * (o.dup + o.ddn) + sizeof(ParamDev) * np), 0);
    return EDK_OK;
}

// <a|dH_q|b> for every parameter, to the host.
int ops_bilinear(Ops &o, const double *a, const double *b, double *out_host)
{
    int rc = o.cuda(launch_bilinear(o.dup, o.ddn, a, b, static_cast<const uint32_t *>(o.st_up.p),
                                    static_cast<const uint32_t *>(o.st_dn.p), o.np,
                                    static_cast<const ParamDev *>(o.params.p), o.partials, o.counter, o.out, o.grid,
                                    o.st),
                    "bilinear kernel");
    edk_internal_add_launches(o.ctx, 1);
    if (rc) return rc;
    if ((rc = o.cuda(cudaMemcpyAsync(out_host, o.out, sizeof(double) * o.np, cudaMemcpyDeviceToHost, o.st), "d2h")))
        return rc;
    return o.cuda(cudaStreamSynchronize(o.st), "sync");
}

// Vector helpers on the sector of `o` (length o.dim).
struct Vec {
    Ops &o;
    int lincomb(double *out, bool acc, const double *x0, double c0, const double *x1 = nullptr, double c1 = 0,
                const double *x2 = nullptr, double c2 = 0, const double *x3 = nullptr, double c3 = 0)
    {
        edk_internal_add_launches(o.ctx, 1);
        return o.cuda(launch_lincomb(o.dim, out, acc, x0, c0, x1, c1, x2, c2, x3, c3, o.grid, o.st), "lincomb");
    }
    // up to 4 dot products in one pass, to the host
    int dots(double *res, const double *x0, const double *y0, const double *x1 = nullptr, const double *y1 = nullptr,
             const double *x2 = nullptr, const double *y2 = nullptr, const double *x3 = nullptr,
             const double *y3 = nullptr)
    {
        edk_internal_add_launches(o.ctx, 1);
        int rc = o.cuda(launch_dots(o.dim, x0, y0, x1, y1, x2, y2, x3, y3, o.partials, o.counter, o.out, o.grid, o.st),
                        "dots");
        if (rc) return rc;
        double t[4];
        if ((rc = o.cuda(cudaMemcpyAsync(t, o.out, sizeof t, cudaMemcpyDeviceToHost, o.st), "d2h"))) return rc;
        if ((rc = o.cuda(cudaStreamSynchronize(o.st), "sync"))) return rc;
        const int n = x3 ? 4 : x2 ? 3 : x1 ? 2 : 1;
        for (int i = 0; i < n; ++i) res[i] = t[i];
        return EDK_OK;
    }
};

// ---- continued-fraction VJP (host) ----------------------------------------
// G(z) = s u_1 with (z - ph (T - e0)) u = e1, s = b1^2; al[k] (0-based) are the
// diagonal, be[k] (k = 1..K-1) couples levels k-1 and k.
void cf_vjp(int K, const double *al, const double *be, double b1, double e0, double ph, int nw, const double *wn,
            const double *gbar, std::vector<double> &abar, std::vector<double> &bbar, double &b1bar, double &e0bar,
            double *G_out)
{
    using cd = std::complex<double>;
    abar.assign(K, 0.0);
    bbar.assign(K + 1, 0.0);
    b1bar = 0.0;
    e0bar = 0.0;
    const double s = b1 * b1;
    std::vector<cd> d(K), u(K), cp(K), dp(K);
    for (int w = 0; w < nw; ++w) {
        const cd z(0.0, wn[w]);
        // tridiagonal solve (Thomas): diagonal z - ph (a_k - e0), off-diagonal -ph b_k
        for (int k = 0; k < K; ++k) d[k] = z - ph * (al[k] - e0);
        cd denom = d[0];
        cp[0] = K > 1 ? cd(-ph * be[1]) / denom : cd(0.0);
        dp[0] = cd(1.0) / denom;
        for (int k = 1; k < K; ++k) {
            const cd off = -ph * be[k];
            denom = d[k] - off * cp[k - 1];
            cp[k] = k + 1 < K ? cd(-ph * be[k + 1]) / denom : cd(0.0);
            dp[k] = (cd(0.0) - off * dp[k - 1]) / denom;
        }
        u[K - 1] = dp[K - 1];
        for (int k = K - 2; k >= 0; --k) u[k] = dp[k] - cp[k] * u[k + 1];
        const cd f = u[0];
        if (G_out) {
            G_out[2 * w] = (s * f).real();
            G_out[2 * w + 1] = (s * f).imag();
        }
        const cd gc = std::conj(cd(gbar[2 * w], gbar[2 * w + 1]));
        cd uu(0.0);
        for (int k = 0; k < K; ++k) {
            abar[k] += (gc * s * ph * u[k] * u[k]).real();
            uu += u[k] * u[k];
            if (k + 1 < K) bbar[k + 1] += (gc * s * 2.0 * ph * u[k] * u[k + 1]).real();
        }
        e0bar += (gc * s * (-ph) * uu).real();
        b1bar += (gc * 2.0 * b1 * f).real();
    }
}

// Forward Lanczos of phi (K steps or until breakdown) keeping checkpoints, CF
// VJP, then the reverse sweep.  Adds to theta_bar (target-sector parameters),
// writes phibar (target sector) and returns the e0bar of this chain.
int chain_vjp(edk_h *ht, Ops &o, const double *phi, int K, double e0, double ph, int nw, const double *wn,
              const double *gbar, double *theta_bar, double *phibar, double &e0bar_out, double *G_out,
              edk_grad_stats *stats)
{
    Vec v{o};
    const int64_t n = o.dim;
    const size_t vb = sizeof(double) * (size_t)n;
    int rc;
    // ---- forward ----
    double nrm2 = 0.0;
    if ((rc = v.dots(&nrm2, phi, phi))) return rc;
    const double b1 = std::sqrt(nrm2);
    if (!(b1 > 1e-300)) return o.fail(EDK_ERR_ZERO_START, "gradient: zero start vector");
    K = (int)std::min<int64_t>(K, n);
    const int m = std::max(2, (int)std::ceil(std::sqrt(2.0 * K)));
    const int nseg = (K + m - 1) / m;
    std::vector<DBuf> ck(2 * nseg);       // (v_{s-1}, v_s) at segment starts s = 1 + j m
    DBuf va(vb), vbuf(vb), vc(vb), hv(vb);
    if (!va.p || !vbuf.p || !vc.p || !hv.p) return o.fail(EDK_ERR_NOMEM, "gradient vectors");
    double *vkm1 = va.d(), *vk = vbuf.d(), *vnext = vc.d();
    if ((rc = o.cuda(cudaMemsetAsync(vkm1, 0, vb, o.st), "memset"))) return rc;
    if ((rc = v.lincomb(vk, false, phi, 1.0 / b1))) return rc;
    std::vector<double> al(K + 1, 0.0), be(K + 2, 0.0);   // al[k-1] = a_k; be[k] = b_k (be[1] = b1)
    be[1] = b1;
    int Keff = K;
    for (int k = 1; k <= K; ++k) {
        if ((k - 1) % m == 0) {
            const int j = (k - 1) / m;
            ck[2 * j] = DBuf(vb);
            ck[2 * j + 1] = DBuf(vb);
            if (!ck[2 * j].p || !ck[2 * j + 1].p) return o.fail(EDK_ERR_NOMEM, "gradient checkpoints");
            if ((rc = o.cuda(cudaMemcpyAsync(ck[2 * j].p, vkm1, vb, cudaMemcpyDeviceToDevice, o.st), "copy"))) return rc;
            if ((rc = o.cuda(cudaMemcpyAsync(ck[2 * j + 1].p, vk, vb, cudaMemcpyDeviceToDevice, o.st), "copy")))
                return rc;
        }
        if ((rc = edk_hmult(ht, EDK_F64, n, vk, hv.p))) return rc;
        // w = H v_k - b_k v_{k-1}; a_k = <w, v_k>
        if ((rc = v.lincomb(hv.d(), true, vkm1, -be[k]))) return rc;
        double a = 0.0;
        if ((rc = v.dots(&a, hv.d(), vk))) return rc;
        al[k - 1] = a;
        // r = w - a v_k; b_{k+1} = |r|; v_{k+1} = r / b_{k+1}
        if ((rc = v.lincomb(vnext, false, hv.d(), 1.0, vk, -a))) return rc;
        double r2 = 0.0;
        if ((rc = v.dots(&r2, vnext, vnext))) return rc;
        const double bn = std::sqrt(std::max(r2, 0.0));
        be[k + 1] = bn;
        if (stats) stats->forward_steps++;
        if (!(bn > 1e-25) || k == K) {
            Keff = k;
            break;
        }
        if ((rc = v.lincomb(vnext, false, vnext, 1.0 / bn))) return rc;
        std::swap(vkm1, vk);
        std::swap(vk, vnext);
    }
    const bool has_next = be[Keff + 1] > 1e-25;
    va = DBuf();   // the forward vectors are not needed any more
    vbuf = DBuf();
    vc = DBuf();
    hv = DBuf();
    // ---- continued fraction and its VJP ----
    std::vector<double> abar, bbar;
    double b1bar = 0.0, e0bar = 0.0;
    cf_vjp(Keff, al.data(), be.data() + 1, b1, e0, ph, nw, wn, gbar, abar, bbar, b1bar, e0bar, G_out);
    // bbar[k] of the 0-based helper is the adjoint of b_{k+1} here
    std::vector<double> bb(Keff + 2, 0.0);
    for (int k = 1; k < Keff; ++k) bb[k + 1] = bbar[k];
    bb[1] = b1bar;
    // ---- reverse sweep over segments, last first ----
    const int mseg = m + 2;
    std::vector<DBuf> seg(mseg);
    for (auto &sg : seg) {
        sg = DBuf(vb);
        if (!sg.p) return o.fail(EDK_ERR_NOMEM, "gradient segment");
    }
    if (stats) stats->stored_vectors = std::max<int32_t>(stats->stored_vectors, 2 * nseg + mseg + 4);
    DBuf vbn_b(vb), vbc_b(vb), wbar_b(vb), rbar_b(vb);
    if (!vbn_b.p || !vbc_b.p || !wbar_b.p || !rbar_b.p) return o.fail(EDK_ERR_NOMEM, "gradient adjoints");
    double *vbn = vbn_b.d(), *vbc = vbc_b.d(), *wbar = wbar_b.d(), *rbar = rbar_b.d();
    if ((rc = o.cuda(cudaMemsetAsync(vbn, 0, vb, o.st), "memset"))) return rc;   // vbar_{Keff+1} = 0
    if ((rc = o.cuda(cudaMemsetAsync(vbc, 0, vb, o.st), "memset"))) return rc;   // vbar_{Keff} (partial)
    std::vector<double> tb(o.np);
    const int jlast = (Keff - 1) / m;
    for (int j = jlast; j >= 0; --j) {
        const int s0 = 1 + j * m, e1 = std::min(s0 + m - 1, Keff);
        // replay: seg[i] = v_{s0-1+i}
        if ((rc = o.cuda(cudaMemcpyAsync(seg[0].p, ck[2 * j].p, vb, cudaMemcpyDeviceToDevice, o.st), "copy")))
            return rc;
        if ((rc = o.cuda(cudaMemcpyAsync(seg[1].p, ck[2 * j + 1].p, vb, cudaMemcpyDeviceToDevice, o.st), "copy")))
            return rc;
        for (int k = s0; k <= e1; ++k) {
            const int i = k - (s0 - 1);
            if (k == Keff && !has_next) {
                if ((rc = o.cuda(cudaMemsetAsync(seg[i + 1].p, 0, vb, o.st), "memset"))) return rc;
                continue;
            }
            if ((rc = edk_hmult(ht, EDK_F64, n, seg[i].p, seg[i + 1].p))) return rc;
            if ((rc = v.lincomb(seg[i + 1].d(), true, seg[i - 1].d(), -be[k], seg[i].d(), -al[k - 1]))) return rc;
            if ((rc = v.lincomb(seg[i + 1].d(), false, seg[i + 1].d(), 1.0 / be[k + 1]))) return rc;
            if (stats) stats->replay_steps++;
        }
        for (int k = e1; k >= s0; --k) {
            const int i = k - (s0 - 1);
            const double *vkp = seg[i + 1].d(), *vkk = seg[i].d(), *vkm = seg[i - 1].d();
            const double ak = al[k - 1], bk = be[k], bk1 = be[k + 1];
            bool have_r = false;
            if (k < Keff) {
                // rbar = vbar_{k+1} / b_{k+1} + (bb_{k+1} - <vbar_{k+1}, v_{k+1}> / b_{k+1}) v_{k+1}
                double d1 = 0.0;
                if ((rc = v.dots(&d1, vbn, vkp))) return rc;
                if ((rc = v.lincomb(rbar, false, vbn, 1.0 / bk1, vkp, bb[k + 1] - d1 / bk1))) return rc;
                have_r = true;
            }
            // abar' = abar_k - <rbar, v_k>; wbar = rbar + abar' v_k
            double d2 = 0.0;
            if (have_r && (rc = v.dots(&d2, rbar, vkk))) return rc;
            const double ab = abar[k - 1] - d2;
            if (have_r) {
                if ((rc = v.lincomb(wbar, false, rbar, 1.0, vkk, ab))) return rc;
                // vbar_k += -a_k rbar + abar' w_k,  w_k = b_{k+1} v_{k+1} + a_k v_k
                if ((rc = v.lincomb(vbc, true, rbar, -ak, vkp, ab * bk1, vkk, ab * ak))) return rc;
            } else {
                if ((rc = v.lincomb(wbar, false, vkk, ab))) return rc;
                if ((rc = v.lincomb(vbc, true, vkp, ab * bk1, vkk, ab * ak))) return rc;
            }
            // vbar_k += H wbar
            if ((rc = edk_hmult(ht, EDK_F64, n, wbar, rbar))) return rc;
            if ((rc = v.lincomb(vbc, true, rbar, 1.0))) return rc;
            // theta_bar += <wbar| dH |v_k>
            if ((rc = ops_bilinear(o, wbar, vkk, tb.data()))) return rc;
            for (int q = 0; q < o.np; ++q) theta_bar[q] += tb[q];
            // bb_k -= <wbar, v_{k-1}>; vbar_{k-1} starts at -b_k wbar
            if (k >= 2) {
                double d3 = 0.0;
                if ((rc = v.dots(&d3, wbar, vkm))) return rc;
                bb[k] -= d3;
            }
            std::swap(vbn, vbc);
            if ((rc = v.lincomb(vbc, false, wbar, -bk))) return rc;
            if (stats) stats->reverse_steps++;
        }
    }
    // vbn = vbar_1; seg[1] = v_1 (replay of the first segment).  v_1 = phi / b1, b1 = |phi|:
    // phibar = (vbar_1 - <vbar_1, v_1> v_1) / b1 + bb_1 v_1
    double d4 = 0.0;
    if ((rc = v.dots(&d4, vbn, seg[1].d()))) return rc;
    if ((rc = v.lincomb(phibar, false, vbn, 1.0 / b1, seg[1].d(), -d4 / b1 + bb[1]))) return rc;
    e0bar_out = e0bar;
    return EDK_OK;
}

}  // namespace

extern "C" {

int edk_dh_bilinear(edk_h *h, const void *a_dev, const void *b_dev, int32_t np, const edk_param *params,
                    double *out_host)
{
    if (!h || !a_dev || !b_dev || !out_host) return EDK_ERR_INVALID;
    Ops o;
    int rc = ops_setup(h, np, params, o);
    if (rc) return rc;
    return ops_bilinear(o, static_cast<const double *>(a_dev), static_cast<const double *>(b_dev), out_host);
}

int edk_grad_e0(edk_h *h, const void *psi_dev, int32_t np, const edk_param *params, double *grad_host)
{
    if (!h || !psi_dev || !grad_host) return EDK_ERR_INVALID;
    Ops o;
    int rc = ops_setup(h, np, params, o);
    if (rc) return rc;
    const double *psi = static_cast<const double *>(psi_dev);
    double n2 = 0.0;
    Vec v{o};
    if ((rc = v.dots(&n2, psi, psi))) return rc;
    if (!(n2 > 0.0)) return o.fail(EDK_ERR_ZERO_START, "zero state vector");
    if ((rc = ops_bilinear(o, psi, psi, grad_host))) return rc;
    for (int q = 0; q < np; ++q) grad_host[q] /= n2;
    return EDK_OK;
}

int edk_grad_green(edk_h *h, const void *psi_dev, double e0, int32_t nchain, const edk_green_spec *chains,
                   int32_t nitergreen, int32_t nw, const double *wn_host, const double *gbar_host, double e0bar,
                   int32_t np, const edk_param *params, double cg_tol, double *grad_host, double *G_host,
                   edk_grad_stats *stats)
{
    if (!h || !psi_dev || !grad_host || nchain < 0 || (nchain > 0 && (!chains || !wn_host || !gbar_host)) ||
        (nchain > 0 && (nw < 1 || nitergreen < 1)))
        return EDK_ERR_INVALID;
    if (stats) std::memset(stats, 0, sizeof *stats);
    Ops o;
    int rc = ops_setup(h, np, params, o);
    if (rc) return rc;
    Vec v{o};
    const int64_t n = o.dim;
    const size_t vb = sizeof(double) * (size_t)n;
    int nc, nb, nup, ndn;
    edk_internal_h_info(h, &nc, &nb, &nup, &ndn);
    const int ns = nc + nb;
    // normalised psi
    DBuf psi_b(vb), psibar_b(vb);
    if (!psi_b.p || !psibar_b.p) return o.fail(EDK_ERR_NOMEM, "gradient vectors");
    double n2 = 0.0;
    if ((rc = v.dots(&n2, static_cast<const double *>(psi_dev), static_cast<const double *>(psi_dev)))) return rc;
    if (!(n2 > 0.0)) return o.fail(EDK_ERR_ZERO_START, "zero state vector");
    const double *psi = psi_b.d();
    if ((rc = v.lincomb(psi_b.d(), false, static_cast<const double *>(psi_dev), 1.0 / std::sqrt(n2)))) return rc;
    if ((rc = o.cuda(cudaMemsetAsync(psibar_b.p, 0, vb, o.st), "memset"))) return rc;
    std::vector<double> grad(np, 0.0), tb(np);
    double e0bar_total = e0bar;
    // ---- chains ----
    for (int c = 0; c < nchain; ++c) {
        const edk_green_spec &g = chains[c];
        if (g.spin < 0 || g.spin > 1 || g.site < 0 || g.site >= nc) return o.fail(EDK_ERR_INVALID, "chain spec");
        const int d = g.dagger ? 1 : -1;
        const int tnu = nup + (g.spin == 0 ? d : 0), tnd = ndn + (g.spin == 1 ? d : 0);
        if (tnu < 0 || tnu > ns || tnd < 0 || tnd > ns) {
            if (G_host) std::memset(G_host + (size_t)c * 2 * nw, 0, sizeof(double) * 2 * nw);
            continue;
        }
        edk_h *ht_raw = nullptr;
        if ((rc = edk_internal_h_sibling(h, tnu, tnd, &ht_raw))) return rc;
        HPtr ht(ht_raw);
        Ops ot;
        if ((rc = ops_setup(ht.get(), np, params, ot))) return rc;
        const size_t tvb = sizeof(double) * (size_t)ot.dim;
        DBuf phi(tvb), phibar(tvb);
        if (!phi.p || !phibar.p) return o.fail(EDK_ERR_NOMEM, "gradient vectors");
        int64_t od = 0;
        if ((rc = edk_apply_c(h, EDK_F64, g.site, g.spin, g.dagger ? 1 : 0, g.site2, g.sign2, psi, phi.p, &od)))
            return rc;
        double e0b = 0.0;
        std::vector<double> tg(np, 0.0);
        if ((rc = chain_vjp(ht.get(), ot, phi.d(), nitergreen, e0, g.dagger ? 1.0 : -1.0, nw, wn_host,
                            gbar_host + (size_t)c * 2 * nw, tg.data(), phibar.d(), e0b,
                            G_host ? G_host + (size_t)c * 2 * nw : nullptr, stats)))
            return rc;
        for (int q = 0; q < np; ++q) grad[q] += tg[q];
        e0bar_total += e0b;
        // psibar += C^T phibar (the map with dagger flipped, from the target sector back)
        DBuf back(vb);
        if (!back.p) return o.fail(EDK_ERR_NOMEM, "gradient vectors");
        if ((rc = edk_apply_c(ht.get(), EDK_F64, g.site, g.spin, g.dagger ? 0 : 1, g.site2, g.sign2, phibar.p, back.p,
                              &od)))
            return rc;
        if ((rc = v.lincomb(psibar_b.d(), true, back.d(), 1.0))) return rc;
    }
    // ---- E0 (Hellmann-Feynman) ----
    if ((rc = ops_bilinear(o, psi, psi, tb.data()))) return rc;
    for (int q = 0; q < np; ++q) grad[q] += e0bar_total * tb[q];
    // ---- eigenvector: (H - E0) lambda = P psibar, lambda orthogonal to psi ----
    if (nchain > 0) {
        double pp[2];
        if ((rc = v.dots(pp, psibar_b.d(), psi, psibar_b.d(), psibar_b.d()))) return rc;
        if (pp[1] > 0.0) {
            DBuf x_b(vb), r_b(vb), p_b(vb), ap_b(vb);
            if (!x_b.p || !r_b.p || !p_b.p || !ap_b.p) return o.fail(EDK_ERR_NOMEM, "gradient CG vectors");
            double *x = x_b.d(), *r = r_b.d(), *p = p_b.d(), *ap = ap_b.d();
            if ((rc = o.cuda(cudaMemsetAsync(x, 0, vb, o.st), "memset"))) return rc;
            if ((rc = v.lincomb(r, false, psibar_b.d(), 1.0, psi, -pp[0]))) return rc;
            if ((rc = v.lincomb(p, false, r, 1.0))) return rc;
            double rr = 0.0;
            if ((rc = v.dots(&rr, r, r))) return rc;
            const double rr0 = rr;
            const double tol = cg_tol > 0.0 ? cg_tol : 1e-10;
            int it = 0;
            const int maxit = 20000;
            while (rr > tol * tol * rr0 && it < maxit) {
                if ((rc = edk_hmult(h, EDK_F64, n, p, ap))) return rc;
                // ap = (H - E0) p, projected off psi
                double t[2];
                if ((rc = v.dots(t, ap, psi, p, psi))) return rc;
                if ((rc = v.lincomb(ap, false, ap, 1.0, p, -e0, psi, -(t[0] - e0 * t[1])))) return rc;
                double pap = 0.0;
                if ((rc = v.dots(&pap, p, ap))) return rc;
                if (!(pap > 0.0)) break;
                const double alpha = rr / pap;
                if ((rc = v.lincomb(x, true, p, alpha))) return rc;
                if ((rc = v.lincomb(r, true, ap, -alpha))) return rc;
                double rn = 0.0;
                if ((rc = v.dots(&rn, r, r))) return rc;
                if ((rc = v.lincomb(p, false, r, 1.0, p, rn / rr))) return rc;
                rr = rn;
                ++it;
            }
            if (stats) {
                stats->cg_iterations = it;
                stats->cg_residual = std::sqrt(rr / rr0);
            }
            if ((rc = ops_bilinear(o, x, psi, tb.data()))) return rc;
            for (int q = 0; q < np; ++q) grad[q] -= tb[q];
        }
    }
    std::memcpy(grad_host, grad.data(), sizeof(double) * np);
    return EDK_OK;
}

}  // extern "C"
