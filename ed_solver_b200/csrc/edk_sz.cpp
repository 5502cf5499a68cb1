// Nambu (Sz) sectors: the host side of HAIMsz (HAIMsz.f90:51-1027).
//
// new_HAIMsz tabulates, per state, QUART_INT_SZ and the quadratic part
// (tab_HAIM2 on the Nambu AIM2, HAIM_offdiag_arrays.f90:210-606); here
// nothing is tabulated per state.  The device kernel (edk_sz.cu) walks, for
// every state, the ordered list of one-body terms c+_tgt c_src built below
// (the order in which tab_HAIM2 or HAIMsz_mult_fly_r visits them), computes
// the target's rank from two small tables (off_h, rank_low), and takes
// QUART_INT_SZ from a table indexed by the impurity configuration.  The
// only per-sector data are 2^ns row offsets.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "edk_internal.h"

namespace edk {

namespace {

struct Buf {
    void *p = nullptr;
    size_t bytes = 0;
    Buf() = default;
    Buf(const Buf &) = delete;
    Buf &operator=(const Buf &) = delete;
    ~Buf() { if (p) cudaFree(p); }
    template <typename T>
    cudaError_t put(const std::vector<T> &v, cudaStream_t st)
    {
        if (p) { cudaFree(p); p = nullptr; bytes = 0; }
        const size_t n = sizeof(T) * (v.empty() ? 1 : v.size());
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) { p = nullptr; return e; }
        bytes = n;
        if (v.empty()) return cudaSuccess;
        e = cudaMemcpyAsync(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return e;
        return cudaStreamSynchronize(st);   // the host vector may go out of scope
    }
    template <typename T> const T *as() const { return static_cast<const T *>(p); }
};

int64_t binom(int n, int k)
{
    if (k < 0 || k > n) return 0;
    int64_t r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

struct Sector {
    SzSectorDev dev;
    Buf row_h, off_h;
};

// Rows of the sector: every high half h with 0 <= npart - |h| <= ns, in
// increasing order, and the rank of each row's first state.
cudaError_t build_sector(int ns, int npart, cudaStream_t st, Sector &S, int64_t &bytes, std::string *err)
{
    const uint32_t nh = 1u << ns;
    std::vector<uint32_t> off(nh, 0u), rows;
    int64_t acc = 0;
    int maxlen = 0;
    for (uint32_t h = 0; h < nh; ++h) {
        const int k = npart - __builtin_popcount(h);
        off[h] = (uint32_t)acc;
        if (k < 0 || k > ns) continue;
        rows.push_back(h);
        const int64_t len = binom(ns, k);
        acc += len;
        if (len > maxlen) maxlen = (int)len;
    }
    if (acc != binom(2 * ns, npart) || acc >= (int64_t(1) << 32)) {
        if (err) *err = "Nambu sector dimension beyond 2^32";
        return cudaErrorInvalidValue;
    }
    cudaError_t e;
    if ((e = S.row_h.put(rows, st)) != cudaSuccess) return e;
    if ((e = S.off_h.put(off, st)) != cudaSuccess) return e;
    bytes += (int64_t)(rows.size() + off.size()) * 4;
    S.dev.npart = npart;
    S.dev.nrows = (int)rows.size();
    S.dev.maxlen = maxlen;
    S.dev.dim = acc;
    S.dev.row_h = S.row_h.as<uint32_t>();
    S.dev.off_h = S.off_h.as<uint32_t>();
    return cudaSuccess;
}

uint32_t between_mask(int a, int b)
{
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    if (hi - lo <= 1) return 0u;
    const uint32_t below_hi = (uint32_t)((uint64_t(1) << hi) - 1u);
    const uint32_t upto_lo = (uint32_t)((uint64_t(1) << (lo + 1)) - 1u);
    return below_hi & ~upto_lo;
}

}  // namespace

struct SzHost {
    int ns = 0, nb = 0, nc = 0;
    double shift = 0.0;
    Buf rank_low, low_states, class_start, terms, diag_bit, diag_e, quart, runs, term_run, ell;
    Sector own;
    std::vector<std::unique_ptr<Sector>> others;
    SzDev dev;
    int64_t bytes = 0;
};

int sz_create(const edk_model_sz *m, int npart, cudaStream_t st, SzHost **out, std::string *err)
{
    *out = nullptr;
    const edk_model &b = m->base;
    const int nc = b.nc, nb = b.nb, ns = nc + nb, NI = 2 * nc, NB = 2 * nb;
    if (nc < 1 || nc > kMaxNc || nb < 0 || ns > kMaxSzNs) {
        *err = "Nambu sector: need 1 <= nc <= 6 and nc + nb <= 16";
        return EDK_ERR_UNSUPPORTED;
    }
    if (npart < 0 || npart > 2 * ns) {
        *err = "Nambu sector: npart outside [0, 2 ns]";
        return EDK_ERR_INVALID;
    }
    if (std::fabs(b.jhund) > 1e-5) {
        *err = "Jhund and Sz basis: not implemented in the reference (HAIMsz.f90:470-473)";
        return EDK_ERR_UNSUPPORTED;
    }
    if (!b.ec || !b.u || (nb > 0 && (!b.eb || !b.vbc))) {
        *err = "Nambu sector: missing model matrices";
        return EDK_ERR_INVALID;
    }
    std::unique_ptr<SzHost> z(new (std::nothrow) SzHost);
    if (!z) return EDK_ERR_NOMEM;
    z->ns = ns;
    z->nb = nb;
    z->nc = nc;

    // ---- Nambu matrices (Nambu_Ec, Nambu_Eb, Nambu_Vbc) and orbital bits ----
    std::vector<double> ecn((size_t)NI * NI, 0.0), ebn((size_t)NB * NB, 0.0), vbcn((size_t)NB * NI, 0.0);
    std::vector<int> ibit(NI), bbit(NB);
    for (int i = 0; i < nc; ++i) {
        ibit[i] = nb + i;
        ibit[nc + i] = ns + nb + i;
        for (int j = 0; j < nc; ++j) {
            ecn[(size_t)i * NI + j] = b.ec[i * nc + j];
            ecn[(size_t)(nc + i) * NI + nc + j] = -b.ec[nc * nc + j * nc + i];
        }
    }
    for (int k = 0; k < nb; ++k) {
        bbit[k] = k;
        bbit[nb + k] = ns + k;
        for (int l = 0; l < nb; ++l) {
            ebn[(size_t)k * NB + l] = b.eb[k * nb + l];
            ebn[(size_t)(nb + k) * NB + nb + l] = -b.eb[nb * nb + l * nb + k];
            if (m->pb) {
                ebn[(size_t)k * NB + nb + l] = m->pb[k * nb + l];
                ebn[(size_t)(nb + k) * NB + l] = m->pb[l * nb + k];
            }
        }
        for (int c = 0; c < nc; ++c) {
            vbcn[(size_t)k * NI + c] = b.vbc[k * nc + c];
            vbcn[(size_t)(nb + k) * NI + nc + c] = -b.vbc[nb * nc + k * nc + c];
            if (m->pvbc) {
                vbcn[(size_t)(nb + k) * NI + c] = m->pvbc[k * nc + c];
                vbcn[(size_t)k * NI + nc + c] = m->pvbc[nb * nc + k * nc + c];
            }
        }
    }
    {
        // energy_global_shift + energy_global_shift2 (impurity_class.f90:1037, bath_class.f90:976)
        double s1 = 0.0, s2 = 0.0;
        for (int c = 0; c < nc; ++c) s1 = s1 + b.ec[nc * nc + c * nc + c];
        for (int k = 0; k < nb; ++k) s2 = s2 + ebn[(size_t)(nb + k) * NB + nb + k];
        z->shift = s1 + (-s2);
    }

    // ---- the ordered one-body terms ----
    std::vector<SzTerm> terms;
    auto add = [&](int tgt_bit, int src_bit, double h) {
        SzTerm t;
        t.src = 1u << src_bit;
        t.tgt = 1u << tgt_bit;
        t.btw = between_mask(src_bit, tgt_bit);
        t.pad = 0u;
        t.h = h;
        terms.push_back(t);
    };
    const double cut = b.cutoff_hamilt_param;
    const bool keep_all = m->on_fly != 0;
    auto kept = [&](double h) { return h != 0.0 && (keep_all || std::fabs(h) > cut); };
    if (!m->on_fly) {
        // tab_HAIM2 (HAIM_offdiag_arrays.f90:448-526): impurity, bath, then per
        // (bath, impurity) pair impurity->bath and bath->impurity
        for (int i = 0; i < NI; ++i)
            for (int j = 0; j < NI; ++j)
                if (i != j && kept(ecn[(size_t)i * NI + j])) add(ibit[i], ibit[j], ecn[(size_t)i * NI + j]);
        for (int i = 0; i < NB; ++i)
            for (int j = 0; j < NB; ++j)
                if (i != j && kept(ebn[(size_t)i * NB + j])) add(bbit[i], bbit[j], ebn[(size_t)i * NB + j]);
        for (int k = 0; k < NB; ++k)
            for (int c = 0; c < NI; ++c) {
                const double h = vbcn[(size_t)k * NI + c];
                if (!kept(h)) continue;
                add(bbit[k], ibit[c], h);
                add(ibit[c], bbit[k], h);
            }
    } else {
        // HAIMsz_mult_fly_r (HAIMsz.f90:686-790): per source orbital its targets
        for (int j = 0; j < NI; ++j)
            for (int i = 0; i < NI; ++i)
                if (i != j && kept(ecn[(size_t)i * NI + j])) add(ibit[i], ibit[j], ecn[(size_t)i * NI + j]);
        for (int j = 0; j < NB; ++j)
            for (int i = 0; i < NB; ++i)
                if (i != j && kept(ebn[(size_t)i * NB + j])) add(bbit[i], bbit[j], ebn[(size_t)i * NB + j]);
        for (int j = 0; j < NI; ++j)
            for (int k = 0; k < NB; ++k)
                if (kept(vbcn[(size_t)k * NI + j])) add(bbit[k], ibit[j], vbcn[(size_t)k * NI + j]);
        for (int k = 0; k < NB; ++k)
            for (int j = 0; j < NI; ++j)
                if (kept(vbcn[(size_t)k * NI + j])) add(ibit[j], bbit[k], vbcn[(size_t)k * NI + j]);
    }
    if ((int)terms.size() > kMaxSzTerms) {
        *err = "Nambu sector: more than 4096 one-body terms";
        return EDK_ERR_UNSUPPORTED;
    }

    // ---- diagonal: occupied impurity Nambu orbitals, then bath (:419-427) ----
    std::vector<uint32_t> dbit;
    std::vector<double> de;
    for (int i = 0; i < NI; ++i) { dbit.push_back(1u << ibit[i]); de.push_back(ecn[(size_t)i * NI + i]); }
    for (int k = 0; k < NB; ++k) { dbit.push_back(1u << bbit[k]); de.push_back(ebn[(size_t)k * NB + k]); }

    // ---- QUART_INT_SZ by impurity configuration (tab_HAIMsz, HAIMsz.f90:133-173) ----
    std::vector<double> quart((size_t)1 << (2 * nc), 0.0);
    {
        std::vector<uint8_t> umask((size_t)nc * nc);
        bool offc = false;
        for (int i = 0; i < nc; ++i)
            for (int j = 0; j < nc; ++j) {
                umask[(size_t)i * nc + j] = b.u[i * nc + j] != 0.0;
                if (i != j && umask[(size_t)i * nc + j]) offc = true;
            }
        for (uint32_t cfg = 0; cfg < quart.size(); ++cfg) {
            auto nocc = [&](int site) { return (int)((cfg >> site) & 1u) + (int)(((cfg >> (nc + site)) & 1u) == 0u); };
            double q = 0.0;
            for (int s1 = 0; s1 < nc; ++s1) {
                const int n1 = nocc(s1);
                if (n1 == 2 && umask[(size_t)s1 * nc + s1]) q = q + b.u[s1 * nc + s1];
                if (offc && n1 != 0)
                    for (int s2 = s1 + 1; s2 < nc; ++s2) {
                        if (!umask[(size_t)s1 * nc + s2]) continue;
                        const double t1 = b.u[s1 * nc + s2] * (double)n1;
                        const double t2 = t1 * (double)nocc(s2);
                        q = q + t2;
                    }
            }
            quart[cfg] = q;
        }
    }

    // ---- rank tables of the low halves ----
    const uint32_t nh = 1u << ns;
    std::vector<int32_t> cstart(ns + 2, 0);
    std::vector<uint16_t> rlow(nh), lst(nh);
    for (uint32_t l = 0; l < nh; ++l) cstart[__builtin_popcount(l) + 1]++;
    for (int k = 0; k <= ns; ++k) cstart[k + 1] += cstart[k];
    {
        std::vector<int32_t> pos(cstart.begin(), cstart.end() - 1);
        for (uint32_t l = 0; l < nh; ++l) {
            const int k = __builtin_popcount(l);
            rlow[l] = (uint16_t)(pos[k] - cstart[k]);
            lst[pos[k]++] = (uint16_t)l;
        }
    }

    // ---- runs of one kind, and the tables of the up-up runs ----
    const uint32_t lowmask = (1u << ns) - 1u;
    std::vector<SzRun> runs;
    std::vector<int32_t> term_run(terms.size());
    for (size_t t = 0; t < terms.size(); ++t) {
        const uint32_t both = terms[t].src | terms[t].tgt;
        const int kind = (both & ~lowmask) == 0u ? 0 : (both & lowmask) == 0u ? 1 : 2;
        if (runs.empty() || runs.back().kind != kind) runs.push_back(SzRun{kind, (int32_t)t, 0, 0, 0});
        runs.back().count++;
        term_run[t] = (int32_t)runs.size() - 1;
    }
    std::vector<uint32_t> ell;
    for (auto &r : runs) {
        if (r.kind != 0) continue;
        std::vector<std::vector<uint32_t>> lists(nh);
        int kmax = 0;
        for (uint32_t p = 0; p < nh; ++p) {
            const uint32_t l = lst[p];
            for (int q = 0; q < r.count; ++q) {
                const SzTerm &tm = terms[(size_t)r.first + q];
                if (!(l & tm.src) || (l & tm.tgt)) continue;
                const uint32_t l2 = l ^ tm.src ^ tm.tgt;
                const uint32_t neg = (uint32_t)(__builtin_popcount(l & tm.btw) & 1);
                lists[p].push_back((uint32_t)rlow[l2] | (neg << 16) | ((uint32_t)q << 17));
            }
            kmax = std::max<int>(kmax, (int)lists[p].size());
        }
        r.kell = kmax;
        r.ell_off = (int64_t)ell.size();
        ell.resize(ell.size() + (size_t)kmax * nh, 0xFFFFFFFFu);
        for (uint32_t p = 0; p < nh; ++p)
            for (size_t q = 0; q < lists[p].size(); ++q) ell[(size_t)r.ell_off + q * nh + p] = lists[p][q];
    }

    cudaError_t e;
    std::string berr;
    if ((e = z->rank_low.put(rlow, st)) != cudaSuccess || (e = z->low_states.put(lst, st)) != cudaSuccess ||
        (e = z->class_start.put(cstart, st)) != cudaSuccess || (e = z->terms.put(terms, st)) != cudaSuccess ||
        (e = z->diag_bit.put(dbit, st)) != cudaSuccess || (e = z->diag_e.put(de, st)) != cudaSuccess ||
        (e = z->quart.put(quart, st)) != cudaSuccess || (e = z->runs.put(runs, st)) != cudaSuccess ||
        (e = z->term_run.put(term_run, st)) != cudaSuccess || (e = z->ell.put(ell, st)) != cudaSuccess ||
        (e = build_sector(ns, npart, st, z->own, z->bytes, &berr)) != cudaSuccess) {
        *err = berr.empty() ? std::string("Nambu sector upload: ") + cudaGetErrorString(e) : berr;
        return e == cudaErrorMemoryAllocation ? EDK_ERR_NOMEM : (berr.empty() ? EDK_ERR_CUDA : EDK_ERR_UNSUPPORTED);
    }
    z->bytes += (int64_t)(rlow.size() * 2 + lst.size() * 2 + cstart.size() * 4 + terms.size() * sizeof(SzTerm) +
                          dbit.size() * 12 + quart.size() * 8 + runs.size() * sizeof(SzRun) +
                          term_run.size() * 4 + ell.size() * 4);
    SzDev &d = z->dev;
    d.ns = ns;
    d.nb = nb;
    d.nc = nc;
    d.order = m->on_fly ? 1 : 0;
    d.sec = z->own.dev;
    d.rank_low = z->rank_low.as<uint16_t>();
    d.low_states = z->low_states.as<uint16_t>();
    d.class_start = z->class_start.as<int32_t>();
    d.nterm = (int)terms.size();
    d.terms = z->terms.as<SzTerm>();
    d.ndiag = (int)dbit.size();
    d.diag_bit = z->diag_bit.as<uint32_t>();
    d.diag_e = z->diag_e.as<double>();
    d.quart = z->quart.as<double>();
    d.nrun = (int)runs.size();
    d.runs = z->runs.as<SzRun>();
    d.term_run = z->term_run.as<int32_t>();
    d.ell = z->ell.as<uint32_t>();
    *out = z.release();
    return EDK_OK;
}

void sz_destroy(SzHost *z) { delete z; }

const SzDev &sz_dev(const SzHost *z) { return z->dev; }

double sz_shift(const SzHost *z) { return z->shift; }

int64_t sz_upload_bytes(const SzHost *z) { return z->bytes; }

int sz_sector(SzHost *z, int npart, cudaStream_t st, const SzSectorDev **out, std::string *err)
{
    if (npart == z->own.dev.npart) { *out = &z->own.dev; return EDK_OK; }
    for (auto &s : z->others)
        if (s->dev.npart == npart) { *out = &s->dev; return EDK_OK; }
    if (npart < 0 || npart > 2 * z->ns) { *err = "Nambu sector: npart outside [0, 2 ns]"; return EDK_ERR_INVALID; }
    std::unique_ptr<Sector> s(new (std::nothrow) Sector);
    if (!s) return EDK_ERR_NOMEM;
    std::string berr;
    cudaError_t e = build_sector(z->ns, npart, st, *s, z->bytes, &berr);
    if (e != cudaSuccess) {
        *err = berr.empty() ? std::string("Nambu sector upload: ") + cudaGetErrorString(e) : berr;
        return e == cudaErrorMemoryAllocation ? EDK_ERR_NOMEM : EDK_ERR_CUDA;
    }
    *out = &s->dev;
    z->others.push_back(std::move(s));
    return EDK_OK;
}

}  // namespace edk
