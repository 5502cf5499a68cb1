// Host-side construction of the sector data the device kernels consume:
// basis enumeration and ranks (quantum_fermion_hilbert_class.f90:346-421),
// one-body hopping tables in tab_HAIM2 order (HAIM_offdiag_arrays.f90:210-606),
// density-term lists (HAIMupdo.f90:784-829), Hund move tables
// (HAIMupdo.f90:1017-1129), the column-major padded up table with its value
// palette, and the L2-friendly row schedule.
#include "edk_tables.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>

namespace edk {

int64_t binom(int n, int k)
{
    if (k < 0 || k > n || n < 0) return 0;
    int64_t r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

// Gosper's hack walks the integers with a fixed popcount in increasing
// order, which is exactly the order the reference fills sector%state in.
std::vector<uint64_t> enumerate_states(int ns, int np)
{
    std::vector<uint64_t> out;
    if (np < 0 || np > ns) return out;
    out.reserve((size_t)binom(ns, np));
    if (np == 0) { out.push_back(0); return out; }
    const uint64_t limit = 1ull << ns;
    uint64_t s = (np == 64) ? ~0ull : ((1ull << np) - 1ull);
    while (s < limit) {
        out.push_back(s);
        const uint64_t c = s & (~s + 1ull);
        const uint64_t r = s + c;
        s = (((r ^ s) >> 2) / c) | r;
    }
    return out;
}

std::vector<int32_t> rank_table(int ns)
{
    std::vector<int32_t> rank((size_t)1 << ns);
    int32_t count[65] = {0};
    for (uint64_t s = 0; s < ((uint64_t)1 << ns); ++s)
        rank[s] = count[__builtin_popcountll(s)]++;
    return rank;
}

// ---------------------------------------------------------------------------

namespace {

struct HopPattern {
    int tgt, src;     // bits
    double val;       // coefficient of c+_tgt c_src
};

// All one-body hops of one spin species, in the order tab_HAIM2 visits them:
// impurity-impurity (row-major over (i,j), i != j), bath-bath, then for each
// (bath k, impurity c): impurity->bath with Vbc(k,c) and bath->impurity with
// conj(Vbc(k,c)).  Zero entries and |t| <= cutoff are skipped.
std::vector<HopPattern> hop_patterns(const ModelHost &m, int spin)
{
    std::vector<HopPattern> p;
    const int nc = m.nc, nb = m.nb;
    auto keep = [&](double h) { return h != 0.0 && std::fabs(h) > m.cutoff; };
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
            const double h = m.ec[(size_t)spin * nc * nc + i * nc + j];
            if (i != j && keep(h)) p.push_back({nb + i, nb + j, h});
        }
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) {
            const double h = m.eb[(size_t)spin * nb * nb + i * nb + j];
            if (i != j && keep(h)) p.push_back({i, j, h});
        }
    for (int k = 0; k < nb; ++k)
        for (int c = 0; c < nc; ++c) {
            const double h = m.vbc[(size_t)spin * nb * nc + k * nc + c];
            if (!keep(h)) continue;
            p.push_back({k, nb + c, h});
            p.push_back({nb + c, k, h});
        }
    return p;
}

// Sign of c+_tgt c_src on |s> with the Jordan-Wigner string counted above
// each orbital (Fermion_sign, quantum_fermion_ket_class.f90:605-618): the
// two strings cancel except between the two orbitals.
inline int hop_sign(uint64_t s, int a, int b)
{
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    if (hi - lo < 2) return 1;
    const uint64_t mask = ((1ull << hi) - 1ull) & ~((1ull << (lo + 1)) - 1ull);
    return (__builtin_popcountll(s & mask) & 1) ? -1 : 1;
}

}  // namespace

SpinTableHost build_spin_table(const ModelHost &m, int spin, int np, const std::vector<int32_t> &rank)
{
    SpinTableHost t;
    const int ns = m.nc + m.nb;
    t.states = enumerate_states(ns, np);
    const int64_t dim = (int64_t)t.states.size();
    const auto pats = hop_patterns(m, spin);
    t.ptr.assign((size_t)dim + 1, 0);
    t.diag.assign((size_t)dim, 0.0);
    t.imp.assign((size_t)dim, 0);
    for (int64_t i = 0; i < dim; ++i) {
        const uint64_t s = t.states[i];
        for (const auto &p : pats) {
            if (!((s >> p.src) & 1ull) || ((s >> p.tgt) & 1ull)) continue;
            const uint64_t o = (s & ~(1ull << p.src)) | (1ull << p.tgt);
            t.tgt.push_back(rank[o]);
            t.val.push_back(p.val * (double)hop_sign(s, p.tgt, p.src));
        }
        t.ptr[i + 1] = (int32_t)t.tgt.size();
        // diagonal: occupied impurity Ec(c,c), then occupied bath Eb(k,k)
        double d = 0.0;
        for (int c = 0; c < m.nc; ++c)
            if ((s >> (m.nb + c)) & 1ull) d = d + m.ec[(size_t)spin * m.nc * m.nc + c * m.nc + c];
        for (int k = 0; k < m.nb; ++k)
            if ((s >> k) & 1ull) d = d + m.eb[(size_t)spin * m.nb * m.nb + k * m.nb + k];
        t.diag[i] = d;
        t.imp[i] = (uint8_t)((s >> m.nb) & ((1ull << m.nc) - 1ull));
    }
    // Hund moves: one electron from impurity site a to b, a != b
    const int nmove = m.nc * (m.nc - 1);
    t.move.assign((size_t)dim * (nmove > 0 ? nmove : 0), 0);
    for (int64_t i = 0; i < dim && nmove > 0; ++i) {
        const uint64_t s = t.states[i];
        for (int a = 0; a < m.nc; ++a)
            for (int b = 0; b < m.nc; ++b) {
                if (a == b) continue;
                const int pa = m.nb + a, pb = m.nb + b;
                const int idx = a * (m.nc - 1) + (b < a ? b : b - 1);
                if (!((s >> pa) & 1ull) || ((s >> pb) & 1ull)) continue;
                const uint64_t o = (s & ~(1ull << pa)) | (1ull << pb);
                const int sg = hop_sign(o, pa, pb);
                t.move[(size_t)i * nmove + idx] = (rank[o] + 1) * sg;
            }
    }
    // column-major padded copy with a value palette
    int kmax = 0;
    for (int64_t i = 0; i < dim; ++i) kmax = std::max(kmax, t.ptr[i + 1] - t.ptr[i]);
    t.ell_k = kmax;
    std::map<uint64_t, int> pal_index;
    std::vector<double> pal{0.0};
    pal_index[0] = 0;
    bool packed = dim < (1 << 24);
    for (double v : t.val) {
        uint64_t key;
        std::memcpy(&key, &v, 8);
        if (pal_index.count(key)) continue;
        if (pal.size() >= 256) { packed = false; break; }
        pal_index[key] = (int)pal.size();
        pal.push_back(v);
    }
    t.packed = packed;
    t.ell.assign((size_t)kmax * dim, 0);
    if (!packed) t.ell_val.assign((size_t)kmax * dim, 0.0);
    for (int64_t i = 0; i < dim; ++i) {
        const int n = t.ptr[i + 1] - t.ptr[i];
        for (int k = 0; k < kmax; ++k) {
            const size_t slot = (size_t)k * dim + i;
            if (k < n) {
                const int32_t j = t.tgt[t.ptr[i] + k];
                const double v = t.val[t.ptr[i] + k];
                if (packed) {
                    uint64_t key;
                    std::memcpy(&key, &v, 8);
                    t.ell[slot] = (uint32_t)j | ((uint32_t)pal_index[key] << 24);
                } else {
                    t.ell[slot] = (uint32_t)j;
                    t.ell_val[slot] = v;
                }
            } else {
                t.ell[slot] = (uint32_t)i;       // padding: value 0 on the state itself
            }
        }
    }
    if (packed) t.palette = pal;
    // lean copy for the FP32 kernel: per column, the entries contiguous and
    // pre-shifted (target << 14 | palette index << 3), the width rounded up to
    // an even count; per 64-column block the largest hop count
    if (spin == 0 && packed && dim % 2 == 0 && dim < (1 << 18) && kmax <= 16) {
        const int ks = kmax + (kmax & 1);
        t.lean_ks = ks;
        t.lean.assign((size_t)ks * dim, 0);
        t.lean_kw.assign((size_t)(dim + 63) / 64, 0);
        for (int64_t i = 0; i < dim; ++i) {
            const int n = t.ptr[i + 1] - t.ptr[i];
            for (int k = 0; k < ks; ++k) {
                const uint32_t e = k < kmax ? t.ell[(size_t)k * dim + i] : 0u;
                const uint32_t tg = k < n ? (e & 0xFFFFFFu) : (uint32_t)i;
                const uint32_t pi = k < n ? (e >> 24) : 0u;
                t.lean[(size_t)i * ks + k] = (tg << 14) | (pi << 3);
            }
            uint8_t &w = t.lean_kw[(size_t)i / 64];
            w = std::max<uint8_t>(w, (uint8_t)n);
        }
        // blocked copy: entry k of column i at (i/64)*64*ks + k*64 + i%64
        t.lean_b.assign((size_t)(dim + 63) / 64 * 64 * ks, 0);
        for (int64_t i = 0; i < dim; ++i)
            for (int k = 0; k < ks; ++k)
                t.lean_b[(size_t)(i / 64) * 64 * ks + (size_t)k * 64 + (size_t)(i % 64)] = t.lean[(size_t)i * ks + k];
    }
    return t;
}

// Ordered density-density terms per pair of impurity configurations
// (HAIMupdo.f90:784-829): U(c,c) for doubly occupied sites, then for each
// pair c1<c2 with U(c1,c2) != 0 and both sites occupied: U*n1*n2, -JJ for an
// up-up pair, -JJ for a down-down pair.  The second group only exists when U
// has an off-diagonal element.  with_jj = false gives the terms of
// HAIMupdo_multr_split (HAIMupdo.f90:1250-1284), which has no -JJ terms.
void density_terms(const ModelHost &m, std::vector<int32_t> &off, std::vector<double> &coef, bool with_jj)
{
    const int nc = m.nc, ncfg = 1 << nc;
    bool offc = false;
    for (int a = 0; a < nc; ++a)
        for (int b = 0; b < nc; ++b)
            if (a != b && m.u[a * nc + b] != 0.0) offc = true;
    off.assign((size_t)ncfg * ncfg + 1, 0);
    coef.clear();
    for (int cu = 0; cu < ncfg; ++cu)
        for (int cd = 0; cd < ncfg; ++cd) {
            for (int c = 0; c < nc; ++c)
                if (m.u[c * nc + c] != 0.0 && ((cu >> c) & 1) && ((cd >> c) & 1))
                    coef.push_back(m.u[c * nc + c]);
            if (offc)
                for (int s1 = 0; s1 < nc - 1; ++s1) {
                    const int u1 = (cu >> s1) & 1, d1 = (cd >> s1) & 1;
                    if (u1 + d1 == 0) continue;
                    for (int s2 = s1 + 1; s2 < nc; ++s2) {
                        if (m.u[s1 * nc + s2] == 0.0) continue;
                        const int u2 = (cu >> s2) & 1, d2 = (cd >> s2) & 1;
                        if (u2 + d2 == 0) continue;
                        coef.push_back(m.u[s1 * nc + s2] * (double)(u1 + d1) * (double)(u2 + d2));
                        if (with_jj && u1 && u2) coef.push_back(-m.jj[s1 * nc + s2]);
                        if (with_jj && d1 && d2) coef.push_back(-m.jj[s1 * nc + s2]);
                    }
                }
            off[(size_t)cu * ncfg + cd + 1] = (int32_t)coef.size();
        }
}

// Down rows are visited sorted by their state with the impurity bits moved
// below the bath bits.  Rows whose bath parts are close then run together,
// and their down-spin hop partners (which differ in one impurity and one
// bath bit) were touched recently, so more of them hit in L2.
std::vector<int32_t> row_schedule(const std::vector<uint64_t> &states, int nc, int nb)
{
    std::vector<int32_t> order(states.size());
    std::iota(order.begin(), order.end(), 0);
    const uint64_t bath_mask = (nb > 0) ? ((1ull << nb) - 1ull) : 0ull;
    auto key = [&](int32_t i) {
        const uint64_t s = states[i];
        return ((s & bath_mask) << nc) | (s >> nb);
    };
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return key(a) < key(b); });
    return order;
}

}  // namespace edk
