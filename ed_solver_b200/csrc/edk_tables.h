// Host-side sector data builders (see edk_tables.cpp).
#pragma once

#include <cstdint>
#include <vector>

namespace edk {

struct ModelHost {
    int nc = 0, nb = 0;
    std::vector<double> ec, eb, vbc, u, jj;
    double jhund = 0.0, cutoff = 1e-3;
};

struct SpinTableHost {
    std::vector<uint64_t> states;
    std::vector<int32_t> ptr, tgt;      // CSR in tab_HAIM2 order
    std::vector<double> val, diag;
    std::vector<uint8_t> imp;
    std::vector<int32_t> move;
    int ell_k = 0;
    bool packed = false;
    std::vector<uint32_t> ell;
    std::vector<double> ell_val;
    std::vector<double> palette;
    // lean copy for the FP32 kernel of kind 3 (see SpinTabDev::lean)
    int lean_ks = 0;
    std::vector<uint32_t> lean;
    std::vector<uint8_t> lean_kw;
    std::vector<uint32_t> lean_b;   // the same entries blocked by 64 columns (see SpinTabDev::lean_b)
};

int64_t binom(int n, int k);
std::vector<uint64_t> enumerate_states(int ns, int np);
std::vector<int32_t> rank_table(int ns);
SpinTableHost build_spin_table(const ModelHost &m, int spin, int np, const std::vector<int32_t> &rank);
void density_terms(const ModelHost &m, std::vector<int32_t> &off, std::vector<double> &coef, bool with_jj = true);
std::vector<int32_t> row_schedule(const std::vector<uint64_t> &states, int nc, int nb);

}  // namespace edk
