// The local two-particle vertex chi~_loc of the reference's vertex tool
// (chi_tilde_loc_, ed_solver/Chiloc_Wenhu_version3.cpp:29-989): for each
// eigenstate i of the sector (nup, ndn), the Lehmann sum over eigenstates
// j, k, l of the neighbouring sectors of
//   coefficient(E_i, E_j, E_k, E_l; w1, w2, w3) x four c+ matrix elements,
// weighted by exp(-beta (E_i - E_gs)) / Z, for the DNDN (op 1) and UPDN
// (op 2) combinations of four operators.
//
// The reference writes one triple loop per term.  Here every term is one row
// of a table (sectors of j, k, l; the one or two Phi kernels with their
// frequency orders and signs; the four matrix factors as (matrix, row index,
// column index)), and one kernel evaluates every (frequency triple, term,
// state i) as a thread block whose threads share the (j, k, l) sum.  Block
// sums go to a buffer that a second kernel reduces in a fixed order: per
// state i the terms in table order, then the states in order with their
// Boltzmann weights.  The table follows the reference's loops one for one;
// the host checks every factor's row and column sectors against the
// matrix's target and source sectors before a launch.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/edk.h"

namespace {

// sectors: i, pup, pdn, mup, mdn, p2dn, m2dn, puppdn, muppdn, pupmdn, mupmdn
enum Sec : int8_t { S_I, S_PUP, S_PDN, S_MUP, S_MDN, S_P2DN, S_M2DN, S_PUPPDN, S_MUPPDN, S_PUPMDN, S_MUPMDN };
// c+ matrices, <target| c+ |source>, row-major target x source
enum Mat : int8_t {
    M_I_CDUP, M_I_CDDN, M_PUP_CDDN, M_PDN_CDUP, M_PDN_CDDN, M_MUP_CDUP, M_MUP_CDDN,
    M_MDN_CDDN, M_MDN_CDUP, M_MUPPDN_CDUP, M_PUPMDN_CDDN, M_MUPMDN_CDUP, M_MUPMDN_CDDN, M_M2DN_CDDN
};
constexpr int8_t kMatTgt[14] = {S_PUP, S_PDN, S_PUPPDN, S_PUPPDN, S_P2DN, S_I, S_MUPPDN,
                                S_I, S_PUPMDN, S_PDN, S_PUP, S_MDN, S_MUP, S_MDN};
constexpr int8_t kMatSrc[14] = {S_I, S_I, S_PUP, S_PDN, S_PDN, S_MUP, S_MUP,
                                S_MDN, S_MDN, S_MUPPDN, S_PUPMDN, S_MUPMDN, S_MUPMDN, S_M2DN};
// Phi kernels (PhiM_ii, PhiM_ji, PhiM_ki, PhiM_li)
enum Phi : int8_t { P_II, P_JI, P_KI, P_LI };
// index variables of a factor
enum Var : int8_t { VI, VJ, VK, VL };
// conditions on (sites, nup, ndn) of the term groups
enum Cond : int8_t {
    C_DN_NOT_FULL,          // ndn != sites
    C_DN_MID,               // ndn != sites && ndn != 0
    C_DN_BELOW_FULL_1,      // ndn < sites - 1
    C_DN_ABOVE_1,           // ndn > 1
    C_DN_NOT_EMPTY,         // ndn != 0
    C_DN_NF_UP_NF,          // ndn != sites && nup != sites
    C_DN_NF_UP_NE,          // ndn != sites && nup != 0
    C_DN_NE_UP_NF,          // ndn != 0 && nup != sites
    C_DN_NE_UP_NE,          // ndn != 0 && nup != 0
};

// Frequency orders: indices into (w1, w2, w3).
#define W123 {0, 1, 2}
#define W321 {2, 1, 0}
#define W213 {1, 0, 2}
#define W231 {1, 2, 0}
#define W312 {2, 0, 1}
#define W132 {0, 2, 1}

struct Term {
    int8_t op, cond;
    int8_t sj, sk, sl;
    int8_t nphi;
    int8_t kind[2];
    int8_t perm[2][3];
    int8_t sgn[2];
    int8_t total;           // +1: c += ..., -1: c -= ...
    int8_t mat[4], row[4], col[4];
};

// One row per loop nest of chi_tilde_loc_, in the reference's order
// (Chiloc_Wenhu_version3.cpp:261-519 for DNDN, 532-986 for UPDN).
const Term kTerms[] = {
    // ---- DNDN ----
    {1, C_DN_NOT_FULL, S_PDN, S_I, S_PDN, 2, {P_II, P_II}, {W123, W321}, {1, -1}, 1,
     {M_I_CDDN, M_I_CDDN, M_I_CDDN, M_I_CDDN}, {VJ, VJ, VL, VL}, {VI, VK, VK, VI}},
    {1, C_DN_NOT_FULL, S_PDN, S_I, S_PDN, 2, {P_KI, P_KI}, {W123, W321}, {1, -1}, 1,
     {M_I_CDDN, M_I_CDDN, M_I_CDDN, M_I_CDDN}, {VL, VL, VJ, VJ}, {VI, VK, VK, VI}},
    {1, C_DN_MID, S_MDN, S_I, S_PDN, 2, {P_II, P_II}, {W213, W231}, {-1, 1}, 1,
     {M_MDN_CDDN, M_MDN_CDDN, M_I_CDDN, M_I_CDDN}, {VI, VK, VL, VL}, {VJ, VJ, VK, VI}},
    {1, C_DN_MID, S_I, S_PDN, S_MDN, 2, {P_LI, P_LI}, {W312, W132}, {1, -1}, 1,
     {M_MDN_CDDN, M_MDN_CDDN, M_I_CDDN, M_I_CDDN}, {VI, VJ, VK, VK}, {VL, VL, VJ, VI}},
    {1, C_DN_MID, S_MDN, S_I, S_PDN, 2, {P_KI, P_KI}, {W213, W231}, {-1, 1}, 1,
     {M_I_CDDN, M_I_CDDN, M_MDN_CDDN, M_MDN_CDDN}, {VL, VL, VK, VI}, {VI, VK, VJ, VJ}},
    {1, C_DN_MID, S_MDN, S_PDN, S_I, 2, {P_JI, P_JI}, {W312, W132}, {1, -1}, 1,
     {M_I_CDDN, M_I_CDDN, M_MDN_CDDN, M_MDN_CDDN}, {VK, VK, VL, VI}, {VI, VL, VJ, VJ}},
    {1, C_DN_BELOW_FULL_1, S_PDN, S_PDN, S_P2DN, 2, {P_JI, P_JI}, {W213, W231}, {-1, 1}, 1,
     {M_I_CDDN, M_PDN_CDDN, M_PDN_CDDN, M_I_CDDN}, {VK, VL, VL, VJ}, {VI, VK, VJ, VI}},
    {1, C_DN_BELOW_FULL_1, S_PDN, S_P2DN, S_PDN, 2, {P_II, P_II}, {W312, W132}, {1, -1}, 1,
     {M_I_CDDN, M_PDN_CDDN, M_PDN_CDDN, M_I_CDDN}, {VJ, VK, VK, VL}, {VI, VJ, VL, VI}},
    {1, C_DN_ABOVE_1, S_M2DN, S_MDN, S_MDN, 2, {P_LI, P_LI}, {W213, W231}, {-1, 1}, 1,
     {M_MDN_CDDN, M_M2DN_CDDN, M_M2DN_CDDN, M_MDN_CDDN}, {VI, VL, VK, VI}, {VL, VJ, VJ, VK}},
    {1, C_DN_ABOVE_1, S_MDN, S_M2DN, S_MDN, 2, {P_KI, P_KI}, {W312, W132}, {1, -1}, 1,
     {M_MDN_CDDN, M_M2DN_CDDN, M_M2DN_CDDN, M_MDN_CDDN}, {VI, VL, VJ, VI}, {VL, VK, VK, VJ}},
    {1, C_DN_NOT_EMPTY, S_MDN, S_MDN, S_I, 2, {P_JI, P_JI}, {W123, W321}, {1, -1}, 1,
     {M_MDN_CDDN, M_MDN_CDDN, M_MDN_CDDN, M_MDN_CDDN}, {VI, VL, VL, VI}, {VK, VK, VJ, VJ}},
    {1, C_DN_NOT_EMPTY, S_I, S_MDN, S_MDN, 2, {P_LI, P_LI}, {W123, W321}, {1, -1}, 1,
     {M_MDN_CDDN, M_MDN_CDDN, M_MDN_CDDN, M_MDN_CDDN}, {VI, VJ, VJ, VI}, {VL, VL, VK, VK}},
    // ---- UPDN ----
    {2, C_DN_NF_UP_NF, S_PUP, S_I, S_PDN, 2, {P_II, P_KI}, {W123, W123}, {1, 1}, 1,
     {M_I_CDUP, M_I_CDUP, M_I_CDDN, M_I_CDDN}, {VJ, VJ, VL, VL}, {VI, VK, VK, VI}},
    {2, C_DN_NF_UP_NF, S_PUP, S_PUP, S_PUPPDN, 1, {P_JI, P_JI}, {W213, W213}, {1, 0}, -1,
     {M_I_CDUP, M_PUP_CDDN, M_PUP_CDDN, M_I_CDUP}, {VK, VL, VL, VJ}, {VI, VK, VJ, VI}},
    {2, C_DN_NF_UP_NF, S_PDN, S_PUPPDN, S_PDN, 1, {P_II, P_II}, {W312, W312}, {1, 0}, 1,
     {M_I_CDDN, M_PDN_CDUP, M_PDN_CDUP, M_I_CDDN}, {VJ, VK, VK, VL}, {VI, VJ, VL, VI}},
    {2, C_DN_NF_UP_NF, S_PUP, S_PUPPDN, S_PDN, 1, {P_II, P_II}, {W132, W132}, {1, 0}, -1,
     {M_I_CDUP, M_PUP_CDDN, M_PDN_CDUP, M_I_CDDN}, {VJ, VK, VK, VL}, {VI, VJ, VL, VI}},
    {2, C_DN_NF_UP_NF, S_PUP, S_PDN, S_PUPPDN, 1, {P_JI, P_JI}, {W231, W231}, {1, 0}, 1,
     {M_I_CDDN, M_PDN_CDUP, M_PUP_CDDN, M_I_CDUP}, {VK, VL, VL, VJ}, {VI, VK, VJ, VI}},
    {2, C_DN_NF_UP_NE, S_MUP, S_MUP, S_MUPPDN, 1, {P_JI, P_JI}, {W123, W123}, {1, 0}, 1,
     {M_MUP_CDUP, M_MUP_CDDN, M_MUP_CDDN, M_MUP_CDUP}, {VI, VL, VL, VI}, {VK, VK, VJ, VJ}},
    {2, C_DN_NF_UP_NE, S_MUP, S_I, S_PDN, 1, {P_II, P_II}, {W213, W213}, {1, 0}, -1,
     {M_MUP_CDUP, M_MUP_CDUP, M_I_CDDN, M_I_CDDN}, {VI, VK, VL, VL}, {VJ, VJ, VK, VI}},
    {2, C_DN_NF_UP_NE, S_MUP, S_I, S_PDN, 1, {P_KI, P_KI}, {W213, W213}, {1, 0}, -1,
     {M_I_CDDN, M_I_CDDN, M_MUP_CDUP, M_MUP_CDUP}, {VL, VL, VK, VI}, {VI, VK, VJ, VJ}},
    {2, C_DN_NF_UP_NE, S_MUP, S_PDN, S_MUPPDN, 1, {P_JI, P_JI}, {W132, W132}, {1, 0}, -1,
     {M_I_CDDN, M_MUPPDN_CDUP, M_MUP_CDDN, M_MUP_CDUP}, {VK, VK, VL, VI}, {VI, VL, VJ, VJ}},
    {2, C_DN_NF_UP_NE, S_MUP, S_MUPPDN, S_PDN, 1, {P_II, P_II}, {W231, W231}, {1, 0}, 1,
     {M_MUP_CDUP, M_MUP_CDDN, M_MUPPDN_CDUP, M_I_CDDN}, {VI, VK, VL, VL}, {VJ, VJ, VK, VI}},
    {2, C_DN_NF_UP_NE, S_PDN, S_MUPPDN, S_PDN, 1, {P_II, P_II}, {W321, W321}, {1, 0}, -1,
     {M_I_CDDN, M_MUPPDN_CDUP, M_MUPPDN_CDUP, M_I_CDDN}, {VJ, VJ, VL, VL}, {VI, VK, VK, VI}},
    {2, C_DN_NE_UP_NF, S_PUPMDN, S_MDN, S_MDN, 1, {P_LI, P_LI}, {W123, W123}, {1, 0}, 1,
     {M_MDN_CDDN, M_MDN_CDUP, M_MDN_CDUP, M_MDN_CDDN}, {VI, VJ, VJ, VI}, {VL, VL, VK, VK}},
    {2, C_DN_NE_UP_NF, S_MDN, S_PUP, S_I, 1, {P_JI, P_JI}, {W312, W312}, {1, 0}, 1,
     {M_I_CDUP, M_I_CDUP, M_MDN_CDDN, M_MDN_CDDN}, {VK, VK, VL, VI}, {VI, VL, VJ, VJ}},
    {2, C_DN_NE_UP_NF, S_I, S_PUP, S_MDN, 1, {P_LI, P_LI}, {W312, W312}, {1, 0}, 1,
     {M_MDN_CDDN, M_MDN_CDDN, M_I_CDUP, M_I_CDUP}, {VI, VJ, VK, VK}, {VL, VL, VJ, VI}},
    {2, C_DN_NE_UP_NF, S_PUPMDN, S_PUP, S_MDN, 1, {P_LI, P_LI}, {W132, W132}, {1, 0}, -1,
     {M_MDN_CDDN, M_MDN_CDUP, M_PUPMDN_CDDN, M_I_CDUP}, {VI, VJ, VK, VK}, {VL, VL, VJ, VI}},
    {2, C_DN_NE_UP_NF, S_MDN, S_PUPMDN, S_PUP, 1, {P_KI, P_KI}, {W231, W231}, {1, 0}, 1,
     {M_I_CDUP, M_PUPMDN_CDDN, M_MDN_CDUP, M_MDN_CDDN}, {VL, VL, VK, VI}, {VI, VK, VJ, VJ}},
    {2, C_DN_NE_UP_NF, S_PUP, S_PUPMDN, S_PUP, 1, {P_KI, P_KI}, {W321, W321}, {1, 0}, -1,
     {M_I_CDUP, M_PUPMDN_CDDN, M_PUPMDN_CDDN, M_I_CDUP}, {VL, VL, VJ, VJ}, {VI, VK, VK, VI}},
    {2, C_DN_NE_UP_NE, S_MUPMDN, S_MDN, S_MDN, 1, {P_LI, P_LI}, {W213, W213}, {1, 0}, -1,
     {M_MDN_CDDN, M_MUPMDN_CDUP, M_MUPMDN_CDUP, M_MDN_CDDN}, {VI, VL, VK, VI}, {VL, VJ, VJ, VK}},
    {2, C_DN_NE_UP_NE, S_MUP, S_MUPMDN, S_MUP, 1, {P_KI, P_KI}, {W312, W312}, {1, 0}, 1,
     {M_MUP_CDUP, M_MUPMDN_CDDN, M_MUPMDN_CDDN, M_MUP_CDUP}, {VI, VL, VJ, VI}, {VL, VK, VK, VJ}},
    {2, C_DN_NE_UP_NE, S_MDN, S_MUPMDN, S_MUP, 1, {P_KI, P_KI}, {W132, W132}, {1, 0}, -1,
     {M_MUP_CDUP, M_MUPMDN_CDDN, M_MUPMDN_CDUP, M_MDN_CDDN}, {VI, VL, VJ, VI}, {VL, VK, VK, VJ}},
    {2, C_DN_NE_UP_NE, S_MUPMDN, S_MUP, S_MDN, 1, {P_LI, P_LI}, {W231, W231}, {1, 0}, 1,
     {M_MDN_CDDN, M_MUPMDN_CDUP, M_MUPMDN_CDDN, M_MUP_CDUP}, {VI, VL, VK, VI}, {VL, VJ, VJ, VK}},
    {2, C_DN_NE_UP_NE, S_MDN, S_MUP, S_I, 1, {P_JI, P_JI}, {W321, W321}, {1, 0}, -1,
     {M_MUP_CDUP, M_MUP_CDUP, M_MDN_CDDN, M_MDN_CDDN}, {VI, VL, VL, VI}, {VK, VK, VJ, VJ}},
    {2, C_DN_NE_UP_NE, S_I, S_MUP, S_MDN, 1, {P_LI, P_LI}, {W321, W321}, {1, 0}, -1,
     {M_MDN_CDDN, M_MDN_CDDN, M_MUP_CDUP, M_MUP_CDUP}, {VI, VJ, VJ, VI}, {VL, VL, VK, VK}},
};
constexpr int kNumTerms = sizeof(kTerms) / sizeof(kTerms[0]);

bool cond_holds(int c, int sites, int nup, int ndn)
{
    switch (c) {
    case C_DN_NOT_FULL: return ndn != sites;
    case C_DN_MID: return ndn != sites && ndn != 0;
    case C_DN_BELOW_FULL_1: return ndn < sites - 1;
    case C_DN_ABOVE_1: return ndn > 1;
    case C_DN_NOT_EMPTY: return ndn != 0;
    case C_DN_NF_UP_NF: return ndn != sites && nup != sites;
    case C_DN_NF_UP_NE: return ndn != sites && nup != 0;
    case C_DN_NE_UP_NF: return ndn != 0 && nup != sites;
    case C_DN_NE_UP_NE: return ndn != 0 && nup != 0;
    }
    return false;
}

// ---------------------------------------------------------------------------
// device: complex arithmetic and the four Phi kernels
// ---------------------------------------------------------------------------
struct Cx {
    double re, im;
};
__device__ __forceinline__ Cx cx(double r, double i = 0.0) { return Cx{r, i}; }
__device__ __forceinline__ Cx operator+(Cx a, Cx b) { return Cx{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Cx operator-(Cx a, Cx b) { return Cx{a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Cx operator-(Cx a) { return Cx{-a.re, -a.im}; }
__device__ __forceinline__ Cx operator+(Cx a, double b) { return Cx{a.re + b, a.im}; }
__device__ __forceinline__ Cx operator-(Cx a, double b) { return Cx{a.re - b, a.im}; }
__device__ __forceinline__ Cx operator*(Cx a, Cx b) { return Cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ Cx operator*(Cx a, double b) { return Cx{a.re * b, a.im * b}; }
// 1 / b with Smith's scaling (no overflow for |b| near the double range)
__device__ __forceinline__ Cx inv(Cx b)
{
    if (fabs(b.re) >= fabs(b.im)) {
        const double r = b.im / b.re, d = b.re + b.im * r;
        return Cx{1.0 / d, -r / d};
    }
    const double r = b.re / b.im, d = b.im + b.re * r;
    return Cx{r / d, -1.0 / d};
}
__device__ __forceinline__ double cabs_(Cx a) { return hypot(a.re, a.im); }
// 1 / b through one reciprocal of |b|^2 (the split kernel's denominators are
// O(1) to O(1e3): no scaling needed)
__device__ __forceinline__ Cx inv_fast(Cx b)
{
    const double d = __drcp_rn(b.re * b.re + b.im * b.im);
    return Cx{b.re * d, -b.im * d};
}
// |z| > eps without the square root
__device__ __forceinline__ bool above(Cx z, double eps2) { return z.re * z.re + z.im * z.im > eps2; }

// Fourier transform of <T c c c c> without the Boltzmann factor for the four
// orderings (the PhiM functions of Chiloc_Wenhu_version3.cpp:29-105); the
// branches taken when a denominator vanishes (|z| <= eps) are the
// reference's.
__device__ Cx phi_ii(double beta, double Ei, double Ej, double Ek, double El, Cx w1, Cx w2, Cx w3, double eps)
{
    const Cx a = inv(w3 + (Ek - El));
    const Cx z = w2 + w3 + (Ej - El);
    const Cx b = inv(w1 + (Ei - Ej));
    const Cx t = cabs_(z) > eps ? inv(z) * (b - inv(w1 + w2 + w3 + Ei - El)) : b * b;
    const Cx y = w1 + w2 + (Ei - Ek);
    const Cx u = cabs_(y) > eps ? -inv(y) : cx(beta);
    return a * (t - inv(w2 + Ej - Ek) * (b + u));
}
__device__ Cx phi_ji(double beta, double Ei, double Ej, double Ek, double El, Cx w1, Cx w2, Cx w3, double eps)
{
    const Cx a = inv(w3 + (Ek - El));
    const Cx z = w2 + w3 + Ei - El;
    const Cx b = inv(w1 + Ej - Ei);
    const Cx t = cabs_(z) > eps ? inv(z) * b : b * b - b * beta;
    return a * (t - inv(w2 + Ei - Ek) * b);
}
__device__ Cx phi_ki(double, double Ei, double Ej, double Ek, double El, Cx w1, Cx w2, Cx w3, double eps)
{
    const Cx y = w1 + w2 + Ek - Ei;
    if (!(cabs_(y) > eps)) return cx(0.0);
    return -inv(w3 + Ei - El) * inv(y) * inv(w2 + Ej - Ei);
}
__device__ Cx phi_li(double, double Ei, double Ej, double Ek, double El, Cx w1, Cx w2, Cx w3, double eps)
{
    const Cx z = w2 + w3 + Ej - Ei;
    if (!(cabs_(z) > eps)) return cx(0.0);
    return -inv((w3 + Ek - Ei) * z * (w1 + w2 + w3 + El - Ei));
}
__device__ __forceinline__ Cx phi(int kind, double beta, double Ei, double Ej, double Ek, double El, Cx w1, Cx w2,
                                  Cx w3, double eps)
{
    switch (kind) {
    case P_II: return phi_ii(beta, Ei, Ej, Ek, El, w1, w2, w3, eps);
    case P_JI: return phi_ji(beta, Ei, Ej, Ek, El, w1, w2, w3, eps);
    case P_KI: return phi_ki(beta, Ei, Ej, Ek, El, w1, w2, w3, eps);
    default: return phi_li(beta, Ei, Ej, Ek, El, w1, w2, w3, eps);
    }
}

struct DevTerm {
    int op, sj, sk, sl, nphi, kind[2], perm[2][3], sgn[2], total;
    int mat[4], row[4], col[4], ld[4];   // ld: the matrix's source-sector dimension
};

struct ChiArgs {
    int nterm, ni, nf;
    double beta, eps;
    const double *E;          // concatenated sector energies
    int eoff[11], dim[11];
    const double *C;          // concatenated matrices
    int64_t moff[14];
    const DevTerm *terms;
    const double *w;          // nf x 6: re, im of w1, w2, w3
    double *part;             // nf x nterm x ni x 2
};

constexpr int kChiBlock = 256;

// One block per (state i, term, frequency triple): the (j, k, l) sum.
__global__ void __launch_bounds__(kChiBlock) chi_terms_kernel(const ChiArgs A)
{
    const int i = blockIdx.x, t = blockIdx.y, f = blockIdx.z;
    const DevTerm T = A.terms[t];
    const int dj = A.dim[T.sj], dk = A.dim[T.sk], dl = A.dim[T.sl];
    const double *Ej = A.E + A.eoff[T.sj], *Ek = A.E + A.eoff[T.sk], *El = A.E + A.eoff[T.sl];
    const double Ei = A.E[A.eoff[S_I] + i];
    const Cx w[3] = {Cx{A.w[6 * f], A.w[6 * f + 1]}, Cx{A.w[6 * f + 2], A.w[6 * f + 3]},
                     Cx{A.w[6 * f + 4], A.w[6 * f + 5]}};
    const double *M[4];
    int ld[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        M[q] = A.C + A.moff[T.mat[q]];
        ld[q] = T.ld[q];
    }
    const int64_t n = (int64_t)dj * dk * dl;
    Cx acc = cx(0.0);
    for (int64_t e = threadIdx.x; e < n; e += blockDim.x) {
        const int l = (int)(e % dl);
        const int k = (int)((e / dl) % dk);
        const int j = (int)(e / ((int64_t)dl * dk));
        const int var[4] = {i, j, k, l};
        double fac = 1.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) fac *= __ldg(M[q] + (int64_t)var[T.row[q]] * ld[q] + var[T.col[q]]);
        if (fac == 0.0) continue;
        Cx c = phi(T.kind[0], A.beta, Ei, Ej[j], Ek[k], El[l], w[T.perm[0][0]], w[T.perm[0][1]], w[T.perm[0][2]],
                   A.eps) * (double)T.sgn[0];
        if (T.nphi == 2)
            c = c + phi(T.kind[1], A.beta, Ei, Ej[j], Ek[k], El[l], w[T.perm[1][0]], w[T.perm[1][1]],
                        w[T.perm[1][2]], A.eps) * (double)T.sgn[1];
        acc = acc + c * (fac * (double)T.total);
    }
    // block sum in a fixed order
    __shared__ double red[2][kChiBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc.re += __shfl_down_sync(0xffffffffu, acc.re, o);
        acc.im += __shfl_down_sync(0xffffffffu, acc.im, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { red[0][warp] = acc.re; red[1][warp] = acc.im; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double re = 0.0, im = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { re += red[0][q]; im += red[1][q]; }
        double *p = A.part + (((int64_t)f * A.nterm + t) * A.ni + i) * 2;
        p[0] = re;
        p[1] = im;
    }
}

// The same sums with the Phi kernels split into their one-index parts, which
// the block computes once into shared memory (complex inverses through one
// reciprocal, the |z| > PHI_EPS tests on |z|^2): per element, phi_ii keeps the
// inverses of w3 + E_k - E_l, w2 + w3 + E_j - E_l and w2 + E_j - E_k (the
// last from a (j, k) table when it fits), phi_ji the inverse of w3 + E_k - E_l,
// and phi_ki, phi_li none.  Same formulas and branches as phi_*.
struct Hoist {
    Cx *J[2], *K[2], *L[2], *JK[2];    // per evaluation: one-index parts, (j, k) table
    unsigned char *fJ[2], *fK[2], *fL[2];
};

__global__ void __launch_bounds__(kChiBlock, 3) chi_terms_hoisted_kernel(const ChiArgs A, int use_jk)
{
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const int i = blockIdx.x, t = blockIdx.y, f = blockIdx.z;
    const DevTerm T = A.terms[t];
    const int dj = A.dim[T.sj], dk = A.dim[T.sk], dl = A.dim[T.sl];
    const double *Ej = A.E + A.eoff[T.sj], *Ek = A.E + A.eoff[T.sk], *El = A.E + A.eoff[T.sl];
    const double Ei = A.E[A.eoff[S_I] + i];
    const Cx w[3] = {Cx{A.w[6 * f], A.w[6 * f + 1]}, Cx{A.w[6 * f + 2], A.w[6 * f + 3]},
                     Cx{A.w[6 * f + 4], A.w[6 * f + 5]}};
    const double beta = A.beta, eps2 = A.eps * A.eps;
    // shared layout: per evaluation J[dj], K[dk], L[dl], JK[dj*dk] (if use_jk), then the flags
    Hoist H{};
    Cx *p = reinterpret_cast<Cx *>(sm_raw);
    for (int e = 0; e < T.nphi; ++e) {
        H.J[e] = p; p += dj;
        H.K[e] = p; p += dk;
        H.L[e] = p; p += dl;
        H.JK[e] = p; p += use_jk ? dj * dk : 0;
    }
    unsigned char *fp = reinterpret_cast<unsigned char *>(p);
    for (int e = 0; e < T.nphi; ++e) {
        H.fJ[e] = fp; fp += dj;
        H.fK[e] = fp; fp += dk;
        H.fL[e] = fp; fp += dl;
    }
    for (int e = 0; e < T.nphi; ++e) {
        const Cx W1 = w[T.perm[e][0]], W2 = w[T.perm[e][1]], W3 = w[T.perm[e][2]];
        const Cx Ws23 = W2 + W3, Ws123 = W1 + W2 + W3, Ws12 = W1 + W2;
        const int kind = T.kind[e];
        for (int x = threadIdx.x; x < dj; x += blockDim.x) {
            if (kind == P_II) H.J[e][x] = inv_fast(W1 + (Ei - Ej[x]));
            else if (kind == P_JI) H.J[e][x] = inv_fast(W1 + Ej[x] - Ei);
            else if (kind == P_KI) H.J[e][x] = inv_fast(W2 + Ej[x] - Ei);
            else {
                const Cx z = Ws23 + Ej[x] - Ei;
                H.fJ[e][x] = above(z, eps2);
                H.J[e][x] = inv_fast(z);
            }
        }
        for (int x = threadIdx.x; x < dk; x += blockDim.x) {
            if (kind == P_II) {
                const Cx y = Ws12 + (Ei - Ek[x]);
                H.K[e][x] = above(y, eps2) ? -inv_fast(y) : cx(beta);
            } else if (kind == P_JI) {
                H.K[e][x] = inv_fast(W2 + Ei - Ek[x]);
            } else if (kind == P_KI) {
                const Cx y = Ws12 + Ek[x] - Ei;
                H.fK[e][x] = above(y, eps2);
                H.K[e][x] = inv_fast(y);
            } else {
                H.K[e][x] = inv_fast(W3 + Ek[x] - Ei);
            }
        }
        for (int x = threadIdx.x; x < dl; x += blockDim.x) {
            if (kind == P_II) {
                H.L[e][x] = inv_fast(Ws123 + Ei - El[x]);
            } else if (kind == P_JI) {
                const Cx z = Ws23 + Ei - El[x];
                H.fL[e][x] = above(z, eps2);
                H.L[e][x] = inv_fast(z);
            } else if (kind == P_KI) {
                H.L[e][x] = -inv_fast(W3 + Ei - El[x]);
            } else {
                H.L[e][x] = inv_fast(Ws123 + El[x] - Ei);
            }
        }
        if (use_jk && kind == P_II)
            for (int x = threadIdx.x; x < dj * dk; x += blockDim.x) {
                const int jj = x / dk, kk = x % dk;
                H.JK[e][x] = inv_fast(W2 + Ej[jj] - Ek[kk]);
            }
    }
    __syncthreads();
    int cf[4][3];                      // address coefficients of j, k, l per factor (i folded in M)
    const double *M[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int ci = (T.row[q] == VI ? T.ld[q] : 0) + (T.col[q] == VI ? 1 : 0);
        M[q] = A.C + A.moff[T.mat[q]] + (int64_t)ci * i;
#pragma unroll
        for (int v = 1; v < 4; ++v) cf[q][v - 1] = (T.row[q] == v ? T.ld[q] : 0) + (T.col[q] == v ? 1 : 0);
    }
    const int64_t n = (int64_t)dj * dk * dl;
    Cx acc = cx(0.0);
    for (int64_t e = threadIdx.x; e < n; e += blockDim.x) {
        const int l = (int)(e % dl);
        const int k = (int)((e / dl) % dk);
        const int j = (int)(e / ((int64_t)dl * dk));
        double fac = 1.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) fac *= __ldg(M[q] + (cf[q][0] * j + cf[q][1] * k + cf[q][2] * l));
        if (fac == 0.0) continue;
        Cx c = cx(0.0);
        for (int ev = 0; ev < T.nphi; ++ev) {
            const Cx W2 = w[T.perm[ev][1]], W3 = w[T.perm[ev][2]];
            Cx r;
            switch (T.kind[ev]) {
            case P_II: {
                const Cx a = inv_fast(W3 + (Ek[k] - El[l]));
                const Cx z = W2 + W3 + (Ej[j] - El[l]);
                const Cx b = H.J[ev][j];
                const Cx tt = above(z, eps2) ? inv_fast(z) * (b - H.L[ev][l]) : b * b;
                const Cx cjk = use_jk ? H.JK[ev][j * dk + k] : inv_fast(W2 + Ej[j] - Ek[k]);
                r = a * (tt - cjk * (b + H.K[ev][k]));
                break;
            }
            case P_JI: {
                const Cx a = inv_fast(W3 + (Ek[k] - El[l]));
                const Cx b = H.J[ev][j];
                const Cx tt = H.fL[ev][l] ? H.L[ev][l] * b : b * b - b * beta;
                r = a * (tt - H.K[ev][k] * b);
                break;
            }
            case P_KI:
                r = H.fK[ev][k] ? H.L[ev][l] * H.K[ev][k] * H.J[ev][j] : cx(0.0);
                break;
            default:
                r = H.fJ[ev][j] ? -(H.K[ev][k] * H.J[ev][j] * H.L[ev][l]) : cx(0.0);
                break;
            }
            c = c + r * (double)T.sgn[ev];
        }
        acc = acc + c * (fac * (double)T.total);
    }
    __shared__ double red[2][kChiBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc.re += __shfl_down_sync(0xffffffffu, acc.re, o);
        acc.im += __shfl_down_sync(0xffffffffu, acc.im, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { red[0][warp] = acc.re; red[1][warp] = acc.im; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double re = 0.0, im = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { re += red[0][q]; im += red[1][q]; }
        double *pp = A.part + (((int64_t)f * A.nterm + t) * A.ni + i) * 2;
        pp[0] = re;
        pp[1] = im;
    }
}

// out[f] = sum_i boltz_i sum_t part[f][t][i] for the terms of one op, in order.
__global__ void chi_reduce_kernel(const ChiArgs A, const double *boltz, int op, double *out)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= A.nf) return;
    double pre = 0.0, pim = 0.0;
    for (int i = 0; i < A.ni; ++i) {
        double cre = 0.0, cim = 0.0;
        for (int t = 0; t < A.nterm; ++t) {
            if (A.terms[t].op != op) continue;
            const double *p = A.part + (((int64_t)f * A.nterm + t) * A.ni + i) * 2;
            cre += p[0];
            cim += p[1];
        }
        pre += cre * boltz[i];
        pim += cim * boltz[i];
    }
    out[2 * f] = pre;
    out[2 * f + 1] = pim;
}

struct DevMem {
    void *p = nullptr;
    ~DevMem() { if (p) cudaFree(p); }
};

template <typename T>
cudaError_t put(DevMem &m, const T *src, size_t count, cudaStream_t st)
{
    cudaError_t e = cudaMalloc(&m.p, sizeof(T) * (count ? count : 1));
    if (e != cudaSuccess) { m.p = nullptr; return e; }
    if (!count) return cudaSuccess;
    return cudaMemcpyAsync(m.p, src, sizeof(T) * count, cudaMemcpyHostToDevice, st);
}

}  // namespace

// 1: always the plain per-element kernel (for A/B checks of the split one)
static int chiloc_plain_kernel = 0;

extern "C" {
cudaStream_t edk_internal_stream(edk_ctx *ctx);

int edk_chiloc_set_kernel(int plain)
{
    chiloc_plain_kernel = plain ? 1 : 0;
    return EDK_OK;
}

int edk_internal_fail(edk_ctx *ctx, int code, const char *msg);
void edk_internal_add_launches(edk_ctx *ctx, int64_t n);
void edk_internal_count(edk_ctx *ctx, int64_t h2d, int64_t d2h);

int edk_chiloc(edk_ctx *ctx, int32_t op_mask, double beta, double Z, double gs_e, double phi_eps, int32_t sites,
               int32_t nup, int32_t ndn, const edk_chiloc_sectors *s, int32_t nf, const double *w_host,
               double *pdndn_host, double *pupdn_host)
{
    if (!ctx || !s || nf < 0 || (nf > 0 && !w_host) || !(Z > 0.0) || (op_mask & ~3) || op_mask == 0)
        return EDK_ERR_INVALID;
    if (((op_mask & 1) && !pdndn_host) || ((op_mask & 2) && !pupdn_host)) return EDK_ERR_INVALID;
    if (nf == 0) return EDK_OK;
    const int ni = s->dim[S_I];
    if (ni < 1 || !s->E[S_I]) return edk_internal_fail(ctx, EDK_ERR_INVALID, "chiloc: empty i sector");
    // the active terms, each checked against the matrices' sectors
    std::vector<DevTerm> terms;
    for (int t = 0; t < kNumTerms; ++t) {
        const Term &T = kTerms[t];
        if (!((op_mask >> (T.op - 1)) & 1) || !cond_holds(T.cond, sites, nup, ndn)) continue;
        const int sec[4] = {S_I, T.sj, T.sk, T.sl};
        for (int v = 1; v < 4; ++v)
            if (s->dim[sec[v]] < 0 || (s->dim[sec[v]] > 0 && !s->E[sec[v]]))
                return edk_internal_fail(ctx, EDK_ERR_INVALID, "chiloc: sector energies missing");
        DevTerm d{};
        d.op = T.op; d.sj = T.sj; d.sk = T.sk; d.sl = T.sl; d.nphi = T.nphi; d.total = T.total;
        for (int q = 0; q < 2; ++q) {
            d.kind[q] = T.kind[q];
            d.sgn[q] = T.sgn[q];
            for (int r = 0; r < 3; ++r) d.perm[q][r] = T.perm[q][r];
        }
        bool empty = false;
        for (int q = 0; q < 4; ++q) {
            const int m = T.mat[q];
            if (sec[T.row[q]] != kMatTgt[m] || sec[T.col[q]] != kMatSrc[m])
                return edk_internal_fail(ctx, EDK_ERR_INVALID, "chiloc: term table inconsistent with the matrices");
            if (s->dim[kMatTgt[m]] > 0 && s->dim[kMatSrc[m]] > 0 && !s->C[m])
                return edk_internal_fail(ctx, EDK_ERR_INVALID, "chiloc: c+ matrix missing");
            d.mat[q] = m;
            d.row[q] = T.row[q];
            d.col[q] = T.col[q];
            d.ld[q] = s->dim[kMatSrc[m]];
        }
        for (int v = 1; v < 4; ++v) empty = empty || s->dim[sec[v]] == 0;
        if (!empty) terms.push_back(d);
    }
    // concatenated energies and matrices
    std::vector<double> E, C;
    ChiArgs A{};
    for (int q = 0; q < 11; ++q) {
        A.eoff[q] = (int)E.size();
        A.dim[q] = s->dim[q] > 0 ? s->dim[q] : 0;
        if (A.dim[q] > 0) E.insert(E.end(), s->E[q], s->E[q] + A.dim[q]);
    }
    for (int m = 0; m < 14; ++m) {
        A.moff[m] = (int64_t)C.size();
        const int64_t sz = (int64_t)A.dim[kMatTgt[m]] * A.dim[kMatSrc[m]];
        if (sz > 0 && s->C[m]) C.insert(C.end(), s->C[m], s->C[m] + sz);
    }
    std::vector<double> boltz(ni);
    for (int i = 0; i < ni; ++i) boltz[i] = std::exp(-(s->E[S_I][i] - gs_e) * beta) / Z;
    cudaStream_t st = edk_internal_stream(ctx);
    const int nterm = (int)terms.size();
    DevMem dE, dC, dT, dW, dP, dB, dO;
    cudaError_t e;
    if ((e = put(dE, E.data(), E.size(), st)) != cudaSuccess || (e = put(dC, C.data(), C.size(), st)) != cudaSuccess ||
        (e = put(dT, terms.data(), terms.size(), st)) != cudaSuccess ||
        (e = put(dW, w_host, (size_t)nf * 6, st)) != cudaSuccess ||
        (e = put(dB, boltz.data(), boltz.size(), st)) != cudaSuccess ||
        (e = cudaMalloc(&dP.p, sizeof(double) * 2 * std::max<size_t>(1, (size_t)nf * nterm * ni))) != cudaSuccess ||
        (e = cudaMalloc(&dO.p, sizeof(double) * 2 * (size_t)nf)) != cudaSuccess)
        return edk_internal_fail(ctx, e == cudaErrorMemoryAllocation ? EDK_ERR_NOMEM : EDK_ERR_CUDA,
                                 cudaGetErrorString(e));
    edk_internal_count(ctx, (int64_t)(E.size() + C.size() + (size_t)nf * 6 + boltz.size()) * 8, 0);
    A.nterm = nterm;
    A.ni = ni;
    A.nf = nf;
    A.beta = beta;
    A.eps = phi_eps;
    A.E = static_cast<const double *>(dE.p);
    A.C = static_cast<const double *>(dC.p);
    A.terms = static_cast<const DevTerm *>(dT.p);
    A.w = static_cast<const double *>(dW.p);
    A.part = static_cast<double *>(dP.p);
    if (nterm > 0) {
        // shared memory of the split kernel: the largest term's one-index parts
        // (and (j, k) tables when they fit)
        size_t smem_1d = 0, smem_jk = 0;
        for (const DevTerm &d : terms) {
            const size_t dj = A.dim[d.sj], dk = A.dim[d.sk], dl = A.dim[d.sl];
            const size_t one = (size_t)d.nphi * ((dj + dk + dl) * (sizeof(Cx) + 1));
            smem_1d = std::max(smem_1d, one + 16);
            smem_jk = std::max(smem_jk, one + (size_t)d.nphi * dj * dk * sizeof(Cx) + 16);
        }
        const size_t cap = 96 * 1024;
        const int use_jk = smem_jk <= cap ? 1 : 0;
        const size_t smem = use_jk ? smem_jk : smem_1d;
        const bool split = smem <= cap;
        if (split && smem > 48 * 1024)
            cudaFuncSetAttribute(chi_terms_hoisted_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        // grid.z is limited to 65535: frequency triples in chunks
        for (int f0 = 0; f0 < nf; f0 += 65535) {
            ChiArgs Ac = A;
            const int nfc = std::min(65535, nf - f0);
            Ac.w = A.w + (size_t)f0 * 6;
            Ac.part = A.part + (size_t)f0 * nterm * ni * 2;
            if (split && !chiloc_plain_kernel)
                chi_terms_hoisted_kernel<<<dim3(ni, nterm, nfc), kChiBlock, smem, st>>>(Ac, use_jk);
            else
                chi_terms_kernel<<<dim3(ni, nterm, nfc), kChiBlock, 0, st>>>(Ac);
            edk_internal_add_launches(ctx, 1);
        }
    } else {
        cudaMemsetAsync(dP.p, 0, sizeof(double) * 2, st);
    }
    for (int op = 1; op <= 2; ++op) {
        if (!((op_mask >> (op - 1)) & 1)) continue;
        double *out = op == 1 ? pdndn_host : pupdn_host;
        if (nterm > 0) {
            chi_reduce_kernel<<<(nf + 127) / 128, 128, 0, st>>>(A, static_cast<const double *>(dB.p), op,
                                                                 static_cast<double *>(dO.p));
            edk_internal_add_launches(ctx, 1);
            if ((e = cudaMemcpyAsync(out, dO.p, sizeof(double) * 2 * nf, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
                return edk_internal_fail(ctx, EDK_ERR_CUDA, cudaGetErrorString(e));
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
                return edk_internal_fail(ctx, EDK_ERR_CUDA, cudaGetErrorString(e));
            edk_internal_count(ctx, 0, (int64_t)nf * 16);
        } else {
            std::memset(out, 0, sizeof(double) * 2 * nf);
        }
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return edk_internal_fail(ctx, EDK_ERR_CUDA, cudaGetErrorString(e));
    return EDK_OK;
}
}  // extern "C"
