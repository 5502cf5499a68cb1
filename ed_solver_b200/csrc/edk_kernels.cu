// Device kernels of the Krylov engine (sm_100a).
//
// The sector vector is a dim_up x dim_dn array, up index contiguous
// ("row" = one down state = dim_up contiguous elements).  The fused row kernel
// evaluates (H x) for a group of R rows per thread block:
//   * the R rows of x are staged in shared memory with 16-byte loads, so the
//     up-spin hops (targets inside the same row, HAIMupdo.f90:865-881) gather
//     from shared memory;
//   * each thread owns columns (up states) and keeps R accumulators, so one
//     read of an up-table entry serves R rows;
//   * the down-spin hops (HAIMupdo.f90:883-900) read whole neighbour rows from
//     global memory, coalesced along the up index; rows are visited in a
//     host-chosen order that keeps neighbour rows resident in L2;
//   * diagonal and density-density terms come from the impurity occupation
//     bits of the two spin states (HAIMupdo.f90:784-848), Hund spin flip and
//     pair hopping from per-state move tables (HAIMupdo.f90:1017-1129).
// Per element the additions happen in the reference's order with separate
// multiply and add (no FMA contraction), so the FP64 result equals a
// sequential FP64 evaluation of HAIMupdo_multr bit for bit.
//
// Lanczos step (kModeStep).  The previous launch stored s = w_k - gamma_k v_k
// (w_k = H v_k - beta_k v_{k-1}, gamma_k a shift known before that launch:
// gamma_1 given, gamma_{k+1} = alpha_k), and its reductions gave alpha_k,
// beta_{k+1}.  With delta_k = alpha_k - gamma_k one pass computes
//   v_{k+1}   = (s - delta_k v_k) / beta_{k+1}
//   H v_{k+1} = (H s - delta_k (s + gamma_k v_k + beta_k v_{k-1})) / beta_{k+1}
//   w_{k+1}   = H v_{k+1} - beta_{k+1} v_k,   s' = w_{k+1} - alpha_k v_{k+1}
// using H v_k = s + gamma_k v_k + beta_k v_{k-1}, plus the sums |s'|^2,
// <s',v_{k+1}>, |v_{k+1}|^2 that give alpha_{k+1} and beta_{k+2}
// (lanc_opt, Lanczos_plain.h:66-173, without its separate orthogonalise and
// normalise passes).  The shift keeps |s| near beta, so the rounding of the
// stored s is not amplified by |alpha|/beta when H s is formed.
// Reductions are deterministic: per-block partials, summed in block order by
// the last block to finish.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include "edk_internal.h"
#include "edk_device.cuh"

namespace edk {

// one electron of one spin moved between impurity sites a -> b
__device__ __forceinline__ int move_index(int a, int b, int nc)
{
    return a * (nc - 1) + (b < a ? b : b - 1);
}

// Hund spin flip and pair hopping for element (iup, ido) (HAIMupdo.f90:1017-1129).
template <typename T>
__device__ __forceinline__ double hund_terms(const HamDev &H, const T *x, int64_t iup, int64_t ido,
                                             int cu, int cd, double acc)
{
    const int nc = H.nc;
    const double *jj = H.jj;
    // spin flip, sites s1 < s2 singly occupied with opposite spins
    for (int s1 = 0; s1 < nc; ++s1) {
        const int b1u = (cu >> s1) & 1, b1d = (cd >> s1) & 1;
        if (b1u + b1d != 1) continue;
        for (int s2 = s1 + 1; s2 < nc; ++s2) {
            if (!H.umask[s1 * nc + s2]) continue;
            const int b2u = (cu >> s2) & 1, b2d = (cd >> s2) & 1;
            if (b2u + b2d != 1) continue;
            int mu = -1, md = -1;
            if (b1u && b2d) { mu = move_index(s1, s2, nc); md = move_index(s2, s1, nc); }
            else if (b1d && b2u) { mu = move_index(s2, s1, nc); md = move_index(s1, s2, nc); }
            if (mu < 0) continue;
            const int32_t pu = H.up.move[iup * H.nmove + mu];
            const int32_t pd = H.dn.move[ido * H.nmove + md];
            if (pu == 0 || pd == 0) continue;
            const int64_t ju = (pu > 0 ? pu : -pu) - 1, jd = (pd > 0 ? pd : -pd) - 1;
            const double t = fmul((double)__ldg(x + ju + jd * H.dup), jj[s1 * nc + s2]);
            acc = ((pu > 0) == (pd > 0)) ? fadd(acc, t) : fsub(acc, t);
        }
    }
    // pair hopping: s1 doubly occupied, s2 empty
    for (int s1 = 0; s1 < nc; ++s1) {
        if (!(((cu >> s1) & 1) && ((cd >> s1) & 1))) continue;
        for (int s2 = 0; s2 < nc; ++s2) {
            if (s2 == s1 || !H.umask[s1 * nc + s2]) continue;
            if (((cu >> s2) & 1) || ((cd >> s2) & 1)) continue;
            const int m = move_index(s1, s2, nc);
            const int32_t pu = H.up.move[iup * H.nmove + m];
            const int32_t pd = H.dn.move[ido * H.nmove + m];
            if (pu == 0 || pd == 0) continue;
            const int64_t ju = (pu > 0 ? pu : -pu) - 1, jd = (pd > 0 ? pd : -pd) - 1;
            const double t = fmul((double)__ldg(x + ju + jd * H.dup), jj[s1 * nc + s2]);
            acc = ((pu > 0) == (pd > 0)) ? fadd(acc, t) : fsub(acc, t);
        }
    }
    return acc;
}

// ---------------------------------------------------------------------------
// fused row kernel
// ---------------------------------------------------------------------------

// Row kernel.  T: element type; R: rows per group (register accumulators);
// STAGE: rows staged in shared memory; PACKED: 24+8-bit up-table entries;
// KM: compile-time bound on up-table width and down-table row length (8 or 16;
// 0 = dynamic loops for wide generic tables).  With KM > 0 every table entry
// and every neighbour-row element of a column is loaded before the in-order
// accumulation starts, so each thread keeps R*KM independent loads in flight.
template <typename T, int R, bool STAGE, bool PACKED, int KM>
__global__ void __launch_bounds__(512, 1) row_kernel(const HamDev H, const RowArgs a)
{
    constexpr int KB = KM > 0 ? KM : 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double pal_s[256];
    __shared__ int s_nd[R];
    __shared__ int s_jd[R][KB];
    __shared__ double s_hd[R][KB];
    T *xs = reinterpret_cast<T *>(smem_raw);
    const int64_t dup = H.dup, ddn = H.ddn;
    const T *__restrict__ x = static_cast<const T *>(a.x);

    // step scalars: s = w_k - gamma_k v_k was stored by the previous launch;
    // delta_k = alpha_k - gamma_k; the new vector is s' = w_{k+1} - gamma_{k+1} v_{k+1}
    // with gamma_{k+1} = alpha_k
    double delta = 0.0, gam = 0.0, gam1 = a.gamma1, beta_k = 0.0, beta_k1 = 0.0, inv_b = 0.0, cpsi = 0.0;
    const int ks = step_index(a);
    if (a.mode == kModeStep) {
        beta_k1 = a.tri_sub[ks];
        // the chain already ended (breakdown recorded by an earlier launch)
        if (!(beta_k1 >= a.cutoff) || a.flags[0] != 0) return;
        const double alpha = a.tri_diag[ks - 1];
        gam = ks >= 2 ? a.tri_diag[ks - 2] : a.gamma1;
        delta = alpha - gam;
        gam1 = alpha;
        beta_k = ks >= 2 ? a.tri_sub[ks - 1] : 0.0;
        inv_b = 1.0 / beta_k1;
        if (a.psi_coef) cpsi = a.psi_coef[ks];
    }
    if (PACKED) {
        for (int i = threadIdx.x; i < H.up.npal; i += blockDim.x) pal_s[i] = H.up.pal[i];
    }

    const uint32_t *__restrict__ ell = H.up.ell;
    const double *__restrict__ ellv = H.up.ell_val;
    const int K = H.up.ell_k;
    const double *__restrict__ dnv = H.dn.val;
    const double *__restrict__ upd = H.up.diag;
    const double *__restrict__ dnd = H.dn.diag;
    const double *__restrict__ icoef = H.int_coef;

    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    const int64_t ngroups = (ddn + R - 1) / R;
    for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        int row[R];
        double dd[R];
        int cd[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int64_t q = g * R + r;
            row[r] = q < ddn ? H.row_order[q] : -1;
            dd[r] = row[r] >= 0 ? dnd[row[r]] : 0.0;
            cd[r] = row[r] >= 0 ? (int)H.dn.imp[row[r]] : 0;
        }
        __syncthreads();                                 // previous group done with shared data
        if (KM > 0) {
            for (int t = threadIdx.x; t < R * KM; t += blockDim.x) {
                const int r = t / KM, f = t % KM;
                int nd = 0, jd = 0;
                double hd = 0.0;
                if (row[r] >= 0) {
                    const int f0 = H.dn.ptr[row[r]];
                    nd = H.dn.ptr[row[r] + 1] - f0;
                    if (f < nd) { jd = H.dn.tgt[f0 + f]; hd = dnv[f0 + f]; }
                }
                s_jd[r][f] = jd;
                s_hd[r][f] = hd;
                if (f == 0) s_nd[r] = nd;
            }
        }
        if (STAGE) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (row[r] >= 0) stage_row<T>(xs + (size_t)r * dup, x + (int64_t)row[r] * dup, dup);
        }
        __syncthreads();
        for (int64_t c = threadIdx.x; c < dup; c += blockDim.x) {
            const int cu = H.up.imp[c];
            const double du = upd[c];
            double acc[R];
            T xo[R];
            if (KM > 0) {
                // ---- issue every load of this column first ----
                uint32_t ent[KB];
                double hv[KB];
#pragma unroll
                for (int k = 0; k < KB; ++k) {
                    if (k < K) {
                        ent[k] = __ldg(ell + (int64_t)k * dup + c);
                        if (!PACKED) hv[k] = __ldg(ellv + (int64_t)k * dup + c);
                    } else {
                        ent[k] = (uint32_t)c;
                        if (!PACKED) hv[k] = 0.0;
                    }
                }
                T xd[R][KB];
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int f = 0; f < KB; ++f)
                        xd[r][f] = (row[r] >= 0 && f < s_nd[r]) ? __ldg(x + (int64_t)s_jd[r][f] * dup + c) : T(0);
#pragma unroll
                for (int r = 0; r < R; ++r)
                    xo[r] = row[r] < 0 ? T(0) : (STAGE ? xs[(size_t)r * dup + c] : __ldg(x + (int64_t)row[r] * dup + c));
                // ---- accumulate in the reference order ----
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int cfg = cu * H.ncfg + cd[r];
                    const int o0 = H.int_off[cfg], o1 = H.int_off[cfg + 1];
                    double ac = 0.0;
                    for (int o = o0; o < o1; ++o) ac = hmadd<T>(ac, icoef[o], xo[r]);
                    acc[r] = hmadd<T>(ac, fadd(du, dd[r]), xo[r]);
                }
#pragma unroll
                for (int k = 0; k < KB; ++k) {
                    if (k >= K) break;
                    const int64_t j = PACKED ? (int64_t)(ent[k] & 0xFFFFFFu) : (int64_t)(int32_t)ent[k];
                    const double h = PACKED ? pal_s[ent[k] >> 24] : hv[k];
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const T xj = STAGE ? xs[(size_t)r * dup + j] : __ldg(x + (int64_t)row[r] * dup + j);
                        acc[r] = hmadd<T>(acc[r], h, xj);
                    }
                }
#pragma unroll
                for (int r = 0; r < R; ++r) {
#pragma unroll
                    for (int f = 0; f < KB; ++f)
                        if (f < s_nd[r]) acc[r] = hmadd<T>(acc[r], s_hd[r][f], xd[r][f]);
                    if (H.hund && row[r] >= 0) acc[r] = hund_terms<T>(H, x, c, row[r], cu, cd[r], acc[r]);
                }
            } else {
                // ---- generic tables: dynamic loops ----
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (row[r] < 0) { acc[r] = 0.0; xo[r] = T(0); continue; }
                    xo[r] = STAGE ? xs[(size_t)r * dup + c] : __ldg(x + (int64_t)row[r] * dup + c);
                    const int cfg = cu * H.ncfg + cd[r];
                    const int o0 = H.int_off[cfg], o1 = H.int_off[cfg + 1];
                    double ac = 0.0;
                    for (int o = o0; o < o1; ++o) ac = hmadd<T>(ac, icoef[o], xo[r]);
                    acc[r] = hmadd<T>(ac, fadd(du, dd[r]), xo[r]);
                }
                for (int k = 0; k < K; ++k) {
                    const uint32_t ent = __ldg(ell + (int64_t)k * dup + c);
                    const int64_t j = PACKED ? (int64_t)(ent & 0xFFFFFFu) : (int64_t)(int32_t)ent;
                    const double h = PACKED ? pal_s[ent >> 24] : __ldg(ellv + (int64_t)k * dup + c);
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        if (row[r] < 0) continue;
                        const T xj = STAGE ? xs[(size_t)r * dup + j] : __ldg(x + (int64_t)row[r] * dup + j);
                        acc[r] = hmadd<T>(acc[r], h, xj);
                    }
                }
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (row[r] < 0) continue;
                    const int f0 = H.dn.ptr[row[r]], f1 = H.dn.ptr[row[r] + 1];
                    for (int f = f0; f < f1; ++f) {
                        const int64_t jd = H.dn.tgt[f];
                        acc[r] = hmadd<T>(acc[r], dnv[f], __ldg(x + jd * dup + c));
                    }
                    if (H.hund) acc[r] = hund_terms<T>(H, x, c, row[r], cu, cd[r], acc[r]);
                }
            }
            // ---- epilogue ----
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (row[r] < 0) continue;
                const int64_t i = (int64_t)row[r] * dup + c;
                if (a.mode == kModeHv) {
                    static_cast<T *>(a.y)[i] = (T)acc[r];
                } else if (a.mode == kModeFirst) {
                    const double v = (double)xo[r];
                    const T st = (T)((double)acc[r] - gam1 * v);
                    static_cast<T *>(a.y)[i] = st;
                    const double sd = (double)st;
                    s0 += sd * sd; s1 += sd * v; s2 += v * v;
                } else if (a.mode == kModeStep) {
                    const double sv = (double)xo[r];
                    const double vk = (double)static_cast<const T *>(a.vk)[i];
                    const double vm = a.vkm1 ? (double)static_cast<const T *>(a.vkm1)[i] : 0.0;
                    const T vt = (T)((sv - delta * vk) * inv_b);
                    const double hv1 = ((double)acc[r] - delta * (sv + gam * vk + beta_k * vm)) * inv_b;
                    const double w = hv1 - beta_k1 * vk;
                    const T wt = (T)(w - gam1 * (double)vt);
                    static_cast<T *>(a.y)[i] = wt;
                    static_cast<T *>(a.vout)[i] = vt;
                    if (a.psi) {
                        T *p = static_cast<T *>(a.psi) + i;
                        *p = (T)((double)*p + cpsi * (double)vt);
                    }
                    const double wd = (double)wt, vd = (double)vt;
                    s0 += wd * wd; s1 += wd * vd; s2 += vd * vd;
                } else {   // kModeResid
                    const double rr = (double)acc[r] - a.eshift * (double)xo[r];
                    s0 += rr * rr; s2 += (double)xo[r] * (double)xo[r];
                }
            }
        }
    }
    if (a.mode == kModeHv) return;

    double v[4] = {s0, s1, s2, s3};
    if (grid_sum<4>(v, a.partials, a.counter, a.sums_out))
        if (a.mode == kModeFirst || a.mode == kModeStep) lanczos_finalize(a, ks);
}

// ---------------------------------------------------------------------------
// start vector, norms, scaling, conversion
// ---------------------------------------------------------------------------
// v(i) = ran_tab(modi(i,10000)) (rcvector_class.f90:43-60) or a copy of a user
// vector; also |v|^2 (deterministic).
template <typename T>
__global__ void start_kernel(int64_t n, const double *tab, const T *user, T *v, double *partials,
                             unsigned *counter, double *sums)
{
    double s[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        T val = user ? user[i] : (T)tab[(i % 10000) + 1];
        v[i] = val;
        s[0] += (double)val * (double)val;
    }
    grid_sum<1>(s, partials, counter, sums);
}

template <typename T>
__global__ void norm2_kernel(int64_t n, const T *v, double *partials, unsigned *counter, double *sums)
{
    double s[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double t = (double)v[i];
        s[0] += t * t;
    }
    grid_sum<1>(s, partials, counter, sums);
}

// v *= 1/sqrt(sums[which]); optionally psi = psi_coef[0] * v and tri_sub[0] = |v|
template <typename T>
__global__ void scale_kernel(int64_t n, T *v, const double *sums, int which, T *psi,
                             const double *psi_coef, double *tri_sub0)
{
    const double nrm = sqrt(sums[which]);
    const double inv = 1.0 / nrm;
    const double c0 = psi_coef ? psi_coef[0] : 0.0;
    if (tri_sub0 && blockIdx.x == 0 && threadIdx.x == 0) *tri_sub0 = nrm;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const T t = (T)((double)v[i] * inv);
        v[i] = t;
        if (psi) psi[i] = (T)(c0 * (double)t);
    }
}

// psi = sum_q coef[q] v_q over stored Krylov vectors, accumulated in the
// order the fused steps of a recomputing pass 2 use: psi = coef[0] v_0, then
// psi += coef[q] v_q for q = 1, 2, ... (each stored in the element type).
template <typename T>
__global__ void combine_kernel(int64_t n, const T *const *vecs, const double *coef, int nv, T *psi)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        T p = (T)(coef[0] * (double)vecs[0][i]);
        for (int q = 1; q < nv; ++q) p = (T)((double)p + coef[q] * (double)__ldg(vecs[q] + i));
        psi[i] = p;
    }
}

template <typename A, typename B>
__global__ void convert_kernel(int64_t n, const A *in, B *out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (B)in[i];
}

// ---------------------------------------------------------------------------
// c / c+ maps (apply_Cupdo, apply_C.f90:497-653), output driven
// ---------------------------------------------------------------------------
template <typename T>
__global__ void apply_c_kernel(int spin, int64_t dother, int64_t dup_src, int64_t dup_tgt,
                               int64_t dim_sigma_tgt, const int32_t *src1, const int8_t *sg1,
                               const int32_t *src2, const int8_t *sg2, int sign2, const T *in, T *out)
{
    const int64_t n = dim_sigma_tgt * dother;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        int64_t jt, other, o_idx;
        if (spin == 0) { jt = e % dup_tgt; other = e / dup_tgt; o_idx = jt + other * dup_tgt; }
        else { other = e % dup_tgt; jt = e / dup_tgt; o_idx = other + jt * dup_tgt; }
        T acc = T(0);
        const int32_t i1 = src1[jt];
        if (i1 >= 0) {
            const int64_t si = spin == 0 ? (i1 + other * dup_src) : (other + (int64_t)i1 * dup_src);
            acc = sg1[jt] > 0 ? in[si] : -in[si];
        }
        if (src2) {
            const int32_t i2 = src2[jt];
            if (i2 >= 0) {
                const int64_t si = spin == 0 ? (i2 + other * dup_src) : (other + (int64_t)i2 * dup_src);
                acc = (sg2[jt] * sign2) > 0 ? fadd(acc, in[si]) : fsub(acc, in[si]);
            }
        }
        out[o_idx] = acc;
    }
}

// ---------------------------------------------------------------------------
// continued fraction (invert_zmtridiag, matrices_tridiag.f90:163-198)
// ---------------------------------------------------------------------------
__global__ void cf_kernel(int nchain, int ld, const int32_t *nlev, const double *diag,
                          const double *sub, const double *e, const double *ph,
                          const double *scale, int nw, const double *wn, double *G, int *flag)
{
    const int64_t total = (int64_t)nchain * nw;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(t / nw), w = (int)(t % nw);
        const int n = nlev[c];
        double gr = 0.0, gi = 0.0;
        if (n > 0) {
            const double *d = diag + (size_t)c * ld;
            const double *s = sub + (size_t)c * ld;
            const double zi = wn[w];
            const double p = ph[c], ee = e[c];
            // r = 1 / (z - ph*(d[n-1]-e))
            double ar = -p * (d[n - 1] - ee), ai = zi;
            double den = ar * ar + ai * ai;
            if (sqrt(den) < 2.220446049250313e-16) { atomicExch(flag, 1); den = 1e-300; }
            double rr = ar / den, ri = -ai / den;
            for (int it = n - 2; it >= 0; --it) {
                const double b2 = s[it + 1] * s[it + 1];
                ar = -p * (d[it] - ee) - rr * b2;
                ai = zi - ri * b2;
                den = ar * ar + ai * ai;
                if (sqrt(den) < 2.220446049250313e-16) { atomicExch(flag, 1); den = 1e-300; }
                rr = ar / den;
                ri = -ai / den;
            }
            gr = scale[c] * rr;
            gi = scale[c] * ri;
        }
        G[2 * t] = gr;
        G[2 * t + 1] = gi;
    }
}

// ---------------------------------------------------------------------------
// double occupancy: sum over elements with both impurity bits set
// ---------------------------------------------------------------------------
template <typename T>
__global__ void docc_kernel(int64_t dup, int64_t ddn, const uint8_t *imp_up, const uint8_t *imp_dn,
                            int mask, const T *psi, double *partials, unsigned *counter, double *sums)
{
    double s[2] = {0.0, 0.0};
    const int64_t n = dup * ddn;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = i % dup, r = i / dup;
        const double v = (double)psi[i];
        const double v2 = v * v;
        s[1] += v2;
        if ((imp_up[c] & mask) && (imp_dn[r] & mask)) s[0] += v2;
    }
    grid_sum<2>(s, partials, counter, sums);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
LaunchCfg plan_rows(const HamDev &H, int elem_bytes, int num_sms)
{
    LaunchCfg c;
    const int64_t rowbytes = H.dup * (int64_t)elem_bytes;
    const int kmax = H.up.ell_k > H.dn_kmax ? H.up.ell_k : H.dn_kmax;
    c.km = kmax <= 8 ? 8 : kmax <= 16 ? 16 : 0;
    // register budget: R*KM loaded values per thread under a 64-register cap
    int rcap = elem_bytes == 4 ? (c.km == 16 ? 2 : 4) : (c.km == 16 ? 1 : 2);
    if (c.km == 0) rcap = 4;
    // two blocks per SM when the staged rows fit in half of the shared memory
    const int64_t half = kMaxSmemBytes / 2;
    int R = 0;
    if (rowbytes <= half) {
        const int64_t cap = half / (rowbytes > 0 ? rowbytes : 1);
        R = cap >= 4 ? 4 : cap >= 2 ? 2 : 1;
        c.stage = true;
    } else if (rowbytes <= kMaxSmemBytes) {
        R = 1;
        c.stage = true;
    } else {
        R = 2;
        c.stage = false;
    }
    if (R > rcap) R = rcap;
    while (R > 1 && (H.ddn + R - 1) / R < num_sms) R >>= 1;   // keep every SM busy
    c.rows = R;
    int block = 512;
    if (H.dup < block) block = (int)(((H.dup + 31) / 32) * 32);
    if (block < 64) block = 64;
    c.block = block;
    c.smem = c.stage ? (size_t)R * (size_t)rowbytes : 0;
    const int64_t groups = (H.ddn + R - 1) / R;
    int per_sm = 1024 / block;
    if (per_sm > 16) per_sm = 16;
    if (c.smem > 0) {
        int by_smem = (int)((228 * 1024) / (c.smem + 4096));
        if (by_smem < per_sm) per_sm = by_smem;
    }
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)num_sms * per_sm;
    if (grid > groups) grid = groups;
    if (grid < 1) grid = 1;
    c.grid = (int)grid;          // upper bound; the launcher trims it to the resident blocks
    c.groups = groups;
    c.num_sms = num_sms;
    return c;
}

template <typename T, int R, bool S, bool P, int KM>
static cudaError_t launch_rows_k(const HamDev &H, const RowArgs &a, const LaunchCfg &cfg, cudaStream_t st)
{
    auto k = row_kernel<T, R, S, P, KM>;
    if (cfg.smem > 0) {
        // static + dynamic shared memory may exceed the 48 KB default
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem);
        if (e != cudaSuccess) return e;
    }
    // grid = resident blocks (registers and shared memory of this instance)
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, cfg.block, cfg.smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)cfg.num_sms * per_sm;
    if (grid > cfg.groups) grid = cfg.groups;
    if (grid > cfg.grid) grid = cfg.grid;
    if (grid < 1) grid = 1;
    k<<<(int)grid, cfg.block, cfg.smem, st>>>(H, a);
    return cudaGetLastError();
}

template <typename T, int R, bool S>
static cudaError_t launch_rows_t(const HamDev &H, const RowArgs &a, const LaunchCfg &cfg, cudaStream_t st)
{
    const bool p = H.up.packed != 0;
    switch (cfg.km) {
        case 8: return p ? launch_rows_k<T, R, S, true, 8>(H, a, cfg, st) : launch_rows_k<T, R, S, false, 8>(H, a, cfg, st);
        case 16: return p ? launch_rows_k<T, R, S, true, 16>(H, a, cfg, st) : launch_rows_k<T, R, S, false, 16>(H, a, cfg, st);
        default: return p ? launch_rows_k<T, R, S, true, 0>(H, a, cfg, st) : launch_rows_k<T, R, S, false, 0>(H, a, cfg, st);
    }
}

template <typename T>
static cudaError_t launch_rows_r(const HamDev &H, const RowArgs &a, const LaunchCfg &cfg, cudaStream_t st)
{
    if (cfg.stage) {
        switch (cfg.rows) {
            case 4: return launch_rows_t<T, 4, true>(H, a, cfg, st);
            case 2: return launch_rows_t<T, 2, true>(H, a, cfg, st);
            default: return launch_rows_t<T, 1, true>(H, a, cfg, st);
        }
    }
    switch (cfg.rows) {
        case 2: return launch_rows_t<T, 2, false>(H, a, cfg, st);
        default: return launch_rows_t<T, 1, false>(H, a, cfg, st);
    }
}

cudaError_t launch_rows(const HamDev &H, int dtype, const RowArgs &a, const LaunchCfg &cfg, cudaStream_t st)
{
    if (cfg.fast) return launch_rows_fast(H, dtype, a, cfg.num_sms, cfg.fast_shape, st);
    return dtype == EDK_F64 ? launch_rows_r<double>(H, a, cfg, st) : launch_rows_r<float>(H, a, cfg, st);
}

__global__ void set_int_kernel(int *p, int v) { *p = v; }

cudaError_t launch_set_int(int *p, int v, cudaStream_t st)
{
    set_int_kernel<<<1, 1, 0, st>>>(p, v);
    return cudaGetLastError();
}

cudaError_t launch_start_vector(int dtype, int64_t n, const double *tab, const void *user, void *v,
                                double *partials, unsigned *counter, double *sums, int grid,
                                cudaStream_t st)
{
    if (dtype == EDK_F64)
        start_kernel<double><<<grid, 256, 0, st>>>(n, tab, (const double *)user, (double *)v,
                                                   partials, counter, sums);
    else
        start_kernel<float><<<grid, 256, 0, st>>>(n, tab, (const float *)user, (float *)v,
                                                  partials, counter, sums);
    return cudaGetLastError();
}

cudaError_t launch_combine(int dtype, int64_t n, const void *const *vecs_dev, const double *coef_dev, int nv,
                           void *psi, int grid, cudaStream_t st)
{
    if (dtype == EDK_F64)
        combine_kernel<double><<<grid, 256, 0, st>>>(n, (const double *const *)vecs_dev, coef_dev, nv, (double *)psi);
    else
        combine_kernel<float><<<grid, 256, 0, st>>>(n, (const float *const *)vecs_dev, coef_dev, nv, (float *)psi);
    return cudaGetLastError();
}

cudaError_t launch_norm2(int dtype, int64_t n, const void *v, double *partials, unsigned *counter,
                         double *sums, int grid, cudaStream_t st)
{
    if (dtype == EDK_F64)
        norm2_kernel<double><<<grid, 256, 0, st>>>(n, (const double *)v, partials, counter, sums);
    else
        norm2_kernel<float><<<grid, 256, 0, st>>>(n, (const float *)v, partials, counter, sums);
    return cudaGetLastError();
}

cudaError_t launch_scale(int dtype, int64_t n, void *v, const double *sums, int which, void *psi,
                         const double *psi_coef, double *tri_sub0, int grid, cudaStream_t st)
{
    if (dtype == EDK_F64)
        scale_kernel<double><<<grid, 256, 0, st>>>(n, (double *)v, sums, which, (double *)psi,
                                                   psi_coef, tri_sub0);
    else
        scale_kernel<float><<<grid, 256, 0, st>>>(n, (float *)v, sums, which, (float *)psi,
                                                  psi_coef, tri_sub0);
    return cudaGetLastError();
}

cudaError_t launch_convert(int from, int to, int64_t n, const void *in, void *out, cudaStream_t st)
{
    const int grid = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    if (from == EDK_F32 && to == EDK_F64)
        convert_kernel<float, double><<<grid > 0 ? grid : 1, 256, 0, st>>>(n, (const float *)in, (double *)out);
    else if (from == EDK_F64 && to == EDK_F32)
        convert_kernel<double, float><<<grid > 0 ? grid : 1, 256, 0, st>>>(n, (const double *)in, (float *)out);
    else
        return cudaMemcpyAsync(out, in, (size_t)n * (from == EDK_F64 ? 8 : 4), cudaMemcpyDeviceToDevice, st);
    return cudaGetLastError();
}

cudaError_t launch_apply_c(int dtype, int spin, int64_t dother, int64_t dup_src, int64_t dup_tgt,
                           int64_t dim_sigma_tgt, const int32_t *src1, const int8_t *sg1,
                           const int32_t *src2, const int8_t *sg2, int sign2, const void *in, void *out,
                           cudaStream_t st)
{
    const int64_t n = dim_sigma_tgt * dother;
    int grid = (int)((n + 255) / 256);
    if (grid > 8192) grid = 8192;
    if (grid < 1) grid = 1;
    if (dtype == EDK_F64)
        apply_c_kernel<double><<<grid, 256, 0, st>>>(spin, dother, dup_src, dup_tgt, dim_sigma_tgt,
                                                     src1, sg1, src2, sg2, sign2, (const double *)in,
                                                     (double *)out);
    else
        apply_c_kernel<float><<<grid, 256, 0, st>>>(spin, dother, dup_src, dup_tgt, dim_sigma_tgt,
                                                    src1, sg1, src2, sg2, sign2, (const float *)in,
                                                    (float *)out);
    return cudaGetLastError();
}

cudaError_t launch_cf(int nchain, int ld, const int32_t *n, const double *diag, const double *sub,
                      const double *e, const double *ph, const double *scale, int nw,
                      const double *wn, double *G, int *flag, cudaStream_t st)
{
    const int64_t total = (int64_t)nchain * nw;
    int grid = (int)((total + 127) / 128);
    if (grid < 1) grid = 1;
    if (grid > 4096) grid = 4096;
    cf_kernel<<<grid, 128, 0, st>>>(nchain, ld, n, diag, sub, e, ph, scale, nw, wn, G, flag);
    return cudaGetLastError();
}

cudaError_t launch_double_occ(int dtype, const HamDev &H, int mask_up, int mask_dn, const void *psi,
                              double *partials, unsigned *counter, double *sums, int grid,
                              cudaStream_t st)
{
    (void)mask_dn;
    if (dtype == EDK_F64)
        docc_kernel<double><<<grid, 256, 0, st>>>(H.dup, H.ddn, H.up.imp, H.dn.imp, mask_up,
                                                  (const double *)psi, partials, counter, sums);
    else
        docc_kernel<float><<<grid, 256, 0, st>>>(H.dup, H.ddn, H.up.imp, H.dn.imp, mask_up,
                                                 (const float *)psi, partials, counter, sums);
    return cudaGetLastError();
}

}  // namespace edk
