// Row kernel with asynchronous row staging (the launch shapes of kind 1).
//
// Same sector shapes, mathematics and, in FP64, the same per-element order of
// additions as the fast row kernel (edk_rows_fast.cuh); what changes is how
// the memory system is kept busy:
//   * the R rows of x that a row group gathers its up-spin hops from are
//     staged into shared memory by one cp.async.bulk copy per row (global ->
//     shared, completed on an mbarrier), into the second half of a double
//     buffer while the block computes the current group; the few elements of
//     a row outside its 16-byte aligned middle are filled by plain loads, so
//     any vector alignment works and nothing past a row is read;
//   * each thread owns one column of the group's R rows.  The loads of the
//     next column it will compute -- up-table entries, the R x KMD down-spin
//     neighbour elements, v_k and v_{k-1} -- are issued before the current
//     column is computed (a two-deep register pipeline), so a warp always has
//     one column's worth of global loads in flight while it does arithmetic;
//   * the next group's neighbour-row table (offsets and values) is prepared
//     in shared memory during the current group.
// All copies read this GPU's own memory; there is no cluster and no multicast.
// Every wait on an mbarrier is bounded: after kMbarSpins failed polls the
// block records EDK's timeout flag (flags[1] = 2) and carries on, so the
// launch always ends.
#pragma once
#include "edk_rows_fast.cuh"   // ld_cols

namespace edk {

constexpr int kMbarSpins = 1 << 24;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *b, uint32_t tx)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(tx) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase with the given parity; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity)
{
    for (int i = 0; i < kMbarSpins; ++i)
        if (mbar_try_wait(b, parity)) return true;
    return false;
}
// 1-D bulk copy global -> this CTA's shared memory; both addresses 16-byte
// aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }


// streaming stores of CPT adjacent elements
__device__ __forceinline__ void st_cs(float *p, const float (&v)[1]) { __stcs(p, v[0]); }
__device__ __forceinline__ void st_cs(double *p, const double (&v)[1]) { __stcs(p, v[0]); }
__device__ __forceinline__ void st_cs(float *p, const float (&v)[2]) { __stcs(reinterpret_cast<float2 *>(p), make_float2(v[0], v[1])); }
__device__ __forceinline__ void st_cs(double *p, const double (&v)[2])
{
    __stcs(reinterpret_cast<double2 *>(p), make_double2(v[0], v[1]));
}

// The 16-byte aligned middle [a16, e16) of a row starting at `src` with n
// elements: offsets in elements from the row start, mid = 0 when the row has
// no aligned 16-byte block.
template <typename T>
__device__ __forceinline__ void row_middle(const T *src, int n, int &c16, int &ce16, uint32_t &bytes)
{
    const uintptr_t a = reinterpret_cast<uintptr_t>(src);
    const uintptr_t e = a + (uintptr_t)n * sizeof(T);
    const uintptr_t a16 = (a + 15) & ~(uintptr_t)15, e16 = e & ~(uintptr_t)15;
    if (e16 > a16) {
        c16 = (int)((a16 - a) / sizeof(T));
        ce16 = (int)((e16 - a) / sizeof(T));
        bytes = (uint32_t)(e16 - a16);
    } else {
        c16 = ce16 = n;   // everything is ragged
        bytes = 0;
    }
}

// T: element type; R: rows per group; KMU/KMD: up/down table-width bounds;
// NTHR threads per block (one column each), at least MINB blocks per SM.
// slot: elements per staged-row slot (a multiple of 16 bytes, >= dup + 16/sizeof(T)).
// STEP: the launch is a fused Lanczos step (mode kModeStep known at compile
// time); otherwise the mode is read from the arguments.
template <typename T, int R, int KMU, int KMD, int NTHR, int MINB, int CPT, bool PIPE, bool S32, bool STEP>
__global__ void __launch_bounds__(NTHR, MINB) row_tma_kernel(const HamDev H, const RowArgs a, const int slot)
{
    static_assert(!S32 || sizeof(T) == 4, "FP32 hop sums are for FP32 vectors");
    constexpr bool EXACT = sizeof(T) == 8;
    constexpr int kMeta = R * KMD;            // threads that prepare the neighbour table
    constexpr int kRagged = 64;               // first thread of the ragged-end fill
    static_assert(NTHR >= kRagged + 32, "block too small");
    static_assert(kMeta + R + 1 <= kRagged, "too many neighbour entries");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double pal_s[256];
    __shared__ float pal32[S32 ? 256 : 1];
    __shared__ int s_ioff[17];
    __shared__ double s_icoef[96];
    __shared__ double s_dsum[16];   // FP32 vectors: the density coefficients of a configuration pair, summed
    __shared__ int s_nofs[2][R][KMD];
    __shared__ double s_hd[2][R][KMD];
    __shared__ int s_row[2][R], s_cd[2][R], s_off[2][R];
    __shared__ double s_dd[2][R];
    __shared__ __align__(8) uint64_t s_bar[2];
    T *rowbuf = reinterpret_cast<T *>(smem_raw);   // [2][R][slot]
    const int dup = (int)H.dup;
    const int64_t ddn = H.ddn;
    const T *__restrict__ x = static_cast<const T *>(a.x);
    const int tid = threadIdx.x;

    const int mode = STEP ? (int)kModeStep : a.mode;
    double delta = 0.0, gam = 0.0, gam1 = a.gamma1, beta_k = 0.0, beta_k1 = 0.0, inv_b = 0.0, cpsi = 0.0;
    const int ks = step_index(a);
    if (mode == kModeStep) {
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
    {
        for (int i = tid; i < H.up.npal; i += NTHR) {
            pal_s[i] = H.up.pal[i];
            if (S32) pal32[i] = (float)H.up.pal[i];
        }
        const int nio = H.ncfg * H.ncfg + 1;
        for (int i = tid; i < nio; i += NTHR) s_ioff[i] = H.int_off[i];
        const int ncoef = H.int_off[nio - 1];
        for (int i = tid; i < ncoef; i += NTHR) s_icoef[i] = H.int_coef[i];
        if (!EXACT && tid < nio - 1) {
            double t = 0.0;
            for (int o2 = H.int_off[tid]; o2 < H.int_off[tid + 1]; ++o2) t += H.int_coef[o2];
            s_dsum[tid] = t;
        }
    }
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();

    const uint64_t keep = l2_keep(), stream = l2_stream();
    const uint32_t *__restrict__ ell = H.up.ell;
    const int K = H.up.ell_k;
    const double *__restrict__ upd = H.up.diag;
    const int ncfg = H.ncfg;
    const int64_t ngroups = (ddn + R - 1) / R;

    // Group g into buffer b: neighbour table and row metadata (threads below
    // kMeta + R), the rows' aligned middles by bulk copy (thread kMeta + R)
    // and their ragged ends by plain loads (threads from kRagged on).
    auto prepare = [&](int64_t g, int b) {
        if (tid < kMeta) {
            const int r = tid / KMD, f = tid % KMD;
            const int64_t q = g * R + r;
            const int rr = q < ddn ? H.row_order[q] : 0;
            const int f0 = H.dn.ptr[rr], nd = H.dn.ptr[rr + 1] - f0;
            const bool ok = f < nd;
            s_nofs[b][r][f] = (ok ? H.dn.tgt[f0 + f] : rr) * dup;
            s_hd[b][r][f] = ok ? H.dn.val[f0 + f] : 0.0;
        } else if (tid < kMeta + R) {
            const int r = tid - kMeta;
            const int64_t q = g * R + r;
            const int row = q < ddn ? H.row_order[q] : -1;
            const int rr = row >= 0 ? row : 0;
            s_row[b][r] = row;
            s_dd[b][r] = H.dn.diag[rr];
            s_cd[b][r] = (int)H.dn.imp[rr];
            s_off[b][r] = (int)((reinterpret_cast<uintptr_t>(x + (int64_t)rr * dup) & 15) / sizeof(T));
        } else if (tid == kMeta + R) {
            // the bulk copies: one expect_tx for the group's total, then one copy per row
            uint32_t total = 0;
            const T *src[R];
            int c16[R], ce16[R];
            uint32_t bytes[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int64_t q = g * R + r;
                const int rr = q < ddn ? H.row_order[q] : 0;
                src[r] = x + (int64_t)rr * dup;
                row_middle(src[r], dup, c16[r], ce16[r], bytes[r]);
                total += bytes[r];
            }
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&s_bar[b], total);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (bytes[r] == 0) continue;
                const int off = (int)((reinterpret_cast<uintptr_t>(src[r]) & 15) / sizeof(T));
                T *dst = rowbuf + ((size_t)b * R + r) * slot + off + c16[r];
                bulk_g2s(dst, src[r] + c16[r], bytes[r], &s_bar[b]);
            }
        } else if (tid >= kRagged) {
            const int nr = NTHR - kRagged;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int64_t q = g * R + r;
                const int rr = q < ddn ? H.row_order[q] : 0;
                const T *src = x + (int64_t)rr * dup;
                int c16, ce16;
                uint32_t bytes;
                row_middle(src, dup, c16, ce16, bytes);
                const int off = (int)((reinterpret_cast<uintptr_t>(src) & 15) / sizeof(T));
                T *dst = rowbuf + ((size_t)b * R + r) * slot + off;
                const int nhead = c16, ntail = dup - ce16;
                for (int i = tid - kRagged; i < nhead + ntail; i += nr) {
                    const int c = i < nhead ? i : ce16 + (i - nhead);
                    dst[c] = __ldg(src + c);
                }
            }
        }
    };

    // per-column loads (the pipeline stage): CPT adjacent columns
    struct Ld {
        uint32_t ent[KMU][CPT];
        T xd[R][KMD][CPT];
        T vk[R][CPT], vm[R][CPT];
        int cu[CPT];
        double du[CPT];
    };
    auto load = [&](int c, const int (&row)[R], const int (&nofs)[R][KMD], Ld &L) {
#pragma unroll
        for (int k = 0; k < KMU; ++k) {
            if (CPT == 2) {
                const uint2 e2 = k < K ? ldu2(ell + (size_t)k * dup + c) : make_uint2((uint32_t)c, (uint32_t)c + 1);
                L.ent[k][0] = e2.x;
                L.ent[k][CPT - 1] = e2.y;
            } else {
                L.ent[k][0] = k < K ? __ldg(ell + (size_t)k * dup + c) : (uint32_t)c;
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int f = 0; f < KMD; ++f) ld_cols(x + nofs[r][f] + c, keep, L.xd[r][f]);
        if (mode == kModeStep) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const size_t i = (size_t)(row[r] >= 0 ? row[r] : 0) * dup + c;
                ld_cols(static_cast<const T *>(a.vk) + i, stream, L.vk[r]);
                if (a.vkm1) ld_cols(static_cast<const T *>(a.vkm1) + i, stream, L.vm[r]);
                else
#pragma unroll
                    for (int e = 0; e < CPT; ++e) L.vm[r][e] = T(0);
            }
        }
#pragma unroll
        for (int e = 0; e < CPT; ++e) {
            L.cu[e] = H.up.imp[c + e];
            L.du[e] = __ldg(upd + c + e);
        }
    };

    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    auto compute = [&](int c, int b, const int (&row)[R], const int (&cd)[R], const double (&dd)[R],
                       const T *(&xs)[R], const float (&hd32)[R][KMD], const Ld &L) {
        T o[R][CPT];
        double acc[R][CPT], accd[R][CPT];
        float u32[R][CPT], d32[R][CPT];
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int e = 0; e < CPT; ++e) o[r][e] = xs[r][c + e];
        // density terms, diagonal (FP64)
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int e = 0; e < CPT; ++e) {
                const int g0 = L.cu[e] * ncfg + cd[r];
                if (EXACT) {
                    // the reference's order: each density term, then the diagonal
                    double a0 = 0.0;
                    for (int o2 = s_ioff[g0]; o2 < s_ioff[g0 + 1]; ++o2) a0 = hmadd<T>(a0, s_icoef[o2], o[r][e]);
                    acc[r][e] = hmadd<T>(a0, fadd(L.du[e], dd[r]), o[r][e]);
                } else {
                    acc[r][e] = (s_dsum[g0] + (L.du[e] + dd[r])) * (double)o[r][e];
                }
                accd[r][e] = 0.0;
                u32[r][e] = 0.f;
                d32[r][e] = 0.f;
            }
        // up-spin hops from the staged rows: one table entry serves the R rows
        // (a table exactly KMU wide runs the unrolled loop without tests)
        const int kend = K == KMU ? KMU : K;
#pragma unroll
        for (int k = 0; k < KMU; ++k) {
            if (K != KMU && k >= kend) break;
#pragma unroll
            for (int e = 0; e < CPT; ++e) {
                const uint32_t t = L.ent[k][e] & 0xFFFFFFu;
                if (S32) {
                    const float h = pal32[L.ent[k][e] >> 24];
#pragma unroll
                    for (int r = 0; r < R; ++r) u32[r][e] = fmaf(h, (float)xs[r][t], u32[r][e]);
                } else {
                    const double h = pal_s[L.ent[k][e] >> 24];
#pragma unroll
                    for (int r = 0; r < R; ++r) acc[r][e] = hmadd<T>(acc[r][e], h, xs[r][t]);
                }
            }
        }
        // down-spin hops (FP32 vectors: a second accumulator)
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int f = 0; f < KMD; ++f)
#pragma unroll
                for (int e = 0; e < CPT; ++e) {
                    if (S32) {
                        d32[r][e] = fmaf(hd32[r][f], (float)L.xd[r][f][e], d32[r][e]);
                    } else {
                        const double h = s_hd[b][r][f];
                        if (EXACT) acc[r][e] = hmadd<T>(acc[r][e], h, L.xd[r][f][e]);
                        else accd[r][e] = hmadd<T>(accd[r][e], h, L.xd[r][f][e]);
                    }
                }
        if (!EXACT) {
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int e = 0; e < CPT; ++e)
                    acc[r][e] += S32 ? (double)u32[r][e] + (double)d32[r][e] : accd[r][e];
        }
        // epilogue
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (row[r] < 0) continue;
            const size_t i = (size_t)row[r] * dup + c;
            T *y = static_cast<T *>(a.y) + i;
            if (mode == kModeHv) {
                T out[CPT];
#pragma unroll
                for (int e = 0; e < CPT; ++e) out[e] = (T)acc[r][e];
                st_cs(y, out);
            } else if (mode == kModeFirst) {
                T st[CPT];
#pragma unroll
                for (int e = 0; e < CPT; ++e) {
                    const double v = (double)o[r][e];
                    st[e] = (T)(acc[r][e] - gam1 * v);
                    const double sd = (double)st[e];
                    s0 += sd * sd; s1 += sd * v; s2 += v * v;
                }
                st_cs(y, st);
            } else if (mode == kModeStep) {
                T wt[CPT], vt[CPT];
#pragma unroll
                for (int e = 0; e < CPT; ++e) {
                    const double sv = (double)o[r][e], vk = (double)L.vk[r][e], vm = (double)L.vm[r][e];
                    vt[e] = (T)((sv - delta * vk) * inv_b);
                    const double hv1 = (acc[r][e] - delta * (sv + gam * vk + beta_k * vm)) * inv_b;
                    const double w = hv1 - beta_k1 * vk;
                    wt[e] = (T)(w - gam1 * (double)vt[e]);
                    const double wd = (double)wt[e], vd = (double)vt[e];
                    s0 += wd * wd; s1 += wd * vd; s2 += vd * vd;
                }
                st_cs(y, wt);
                st_cs(static_cast<T *>(a.vout) + i, vt);
                if (a.psi) {
#pragma unroll
                    for (int e = 0; e < CPT; ++e) {
                        T *p = static_cast<T *>(a.psi) + i + e;
                        *p = (T)((double)*p + cpsi * (double)vt[e]);
                    }
                }
            } else {
#pragma unroll
                for (int e = 0; e < CPT; ++e) {
                    const double rr = acc[r][e] - a.eshift * (double)o[r][e];
                    s0 += rr * rr; s2 += (double)o[r][e] * (double)o[r][e];
                }
            }
        }
    };

    if ((int64_t)blockIdx.x < ngroups) prepare(blockIdx.x, 0);
    __syncthreads();
    int it = 0;
    for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x, ++it) {
        const int b = it & 1;
        const int64_t gn = g + gridDim.x;
        // buffer b ^ 1 was last read in the previous group (before the barrier below)
        if (gn < ngroups) prepare(gn, b ^ 1);
        int row[R], cd[R], nofs[R][KMD];
        double dd[R];
        float hd32[R][KMD];
        const T *xs[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            row[r] = s_row[b][r];
            cd[r] = s_cd[b][r];
            dd[r] = s_dd[b][r];
            xs[r] = rowbuf + ((size_t)b * R + r) * slot + s_off[b][r];
#pragma unroll
            for (int f = 0; f < KMD; ++f) {
                nofs[r][f] = s_nofs[b][r][f];
                hd32[r][f] = S32 ? (float)s_hd[b][r][f] : 0.f;
            }
        }
        if (!mbar_wait(&s_bar[b], (uint32_t)((it >> 1) & 1))) atomicExch(&a.flags[1], 2);
        // the group's columns, CPT adjacent ones per thread
        constexpr int STRIDE = NTHR * CPT;
        if (PIPE) {
            // the loads of the next columns in flight while these are computed
            Ld A, B;
            int c = tid * CPT;
            if (c < dup) load(c, row, nofs, A);
            while (c < dup) {
                const int c1 = c + STRIDE;
                if (c1 < dup) load(c1, row, nofs, B);
                compute(c, b, row, cd, dd, xs, hd32, A);
                if (c1 >= dup) break;
                const int c2 = c1 + STRIDE;
                if (c2 < dup) load(c2, row, nofs, A);
                compute(c1, b, row, cd, dd, xs, hd32, B);
                c = c2;
            }
        } else {
            for (int c = tid * CPT; c < dup; c += STRIDE) {
                Ld A;
                load(c, row, nofs, A);
                compute(c, b, row, cd, dd, xs, hd32, A);
            }
        }
        __syncthreads();
    }
    if (mode == kModeHv) return;
    double v[4] = {s0, s1, s2, 0.0};
    if (grid_sum<4>(v, a.partials, a.counter, a.sums_out))
        if (mode == kModeFirst || mode == kModeStep) lanczos_finalize(a, ks);
}

// Staged-row slot of the kernel above: dup elements plus up to 15 bytes of
// alignment offset, rounded to 16 bytes.
inline int tma_slot_elems(int64_t dup, int elem_bytes)
{
    const int v = 16 / elem_bytes;
    return (int)((dup + v + v - 1) / v * v);
}

template <typename T, int R, int KMU, int KMD, int NTHR, int MINB, int CPT, bool PIPE, bool S32>
cudaError_t launch_tma_t(const HamDev &H, const RowArgs &a, int num_sms, cudaStream_t st)
{
    auto k = a.mode == kModeStep ? row_tma_kernel<T, R, KMU, KMD, NTHR, MINB, CPT, PIPE, S32, true>
                                 : row_tma_kernel<T, R, KMU, KMD, NTHR, MINB, CPT, PIPE, S32, false>;
    const int slot = tma_slot_elems(H.dup, sizeof(T));
    const size_t smem = (size_t)2 * R * slot * sizeof(T);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NTHR, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int64_t groups = (H.ddn + R - 1) / R;
    int64_t grid = (int64_t)num_sms * per_sm;
    if (grid > groups) grid = groups;
    if (grid < 1) grid = 1;
    k<<<(int)grid, NTHR, smem, st>>>(H, a, slot);
    return cudaGetLastError();
}

cudaError_t launch_tma_f32(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st);
cudaError_t launch_tma_f64(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st);

}  // namespace edk
