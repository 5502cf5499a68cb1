// Fast row kernel for the common sector shape: impurity of at most 2 sites
// without Hund spin-flip/pair-hop terms, even dim_up (aligned column pairs),
// table widths of at most 16, fewer than 2^31 elements.  Same mathematics
// and, in FP64, the same per-element order of additions as the generic row
// kernel (edk_kernels.cu); what differs is instruction economy:
//   * each thread owns CPT adjacent columns (CPT = 2: 8- or 16-byte loads and
//     stores; CPT = 1: half the registers, so twice the resident warps);
//   * the down-spin neighbour rows of the R staged rows (offsets and values)
//     sit in shared memory for the whole group, padded to KMD entries of
//     value 0 on the own row; the up-table entries are padded to KMU with the
//     own column (loads stay unconditional, so they issue back to back);
//   * all table entries and neighbour elements of a column pair are loaded
//     before the ordered accumulation;
//   * x is read with an L2 evict_last policy, the streamed vectors and all
//     outputs with evict_first, so the neighbour rows stay resident longer;
//   * coefficients and accumulators are FP64 for both vector types (hmadd):
//     FP32 vectors are widened and fused into FP64 accumulators, with the
//     down-spin hops in a second accumulator (two independent FMA chains);
//     FP64 keeps one chain with separate multiply and add so the result stays
//     bit-identical to a sequential HAIMupdo_multr.
// The launch shape (threads per block and blocks per SM, rows per group) is
// a template choice; the host times the feasible shapes once per sector
// Hamiltonian and element type and keeps the fastest.
#pragma once
#include "edk_device.cuh"

namespace edk {

template <typename T> struct V2;
template <> struct V2<float> { using t = float2; };
template <> struct V2<double> { using t = double2; };

// The R staged rows are interleaved element by element in shared memory
// (xs[j*R + r]), so the R values a gather needs at target j are one aligned
// vector load; RowVec<T,R> is that vector.
template <typename T, int R> struct alignas(sizeof(T) * R <= 16 ? sizeof(T) * R : 16) RowVec { T v[R]; };

template <typename T, int R>
__device__ __forceinline__ RowVec<T, R> lds_rows(const T *xs, uint32_t j)
{
    return *reinterpret_cast<const RowVec<T, R> *>(xs + (size_t)j * R);
}

template <typename T> __device__ __forceinline__ void ld_cols(const T *p, uint64_t pol, T (&v)[2])
{
    const auto t = ld2(p, pol);
    v[0] = t.x;
    v[1] = t.y;
}
template <typename T> __device__ __forceinline__ void ld_cols(const T *p, uint64_t pol, T (&v)[1]) { v[0] = ld1(p, pol); }
template <typename T> __device__ __forceinline__ void st_cols(T *p, const T (&v)[2], uint64_t pol)
{
    st2(p, v[0], v[1], pol);
}
template <typename T> __device__ __forceinline__ void st_cols(T *p, const T (&v)[1], uint64_t pol) { st1(p, v[0], pol); }

// T: element type; R: staged rows per group; KMU: bound on the up-table width;
// KMD: bound on the down-table row length; NTHR threads per block, at least
// MINB blocks per SM; CPT columns per thread.
template <typename T, int R, int KMU, int KMD, int NTHR, int MINB, int CPT = 2>
__global__ void __launch_bounds__(NTHR, MINB) row_fast_kernel(const HamDev H, const RowArgs a)
{
    constexpr bool EXACT = sizeof(T) == 8;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double pal_s[256];
    __shared__ int s_ioff[17];
    __shared__ double s_icoef[96];
    __shared__ int s_nofs[R][KMD];
    __shared__ double s_hd[R][KMD];
    T *xs = reinterpret_cast<T *>(smem_raw);
    const int dup = (int)H.dup;
    const int64_t ddn = H.ddn;
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
    {
        for (int i = threadIdx.x; i < H.up.npal; i += blockDim.x) pal_s[i] = H.up.pal[i];
        const int nio = H.ncfg * H.ncfg + 1;
        for (int i = threadIdx.x; i < nio; i += blockDim.x) s_ioff[i] = H.int_off[i];
        const int ncoef = H.int_off[nio - 1];
        for (int i = threadIdx.x; i < ncoef; i += blockDim.x) s_icoef[i] = H.int_coef[i];
    }
    const uint64_t keep = l2_keep(), stream = l2_stream();
    const uint32_t *__restrict__ ell = H.up.ell;
    const int K = H.up.ell_k;
    const double *__restrict__ dnv = H.dn.val;
    const double *__restrict__ upd = H.up.diag;
    const double *__restrict__ dnd = H.dn.diag;
    const int ncfg = H.ncfg;

    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    const int64_t ngroups = (ddn + R - 1) / R;
    for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        int row[R], cd[R];
        double dd[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int64_t q = g * R + r;
            row[r] = q < ddn ? H.row_order[q] : -1;
            const int rr = row[r] >= 0 ? row[r] : 0;
            dd[r] = dnd[rr];
            cd[r] = (int)H.dn.imp[rr];
        }
        __syncthreads();
        // neighbour rows (offsets, values) of the group, padded with value 0 on the own row
        for (int t = threadIdx.x; t < R * KMD; t += blockDim.x) {
            const int r = t / KMD, f = t % KMD;
            const int64_t q = g * R + r;
            const int rr = q < ddn ? H.row_order[q] : 0;
            const int f0 = H.dn.ptr[rr], nd = H.dn.ptr[rr + 1] - f0;
            const bool ok = f < nd;
            s_nofs[r][f] = (ok ? H.dn.tgt[f0 + f] : rr) * dup;
            s_hd[r][f] = ok ? dnv[f0 + f] : 0.0;
        }
        // stage the R rows interleaved: xs[c*R + r]
        {
            constexpr int V = 16 / sizeof(T);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const T *src = x + (int64_t)(row[r] >= 0 ? row[r] : 0) * dup;
                const uintptr_t addr = reinterpret_cast<uintptr_t>(src);
                int head = (int)(((16u - (addr & 15u)) & 15u) / sizeof(T));
                if (head > dup) head = dup;
                for (int i = threadIdx.x; i < head; i += blockDim.x) xs[i * R + r] = __ldg(src + i);
                const int nv = (dup - head) / V;
                const int4 *sv = reinterpret_cast<const int4 *>(src + head);
                for (int i = threadIdx.x; i < nv; i += blockDim.x) {
                    const int4 q = __ldg(sv + i);
                    T tmp[V];
                    memcpy(tmp, &q, 16);
#pragma unroll
                    for (int v = 0; v < V; ++v) xs[(head + i * V + v) * R + r] = tmp[v];
                }
                for (int i = head + nv * V + threadIdx.x; i < dup; i += blockDim.x) xs[i * R + r] = __ldg(src + i);
            }
        }
        __syncthreads();

        for (int c = CPT * threadIdx.x; c < dup; c += CPT * blockDim.x) {
            // ---- loads ----
            uint32_t ent[KMU][CPT];
#pragma unroll
            for (int k = 0; k < KMU; ++k) {
                if (CPT == 2) {
                    const uint2 e2 = k < K ? ldu2(ell + (size_t)k * dup + c) : make_uint2((uint32_t)c, (uint32_t)(c + 1));
                    ent[k][0] = e2.x;
                    ent[k][CPT - 1] = e2.y;
                } else {
                    ent[k][0] = k < K ? __ldg(ell + (size_t)k * dup + c) : (uint32_t)c;
                }
            }
            T xd[R][KMD][CPT];
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int f = 0; f < KMD; ++f) ld_cols(x + s_nofs[r][f] + c, keep, xd[r][f]);
            // bring the next iteration's neighbour elements towards L2 while this one computes
            if (c + CPT * (int)blockDim.x < dup) {
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int f = 0; f < KMD; ++f) prefetch_l2(x + s_nofs[r][f] + c + CPT * blockDim.x);
            }
            int cu[CPT];
            double du[CPT];
            RowVec<T, R> o[CPT];
#pragma unroll
            for (int e = 0; e < CPT; ++e) {
                cu[e] = H.up.imp[c + e];
                du[e] = upd[c + e];
                o[e] = lds_rows<T, R>(xs, c + e);
            }
            double acc[R][CPT], accd[R][CPT];
            // ---- ordered accumulation: density terms, diagonal ----
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int e = 0; e < CPT; ++e) {
                    double a0 = 0.0;
                    const int g0 = cu[e] * ncfg + cd[r];
                    for (int o2 = s_ioff[g0]; o2 < s_ioff[g0 + 1]; ++o2) a0 = hmadd<T>(a0, s_icoef[o2], o[e].v[r]);
                    acc[r][e] = hmadd<T>(a0, fadd(du[e], dd[r]), o[e].v[r]);
                    accd[r][e] = 0.0;
                }
            // ---- up-spin hops: one vector load serves the R rows ----
#pragma unroll
            for (int k = 0; k < KMU; ++k) {
                if (k >= K) break;
#pragma unroll
                for (int e = 0; e < CPT; ++e) {
                    const RowVec<T, R> g = lds_rows<T, R>(xs, ent[k][e] & 0xFFFFFFu);
                    const double h = pal_s[ent[k][e] >> 24];
#pragma unroll
                    for (int r = 0; r < R; ++r) acc[r][e] = hmadd<T>(acc[r][e], h, g.v[r]);
                }
            }
            // ---- down-spin hops (FP32 vectors: second accumulator) ----
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int f = 0; f < KMD; ++f) {
                    const double h = s_hd[r][f];
#pragma unroll
                    for (int e = 0; e < CPT; ++e) {
                        if (EXACT) acc[r][e] = hmadd<T>(acc[r][e], h, xd[r][f][e]);
                        else accd[r][e] = hmadd<T>(accd[r][e], h, xd[r][f][e]);
                    }
                }
            if (!EXACT) {
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int e = 0; e < CPT; ++e) acc[r][e] += accd[r][e];
            }
            // ---- epilogue ----
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (row[r] < 0) continue;
                const size_t i = (size_t)row[r] * dup + c;
                T *y = static_cast<T *>(a.y) + i;
                T xo[CPT];
#pragma unroll
                for (int e = 0; e < CPT; ++e) xo[e] = o[e].v[r];
                if (a.mode == kModeHv) {
                    T out[CPT];
#pragma unroll
                    for (int e = 0; e < CPT; ++e) out[e] = (T)acc[r][e];
                    st_cols(y, out, stream);
                } else if (a.mode == kModeFirst) {
                    T st[CPT];
#pragma unroll
                    for (int e = 0; e < CPT; ++e) {
                        const double v = (double)xo[e];
                        st[e] = (T)(acc[r][e] - gam1 * v);
                        const double sd = (double)st[e];
                        s0 += sd * sd; s1 += sd * v; s2 += v * v;
                    }
                    st_cols(y, st, stream);
                } else if (a.mode == kModeStep) {
                    T vkt[CPT], vmt[CPT];
                    ld_cols(static_cast<const T *>(a.vk) + i, stream, vkt);
                    if (a.vkm1) ld_cols(static_cast<const T *>(a.vkm1) + i, stream, vmt);
                    else
#pragma unroll
                        for (int e = 0; e < CPT; ++e) vmt[e] = T(0);
                    T wt[CPT], vt[CPT];
#pragma unroll
                    for (int e = 0; e < CPT; ++e) {
                        const double sv = (double)xo[e], vk = (double)vkt[e], vm = (double)vmt[e];
                        vt[e] = (T)((sv - delta * vk) * inv_b);
                        const double hv1 = (acc[r][e] - delta * (sv + gam * vk + beta_k * vm)) * inv_b;
                        const double w = hv1 - beta_k1 * vk;
                        wt[e] = (T)(w - gam1 * (double)vt[e]);
                        const double wd = (double)wt[e], vd = (double)vt[e];
                        s0 += wd * wd; s1 += wd * vd; s2 += vd * vd;
                    }
                    st_cols(y, wt, stream);
                    st_cols(static_cast<T *>(a.vout) + i, vt, stream);
                    if (a.psi) {
                        T *p = static_cast<T *>(a.psi) + i;
                        T pv[CPT];
                        ld_cols(p, stream, pv);
#pragma unroll
                        for (int e = 0; e < CPT; ++e) pv[e] = (T)((double)pv[e] + cpsi * (double)vt[e]);
                        st_cols(p, pv, stream);
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < CPT; ++e) {
                        const double rr = acc[r][e] - a.eshift * (double)xo[e];
                        s0 += rr * rr; s2 += (double)xo[e] * (double)xo[e];
                    }
                }
            }
        }
    }
    if (a.mode == kModeHv) return;
    double v[4] = {s0, s1, s2, 0.0};
    if (grid_sum<4>(v, a.partials, a.counter, a.sums_out))
        if (a.mode == kModeFirst || a.mode == kModeStep) lanczos_finalize(a, ks);
}

// Launch of one instance: grid = SMs x resident blocks, at most one block per
// row group; blocks narrower than NTHR when dim_up is small.
template <typename T, int R, int KMU, int KMD, int NTHR, int MINB, int CPT = 2>
cudaError_t launch_fast_t(const HamDev &H, const RowArgs &a, int num_sms, cudaStream_t st)
{
    auto k = row_fast_kernel<T, R, KMU, KMD, NTHR, MINB, CPT>;
    const size_t smem = (size_t)R * (size_t)H.dup * sizeof(T);
    // static + dynamic shared memory may exceed the 48 KB default
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int cols = (int)((H.dup + CPT - 1) / CPT);
    int block = NTHR;
    if (cols < block) block = ((cols + 31) / 32) * 32;
    if (block < 32) block = 32;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const int64_t groups = (H.ddn + R - 1) / R;
    int64_t grid = (int64_t)num_sms * per_sm;
    if (grid > groups) grid = groups;
    if (grid < 1) grid = 1;
    k<<<(int)grid, block, smem, st>>>(H, a);
    return cudaGetLastError();
}

// Shape dispatch for one element type (edk_rows_fast.cu: FP32, edk_rows_fast64.cu: FP64).
cudaError_t launch_fast_f32(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st);
cudaError_t launch_fast_f64(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st);

}  // namespace edk
