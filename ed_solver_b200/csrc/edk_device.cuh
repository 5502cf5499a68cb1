// Device helpers shared by the row kernels (edk_kernels.cu, edk_rows_fast.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include "edk_internal.h"

namespace edk {

// ---------------------------------------------------------------------------
// arithmetic without contraction
// ---------------------------------------------------------------------------
__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }

// One term of an H*v accumulation.  Coefficients and accumulators are FP64
// for both vector types.  FP64 vectors: separate multiply and add, so the sum
// equals a sequential FP64 HAIMupdo_multr bit for bit; FP32 vectors: the
// element is widened and fused into the FP64 accumulator.  The FP32 path
// therefore applies exactly the FP64 operator to FP32-stored vectors; only
// the storage of the Krylov vectors is rounded.
template <typename T>
__device__ __forceinline__ double hmadd(double acc, double h, T x)
{
    if (sizeof(T) == 8) return fadd(acc, fmul(h, (double)x));
    return fma(h, (double)x, acc);
}

// ---------------------------------------------------------------------------
// deterministic block / grid reductions of NQ doubles
// ---------------------------------------------------------------------------
template <int NQ>
__device__ __forceinline__ void block_sum(double (&v)[NQ], double (*red)[32])
{
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NQ; ++q) red[q][warp] = v[q];
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double t = lane < nw ? red[q][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            v[q] = t;
        }
    }
}

// Writes this block's NQ partial sums; the last block to arrive sums all
// partials in block order into `out` and returns true (in thread 0 only).
template <int NQ>
__device__ bool grid_sum(double (&v)[NQ], double *partials, unsigned *counter, double *out)
{
    __shared__ double red[NQ][32];
    __shared__ bool last;
    block_sum<NQ>(v, red);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) partials[(size_t)blockIdx.x * NQ + q] = v[q];
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double t = 0.0;
            for (unsigned b = lane; b < gridDim.x; b += 32)
                t += __ldcg(&partials[(size_t)b * NQ + q]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (lane == 0) out[q] = t;
        }
    }
    if (threadIdx.x == 0) *counter = 0u;
    return threadIdx.x == 0;
}

// ---------------------------------------------------------------------------
// row staging: 16-byte global loads, scalar shared stores (any alignment)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void stage_row(T *dst, const T *src, int64_t n)
{
    constexpr int V = 16 / sizeof(T);
    const uintptr_t addr = reinterpret_cast<uintptr_t>(src);
    int64_t head = (int64_t)(((16u - (addr & 15u)) & 15u) / sizeof(T));
    if (head > n) head = n;
    for (int64_t i = threadIdx.x; i < head; i += blockDim.x) dst[i] = __ldg(src + i);
    const int64_t nv = (n - head) / V;
    const int4 *sv = reinterpret_cast<const int4 *>(src + head);
    for (int64_t i = threadIdx.x; i < nv; i += blockDim.x) {
        int4 q = __ldg(sv + i);
        T tmp[V];
        memcpy(tmp, &q, 16);
#pragma unroll
        for (int v = 0; v < V; ++v) dst[head + i * V + v] = tmp[v];
    }
    for (int64_t i = head + nv * V + threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(src + i);
}


// L2 eviction-priority policies (createpolicy) and loads/stores carrying them.
__device__ __forceinline__ uint64_t l2_keep()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_stream()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ float2 ld2(const float *p, uint64_t pol)
{
    float2 v;
    asm volatile("ld.global.nc.L2::cache_hint.v2.f32 {%0,%1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double2 ld2(const double *p, uint64_t pol)
{
    double2 v;
    asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ void st2(float *p, float a, float b, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1,%2}, %3;" :: "l"(p), "f"(a), "f"(b), "l"(pol) : "memory");
}
__device__ __forceinline__ void st2(double *p, double a, double b, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1,%2}, %3;" :: "l"(p), "d"(a), "d"(b), "l"(pol) : "memory");
}
__device__ __forceinline__ float4 ld4(const float *p, uint64_t pol)
{
    float4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ void st4(float *p, float a, float b, float c, float d, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1,%2,%3,%4}, %5;"
                 :: "l"(p), "f"(a), "f"(b), "f"(c), "f"(d), "l"(pol) : "memory");
}
__device__ __forceinline__ float ld1(const float *p, uint64_t pol)
{
    float v;
    asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double ld1(const double *p, uint64_t pol)
{
    double v;
    asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ void st1(float *p, float a, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" :: "l"(p), "f"(a), "l"(pol) : "memory");
}
__device__ __forceinline__ void st1(double *p, double a, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" :: "l"(p), "d"(a), "l"(pol) : "memory");
}
__device__ __forceinline__ void prefetch_l2(const void *p)
{
    asm volatile("prefetch.global.L2::evict_last [%0];" :: "l"(p));
}
__device__ __forceinline__ uint2 ldu2(const uint32_t *p)
{
    return __ldg(reinterpret_cast<const uint2 *>(p));
}

// Lanczos coefficients from the grid sums, written by thread 0 of the last
// block.  The stored vector is s' = w - gamma v' (gamma known before the
// launch: gamma1 for the first step, alpha_k for step k), so
//   alpha = <s',v'> + gamma |v'|^2,  delta = alpha - gamma,
//   beta^2 = |s'|^2 - 2 delta <s',v'> + delta^2 |v'|^2,
// a difference of numbers of size beta^2 + delta^2 instead of |w|^2.
// The step index of a launch: the argument, or the device counter.
__device__ __forceinline__ int step_index(const RowArgs &a) { return a.kdev ? *a.kdev : a.k; }
__device__ __forceinline__ double step_gamma(const RowArgs &a, int k)
{
    return a.mode == kModeFirst ? a.gamma1 : a.tri_diag[k - 1];
}
__device__ __forceinline__ void lanczos_finalize(const RowArgs &a, int k)
{
    const double sss = a.sums_out[0], ssv = a.sums_out[1], svv = a.sums_out[2];
    const double g = step_gamma(a, k);
    const double al = ssv + g * svv;
    const double de = al - g;
    const double b2 = sss - 2.0 * de * ssv + de * de * svv;
    const int slot = (a.mode == kModeFirst) ? 0 : k;
    double b = b2 > 0.0 ? sqrt(b2) : 0.0;
    const bool finite = isfinite(al) && isfinite(b2);
    if (!finite) { a.flags[1] = 1; b = 0.0; }
    // relative breakdown: beta at rounding level of |w| = |s' + gamma v'|
    const double ww = sss + 2.0 * g * ssv + g * g * svv;
    if (b2 <= 1e-28 * ww) b = 0.0;
    a.tri_diag[slot] = finite ? al : 0.0;
    a.tri_sub[slot + 1] = b;
    if (!(b >= a.cutoff) && a.flags[0] == 0) a.flags[0] = slot + 1;
    if (a.kdev && a.mode == kModeStep) *a.kdev = k + 1;
}


// Per-launch scalars of the fused Lanczos step (kModeStep, see edk_kernels.cu):
// s = w_k - gamma_k v_k was stored by the previous launch, delta_k = alpha_k -
// gamma_k, and the new stored vector is s' = w_{k+1} - alpha_k v_{k+1}.
struct StepScalars {
    double delta = 0.0, gam = 0.0, gam1 = 0.0, beta_k = 0.0, beta_k1 = 0.0, inv_b = 0.0, cpsi = 0.0;
};
// false: a step launch after the chain ended (breakdown recorded earlier).
__device__ __forceinline__ bool step_scalars(const RowArgs &a, int ks, StepScalars &sc)
{
    sc.gam1 = a.gamma1;
    if (a.mode != kModeStep) return true;
    sc.beta_k1 = a.tri_sub[ks];
    if (!(sc.beta_k1 >= a.cutoff) || a.flags[0] != 0) return false;
    const double alpha = a.tri_diag[ks - 1];
    sc.gam = ks >= 2 ? a.tri_diag[ks - 2] : a.gamma1;
    sc.delta = alpha - sc.gam;
    sc.gam1 = alpha;
    sc.beta_k = ks >= 2 ? a.tri_sub[ks - 1] : 0.0;
    sc.inv_b = 1.0 / sc.beta_k1;
    if (a.psi_coef) sc.cpsi = a.psi_coef[ks];
    return true;
}

// Writes element i of the launch's outputs from acc = (H x)_i and x_i, and
// adds its contribution to the reduction sums (the epilogue of every mode).
template <typename T>
__device__ __forceinline__ void row_epilogue(const RowArgs &a, const StepScalars &sc, int64_t i, double acc, T xo,
                                             double &s0, double &s1, double &s2)
{
    if (a.mode == kModeHv) {
        static_cast<T *>(a.y)[i] = (T)acc;
    } else if (a.mode == kModeFirst) {
        const double v = (double)xo;
        const T st = (T)(acc - sc.gam1 * v);
        static_cast<T *>(a.y)[i] = st;
        const double sd = (double)st;
        s0 += sd * sd; s1 += sd * v; s2 += v * v;
    } else if (a.mode == kModeStep) {
        const double sv = (double)xo;
        const double vk = (double)static_cast<const T *>(a.vk)[i];
        const double vm = a.vkm1 ? (double)static_cast<const T *>(a.vkm1)[i] : 0.0;
        const T vt = (T)((sv - sc.delta * vk) * sc.inv_b);
        const double hv1 = (acc - sc.delta * (sv + sc.gam * vk + sc.beta_k * vm)) * sc.inv_b;
        const double w = hv1 - sc.beta_k1 * vk;
        const T wt = (T)(w - sc.gam1 * (double)vt);
        static_cast<T *>(a.y)[i] = wt;
        static_cast<T *>(a.vout)[i] = vt;
        if (a.psi) {
            T *p = static_cast<T *>(a.psi) + i;
            *p = (T)((double)*p + sc.cpsi * (double)vt);
        }
        const double wd = (double)wt, vd = (double)vt;
        s0 += wd * wd; s1 += wd * vd; s2 += vd * vd;
    } else {   // kModeResid
        const double rr = acc - a.eshift * (double)xo;
        s0 += rr * rr; s2 += (double)xo * (double)xo;
    }
}

}  // namespace edk
