// Row kernel for FP32 vectors with FP32 hop sums (launch shapes of kind 3).
//
// Same sector shapes and mathematics as the other row kernels; it is built
// for instruction economy, since the FP32 fused Lanczos step of the other
// kinds is bound by instruction issue, not by bytes:
//   * a block owns two down rows d0, d1 at a time; they are staged in shared
//     memory interleaved by column, xs2[u] = {x[u,d0], x[u,d1]}, so one 8-byte
//     shared load serves both rows of an up-spin gather and one packed FP32x2
//     FMA (fma.rn.f32x2) accumulates it;
//   * the up table is a copy in which the KS entries of a column are
//     contiguous and pre-shifted: (target << 14) | (palette index << 3), so a
//     gather needs one shift for its shared-memory byte address and one AND
//     for the palette's; the palette holds {h, h} pairs;
//   * the hop count is uniform over a warp's 64 columns (stored per 64-column
//     block), so padding entries are skipped by a uniform branch;
//   * the down-spin hops of a row read the neighbour rows' elements at the
//     thread's column pair (8-byte loads, L2 evict_last) and accumulate them
//     as column pairs with packed FMAs;
//   * the diagonal, the Lanczos epilogue and the reductions stay FP64, as in
//     the FP32-sum mode of the other kinds.
// No cluster, no multicast, no inter-block waits: the reduction is the
// last-block-done sum of edk_device.cuh.
#pragma once
#include "edk_device.cuh"

namespace edk {

__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c)
{
    unsigned long long d;
    const unsigned long long A = *reinterpret_cast<const unsigned long long *>(&a);
    const unsigned long long B = *reinterpret_cast<const unsigned long long *>(&b);
    const unsigned long long C = *reinterpret_cast<const unsigned long long *>(&c);
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(A), "l"(B), "l"(C));
    return *reinterpret_cast<const float2 *>(&d);
}

// KS: entries per column in the lean up table (even); KMD: the down rows'
// length bound (rows with fewer hops are padded with value 0 on the own row,
// so every neighbour load is unconditional); NT threads per block, MINB
// blocks per SM; STEP: fused Lanczos step known at compile time.
// Every global load of a column pair (table entries, neighbour elements,
// v_k, v_{k-1}, the diagonal) is issued at the top of its iteration, before
// any shared-memory gather or branch, so a warp waits for one round trip per
// iteration instead of one per dependent stage.
template <int KS, int KMD, int NT, int MINB, bool STEP>
__global__ void __launch_bounds__(NT, MINB) row_lean_kernel(const HamDev H, const RowArgs a)
{
    static_assert(2 * KMD <= NT, "neighbour table preparation");
    extern __shared__ __align__(16) float2 xs2[];    // [dup]: {x[u,d0], x[u,d1]}
    __shared__ __align__(16) float2 pal2[256];       // {h, h}
    __shared__ __align__(16) float2 s_hd2[2][KMD];   // {h, h} of each neighbour row
    __shared__ double s_dsum[16];
    __shared__ int s_nofs[2][KMD];
    __shared__ int s_cd[2];
    __shared__ double s_dd[2];
    const int dup = (int)H.dup;
    const int64_t ddn = H.ddn;
    const float *__restrict__ x = static_cast<const float *>(a.x);
    const int tid = threadIdx.x;
    const int mode = STEP ? (int)kModeStep : a.mode;

    StepScalars sc;
    const int ks = step_index(a);
    if (!step_scalars(a, ks, sc)) return;
    {
        for (int i = tid; i < H.up.npal; i += NT) {
            const float h = (float)H.up.pal[i];
            pal2[i] = make_float2(h, h);
        }
        const int nio = H.ncfg * H.ncfg;
        if (tid < nio) {
            double t = 0.0;
            for (int o2 = H.int_off[tid]; o2 < H.int_off[tid + 1]; ++o2) t += H.int_coef[o2];
            s_dsum[tid] = t;
        }
    }
    const uint64_t keep = l2_keep(), stream = l2_stream();
    const uint32_t *__restrict__ lt = H.up.lean;
    const uint8_t *__restrict__ kwb = H.up.lean_kw;
    const double *__restrict__ upd = H.up.diag;
    const uint8_t *__restrict__ upi = H.up.imp;
    const float *__restrict__ vkp = static_cast<const float *>(a.vk);
    const float *__restrict__ vmp = static_cast<const float *>(a.vkm1);
    const int ncfg = H.ncfg;
    const unsigned char *xsb = reinterpret_cast<const unsigned char *>(xs2);
    const unsigned char *palb = reinterpret_cast<const unsigned char *>(pal2);

    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    const int64_t ngroups = (ddn + 1) / 2;
    for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const int d0 = H.row_order[2 * g];
        const bool has1 = 2 * g + 1 < ddn;
        const int d1 = has1 ? H.row_order[2 * g + 1] : d0;
        __syncthreads();   // the previous group's readers are done with xs2 and the row tables
        if (tid < 2 * KMD) {
            const int r = tid / KMD, f = tid - r * KMD;
            const int rr = r == 0 ? d0 : d1;
            const int f0 = H.dn.ptr[rr], nd = H.dn.ptr[rr + 1] - f0;
            const bool ok = f < nd;
            const float h = ok ? (float)H.dn.val[f0 + f] : 0.f;
            s_nofs[r][f] = (ok ? H.dn.tgt[f0 + f] : rr) * dup;
            s_hd2[r][f] = make_float2(h, h);
            if (f == 0) {
                s_cd[r] = (int)H.dn.imp[rr];
                s_dd[r] = H.dn.diag[rr];
            }
        }
        {
            // stage the two rows interleaved by column
            const float *x0 = x + (int64_t)d0 * dup, *x1 = x + (int64_t)d1 * dup;
#pragma unroll 4
            for (int u = 2 * tid; u < dup; u += 2 * NT) {
                const float2 p = ld2(x0 + u, keep), q = ld2(x1 + u, keep);
                *reinterpret_cast<float4 *>(xs2 + u) = make_float4(p.x, q.x, p.y, q.y);
            }
        }
        __syncthreads();
        int nofs[2][KMD];
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int f = 0; f < KMD; ++f) nofs[r][f] = s_nofs[r][f];
        const int cd0 = s_cd[0], cd1 = s_cd[1];
        const double dd0 = s_dd[0], dd1 = s_dd[1];
        const size_t ib0 = (size_t)d0 * dup, ib1 = (size_t)d1 * dup;

        // ---- every global load of a column pair, issued before its computation ----
        struct Ld {
            float2 xd[2][KMD];
            float2 vk[2], vm[2];
            uint4 tq[KS / 2];
            double2 du;
            uchar2 cu;
            int kw;
        };
        auto load = [&](int c, Ld &L) {
#pragma unroll
            for (int f = 0; f < KMD; ++f) {
                L.xd[0][f] = ld2(x + nofs[0][f] + c, keep);
                L.xd[1][f] = ld2(x + nofs[1][f] + c, keep);
            }
            if (mode == kModeStep) {
                L.vk[0] = ld2(vkp + ib0 + c, stream);
                L.vk[1] = ld2(vkp + ib1 + c, stream);
                if (vmp) {
                    L.vm[0] = ld2(vmp + ib0 + c, stream);
                    L.vm[1] = ld2(vmp + ib1 + c, stream);
                } else {
                    L.vm[0] = L.vm[1] = make_float2(0.f, 0.f);
                }
            }
            const uint4 *tp = reinterpret_cast<const uint4 *>(lt + (size_t)c * KS);
#pragma unroll
            for (int q = 0; q < KS / 2; ++q) L.tq[q] = __ldg(tp + q);
            L.du = __ldg(reinterpret_cast<const double2 *>(upd + c));
            L.cu = *reinterpret_cast<const uchar2 *>(upi + c);
            L.kw = kwb[c >> 6];
        };
        auto compute = [&](int c, const Ld &L) {
            // up-spin hops of the column pair from the staged rows
            const uint32_t *ent = reinterpret_cast<const uint32_t *>(L.tq);
            float2 U0 = make_float2(0.f, 0.f), U1 = make_float2(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < KS; ++k) {
                if (k < L.kw) {
                    const uint32_t e0 = ent[k], e1 = ent[KS + k];
                    const float2 g0 = *reinterpret_cast<const float2 *>(xsb + (e0 >> 11));
                    const float2 g1 = *reinterpret_cast<const float2 *>(xsb + (e1 >> 11));
                    const float2 h0 = *reinterpret_cast<const float2 *>(palb + (e0 & 0x7F8u));
                    const float2 h1 = *reinterpret_cast<const float2 *>(palb + (e1 & 0x7F8u));
                    U0 = ffma2(h0, g0, U0);
                    U1 = ffma2(h1, g1, U1);
                }
            }
            // down-spin hops: neighbour rows at the column pair
            float2 D0 = make_float2(0.f, 0.f), D1 = make_float2(0.f, 0.f);
#pragma unroll
            for (int f = 0; f < KMD; ++f) {
                D0 = ffma2(s_hd2[0][f], L.xd[0][f], D0);
                D1 = ffma2(s_hd2[1][f], L.xd[1][f], D1);
            }
            // own elements, diagonal (FP64), epilogue
            const float4 o = *reinterpret_cast<const float4 *>(xs2 + c);   // {c:d0, c:d1, c+1:d0, c+1:d1}
            const float hop[2][2] = {{U0.x + D0.x, U1.x + D0.y}, {U0.y + D1.x, U1.y + D1.y}};
            const float ov[2][2] = {{o.x, o.z}, {o.y, o.w}};
            const double due[2] = {L.du.x, L.du.y};
            const int cue[2] = {(int)L.cu.x, (int)L.cu.y};
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                if (r == 1 && !has1) break;
                const int cd = r == 0 ? cd0 : cd1;
                const double dd = r == 0 ? dd0 : dd1;
                const size_t i = (r == 0 ? ib0 : ib1) + c;
                double acc[2], sv[2];
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    sv[e] = (double)ov[r][e];
                    acc[e] = fma(s_dsum[cue[e] * ncfg + cd] + (due[e] + dd), sv[e], (double)hop[r][e]);
                }
                if (mode == kModeHv) {
                    st2(static_cast<float *>(a.y) + i, (float)acc[0], (float)acc[1], stream);
                } else if (mode == kModeFirst) {
                    float st[2];
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        st[e] = (float)(acc[e] - sc.gam1 * sv[e]);
                        const double sd = (double)st[e];
                        s0 += sd * sd; s1 += sd * sv[e]; s2 += sv[e] * sv[e];
                    }
                    st2(static_cast<float *>(a.y) + i, st[0], st[1], stream);
                } else if (mode == kModeStep) {
                    const double vk[2] = {(double)L.vk[r].x, (double)L.vk[r].y};
                    const double vm[2] = {(double)L.vm[r].x, (double)L.vm[r].y};
                    float wt[2], vt[2];
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        vt[e] = (float)((sv[e] - sc.delta * vk[e]) * sc.inv_b);
                        const double hv1 = (acc[e] - sc.delta * (sv[e] + sc.gam * vk[e] + sc.beta_k * vm[e])) * sc.inv_b;
                        const double w = hv1 - sc.beta_k1 * vk[e];
                        const double vd = (double)vt[e];
                        wt[e] = (float)(w - sc.gam1 * vd);
                        const double wd = (double)wt[e];
                        s0 += wd * wd; s1 += wd * vd; s2 += vd * vd;
                    }
                    st2(static_cast<float *>(a.y) + i, wt[0], wt[1], stream);
                    st2(static_cast<float *>(a.vout) + i, vt[0], vt[1], stream);
                    if (a.psi) {
                        float *p = static_cast<float *>(a.psi) + i;
                        const float2 pv = ld2(p, stream);
                        st2(p, (float)((double)pv.x + sc.cpsi * (double)vt[0]), (float)((double)pv.y + sc.cpsi * (double)vt[1]),
                            stream);
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const double rr = acc[e] - a.eshift * sv[e];
                        s0 += rr * rr; s2 += sv[e] * sv[e];
                    }
                }
            }
        };
        for (int c = 2 * tid; c < dup; c += 2 * NT) {
            Ld A;
            load(c, A);
            compute(c, A);
        }
    }
    if (mode == kModeHv) return;
    double v[4] = {s0, s1, s2, 0.0};
    if (grid_sum<4>(v, a.partials, a.counter, a.sums_out))
        if (mode == kModeFirst || mode == kModeStep) lanczos_finalize(a, ks);
}

// Dynamic shared memory of one block: the two interleaved rows.
inline size_t lean_smem_bytes(int64_t dup) { return (size_t)dup * 8; }

template <int KS, int KMD, int NT, int MINB>
cudaError_t launch_lean_t(const HamDev &H, const RowArgs &a, int num_sms, cudaStream_t st)
{
    auto k = a.mode == kModeStep ? row_lean_kernel<KS, KMD, NT, MINB, true> : row_lean_kernel<KS, KMD, NT, MINB, false>;
    const size_t smem = lean_smem_bytes(H.dup);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NT, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int64_t groups = (H.ddn + 1) / 2;
    int64_t grid = (int64_t)num_sms * per_sm;
    if (grid > groups) grid = groups;
    if (grid < 1) grid = 1;
    k<<<(int)grid, NT, smem, st>>>(H, a);
    return cudaGetLastError();
}

cudaError_t launch_lean_f32(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st);

}  // namespace edk
