// Two-pass FP32 row step with FP32 hop sums (launch shapes of kind 5): the
// down-spin hops gathered from column tiles of x while the tile is resident
// in L2.
//
// The fused row kernels gather the down-spin neighbours of a row at the full
// width of x: about two thirds of those rows come from DRAM (a row-order
// simulation of the neighbour graph gives about three reads of each row per
// step), at DRAM latency.  Here the step is split the way the reference's
// HAIMupdo_multr_split separates the two hop directions
// (ed_solver/HAIMupdo.f90:1221-1347), without its transposes:
//   1. up_pass_kernel: the up-spin hops and the diagonal of every element,
//      rows staged in shared memory two at a time interleaved by column (the
//      lean kernel's gathers), written to a scratch vector y1 (FP32);
//   2. down_pass_kernel: column tiles of kTileW up-spin columns swept over all
//      down rows, tile by tile across the whole grid (work unit = a tile and
//      kTileRows rows, taken in tile-major order), so that every block
//      gathers the neighbour rows' pieces of the tile -- kTileW x dim_dn x 4 B
//      = 26 MB at ns=16, resident in L2 after its first touch -- and adds them
//      to y1, then runs the Lanczos epilogue of the mode and the reductions.
// x is read from DRAM about once per pass, at the price of writing and reading
// y1.  All arithmetic as in the lean kernel: hop sums in FP32 (packed FP32x2
// FMAs), the diagonal, the epilogue and the reductions in FP64.  No cluster,
// no multicast, no inter-block waits.
#pragma once
#include "edk_rows_lean.cuh"

namespace edk {

constexpr int kTileW = 512;      // up-spin columns per tile (2 per thread of a 256-thread block)
constexpr int kTileRows = 16;    // down rows per work unit
constexpr int kQuadMaxBlocks = 256;   // 64-column blocks of a row the four-row up pass takes

// Pass 1: y1 = (diagonal + density) x + up-spin hops, FP32 out.  NP row
// pairs per group, each staged interleaved by column in its own buffer, so one
// table entry and palette value serve 2*NP rows.
// SP: the palette has at most 32 values; lane l of every warp holds value l
// in a register and a hop's value comes by a shuffle instead of a shared
// load (the pass is bound by L1 / shared-memory throughput).
template <int KS, int NP, int NT, int MINB, bool SP>
__global__ void __launch_bounds__(NT, MINB) up_pass_kernel(const HamDev H, const float *__restrict__ x,
                                                           float *__restrict__ y1)
{
    extern __shared__ __align__(16) float2 xs2[];    // [NP][dup]: {x[u,d0], x[u,d1]} per pair
    __shared__ __align__(16) float2 pal2[256];
    __shared__ double s_dsum[16];
    constexpr int R = 2 * NP;
    const int dup = (int)H.dup;
    const int64_t ddn = H.ddn;
    const int tid = threadIdx.x;
    for (int i = tid; i < H.up.npal; i += NT) {
        const float h = (float)H.up.pal[i];
        pal2[i] = make_float2(h, h);
    }
    if (tid < H.ncfg * H.ncfg) {
        double t = 0.0;
        for (int o2 = H.int_off[tid]; o2 < H.int_off[tid + 1]; ++o2) t += H.int_coef[o2];
        s_dsum[tid] = t;
    }
    const uint64_t keep = l2_keep(), stream = l2_stream();
    const uint32_t *__restrict__ lt = H.up.lean_b;
    const uint8_t *__restrict__ kwb = H.up.lean_kw;
    const double *__restrict__ upd = H.up.diag;
    const uint8_t *__restrict__ upi = H.up.imp;
    const int ncfg = H.ncfg;
    const unsigned char *palb = reinterpret_cast<const unsigned char *>(pal2);
    const float palr = SP && (tid & 31) < H.up.npal ? (float)H.up.pal[tid & 31] : 0.f;
    const int64_t ngroups = (ddn + R - 1) / R;
    for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        int d[R];
#pragma unroll
        for (int r = 0; r < R; ++r) d[r] = (int)(R * g + r < ddn ? R * g + r : R * g);
        __syncthreads();
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const float *x0 = x + (int64_t)d[2 * p] * dup, *x1 = x + (int64_t)d[2 * p + 1] * dup;
            float2 *dst = xs2 + (size_t)p * dup;
#pragma unroll 4
            for (int u = 2 * tid; u < dup; u += 2 * NT) {
                const float2 a0 = ld2(x0 + u, keep), a1 = ld2(x1 + u, keep);
                *reinterpret_cast<float4 *>(dst + u) = make_float4(a0.x, a1.x, a0.y, a1.y);
            }
        }
        __syncthreads();
        int cd[R];
        double dd[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            cd[r] = (int)H.dn.imp[d[r]];
            dd[r] = H.dn.diag[d[r]];
        }
        // a warp's lanes iterate together (the shuffles need the whole warp):
        // the loop runs on the warp's first column, lanes past the row end
        // compute on the warp's first column and store nothing
        const int lane = tid & 31;
        for (int cw = 2 * (tid - lane); cw < dup; cw += 2 * NT) {
            const int cl = cw + 2 * lane;
            const bool valid = cl < dup;
            const int c = valid ? cl : cw;
            // entry k of the column pair: one 8-byte load, contiguous over the warp
            uint2 ent[KS];
            const uint2 *tp = reinterpret_cast<const uint2 *>(lt + (size_t)(c >> 6) * 64 * KS + (c & 63));
#pragma unroll
            for (int k = 0; k < KS; ++k) ent[k] = __ldg(tp + k * 32);
            const double2 du = __ldg(reinterpret_cast<const double2 *>(upd + c));
            const uchar2 cu = *reinterpret_cast<const uchar2 *>(upi + c);
            const int kw = kwb[cw >> 6];
            float2 U[NP][2];
#pragma unroll
            for (int p = 0; p < NP; ++p) U[p][0] = U[p][1] = make_float2(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < KS; ++k) {
                if (k < kw) {
                    const uint32_t e0 = ent[k].x, e1 = ent[k].y;
                    float2 h0, h1;
                    if (SP) {
                        const float a0 = __shfl_sync(0xffffffffu, palr, (int)((e0 >> 3) & 31u));
                        const float a1 = __shfl_sync(0xffffffffu, palr, (int)((e1 >> 3) & 31u));
                        h0 = make_float2(a0, a0);
                        h1 = make_float2(a1, a1);
                    } else {
                        h0 = *reinterpret_cast<const float2 *>(palb + (e0 & 0x7F8u));
                        h1 = *reinterpret_cast<const float2 *>(palb + (e1 & 0x7F8u));
                    }
#pragma unroll
                    for (int p = 0; p < NP; ++p) {
                        const unsigned char *xb = reinterpret_cast<const unsigned char *>(xs2 + (size_t)p * dup);
                        U[p][0] = ffma2(h0, *reinterpret_cast<const float2 *>(xb + (e0 >> 11)), U[p][0]);
                        U[p][1] = ffma2(h1, *reinterpret_cast<const float2 *>(xb + (e1 >> 11)), U[p][1]);
                    }
                }
            }
            const double due[2] = {du.x, du.y};
            const int cue[2] = {(int)cu.x, (int)cu.y};
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const float4 o = *reinterpret_cast<const float4 *>(xs2 + (size_t)p * dup + c);
                const float up[2][2] = {{U[p][0].x, U[p][1].x}, {U[p][0].y, U[p][1].y}};
                const float ov[2][2] = {{o.x, o.z}, {o.y, o.w}};
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int r = 2 * p + q;
                    if (R * g + r >= ddn || !valid) break;
                    float out[2];
#pragma unroll
                    for (int e = 0; e < 2; ++e)
                        out[e] = (float)fma(s_dsum[cue[e] * ncfg + cd[r]] + (due[e] + dd[r]), (double)ov[q][e],
                                            (double)up[q][e]);
                    st2(y1 + (size_t)d[r] * dup + c, out[0], out[1], stream);
                }
            }
        }
    }
}

// Pass 1 with four rows interleaved by column in one buffer
// ({x[u,d0], x[u,d1], x[u,d2], x[u,d3]} per column): one 16-byte shared load
// per hop serves the four rows, where the two-buffer form issues two 8-byte
// loads, so the random gathers take fewer shared-memory wavefronts.  The FMAs
// and their order per element are those of up_pass_kernel.
template <int KS, int NT, bool SP>
__global__ void __launch_bounds__(NT, 1) up_pass_quad_kernel(const HamDev H, const float *__restrict__ x,
                                                             float *__restrict__ y1)
{
    extern __shared__ __align__(16) float4 xs4[];    // [dup]
    __shared__ __align__(16) float2 pal2[256];
    __shared__ double s_dsum[16];
    __shared__ uint8_t s_kw[kQuadMaxBlocks];          // hop count per 64-column block
    constexpr int R = 4;
    const int dup = (int)H.dup;
    const int64_t ddn = H.ddn;
    const int tid = threadIdx.x;
    for (int i = tid; i < H.up.npal; i += NT) {
        const float h = (float)H.up.pal[i];
        pal2[i] = make_float2(h, h);
    }
    for (int i = tid; i < (dup + 63) / 64; i += NT) s_kw[i] = H.up.lean_kw[i];
    if (tid < H.ncfg * H.ncfg) {
        double t = 0.0;
        for (int o2 = H.int_off[tid]; o2 < H.int_off[tid + 1]; ++o2) t += H.int_coef[o2];
        s_dsum[tid] = t;
    }
    const uint64_t keep = l2_keep(), stream = l2_stream();
    const uint32_t *__restrict__ lt = H.up.lean_b;
    const double *__restrict__ upd = H.up.diag;
    const uint8_t *__restrict__ upi = H.up.imp;
    const int ncfg = H.ncfg;
    const unsigned char *palb = reinterpret_cast<const unsigned char *>(pal2);
    const unsigned char *xb = reinterpret_cast<const unsigned char *>(xs4);
    const float palr = SP && (tid & 31) < H.up.npal ? (float)H.up.pal[tid & 31] : 0.f;
    const int64_t ngroups = (ddn + R - 1) / R;
    for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        int d[R];
#pragma unroll
        for (int r = 0; r < R; ++r) d[r] = (int)(R * g + r < ddn ? R * g + r : R * g);
        __syncthreads();
        {
            // one column per lane: the 16-byte stores of a warp are contiguous
            const float *x0 = x + (int64_t)d[0] * dup, *x1 = x + (int64_t)d[1] * dup;
            const float *x2 = x + (int64_t)d[2] * dup, *x3 = x + (int64_t)d[3] * dup;
#pragma unroll 2
            for (int u = tid; u < dup; u += NT)
                xs4[u] = make_float4(ld1(x0 + u, keep), ld1(x1 + u, keep), ld1(x2 + u, keep), ld1(x3 + u, keep));
        }
        __syncthreads();
        int cd[R];
        double dd[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            cd[r] = (int)H.dn.imp[d[r]];
            dd[r] = H.dn.diag[d[r]];
        }
        const int lane = tid & 31;
        for (int cw = 2 * (tid - lane); cw < dup; cw += 2 * NT) {
            const int cl = cw + 2 * lane;
            const bool valid = cl < dup;
            const int c = valid ? cl : cw;
            // the block's hop count is uniform over the warp: entries past it
            // are padding and not loaded
            const int kw = s_kw[cw >> 6];
            uint2 ent[KS];
            const uint2 *tp = reinterpret_cast<const uint2 *>(lt + (size_t)(c >> 6) * 64 * KS + (c & 63));
#pragma unroll
            for (int k = 0; k < KS; ++k) ent[k] = k < kw ? __ldg(tp + k * 32) : make_uint2(0u, 0u);
            const double2 du = __ldg(reinterpret_cast<const double2 *>(upd + c));
            const uchar2 cu = *reinterpret_cast<const uchar2 *>(upi + c);
            // U[p][e]: rows 2p, 2p+1 of column c+e
            float2 U[2][2];
            U[0][0] = U[0][1] = U[1][0] = U[1][1] = make_float2(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < KS; ++k) {
                if (k < kw) {
                    const uint32_t e0 = ent[k].x, e1 = ent[k].y;
                    float2 h0, h1;
                    if (SP) {
                        const float a0 = __shfl_sync(0xffffffffu, palr, (int)((e0 >> 3) & 31u));
                        const float a1 = __shfl_sync(0xffffffffu, palr, (int)((e1 >> 3) & 31u));
                        h0 = make_float2(a0, a0);
                        h1 = make_float2(a1, a1);
                    } else {
                        h0 = *reinterpret_cast<const float2 *>(palb + (e0 & 0x7F8u));
                        h1 = *reinterpret_cast<const float2 *>(palb + (e1 & 0x7F8u));
                    }
                    // byte offset target * 16: entry >> 10 puts the target (from
                    // bit 14) at bit 4, and the mask drops the palette index's top
                    // bit, which lands in bit 0
                    const float4 g0 = *reinterpret_cast<const float4 *>(xb + ((e0 >> 10) & ~15u));
                    const float4 g1 = *reinterpret_cast<const float4 *>(xb + ((e1 >> 10) & ~15u));
                    U[0][0] = ffma2(h0, make_float2(g0.x, g0.y), U[0][0]);
                    U[1][0] = ffma2(h0, make_float2(g0.z, g0.w), U[1][0]);
                    U[0][1] = ffma2(h1, make_float2(g1.x, g1.y), U[0][1]);
                    U[1][1] = ffma2(h1, make_float2(g1.z, g1.w), U[1][1]);
                }
            }
            const double due[2] = {du.x, du.y};
            const int cue[2] = {(int)cu.x, (int)cu.y};
            const float4 o0 = xs4[c], o1 = xs4[c + 1];
            const float ov[R][2] = {{o0.x, o1.x}, {o0.y, o1.y}, {o0.z, o1.z}, {o0.w, o1.w}};
            const float up[R][2] = {{U[0][0].x, U[0][1].x}, {U[0][0].y, U[0][1].y},
                                    {U[1][0].x, U[1][1].x}, {U[1][0].y, U[1][1].y}};
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (R * g + r >= ddn || !valid) break;
                float out[2];
#pragma unroll
                for (int e = 0; e < 2; ++e)
                    out[e] = (float)fma(s_dsum[cue[e] * ncfg + cd[r]] + (due[e] + dd[r]), (double)ov[r][e],
                                        (double)up[r][e]);
                st2(y1 + (size_t)d[r] * dup + c, out[0], out[1], stream);
            }
        }
    }
}

// Pass 2: the down-spin hops from L2-resident column tiles, added to y1, and
// the epilogue of the mode.  KMD: bound on the down rows' lengths.
template <int KMD, bool STEP>
__global__ void __launch_bounds__(256, 4) down_pass_kernel(const HamDev H, const RowArgs a, const float *__restrict__ y1)
{
    constexpr int NT = 256;
    __shared__ int s_nofs[kTileRows][KMD];
    __shared__ __align__(16) float2 s_hd2[kTileRows][KMD];
    __shared__ int s_nd[kTileRows];
    const int dup = (int)H.dup;
    const int64_t ddn = H.ddn;
    const float *__restrict__ x = static_cast<const float *>(a.x);
    const float *__restrict__ vkp = static_cast<const float *>(a.vk);
    const float *__restrict__ vmp = static_cast<const float *>(a.vkm1);
    const int tid = threadIdx.x;
    const int mode = STEP ? (int)kModeStep : a.mode;
    StepScalars sc;
    const int ks = step_index(a);
    if (!step_scalars(a, ks, sc)) return;
    const uint64_t keep = l2_keep(), stream = l2_stream();
    const int ntiles = (dup + kTileW - 1) / kTileW;
    const int nchunks = (int)((ddn + kTileRows - 1) / kTileRows);
    const int64_t nunits = (int64_t)ntiles * nchunks;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int64_t q = blockIdx.x; q < nunits; q += gridDim.x) {
        const int tile = (int)(q / nchunks), chunk = (int)(q - (int64_t)tile * nchunks);
        const int r0 = chunk * kTileRows;
        const int nr = (int)(ddn - r0 < kTileRows ? ddn - r0 : kTileRows);
        __syncthreads();   // the previous unit is done with the row tables
        for (int t = tid; t < kTileRows * KMD; t += NT) {
            const int r = t / KMD, f = t - r * KMD;
            const int d = r0 + (r < nr ? r : 0);
            const int f0 = H.dn.ptr[d], nd = H.dn.ptr[d + 1] - f0;
            const bool ok = r < nr && f < nd;
            const float h = ok ? (float)H.dn.val[f0 + f] : 0.f;
            s_nofs[r][f] = (ok ? H.dn.tgt[f0 + f] : d) * dup;
            s_hd2[r][f] = make_float2(h, h);
            if (f == 0) s_nd[r] = r < nr ? nd : 0;
        }
        __syncthreads();
        const int c = tile * kTileW + 2 * tid;
        if (c >= dup) continue;
        for (int r = 0; r < nr; ++r) {
            const int d = r0 + r;
            const size_t i = (size_t)d * dup + c;
            // every global load of the element pair first
            float2 xd[KMD];
#pragma unroll
            for (int f = 0; f < KMD; ++f) xd[f] = ld2(x + s_nofs[r][f] + c, keep);
            const float2 own = ld2(x + i, keep);
            const float2 yv = ld2(y1 + i, stream);
            float2 vk2 = make_float2(0.f, 0.f), vm2 = make_float2(0.f, 0.f);
            if (mode == kModeStep) {
                vk2 = ld2(vkp + i, stream);
                if (vmp) vm2 = ld2(vmp + i, stream);
            }
            const int nd = s_nd[r];
            float2 D = make_float2(0.f, 0.f);
#pragma unroll
            for (int f = 0; f < KMD; ++f)
                if (f < nd) D = ffma2(s_hd2[r][f], xd[f], D);
            const double acc[2] = {(double)yv.x + (double)D.x, (double)yv.y + (double)D.y};
            const double sv[2] = {(double)own.x, (double)own.y};
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
                const double vk[2] = {(double)vk2.x, (double)vk2.y}, vm[2] = {(double)vm2.x, (double)vm2.y};
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
    }
    if (mode == kModeHv) return;
    double v[4] = {s0, s1, s2, 0.0};
    if (grid_sum<4>(v, a.partials, a.counter, a.sums_out))
        if (mode == kModeFirst || mode == kModeStep) lanczos_finalize(a, ks);
}

// Pass 2 with four columns per thread: every vector access is one 16-byte
// load or store.  The block's 256 threads cover the tile's 512 columns twice,
// and the two halves take alternate rows of the unit.  Needs dim_up a
// multiple of 4 and 16-byte aligned vectors (checked at the launch).  Per
// element the arithmetic is that of down_pass_kernel; only the order in which
// a thread adds its elements into the reduction sums differs.
template <int KMD, bool STEP>
__global__ void __launch_bounds__(256, 3) down_pass4_kernel(const HamDev H, const RowArgs a,
                                                            const float *__restrict__ y1)
{
    constexpr int NT = 256;
    __shared__ int s_nofs[kTileRows][KMD];
    __shared__ __align__(16) float2 s_hd2[kTileRows][KMD];
    __shared__ int s_nd[kTileRows];
    const int dup = (int)H.dup;
    const int64_t ddn = H.ddn;
    const float *__restrict__ x = static_cast<const float *>(a.x);
    const float *__restrict__ vkp = static_cast<const float *>(a.vk);
    const float *__restrict__ vmp = static_cast<const float *>(a.vkm1);
    const int tid = threadIdx.x;
    const int mode = STEP ? (int)kModeStep : a.mode;
    StepScalars sc;
    const int ks = step_index(a);
    if (!step_scalars(a, ks, sc)) return;
    const uint64_t keep = l2_keep(), stream = l2_stream();
    const int ntiles = (dup + kTileW - 1) / kTileW;
    const int nchunks = (int)((ddn + kTileRows - 1) / kTileRows);
    const int64_t nunits = (int64_t)ntiles * nchunks;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int64_t q = blockIdx.x; q < nunits; q += gridDim.x) {
        const int tile = (int)(q / nchunks), chunk = (int)(q - (int64_t)tile * nchunks);
        const int r0 = chunk * kTileRows;
        const int nr = (int)(ddn - r0 < kTileRows ? ddn - r0 : kTileRows);
        __syncthreads();   // the previous unit is done with the row tables
        for (int t = tid; t < kTileRows * KMD; t += NT) {
            const int r = t / KMD, f = t - r * KMD;
            const int d = r0 + (r < nr ? r : 0);
            const int f0 = H.dn.ptr[d], nd = H.dn.ptr[d + 1] - f0;
            const bool ok = r < nr && f < nd;
            const float h = ok ? (float)H.dn.val[f0 + f] : 0.f;
            s_nofs[r][f] = (ok ? H.dn.tgt[f0 + f] : d) * dup;
            s_hd2[r][f] = make_float2(h, h);
            if (f == 0) s_nd[r] = r < nr ? nd : 0;
        }
        __syncthreads();
        const int c = tile * kTileW + 4 * (tid & 127);
        if (c >= dup) continue;
        for (int r = tid >> 7; r < nr; r += 2) {
            const int d = r0 + r;
            const size_t i = (size_t)d * dup + c;
            // every global load of the four elements first
            float4 xd[KMD];
#pragma unroll
            for (int f = 0; f < KMD; ++f) xd[f] = ld4(x + s_nofs[r][f] + c, keep);
            const float4 own = ld4(x + i, keep);
            const float4 yv = ld4(y1 + i, stream);
            float4 vk4 = make_float4(0.f, 0.f, 0.f, 0.f), vm4 = make_float4(0.f, 0.f, 0.f, 0.f);
            if (mode == kModeStep) {
                vk4 = ld4(vkp + i, stream);
                if (vmp) vm4 = ld4(vmp + i, stream);
            }
            const int nd = s_nd[r];
            float2 Dl = make_float2(0.f, 0.f), Dh = make_float2(0.f, 0.f);
#pragma unroll
            for (int f = 0; f < KMD; ++f)
                if (f < nd) {
                    Dl = ffma2(s_hd2[r][f], make_float2(xd[f].x, xd[f].y), Dl);
                    Dh = ffma2(s_hd2[r][f], make_float2(xd[f].z, xd[f].w), Dh);
                }
            const double acc[4] = {(double)yv.x + (double)Dl.x, (double)yv.y + (double)Dl.y,
                                   (double)yv.z + (double)Dh.x, (double)yv.w + (double)Dh.y};
            const double sv[4] = {(double)own.x, (double)own.y, (double)own.z, (double)own.w};
            if (mode == kModeHv) {
                st4(static_cast<float *>(a.y) + i, (float)acc[0], (float)acc[1], (float)acc[2], (float)acc[3], stream);
            } else if (mode == kModeFirst) {
                float st[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    st[e] = (float)(acc[e] - sc.gam1 * sv[e]);
                    const double sd = (double)st[e];
                    s0 += sd * sd; s1 += sd * sv[e]; s2 += sv[e] * sv[e];
                }
                st4(static_cast<float *>(a.y) + i, st[0], st[1], st[2], st[3], stream);
            } else if (mode == kModeStep) {
                const double vk[4] = {(double)vk4.x, (double)vk4.y, (double)vk4.z, (double)vk4.w};
                const double vm[4] = {(double)vm4.x, (double)vm4.y, (double)vm4.z, (double)vm4.w};
                float wt[4], vt[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    vt[e] = (float)((sv[e] - sc.delta * vk[e]) * sc.inv_b);
                    const double hv1 = (acc[e] - sc.delta * (sv[e] + sc.gam * vk[e] + sc.beta_k * vm[e])) * sc.inv_b;
                    const double w = hv1 - sc.beta_k1 * vk[e];
                    const double vd = (double)vt[e];
                    wt[e] = (float)(w - sc.gam1 * vd);
                    const double wd = (double)wt[e];
                    s0 += wd * wd; s1 += wd * vd; s2 += vd * vd;
                }
                st4(static_cast<float *>(a.y) + i, wt[0], wt[1], wt[2], wt[3], stream);
                st4(static_cast<float *>(a.vout) + i, vt[0], vt[1], vt[2], vt[3], stream);
                if (a.psi) {
                    float *p = static_cast<float *>(a.psi) + i;
                    const float4 pv = ld4(p, stream);
                    st4(p, (float)((double)pv.x + sc.cpsi * (double)vt[0]), (float)((double)pv.y + sc.cpsi * (double)vt[1]),
                        (float)((double)pv.z + sc.cpsi * (double)vt[2]), (float)((double)pv.w + sc.cpsi * (double)vt[3]),
                        stream);
                }
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const double rr = acc[e] - a.eshift * sv[e];
                    s0 += rr * rr; s2 += sv[e] * sv[e];
                }
            }
        }
    }
    if (mode == kModeHv) return;
    double v[4] = {s0, s1, s2, 0.0};
    if (grid_sum<4>(v, a.partials, a.counter, a.sums_out))
        if (mode == kModeFirst || mode == kModeStep) lanczos_finalize(a, ks);
}

// variant & 7 -- 0: two row pairs per up-pass block when they fit, 1: one
// pair, 2 to 5: four rows interleaved in one buffer when they fit (else one
// pair), 512, 640, 768 or 1024 threads; variant & 8: the down pass with four
// columns per thread where dim_up is a multiple of 4 and every vector is
// 16-byte aligned (else two)
template <int KS, int KMD>
cudaError_t launch_tiled_t(const HamDev &H, const RowArgs &a, int num_sms, int variant_in, cudaStream_t st)
{
    if (!a.scratch) return cudaErrorInvalidValue;
    float *y1 = static_cast<float *>(a.scratch);
    const int variant = variant_in & 7;
    const uintptr_t align = reinterpret_cast<uintptr_t>(a.x) | reinterpret_cast<uintptr_t>(a.vk) |
                            reinterpret_cast<uintptr_t>(a.vkm1) | reinterpret_cast<uintptr_t>(a.y) |
                            reinterpret_cast<uintptr_t>(a.vout) | reinterpret_cast<uintptr_t>(a.psi) |
                            reinterpret_cast<uintptr_t>(y1);
    const bool four = (variant_in & 8) && H.dup % 4 == 0 && (align & 15u) == 0;
    // pass 1: rows staged in pairs interleaved by column -- two pairs per block
    // (one block of 512 threads per SM) or one pair (two blocks per SM)
    {
        const size_t pair = lean_smem_bytes(H.dup);
        const bool two = variant != 1 && 2 * pair + 8 * 1024 <= 227 * 1024;
        const bool quad = two && variant >= 2 && (H.dup + 63) / 64 <= kQuadMaxBlocks;
        const int nt = !quad ? 512 : variant == 3 ? 640 : variant == 4 ? 768 : variant == 5 ? 1024 : 512;
        const bool sp = H.up.npal <= 32;
        auto k = quad && nt == 1024 ? (sp ? up_pass_quad_kernel<KS, 1024, true> : up_pass_quad_kernel<KS, 1024, false>)
                 : quad && nt == 768 ? (sp ? up_pass_quad_kernel<KS, 768, true> : up_pass_quad_kernel<KS, 768, false>)
                 : quad && nt == 640 ? (sp ? up_pass_quad_kernel<KS, 640, true> : up_pass_quad_kernel<KS, 640, false>)
                 : quad ? (sp ? up_pass_quad_kernel<KS, 512, true> : up_pass_quad_kernel<KS, 512, false>)
                 : two  ? (sp ? up_pass_kernel<KS, 2, 512, 1, true> : up_pass_kernel<KS, 2, 512, 1, false>)
                        : (sp ? up_pass_kernel<KS, 1, 512, 2, true> : up_pass_kernel<KS, 1, 512, 2, false>);
        const size_t smem = two ? 2 * pair : pair;
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, nt, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorInvalidConfiguration;
        const int64_t groups = (H.ddn + (two ? 3 : 1)) / (two ? 4 : 2);
        int64_t grid = (int64_t)num_sms * per_sm;
        if (grid > groups) grid = groups;
        k<<<(int)grid, nt, smem, st>>>(H, static_cast<const float *>(a.x), y1);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    auto k2 = four ? (a.mode == kModeStep ? down_pass4_kernel<KMD, true> : down_pass4_kernel<KMD, false>)
                   : (a.mode == kModeStep ? down_pass_kernel<KMD, true> : down_pass_kernel<KMD, false>);
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2, 256, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    k2<<<num_sms * per_sm, 256, 0, st>>>(H, a, y1);
    return cudaGetLastError();
}

cudaError_t launch_tiled_f32(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st);

}  // namespace edk
