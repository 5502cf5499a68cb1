// Device kernels of the adjoint (parameter gradients): FP64 vector updates,
// multi-dot products, and the bilinear forms <a| dH/dtheta_q |b> of every
// requested parameter in one pass over a sector vector.
//
// The Hamiltonian is linear in its parameters, so dH/dtheta_q is a fixed
// operator: a one-body number operator n_p (Ec(c,c), Eb(k,k)), a symmetric
// one-body hop c+_p c_q + c+_q c_p (Ec(i,j), Eb(i,j), Vbc(k,c); the terms of
// HAIM_offdiag_arrays.f90:419-524), n_up n_dn of one impurity site (U(c,c),
// HAIMupdo.f90:784-796) or n_i n_j of two (U(i,j), HAIMupdo.f90:798-829).
// Hops act on one spin species through a per-parameter map of that spin's
// basis: (rank of the target + 1) * Jordan-Wigner sign, or 0.
#include "edk_device.cuh"
#include "edk_grad.h"

namespace edk {

namespace {

__global__ void lincomb_kernel(int64_t n, double *out, int accumulate, const double *x0, double c0,
                               const double *x1, double c1, const double *x2, double c2, const double *x3,
                               double c3)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double v = accumulate ? out[i] : 0.0;
        if (x0) v += c0 * x0[i];
        if (x1) v += c1 * x1[i];
        if (x2) v += c2 * x2[i];
        if (x3) v += c3 * x3[i];
        out[i] = v;
    }
}

__global__ void dots_kernel(int64_t n, const double *x0, const double *y0, const double *x1, const double *y1,
                            const double *x2, const double *y2, const double *x3, const double *y3,
                            double *partials, unsigned *counter, double *out)
{
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (x0) s[0] += x0[i] * y0[i];
        if (x1) s[1] += x1[i] * y1[i];
        if (x2) s[2] += x2[i] * y2[i];
        if (x3) s[3] += x3[i] * y3[i];
    }
    grid_sum<4>(s, partials, counter, out);
}

// One block per row; the rows of a and b are staged in shared memory when
// STAGE.  Per parameter, each warp accumulates its columns in a fixed order
// into its own slot; blocks write per-parameter partials and the last block
// sums them in block order (deterministic).
template <bool STAGE>
__global__ void __launch_bounds__(512, 1) bilinear_kernel(int dup, int ddn, const double *__restrict__ a,
                                                          const double *__restrict__ b,
                                                          const uint32_t *__restrict__ st_up,
                                                          const uint32_t *__restrict__ st_dn, int np,
                                                          const ParamDev *__restrict__ P, double *partials,
                                                          unsigned *counter, double *out)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ ParamDev sp[kMaxGradParams];
    __shared__ double s_part[kMaxGradParams][16];
    __shared__ bool last;
    const int nwarp = (blockDim.x + 31) >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = threadIdx.x; q < np; q += blockDim.x) sp[q] = P[q];
    for (int t = threadIdx.x; t < np * 16; t += blockDim.x) s_part[t / 16][t % 16] = 0.0;
    double *as = reinterpret_cast<double *>(smem_raw);
    double *bs = as + dup;
    for (int row = blockIdx.x; row < ddn; row += gridDim.x) {
        __syncthreads();
        const double *arow = a + (size_t)row * dup, *brow = b + (size_t)row * dup;
        if (STAGE) {
            for (int c = threadIdx.x; c < dup; c += blockDim.x) {
                as[c] = arow[c];
                bs[c] = brow[c];
            }
            __syncthreads();
        }
        const double *ar = STAGE ? as : arow;
        const double *br = STAGE ? bs : brow;
        const uint32_t sdn = st_dn[row];
        for (int q = 0; q < np; ++q) {
            const ParamDev p = sp[q];
            double t = 0.0;
            if (p.kind == kParamNumber) {
                const int fdn = ((p.spin_mask & 2) && (sdn & p.bp)) ? 1 : 0;
                for (int c = threadIdx.x; c < dup; c += blockDim.x) {
                    const int f = (((p.spin_mask & 1) && (st_up[c] & p.bp)) ? 1 : 0) + fdn;
                    if (f) t += (double)f * ar[c] * br[c];
                }
            } else if (p.kind == kParamDouble) {
                if (sdn & p.bp)
                    for (int c = threadIdx.x; c < dup; c += blockDim.x)
                        if (st_up[c] & p.bp) t += ar[c] * br[c];
            } else if (p.kind == kParamPair) {
                const int di = (sdn & p.bp) ? 1 : 0, dj = (sdn & p.bq) ? 1 : 0;
                for (int c = threadIdx.x; c < dup; c += blockDim.x) {
                    const uint32_t su = st_up[c];
                    const int f = (((su & p.bp) ? 1 : 0) + di) * (((su & p.bq) ? 1 : 0) + dj);
                    if (f) t += (double)f * ar[c] * br[c];
                }
            } else {   // kParamHop
                if (p.mapu)
                    for (int c = threadIdx.x; c < dup; c += blockDim.x) {
                        const int32_t m = p.mapu[c];
                        if (m) t += (m > 0 ? ar[c] : -ar[c]) * br[(m > 0 ? m : -m) - 1];
                    }
                if (p.mapd) {
                    const int32_t m = p.mapd[row];
                    if (m) {
                        const double *bo = b + (size_t)((m > 0 ? m : -m) - 1) * dup;
                        double u = 0.0;
                        for (int c = threadIdx.x; c < dup; c += blockDim.x) u += ar[c] * bo[c];
                        t += m > 0 ? u : -u;
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (lane == 0) s_part[q][warp] += t;
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < np; q += blockDim.x) {
        double v = 0.0;
        for (int w = 0; w < nwarp; ++w) v += s_part[q][w];
        partials[(size_t)blockIdx.x * np + q] = v;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int q = threadIdx.x; q < np; q += blockDim.x) {
        double v = 0.0;
        for (unsigned g = 0; g < gridDim.x; ++g) v += __ldcg(&partials[(size_t)g * np + q]);
        out[q] = v;
    }
    if (threadIdx.x == 0) *counter = 0u;
}

// out[i] = tab[(i + offset) % 10000 + 1] (the reference's periodic start
// vector, rcvector_class.f90:43-60, shifted by `offset` for a block column)
__global__ void fill_periodic_kernel(int64_t n, const double *tab, int64_t offset, double *out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = tab[(i + offset) % 10000 + 1];
}

}  // namespace

cudaError_t launch_fill_periodic(int64_t n, const double *tab, int64_t offset, double *out, int grid, cudaStream_t st)
{
    fill_periodic_kernel<<<grid, 256, 0, st>>>(n, tab, offset, out);
    return cudaGetLastError();
}

cudaError_t launch_lincomb(int64_t n, double *out, bool accumulate, const double *x0, double c0,
                           const double *x1, double c1, const double *x2, double c2, const double *x3,
                           double c3, int grid, cudaStream_t st)
{
    lincomb_kernel<<<grid, 256, 0, st>>>(n, out, accumulate ? 1 : 0, x0, c0, x1, c1, x2, c2, x3, c3);
    return cudaGetLastError();
}

cudaError_t launch_dots(int64_t n, const double *x0, const double *y0, const double *x1, const double *y1,
                        const double *x2, const double *y2, const double *x3, const double *y3, double *partials,
                        unsigned *counter, double *out, int grid, cudaStream_t st)
{
    dots_kernel<<<grid, 256, 0, st>>>(n, x0, y0, x1, y1, x2, y2, x3, y3, partials, counter, out);
    return cudaGetLastError();
}

cudaError_t launch_bilinear(int64_t dup, int64_t ddn, const double *a, const double *b, const uint32_t *st_up,
                            const uint32_t *st_dn, int np, const ParamDev *P, double *partials, unsigned *counter,
                            double *out, int grid, cudaStream_t st)
{
    if (np < 1 || np > kMaxGradParams) return cudaErrorInvalidValue;
    if (grid > ddn) grid = (int)ddn;
    if (grid < 1) grid = 1;
    const size_t smem = 2 * (size_t)dup * sizeof(double);
    // the kernel's static shared memory is about 11 KB of the 227 KB a block may use
    if (smem <= (size_t)(227 - 12) * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bilinear_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        bilinear_kernel<true><<<grid, 512, smem, st>>>((int)dup, (int)ddn, a, b, st_up, st_dn, np, P, partials,
                                                       counter, out);
    } else {
        bilinear_kernel<false><<<grid, 512, 0, st>>>((int)dup, (int)ddn, a, b, st_up, st_dn, np, P, partials,
                                                     counter, out);
    }
    return cudaGetLastError();
}

}  // namespace edk
