// H*v in the reference's split form, HAIMupdo_multr_split
// (ed_solver/HAIMupdo.f90:1221-1347) on one GPU:
//   1. y = [U(c,c) terms] + [U(c1,c2) n1 n2 terms] + (diag_up + diag_dn) x
//      + up hops, per element in that order (split_up_kernel);
//   2. x and y transposed (dim_up x dim_dn with up fastest -> down fastest);
//   3. the down hops added as up hops of the transposed arrays
//      (split_dn_kernel);
//   4. y transposed back.
// The split form has no -JJ density terms (HAIMupdo_multr has them) and the
// reference STOPs in it when |Jhund| > 1e-5; the host checks that.  In FP64
// every element is accumulated with separate multiply and add in the
// reference's order, so the result equals a sequential FP64 evaluation bit
// for bit; FP32 vectors are widened into FP64 accumulators, and the partial
// sums of step 1 are stored as FP32 between the passes.
#include "edk_device.cuh"

namespace edk {

namespace {

template <typename T>
__global__ void split_up_kernel(const HamDev H, const int32_t *__restrict__ soff, const double *__restrict__ scoef,
                                const T *__restrict__ x, T *__restrict__ y)
{
    const int64_t dup = H.dup, n = H.dup * H.ddn;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = i / dup, u = i - d * dup;
        const T xi = x[i];
        double acc = 0.0;
        const int g = (int)H.up.imp[u] * H.ncfg + (int)H.dn.imp[d];
        for (int o = soff[g]; o < soff[g + 1]; ++o) acc = hmadd<T>(acc, scoef[o], xi);
        acc = hmadd<T>(acc, fadd(H.up.diag[u], H.dn.diag[d]), xi);
        const T *xr = x + d * dup;
        for (int p = H.up.ptr[u]; p < H.up.ptr[u + 1]; ++p) acc = hmadd<T>(acc, H.up.val[p], xr[H.up.tgt[p]]);
        y[i] = (T)acc;
    }
}

// the transposed arrays hold element (u, d) at d + u*ddn
template <typename T>
__global__ void split_dn_kernel(const HamDev H, const T *__restrict__ xt, T *__restrict__ yt)
{
    const int64_t ddn = H.ddn, n = H.dup * H.ddn;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t u = i / ddn, d = i - u * ddn;
        double acc = (double)yt[i];
        const T *xr = xt + u * ddn;
        for (int p = H.dn.ptr[d]; p < H.dn.ptr[d + 1]; ++p) acc = hmadd<T>(acc, H.dn.val[p], xr[H.dn.tgt[p]]);
        yt[i] = (T)acc;
    }
}

// out[r + c*nrow] = in[c + r*ncol] through 32 x 32 shared-memory tiles
template <typename T>
__global__ void transpose_kernel(const T *__restrict__ in, T *__restrict__ out, int64_t ncol, int64_t nrow)
{
    __shared__ T tile[32][33];
    const int64_t c0 = (int64_t)blockIdx.x * 32;
    for (int64_t r0 = (int64_t)blockIdx.y * 32; r0 < nrow; r0 += (int64_t)gridDim.y * 32) {
        for (int j = threadIdx.y; j < 32; j += blockDim.y) {
            const int64_t r = r0 + j, c = c0 + threadIdx.x;
            if (r < nrow && c < ncol) tile[j][threadIdx.x] = in[c + r * ncol];
        }
        __syncthreads();
        for (int j = threadIdx.y; j < 32; j += blockDim.y) {
            const int64_t c = c0 + j, r = r0 + threadIdx.x;
            if (r < nrow && c < ncol) out[r + c * nrow] = tile[threadIdx.x][j];
        }
        __syncthreads();
    }
}

template <typename T>
cudaError_t transpose(const T *in, T *out, int64_t ncol, int64_t nrow, cudaStream_t st)
{
    const int64_t gx = (ncol + 31) / 32, gy = (nrow + 31) / 32;
    if (gx > 0x7fffffffLL) return cudaErrorInvalidValue;
    dim3 grid((unsigned)gx, (unsigned)(gy < 65535 ? gy : 65535));
    transpose_kernel<T><<<grid, dim3(32, 8), 0, st>>>(in, out, ncol, nrow);
    return cudaGetLastError();
}

template <typename T>
cudaError_t split_hv(const HamDev &H, const int32_t *soff, const double *scoef, const T *x, T *y, T *xt, T *yt,
                     int num_sms, cudaStream_t st)
{
    const int grid = num_sms * 8;
    split_up_kernel<T><<<grid, 256, 0, st>>>(H, soff, scoef, x, y);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = transpose<T>(x, xt, H.dup, H.ddn, st);
    if (e == cudaSuccess) e = transpose<T>(y, yt, H.dup, H.ddn, st);
    if (e != cudaSuccess) return e;
    split_dn_kernel<T><<<grid, 256, 0, st>>>(H, xt, yt);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = transpose<T>(yt, y, H.ddn, H.dup, st);
    return e;
}

}  // namespace

cudaError_t launch_split_hv(const HamDev &H, int dtype, const int32_t *soff, const double *scoef, const void *x,
                            void *y, void *xt, void *yt, int num_sms, cudaStream_t st)
{
    if (dtype == EDK_F64)
        return split_hv<double>(H, soff, scoef, static_cast<const double *>(x), static_cast<double *>(y),
                                static_cast<double *>(xt), static_cast<double *>(yt), num_sms, st);
    return split_hv<float>(H, soff, scoef, static_cast<const float *>(x), static_cast<float *>(y),
                           static_cast<float *>(xt), static_cast<float *>(yt), num_sms, st);
}

}  // namespace edk
