// Internal declarations of the adjoint kernels (edk_grad_kernels.cu) used by
// the gradient drivers (edk_grad.cpp).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace edk {

constexpr int kMaxGradParams = 64;

enum ParamKind : int {
    kParamNumber = 0,   // n_p on the spins of spin_mask
    kParamHop = 1,      // c+_p c_q + c+_q c_p through the maps
    kParamDouble = 2,   // n_p,up n_p,dn
    kParamPair = 3,     // (n_p,up + n_p,dn)(n_q,up + n_q,dn)
};

struct ParamDev {
    int kind;
    int spin_mask;                  // bit 0 up, bit 1 down
    uint32_t bp, bq;                // orbital bit masks
    const int32_t *mapu, *mapd;     // hop maps per spin (null when that spin is not included)
};

cudaError_t launch_lincomb(int64_t n, double *out, bool accumulate, const double *x0, double c0,
                           const double *x1, double c1, const double *x2, double c2, const double *x3,
                           double c3, int grid, cudaStream_t st);
cudaError_t launch_dots(int64_t n, const double *x0, const double *y0, const double *x1, const double *y1,
                        const double *x2, const double *y2, const double *x3, const double *y3, double *partials,
                        unsigned *counter, double *out, int grid, cudaStream_t st);
cudaError_t launch_fill_periodic(int64_t n, const double *tab, int64_t offset, double *out, int grid, cudaStream_t st);
cudaError_t launch_bilinear(int64_t dup, int64_t ddn, const double *a, const double *b, const uint32_t *st_up,
                            const uint32_t *st_dn, int np, const ParamDev *P, double *partials, unsigned *counter,
                            double *out, int grid, cudaStream_t st);

}  // namespace edk
