// Row kernel with bulk-copy row staging: FP64 instances.
#include "edk_rows_tma_inst.cuh"

namespace edk {

cudaError_t launch_tma_f64(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st)
{
    EDK_TMA_KIND1(double, 2, 8, 4, false) EDK_TMA_KIND1(double, 2, 16, 4, false)
    EDK_TMA_KIND1(double, 1, 8, 4, false) EDK_TMA_KIND1(double, 1, 16, 4, false)
    EDK_TMA_KIND1(double, 1, 8, 8, false) EDK_TMA_KIND1(double, 1, 16, 8, false)
    EDK_TMA_KIND1(double, 1, 8, 12, false) EDK_TMA_KIND1(double, 1, 16, 12, false)
    EDK_TMA_KIND1(double, 1, 8, 16, false) EDK_TMA_KIND1(double, 1, 16, 16, false)
    EDK_TMA_KIND(double, 1, 8, 8, false, 2, 2, false) EDK_TMA_KIND(double, 1, 16, 8, false, 2, 2, false)
    EDK_TMA_KIND(double, 1, 8, 12, false, 2, 2, false) EDK_TMA_KIND(double, 1, 16, 12, false, 2, 2, false)
    return cudaErrorInvalidValue;
}

}  // namespace edk
