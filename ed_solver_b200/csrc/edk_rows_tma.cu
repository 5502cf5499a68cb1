// Row kernel with bulk-copy row staging: FP32 instances with FP64 hop sums,
// and the FP32 dispatch.  The kernel itself is in edk_rows_tma.cuh.
#include "edk_rows_tma_inst.cuh"

namespace edk {

cudaError_t launch_tma_f32_s32(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st);

cudaError_t launch_tma_f32(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st)
{
    if (a.sum32) return launch_tma_f32_s32(H, a, num_sms, s, st);
    EDK_TMA_F32_ALL(false)
    return cudaErrorInvalidValue;
}

}  // namespace edk
