// Row kernel with bulk-copy row staging: FP32 instances whose up- and
// down-spin hop terms are summed in FP32 (the diagonal, the Lanczos epilogue
// and the reductions stay FP64).
#include "edk_rows_tma_inst.cuh"

namespace edk {

cudaError_t launch_tma_f32_s32(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st)
{
    EDK_TMA_F32_ALL(true)
    return cudaErrorInvalidValue;
}

}  // namespace edk
