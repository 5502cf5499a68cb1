// Two-pass tiled FP32 row step (kind 5): instances and shape dispatch.
// The kernels are in edk_rows_tiled.cuh.
#include "edk_rows_tiled.cuh"

namespace edk {

#define EDK_TILED_V(KS, KMD) \
    if (s.kmu == KS && s.kmd == KMD) return launch_tiled_t<KS, KMD>(H, a, num_sms, s.variant, st);
#define EDK_TILED_KS(KS) EDK_TILED_V(KS, 7) EDK_TILED_V(KS, 8) EDK_TILED_V(KS, 9)

cudaError_t launch_tiled_f32(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st)
{
    if (!a.sum32 || !H.up.lean || !H.up.lean_b || !a.scratch) return cudaErrorInvalidValue;
    EDK_TILED_KS(8)
    EDK_TILED_KS(10)
    return cudaErrorInvalidValue;
}

}  // namespace edk
