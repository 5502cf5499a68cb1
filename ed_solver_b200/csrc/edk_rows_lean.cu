// Lean FP32 row kernel (kind 3): instances and shape dispatch.
// The kernel itself is in edk_rows_lean.cuh.
#include "edk_rows_lean.cuh"

namespace edk {

#define EDK_LEAN_V(KS, KMD)                                                                     \
    if (s.kmu == KS && s.kmd == KMD)                                                            \
        return s.variant == 0 ? launch_lean_t<KS, KMD, 256, 2>(H, a, num_sms, st)               \
                              : launch_lean_t<KS, KMD, 512, 1>(H, a, num_sms, st);
#define EDK_LEAN_KS(KS) EDK_LEAN_V(KS, 7) EDK_LEAN_V(KS, 8) EDK_LEAN_V(KS, 9)

cudaError_t launch_lean_f32(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st)
{
    if (!a.sum32 || !H.up.lean) return cudaErrorInvalidValue;
    EDK_LEAN_KS(8)
    EDK_LEAN_KS(10)
    return cudaErrorInvalidValue;
}

}  // namespace edk
