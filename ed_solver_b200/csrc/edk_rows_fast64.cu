// Fast row kernel: FP64 instances (the kernel is in edk_rows_fast.cuh).
#include "edk_rows_fast.cuh"

namespace edk {

#define EDK_FAST_V(T, R, KMU, KMD)                                                                \
    if (s.r == R && s.kmu == KMU && s.kmd == KMD)                                                 \
        return s.variant == 0   ? launch_fast_t<T, R, KMU, KMD, 512, 1, 2>(H, a, num_sms, st)     \
               : s.variant == 1 ? launch_fast_t<T, R, KMU, KMD, 256, 2, 2>(H, a, num_sms, st)     \
                                : launch_fast_t<T, R, KMU, KMD, 128, 4, 2>(H, a, num_sms, st);
#define EDK_FAST_KMU(T, R, KMD) EDK_FAST_V(T, R, 8, KMD) EDK_FAST_V(T, R, 16, KMD)

cudaError_t launch_fast_f64(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st)
{
    EDK_FAST_KMU(double, 2, 4)
    EDK_FAST_KMU(double, 1, 4)
    EDK_FAST_KMU(double, 1, 8)
    EDK_FAST_KMU(double, 1, 12)
    EDK_FAST_KMU(double, 1, 16)
    return cudaErrorInvalidValue;
}

}  // namespace edk
