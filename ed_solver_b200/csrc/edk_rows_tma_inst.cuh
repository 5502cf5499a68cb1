// Instance lists of the bulk-copy row kernel (edk_rows_tma.cuh), shared by
// the per-element-type dispatch files.
#pragma once
#include "edk_rows_tma.cuh"

// kind 1 (one column, pipelined) for every block variant; kinds 2-4 for the
// 512- and 256-thread variants
#define EDK_TMA_KIND1(T, R, KMU, KMD, S)                                                                     \
    if (s.kind == 1 && s.r == R && s.kmu == KMU && s.kmd == KMD)                                             \
        return s.variant == 0   ? launch_tma_t<T, R, KMU, KMD, 512, 1, 1, true, S>(H, a, num_sms, st)        \
               : s.variant == 1 ? launch_tma_t<T, R, KMU, KMD, 256, 2, 1, true, S>(H, a, num_sms, st)        \
                                : launch_tma_t<T, R, KMU, KMD, 128, 4, 1, true, S>(H, a, num_sms, st);
#define EDK_TMA_KIND(T, R, KMU, KMD, S, KIND, CPT, PIPE)                                                     \
    if (s.kind == KIND && s.r == R && s.kmu == KMU && s.kmd == KMD)                                          \
        return s.variant == 0   ? launch_tma_t<T, R, KMU, KMD, 512, 1, CPT, PIPE, S>(H, a, num_sms, st)      \
               : s.variant == 1 ? launch_tma_t<T, R, KMU, KMD, 256, 2, CPT, PIPE, S>(H, a, num_sms, st)      \
               : s.variant == 3 ? launch_tma_t<T, R, KMU, KMD, 768, 1, CPT, PIPE, S>(H, a, num_sms, st)      \
                                : launch_tma_t<T, R, KMU, KMD, 640, 1, CPT, PIPE, S>(H, a, num_sms, st);
// kind 2 (two columns per thread): rows per group 2 or 1
#define EDK_TMA_MORE(T, KMU, KMD, S)                                                                         \
    EDK_TMA_KIND(T, 2, KMU, KMD, S, 2, 2, false)                                                             \
    EDK_TMA_KIND(T, 1, KMU, KMD, S, 2, 2, false)

#define EDK_TMA_F32_ALL(S)                                                                                   \
    EDK_TMA_KIND1(float, 2, 8, 4, S) EDK_TMA_KIND1(float, 2, 16, 4, S)                                       \
    EDK_TMA_KIND1(float, 1, 8, 4, S) EDK_TMA_KIND1(float, 1, 16, 4, S)                                       \
    EDK_TMA_KIND1(float, 2, 8, 8, S) EDK_TMA_KIND1(float, 2, 16, 8, S)                                       \
    EDK_TMA_KIND1(float, 1, 8, 8, S) EDK_TMA_KIND1(float, 1, 16, 8, S)                                       \
    EDK_TMA_KIND1(float, 2, 8, 12, S) EDK_TMA_KIND1(float, 2, 16, 12, S)                                     \
    EDK_TMA_KIND1(float, 1, 8, 12, S) EDK_TMA_KIND1(float, 1, 16, 12, S)                                     \
    EDK_TMA_KIND1(float, 1, 8, 16, S) EDK_TMA_KIND1(float, 1, 16, 16, S)                                     \
    EDK_TMA_MORE(float, 8, 8, S) EDK_TMA_MORE(float, 16, 8, S)                                               \
    EDK_TMA_MORE(float, 8, 12, S) EDK_TMA_MORE(float, 16, 12, S)                                             \
    EDK_TMA_KIND(float, 1, 9, 8, S, 2, 2, false) EDK_TMA_KIND(float, 1, 8, 9, S, 2, 2, false)                \
    EDK_TMA_KIND(float, 1, 9, 9, S, 2, 2, false)
