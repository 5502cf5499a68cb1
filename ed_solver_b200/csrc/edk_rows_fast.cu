// Fast row kernel: FP32 instances, launch-shape enumeration and dispatch.
// The kernel itself is in edk_rows_fast.cuh.
#include "edk_rows_fast.cuh"

namespace edk {

namespace {

// Rows per group allowed for (element bytes, down-table bound): the R*KMD
// neighbour pairs and the up-table entries stay in registers.
int rows_allowed(int eb, int kmd, int *out)
{
    if (eb == 4) {
        if (kmd == 4) { out[0] = 4; out[1] = 2; out[2] = 1; return 3; }
        if (kmd == 8 || kmd == 12) { out[0] = 2; out[1] = 1; return 2; }
        out[0] = 1;
        return 1;
    }
    if (kmd == 4) { out[0] = 2; out[1] = 1; return 2; }
    out[0] = 1;
    return 1;
}

}  // namespace

bool fast_rows_ok(const HamDev &H, int elem_bytes)
{
    const int kmax = H.up.ell_k > H.dn_kmax ? H.up.ell_k : H.dn_kmax;
    const int64_t rowbytes = H.dup * (int64_t)elem_bytes;
    return !H.hund && H.nc <= 2 && (H.dup % 2) == 0 && kmax <= 16 && rowbytes <= kMaxSmemBytes &&
           H.up.packed && H.dup * H.ddn < (int64_t)1 << 31 && H.up.ell_k >= 0;
}

int fast_shapes(const HamDev &H, int elem_bytes, int num_sms, FastShape *out, int cap)
{
    if (!fast_rows_ok(H, elem_bytes)) return 0;
    const int kmu = H.up.ell_k <= 8 ? 8 : 16;
    const int kmd = H.dn_kmax <= 4 ? 4 : H.dn_kmax <= 8 ? 8 : H.dn_kmax <= 12 ? 12 : 16;
    const int64_t rowbytes = H.dup * (int64_t)elem_bytes;
    int rs[3];
    const int nr = rows_allowed(elem_bytes, kmd, rs);
    int n = 0;
    for (int variant = 0; variant < 3; ++variant) {
        // shared memory per block when 1, 2 or 4 blocks share an SM
        const int64_t smem_cap = kMaxSmemBytes / (variant == 0 ? 1 : variant == 1 ? 2 : 4);
        // 128-thread blocks only pay off for short rows
        if (variant == 2 && H.dup > 4096) continue;
        for (int i = 0; i < nr && n < cap; ++i) {
            const int r = rs[i];
            if ((int64_t)r * rowbytes > smem_cap) continue;
            // keep every SM busy: no multi-row groups when there are too few rows
            if (r > 1 && (H.ddn + r - 1) / r < num_sms) continue;
            out[n++] = FastShape{r, kmu, kmd, variant};
        }
    }
    return n;
}

cudaError_t launch_rows_fast(const HamDev &H, int dtype, const RowArgs &a, int num_sms, const FastShape &s,
                             cudaStream_t st)
{
    return dtype == EDK_F64 ? launch_fast_f64(H, a, num_sms, s, st) : launch_fast_f32(H, a, num_sms, s, st);
}

#define EDK_FAST_V(T, R, KMU, KMD)                                                                \
    if (s.r == R && s.kmu == KMU && s.kmd == KMD)                                                 \
        return s.variant == 0   ? launch_fast_t<T, R, KMU, KMD, 512, 1, 2>(H, a, num_sms, st)     \
               : s.variant == 1 ? launch_fast_t<T, R, KMU, KMD, 256, 2, 2>(H, a, num_sms, st)     \
                                : launch_fast_t<T, R, KMU, KMD, 128, 4, 2>(H, a, num_sms, st);
#define EDK_FAST_KMU(T, R, KMD) EDK_FAST_V(T, R, 8, KMD) EDK_FAST_V(T, R, 16, KMD)

cudaError_t launch_fast_f32(const HamDev &H, const RowArgs &a, int num_sms, const FastShape &s, cudaStream_t st)
{
    EDK_FAST_KMU(float, 4, 4)
    EDK_FAST_KMU(float, 2, 4)
    EDK_FAST_KMU(float, 1, 4)
    EDK_FAST_KMU(float, 2, 8)
    EDK_FAST_KMU(float, 1, 8)
    EDK_FAST_KMU(float, 2, 12)
    EDK_FAST_KMU(float, 1, 12)
    EDK_FAST_KMU(float, 1, 16)
    return cudaErrorInvalidValue;
}

}  // namespace edk
