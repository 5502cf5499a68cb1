// Fast row kernel: FP32 instances, launch-shape enumeration and dispatch.
// The kernel itself is in edk_rows_fast.cuh.
#include "edk_rows_fast.cuh"
#include "edk_rows_tma.cuh"
#include "edk_rows_lean.cuh"
#include "edk_rows_tiled.cuh"

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

// Rows per group of the bulk-copy kernel (one column per thread, the loads of
// the next column in registers): two rows while the neighbour loads fit.
int tma_rows_allowed(int eb, int kmd, int *out)
{
    if (eb == 4 && kmd <= 12) { out[0] = 2; out[1] = 1; return 2; }
    if (eb == 8 && kmd == 4) { out[0] = 2; out[1] = 1; return 2; }
    out[0] = 1;
    return 1;
}

}  // namespace

bool fast_rows_ok(const HamDev &H, int elem_bytes)
{
    const int kmax = H.up.ell_k > H.dn_kmax ? H.up.ell_k : H.dn_kmax;
    const int64_t rowbytes = H.dup * (int64_t)elem_bytes;
    return !H.hund && H.nc <= 2 && kmax <= 16 && rowbytes <= kMaxSmemBytes && H.up.packed &&
           H.dup * H.ddn < (int64_t)1 << 31 && H.up.ell_k >= 0;
}

int fast_shapes(const HamDev &H, int elem_bytes, int num_sms, FastShape *out, int cap, int sum32)
{
    if (!fast_rows_ok(H, elem_bytes)) return 0;
    const int kmu = H.up.ell_k <= 8 ? 8 : 16;
    const int kmd = H.dn_kmax <= 4 ? 4 : H.dn_kmax <= 8 ? 8 : H.dn_kmax <= 12 ? 12 : 16;
    const int64_t rowbytes = H.dup * (int64_t)elem_bytes;
    int rs[3];
    const int nr = rows_allowed(elem_bytes, kmd, rs);
    int n = 0;
    // the register-staged kernel reads column pairs: even rows only
    for (int variant = 0; variant < 3 && (H.dup % 2) == 0; ++variant) {
        // shared memory per block when 1, 2 or 4 blocks share an SM
        const int64_t smem_cap = kMaxSmemBytes / (variant == 0 ? 1 : variant == 1 ? 2 : 4);
        // 128-thread blocks only pay off for short rows
        if (variant == 2 && H.dup > 4096) continue;
        for (int i = 0; i < nr && n < cap; ++i) {
            const int r = rs[i];
            if ((int64_t)r * rowbytes > smem_cap) continue;
            // keep every SM busy: no multi-row groups when there are too few rows
            if (r > 1 && (H.ddn + r - 1) / r < num_sms) continue;
            out[n++] = FastShape{r, kmu, kmd, variant, 0};
        }
    }
    // the bulk-copy kernels: two staged-row buffers of R rows per block
    const int64_t slotb = (int64_t)tma_slot_elems(H.dup, elem_bytes) * elem_bytes;
    auto feasible = [&](int r, int variant) {
        const int64_t smem_cap = kMaxSmemBytes / (variant == 0 ? 1 : variant == 1 ? 2 : 4);
        if (variant == 2 && H.dup > 4096) return false;
        if (2 * r * slotb > smem_cap) return false;
        return !(r > 1 && (H.ddn + r - 1) / r < num_sms);
    };
    const int nr2 = tma_rows_allowed(elem_bytes, kmd, rs);
    for (int variant = 0; variant < 3; ++variant)
        for (int i = 0; i < nr2 && n < cap; ++i)
            if (feasible(rs[i], variant)) out[n++] = FastShape{rs[i], kmu, kmd, variant, 1};
    // kind 2 (instantiated for down-table bounds 8 and 12, and in FP32 with
    // one row per group for tables exactly 9 wide): variants 0, 1, 3 (768
    // threads, one block per SM) and 4 (640 threads, one block per SM)
    if ((kmd == 8 || kmd == 12) && (H.dup % 2) == 0) {
        const int kmu9 = elem_bytes == 4 && H.up.ell_k == 9 ? 9 : kmu;
        const int kmd9 = elem_bytes == 4 && H.dn_kmax == 9 ? 9 : kmd;
        const int rr[2] = {2, 1};
        for (int i = 0; i < 2; ++i) {
            const int r = rr[i];
            if (elem_bytes == 8 && r > 1) continue;
            int ku = r == 1 ? kmu9 : kmu, kd = r == 1 ? kmd9 : kmd;
            // exact-9 instances: (9, 8), (8, 9), (9, 9)
            if ((ku == 9 && kd == 12) || (kd == 9 && ku == 16)) { ku = kmu; kd = kmd; }
            for (int variant : {0, 1, 3, 4})
                if (n < cap && feasible(r, variant >= 3 ? 0 : variant)) out[n++] = FastShape{r, ku, kd, variant, 2};
        }
    }
    // kind 3, the lean FP32 kernel (FP32 hop sums only): two interleaved rows
    // per block; 256 threads x 2 blocks or 512 x 1 per SM; down-row
    // bounds 7, 8 and 9, lean table widths 8 and 10
    if (elem_bytes == 4 && sum32 && H.up.lean && (H.dup % 2) == 0 && H.dn_kmax <= 9 &&
        (H.up.lean_ks == 8 || H.up.lean_ks == 10) && (H.ddn + 1) / 2 >= num_sms) {
        const int ks = H.up.lean_ks;   // the table's stride: instances 8 and 10
        const int kd = H.dn_kmax <= 7 ? 7 : H.dn_kmax;
        const int64_t smem = lean_smem_bytes(H.dup);
        if (n < cap && 2 * smem + 16 * 1024 <= 228 * 1024) out[n++] = FastShape{2, ks, kd, 0, 3};
        if (n < cap && smem + 8 * 1024 <= 228 * 1024) out[n++] = FastShape{2, ks, kd, 1, 3};
        // kind 5: up-spin pass with the rows staged (two row pairs or one per
        // block, or four rows interleaved in one buffer), down-spin pass over
        // L2-resident column tiles
        if (n < cap && 2 * smem + 8 * 1024 <= 227 * 1024) out[n++] = FastShape{2, ks, kd, 0, 5};
        if (n < cap && smem + 8 * 1024 <= 228 * 1024) out[n++] = FastShape{2, ks, kd, 1, 5};
        for (int v = 2; v <= 5; ++v)
            if (n < cap && 2 * smem + 8 * 1024 <= 227 * 1024) out[n++] = FastShape{2, ks, kd, v, 5};
        // the same with the down pass on four columns per thread (16-byte accesses)
        if (H.dup % 4 == 0)
            for (int v = 1; v <= 5; ++v)
                if (n < cap && (v == 1 ? smem + 8 * 1024 <= 228 * 1024 : 2 * smem + 8 * 1024 <= 227 * 1024))
                    out[n++] = FastShape{2, ks, kd, v | 8, 5};
    }
    return n;
}

cudaError_t launch_rows_fast(const HamDev &H, int dtype, const RowArgs &a, int num_sms, const FastShape &s,
                             cudaStream_t st)
{
    if (s.kind == 3) return dtype == EDK_F32 ? launch_lean_f32(H, a, num_sms, s, st) : cudaErrorInvalidValue;
    if (s.kind == 5) return dtype == EDK_F32 ? launch_tiled_f32(H, a, num_sms, s, st) : cudaErrorInvalidValue;
    if (s.kind >= 1)
        return dtype == EDK_F64 ? launch_tma_f64(H, a, num_sms, s, st) : launch_tma_f32(H, a, num_sms, s, st);
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
