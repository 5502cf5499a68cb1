// edk_cf_eval_noalloc: the continued fractions of edk_cf_eval without any
// device allocation.  It has no counterpart in the reference.
//
// All device memory the call needs -- copies of the host inputs, the output
// and the zero-denominator flag -- lives in one file-scope static device array
// (kScratchBytes per device, created with the module), cut into 256-byte
// aligned regions per call.  Each call runs with the context's device current
// (the caller's current device is restored before it returns), so the array,
// the stream and the copies always belong to one device.  The array's address
// is resolved once per device with cudaGetSymbolAddress, with that device
// current, by the first call made on it; that first call should come before
// any stream capture.  Every call on a device shares the one array: the flag,
// which must start at zero, is cleared at the start of each call, and calls
// whose GPU work overlaps race on the array.  No cudaMalloc, cudaFree or allocating library routine is called.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "edk_internal.h"

extern "C" {
cudaStream_t edk_internal_stream(edk_ctx *ctx);
int edk_internal_fail(edk_ctx *ctx, int code, const char *msg);
int edk_internal_ctx_device(const edk_ctx *ctx);
}

namespace {

constexpr size_t kScratchBytes = EDK_NOALLOC_SCRATCH_BYTES;
constexpr size_t kAlign = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void *g_scratch_ptr[kMaxDevices] = {};

size_t round_up(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

// Makes the context's device current for the lifetime of the guard and puts
// the caller's current device back afterwards.
struct DeviceGuard {
    int prev = -1;
    bool switched = false;
    cudaError_t enter(int dev)
    {
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) return e;
        if (prev == dev) return cudaSuccess;
        e = cudaSetDevice(dev);
        switched = e == cudaSuccess;
        return e;
    }
    ~DeviceGuard()
    {
        if (switched) cudaSetDevice(prev);
    }
};

// Once per device, with that device current: the device address of g_scratch.
int scratch_of_device(edk_ctx *ctx, int dev, unsigned char **out)
{
    if (dev < 0 || dev >= kMaxDevices)
        return edk_internal_fail(ctx, EDK_ERR_CUDA, "edk_cf_eval_noalloc: device ordinal outside the table");
    cudaError_t e;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            char msg[256];
            snprintf(msg, sizeof msg, "edk_cf_eval_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                     cudaGetErrorString(e));
            return edk_internal_fail(ctx, EDK_ERR_CUDA, msg);
        }
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<unsigned char *>(g_scratch_ptr[dev]);
    return EDK_OK;
}

}  // namespace

extern "C" int edk_cf_eval_noalloc(edk_ctx *ctx, int32_t nchain, int32_t ld, const int32_t *n_host,
                                   const double *diag_host, const double *subdiag_host, const double *e_host,
                                   const double *ph_host, const double *scale_host, int32_t nw,
                                   const double *wn_host, double *G_host)
{
    if (!ctx || nchain < 1 || ld < 1 || nw < 1 || !n_host || !diag_host || !subdiag_host || !e_host || !ph_host ||
        !scale_host || !wn_host || !G_host)
        return EDK_ERR_INVALID;
    for (int i = 0; i < nchain; ++i)
        if (n_host[i] < 0 || n_host[i] > ld)
            return edk_internal_fail(ctx, EDK_ERR_INVALID, "edk_cf_eval_noalloc: chain length outside [0,ld]");

    // regions of the scratch array, in order
    const size_t nc = (size_t)nchain, L = (size_t)ld, W = (size_t)nw;
    const size_t b_flag = round_up(sizeof(int));
    const size_t b_n = round_up(sizeof(int32_t) * nc);
    const size_t b_tri = round_up(sizeof(double) * nc * L);
    const size_t b_chain = round_up(sizeof(double) * nc);
    const size_t b_wn = round_up(sizeof(double) * W);
    const size_t b_G = round_up(sizeof(double) * 2 * nc * W);
    const size_t need = b_flag + b_n + 2 * b_tri + 3 * b_chain + b_wn + b_G;
    if (need > kScratchBytes) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "edk_cf_eval_noalloc: %d chains x %d levels at %d frequencies need %zu bytes of scratch; "
                 "the static maximum is %zu bytes (EDK_NOALLOC_SCRATCH_BYTES)",
                 nchain, ld, nw, need, kScratchBytes);
        return edk_internal_fail(ctx, EDK_ERR_INVALID, msg);
    }
    // the context's device, not whichever device the caller left current
    const int dev = edk_internal_ctx_device(ctx);
    DeviceGuard guard;
    if (guard.enter(dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return edk_internal_fail(ctx, EDK_ERR_CUDA, "edk_cf_eval_noalloc: cannot make the context's device current");
    }
    unsigned char *base = nullptr;
    int rc = scratch_of_device(ctx, dev, &base);
    if (rc) return rc;
    unsigned char *q = base;
    auto take = [&](size_t bytes) { unsigned char *p = q; q += bytes; return p; };
    int *flag = reinterpret_cast<int *>(take(b_flag));
    int32_t *n = reinterpret_cast<int32_t *>(take(b_n));
    double *diag = reinterpret_cast<double *>(take(b_tri));
    double *sub = reinterpret_cast<double *>(take(b_tri));
    double *e = reinterpret_cast<double *>(take(b_chain));
    double *ph = reinterpret_cast<double *>(take(b_chain));
    double *scale = reinterpret_cast<double *>(take(b_chain));
    double *wn = reinterpret_cast<double *>(take(b_wn));
    double *G = reinterpret_cast<double *>(take(b_G));

    cudaStream_t st = edk_internal_stream(ctx);
    cudaError_t ce = cudaMemsetAsync(flag, 0, sizeof(int), st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(n, n_host, sizeof(int32_t) * nc, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(diag, diag_host, sizeof(double) * nc * L, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(sub, subdiag_host, sizeof(double) * nc * L, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(e, e_host, sizeof(double) * nc, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(ph, ph_host, sizeof(double) * nc, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(scale, scale_host, sizeof(double) * nc, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(wn, wn_host, sizeof(double) * W, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = edk::launch_cf(nchain, ld, n, diag, sub, e, ph, scale, nw, wn, G, flag, st);
    int hflag = 0;
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(G_host, G, sizeof(double) * 2 * nc * W, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) {
        char msg[256];
        snprintf(msg, sizeof msg, "edk_cf_eval_noalloc: %s", cudaGetErrorString(ce));
        return edk_internal_fail(ctx, EDK_ERR_CUDA, msg);
    }
    if (hflag) return edk_internal_fail(ctx, EDK_ERR_CF_ZERO_DEN, "zero denominator in the continued fraction");
    return EDK_OK;
}
