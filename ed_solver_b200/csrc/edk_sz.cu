// Device kernels of the Nambu (Sz) sectors: H*v of HAIMsz_multr /
// HAIMsz_mult_fly_r (HAIMsz.f90:453-808) fused with the Lanczos modes of the
// row kernel, and c / c+ of apply_Csz_updo / apply_Csz_N_updo
// (apply_C.f90:344-483).
//
// One thread block per row of equal high half h (the down holes), threads
// over the row's low halves, so the x reads of the own row and of targets
// that keep h are coalesced.  Per element:
//   acc = QUART_INT_SZ * x                               (table by impurity configuration)
//   tabulated order: acc += (sum of the occupied orbitals' diagonal energies) * x
//   on-the-fly order: acc += e_o * x for each occupied orbital o in turn
//   acc += (+-t) * x[rank(target)] for each term c+_tgt c_src in the list whose
//          source is occupied and target empty (sign: parity of the occupied
//          orbitals strictly between)
// in the reference's order with separate multiply and add, so the FP64 result
// equals a sequential FP64 evaluation bit for bit.
#include <cuda_runtime.h>
#include <cstdint>
#include "edk_internal.h"
#include "edk_device.cuh"

namespace edk {

namespace {

constexpr int kSzBlock = 256;
constexpr int kSeg = 4;        // hole-hole / pairing terms whose gathers are issued together

// One entry of a row's list, in the order of the terms:
//   kind 0: a whole up-up run (the per-state table of the run applies);
//   kind 1: a hole-hole term active on the row: the same column of row joff;
//   kind 2: a pairing term whose high-half condition holds on the row; the
//           low-half condition (lsrc set, ltgt empty) is checked per state.
struct RowTerm {
    uint32_t lsrc, ltgt;   // low-half masks the state must have / lack
    uint32_t lbtw;         // low-half orbitals between source and target (sign)
    uint32_t lflip;        // lsrc | ltgt: the low-half bits the term flips
    uint32_t joff;         // rank of the first state of the target row
    uint32_t kr;           // kind | run << 2
    double hv;             // the term's value with the high-half sign applied
};

// Ordered compaction over a block: returns the position of this thread's
// element among the passing ones of its chunk (valid when pass) and adds the
// chunk's count to *total (read after the call by every thread).
__device__ __forceinline__ int block_compact(bool pass, int *warp_cnt, int *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    const unsigned b = __ballot_sync(0xffffffffu, pass);
    if (lane == 0) warp_cnt[warp] = __popc(b);
    __syncthreads();
    int before = *total;
    for (int w = 0; w < warp; ++w) before += warp_cnt[w];
    const int pos = before + __popc(b & ((1u << lane) - 1u));
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = *total;
        for (int w = 0; w < nw; ++w) t += warp_cnt[w];
        *total = t;
    }
    __syncthreads();
    return pos;
}

constexpr uint32_t kEllEnd = 0xFFFFFFFFu;

// Row kernel on per-row lists (see RowTerm); the own row is staged in shared
// memory when STAGE.  Same arithmetic, in the same order, as
// sz_row_simple_kernel.
template <typename T, bool STAGE>
__global__ void __launch_bounds__(kSzBlock, 4) sz_row_kernel(const SzDev S, const RowArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int warp_cnt[32];
    __shared__ int n_terms, n_diag;
    const int nq = 1 << (2 * S.nc);
    RowTerm *rt = reinterpret_cast<RowTerm *>(smem_raw);
    SzRun *runs = reinterpret_cast<SzRun *>(rt + S.nterm);
    double *hs = reinterpret_cast<double *>(runs + S.nrun);         // term values
    double *qs = hs + S.nterm;
    double *de = qs + nq;                                           // row's diagonal energies
    uint32_t *db = reinterpret_cast<uint32_t *>(de + S.ndiag);       // their low-half bit (0: hole, occupied)
    T *xs = reinterpret_cast<T *>(db + ((S.ndiag + 3) & ~3));
    for (int t = threadIdx.x; t < nq; t += blockDim.x) qs[t] = S.quart[t];
    for (int t = threadIdx.x; t < S.nterm; t += blockDim.x) hs[t] = S.terms[t].h;
    for (int t = threadIdx.x; t < S.nrun; t += blockDim.x) runs[t] = S.runs[t];

    const int ks = step_index(a);
    StepScalars sc;
    if (!step_scalars(a, ks, sc)) return;

    const T *__restrict__ x = static_cast<const T *>(a.x);
    const int ns = S.ns, nb = S.nb, nc = S.nc, nterm = S.nterm, ndiag = S.ndiag;
    const uint32_t lowmask = (1u << ns) - 1u, cm = (1u << nc) - 1u;
    const size_t nlow = (size_t)1 << ns;
    const uint32_t *__restrict__ off_h = S.sec.off_h;
    const uint16_t *__restrict__ rank_low = S.rank_low;
    const uint32_t *__restrict__ ell = S.ell;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int r = blockIdx.x; r < S.sec.nrows; r += gridDim.x) {
        const uint32_t h = S.sec.row_h[r];
        const int k = S.sec.npart - __popc(h);
        const int c0 = S.class_start[k], len = S.class_start[k + 1] - c0;
        const uint32_t base = off_h[h];
        __syncthreads();                       // the previous row is done with the lists
        if (threadIdx.x == 0) { n_terms = 0; n_diag = 0; }
        // ---- the row's list ----
        for (int t0 = 0; t0 < nterm; t0 += blockDim.x) {
            const int t = t0 + threadIdx.x;
            bool pass = false;
            SzTerm tm;
            int run = 0, kind = 0;
            if (t < nterm) {
                tm = S.terms[t];
                run = S.term_run[t];
                kind = runs[run].kind;
                if (kind == 0) {
                    pass = runs[run].first == t;
                } else {
                    const uint32_t hsrc = tm.src >> ns, htgt = tm.tgt >> ns;
                    pass = (h & hsrc) == hsrc && (h & htgt) == 0u;
                }
            }
            const int pos = block_compact(pass, warp_cnt, &n_terms);
            if (pass) {
                RowTerm o;
                o.kr = (uint32_t)kind | ((uint32_t)run << 2);
                if (kind == 0) {
                    o.lsrc = o.ltgt = o.lbtw = o.lflip = o.joff = 0u;
                    o.hv = 0.0;
                } else {
                    const uint32_t h2 = h ^ (tm.src >> ns) ^ (tm.tgt >> ns);
                    o.lsrc = tm.src & lowmask;
                    o.ltgt = tm.tgt & lowmask;
                    o.lbtw = tm.btw & lowmask;
                    o.lflip = o.lsrc | o.ltgt;
                    o.joff = off_h[h2];
                    o.hv = (__popc(h & (tm.btw >> ns)) & 1) ? -tm.h : tm.h;
                }
                rt[pos] = o;
            }
        }
        // ---- the diagonal orbitals: low-half ones kept, occupied holes kept ----
        for (int t0 = 0; t0 < ndiag; t0 += blockDim.x) {
            const int t = t0 + threadIdx.x;
            bool pass = false;
            uint32_t bit = 0u;
            if (t < ndiag) {
                bit = S.diag_bit[t];
                pass = (bit & lowmask) != 0u || (h & (bit >> ns)) != 0u;
            }
            const int pos = block_compact(pass, warp_cnt, &n_diag);
            if (pass) { de[pos] = S.diag_e[t]; db[pos] = bit & lowmask; }
        }
        if (STAGE) stage_row<T>(xs, x + base, len);
        __syncthreads();
        const int nt = n_terms, nd = n_diag;
        const uint32_t hcfg = ((h >> nb) & cm) << nc;
        for (int c = threadIdx.x; c < len; c += blockDim.x) {
            const uint32_t l = (uint32_t)S.low_states[c0 + c];
            const int64_t i = (int64_t)base + c;
            const T xo = STAGE ? xs[c] : x[i];
            double acc = fmul(qs[((l >> nb) & cm) | hcfg], (double)xo);
            if (S.order == 0) {
                double d = 0.0;
                for (int o = 0; o < nd; ++o)
                    if (!db[o] || (l & db[o])) d = fadd(d, de[o]);
                acc = hmadd<T>(acc, d, xo);
            } else {
                for (int o = 0; o < nd; ++o)
                    if (!db[o] || (l & db[o])) acc = hmadd<T>(acc, de[o], xo);
            }
            for (int e = 0; e < nt;) {
                const uint32_t kr = rt[e].kr;
                if ((kr & 3u) != 0u) {
                    // up to kSeg consecutive hole-hole / pairing terms: every
                    // target rank looked up, then every x gathered, then the
                    // terms added in list order (the order of the reference)
                    double hq[kSeg];
                    int64_t jq[kSeg];
                    bool on[kSeg];
                    bool run = true;
                    int taken = 0;
#pragma unroll
                    for (int q = 0; q < kSeg; ++q) {
                        const int eq = e + q;
                        run = run && eq < nt && (rt[eq].kr & 3u) != 0u;
                        on[q] = false;
                        hq[q] = 0.0;
                        jq[q] = i;
                        if (run) {
                            ++taken;
                            const RowTerm &t = rt[eq];
                            if ((t.kr & 3u) == 1u) {
                                on[q] = true;
                                hq[q] = t.hv;
                                jq[q] = (int64_t)t.joff + c;
                            } else if ((l & t.lsrc) == t.lsrc && !(l & t.ltgt)) {
                                on[q] = true;
                                hq[q] = (__popc(l & t.lbtw) & 1) ? -t.hv : t.hv;
                                jq[q] = (int64_t)t.joff + rank_low[l ^ t.lflip];
                            }
                        }
                    }
                    T xq[kSeg];
#pragma unroll
                    for (int q = 0; q < kSeg; ++q) xq[q] = on[q] ? __ldg(x + jq[q]) : T(0);
#pragma unroll
                    for (int q = 0; q < kSeg; ++q)
                        if (on[q]) acc = hmadd<T>(acc, hq[q], xq[q]);
                    e += taken;
                    continue;
                }
                ++e;
                {
                    // up-up run: this state's active terms from the run's table,
                    // four entries loaded ahead of their use
                    const SzRun &R = runs[kr >> 2];
                    const uint32_t *tab = ell + R.ell_off + (size_t)(c0 + c);
                    const double *hr = hs + R.first;
                    for (int q0 = 0; q0 < R.kell; q0 += 4) {
                        uint32_t u[4];
#pragma unroll
                        for (int v = 0; v < 4; ++v) u[v] = q0 + v < R.kell ? __ldg(tab + (size_t)(q0 + v) * nlow) : kEllEnd;
                        T xv[4];
#pragma unroll
                        for (int v = 0; v < 4; ++v) {
                            const int col = (int)(u[v] & 0xFFFFu);
                            xv[v] = u[v] == kEllEnd ? T(0) : (STAGE ? xs[col] : __ldg(x + (int64_t)base + col));
                        }
#pragma unroll
                        for (int v = 0; v < 4; ++v) {
                            if (u[v] == kEllEnd) break;
                            const double hv = hr[u[v] >> 17];
                            acc = hmadd<T>(acc, (u[v] & 0x10000u) ? -hv : hv, xv[v]);
                        }
                        if (u[3] == kEllEnd) break;
                    }
                }
            }
            row_epilogue<T>(a, sc, i, acc, xo, s0, s1, s2);
        }
    }
    if (a.mode == kModeHv) return;
    double v[4] = {s0, s1, s2, 0.0};
    if (grid_sum<4>(v, a.partials, a.counter, a.sums_out))
        if (a.mode == kModeFirst || a.mode == kModeStep) lanczos_finalize(a, ks);
}

// Reference form: every state walks the whole term list (kernel path 1).
template <typename T>
__global__ void __launch_bounds__(kSzBlock) sz_row_simple_kernel(const SzDev S, const RowArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SzTerm *ts = reinterpret_cast<SzTerm *>(smem_raw);
    const int nq = 1 << (2 * S.nc);
    double *qs = reinterpret_cast<double *>(ts + S.nterm);
    double *des = qs + nq;
    uint32_t *dbs = reinterpret_cast<uint32_t *>(des + S.ndiag);
    for (int t = threadIdx.x; t < S.nterm; t += blockDim.x) ts[t] = S.terms[t];
    for (int t = threadIdx.x; t < nq; t += blockDim.x) qs[t] = S.quart[t];
    for (int t = threadIdx.x; t < S.ndiag; t += blockDim.x) { des[t] = S.diag_e[t]; dbs[t] = S.diag_bit[t]; }

    const int ks = step_index(a);
    StepScalars sc;
    if (!step_scalars(a, ks, sc)) return;
    __syncthreads();

    const T *__restrict__ x = static_cast<const T *>(a.x);
    const int ns = S.ns, nb = S.nb, nc = S.nc, nterm = S.nterm, ndiag = S.ndiag;
    const uint32_t lowmask = (1u << ns) - 1u, cm = (1u << nc) - 1u;
    const uint32_t *__restrict__ off_h = S.sec.off_h;
    const uint16_t *__restrict__ rank_low = S.rank_low;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int r = blockIdx.x; r < S.sec.nrows; r += gridDim.x) {
        const uint32_t h = S.sec.row_h[r];
        const int k = S.sec.npart - __popc(h);
        const int c0 = S.class_start[k], len = S.class_start[k + 1] - c0;
        const int64_t base = off_h[h];
        const uint32_t hs = h << ns;
        for (int c = threadIdx.x; c < len; c += blockDim.x) {
            const uint32_t s = (uint32_t)S.low_states[c0 + c] | hs;
            const int64_t i = base + c;
            const T xo = x[i];
            const uint32_t cfg = ((s >> nb) & cm) | (((s >> (ns + nb)) & cm) << nc);
            double acc = fmul(qs[cfg], (double)xo);
            if (S.order == 0) {
                double d = 0.0;
                for (int o = 0; o < ndiag; ++o)
                    if (s & dbs[o]) d = fadd(d, des[o]);
                acc = hmadd<T>(acc, d, xo);
            } else {
                for (int o = 0; o < ndiag; ++o)
                    if (s & dbs[o]) acc = hmadd<T>(acc, des[o], xo);
            }
            for (int t = 0; t < nterm; ++t) {
                const uint32_t src = ts[t].src, tgt = ts[t].tgt;
                if (!(s & src) || (s & tgt)) continue;
                const uint32_t s2t = s ^ src ^ tgt;
                const int64_t j = (int64_t)off_h[s2t >> ns] + rank_low[s2t & lowmask];
                const double hv = (__popc(s & ts[t].btw) & 1) ? -ts[t].h : ts[t].h;
                acc = hmadd<T>(acc, hv, __ldg(x + j));
            }
            row_epilogue<T>(a, sc, i, acc, xo, s0, s1, s2);
        }
    }
    if (a.mode == kModeHv) return;
    double v[4] = {s0, s1, s2, 0.0};
    if (grid_sum<4>(v, a.partials, a.counter, a.sums_out))
        if (a.mode == kModeFirst || a.mode == kModeStep) lanczos_finalize(a, ks);
}

// Gather form of the reference's scatter: every target state looks up its
// source; the map is one-to-one, so each target receives at most one term per
// operator, in operator order.
template <typename T>
__global__ void sz_apply_c_kernel(const SzDev S, const SzSectorDev tgt, int nop, SzOp o0, SzOp o1,
                                  const T *__restrict__ in, T *__restrict__ out)
{
    const int ns = S.ns;
    const uint32_t lowmask = (1u << ns) - 1u;
    for (int r = blockIdx.x; r < tgt.nrows; r += gridDim.x) {
        const uint32_t h = tgt.row_h[r];
        const int k = tgt.npart - __popc(h);
        const int c0 = S.class_start[k], len = S.class_start[k + 1] - c0;
        const int64_t base = tgt.off_h[h];
        for (int c = threadIdx.x; c < len; c += blockDim.x) {
            const uint32_t t = (uint32_t)S.low_states[c0 + c] | (h << ns);
            T acc = T(0);
            for (int q = 0; q < nop; ++q) {
                const SzOp o = q == 0 ? o0 : o1;
                if (((t & o.bit) != 0u) != (o.create != 0)) continue;
                const uint32_t s = t ^ o.bit;
                if ((s & o.pmask) != o.pwant) continue;
                // create / destroy sign: occupied orbitals above the bit, on the result
                const uint32_t above = t & ~((o.bit << 1) - 1u);
                const int sg = (__popc(above) & 1) ? -o.sgn : o.sgn;
                const T v = in[(int64_t)S.sec.off_h[s >> ns] + S.rank_low[s & lowmask]];
                if (q == 0) acc = sg > 0 ? v : -v;
                else acc = sg > 0 ? fadd(acc, v) : fsub(acc, v);
            }
            out[base + c] = acc;
        }
    }
}

size_t sz_smem(const SzDev &S)
{
    return (size_t)S.nterm * sizeof(SzTerm) + sizeof(double) * ((size_t)1 << (2 * S.nc)) +
           (size_t)S.ndiag * (sizeof(double) + sizeof(uint32_t));
}

int sz_block(int maxlen)
{
    int b = ((maxlen + 31) / 32) * 32;
    if (b > kSzBlock) b = kSzBlock;
    if (b < 32) b = 32;
    return b;
}

template <typename K>
cudaError_t launch_one(K kern, int grid, int block, size_t smem, const SzDev &S, const RowArgs &a, cudaStream_t st)
{
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<grid, block, smem, st>>>(S, a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_sz_rows(const SzDev &S, int dtype, const RowArgs &a, int num_sms, int simple, cudaStream_t st)
{
    const int block = sz_block(S.sec.maxlen);
    int per_sm = 2048 / block;
    if (per_sm > 16) per_sm = 16;
    const size_t eb = dtype == EDK_F64 ? 8 : 4;
    if (simple) {
        int grid = num_sms * per_sm;
        if (grid > S.sec.nrows) grid = S.sec.nrows;
        if (grid < 1) grid = 1;
        const size_t smem = sz_smem(S);
        return dtype == EDK_F64 ? launch_one(sz_row_simple_kernel<double>, grid, block, smem, S, a, st)
                                : launch_one(sz_row_simple_kernel<float>, grid, block, smem, S, a, st);
    }
    size_t smem = (size_t)S.nterm * (sizeof(RowTerm) + sizeof(double)) + (size_t)S.nrun * sizeof(SzRun) +
                  sizeof(double) * ((size_t)1 << (2 * S.nc)) + (size_t)S.ndiag * sizeof(double) +
                  (size_t)((S.ndiag + 3) & ~3) * sizeof(uint32_t);
    // stage the own row when it leaves room for four blocks per SM
    const size_t row_bytes = (size_t)S.sec.maxlen * eb;
    const bool stage = smem + row_bytes <= 52 * 1024;
    if (stage) smem += row_bytes;
    int by_smem = (int)((228 * 1024) / (smem + 1024));
    if (by_smem < per_sm) per_sm = by_smem;
    const int reg_cap = 4 * kSzBlock / block;   // the register budget of __launch_bounds__(256, 4)
    if (per_sm > reg_cap) per_sm = reg_cap;
    if (per_sm < 1) per_sm = 1;
    int grid = num_sms * per_sm;
    if (grid > S.sec.nrows) grid = S.sec.nrows;
    if (grid < 1) grid = 1;
    if (dtype == EDK_F64)
        return stage ? launch_one(sz_row_kernel<double, true>, grid, block, smem, S, a, st)
                     : launch_one(sz_row_kernel<double, false>, grid, block, smem, S, a, st);
    return stage ? launch_one(sz_row_kernel<float, true>, grid, block, smem, S, a, st)
                 : launch_one(sz_row_kernel<float, false>, grid, block, smem, S, a, st);
}

cudaError_t launch_sz_apply_c(int dtype, const SzDev &src, const SzSectorDev &tgt, int nop, const SzOp *ops,
                              const void *in, void *out, int num_sms, cudaStream_t st)
{
    if (nop < 1 || nop > 2) return cudaErrorInvalidValue;
    const SzOp o0 = ops[0], o1 = nop > 1 ? ops[1] : SzOp();
    const int block = sz_block(tgt.maxlen);
    int grid = num_sms * (2048 / block);
    if (grid > tgt.nrows) grid = tgt.nrows;
    if (grid < 1) grid = 1;
    if (dtype == EDK_F64)
        sz_apply_c_kernel<double><<<grid, block, 0, st>>>(src, tgt, nop, o0, o1, static_cast<const double *>(in),
                                                          static_cast<double *>(out));
    else
        sz_apply_c_kernel<float><<<grid, block, 0, st>>>(src, tgt, nop, o0, o1, static_cast<const float *>(in),
                                                         static_cast<float *>(out));
    return cudaGetLastError();
}

}  // namespace edk
