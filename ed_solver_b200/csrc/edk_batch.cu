// Batched Green-function chains: one persistent launch over a work queue.
//
// compute_greenAA (green_class_computeAA.f90:105-126) loops over sectors,
// particle/hole parts, eigenstates and orbital combinations, and runs one
// compute_dynamic chain (green_class_compute_dynamic.f90:191-334) per item.
// For the many small, uneven sectors of a finite-temperature solve those
// chains are launch-bound when each Lanczos step is its own grid.  Here every
// chain is a work item: a thread block takes the next item from an atomic
// queue (items sorted largest first) and runs all of its Lanczos steps alone,
// with block-level reductions only -- no block ever waits on another, so the
// kernel has no spin loop.  Vectors written inside the kernel are re-read with
// L2-coherent loads (ld.global.cg), never through the read-only path.
#include "edk_device.cuh"

namespace edk {

template <typename T> __device__ __forceinline__ T ldcg(const T *p) { return __ldcg(p); }

// (H x) for all rows of one sector by one block, in the reference's order of
// terms per element, fused with the Lanczos epilogue of `mode`.
// npsi > 0 (step mode): psi[j] += cpsi[j] * v_{k+1} for j < npsi, the
// accumulation of a recomputing pass 2.
template <typename T, int R>
__device__ void block_rows(const HamDev &H, int mode, const T *x, T *y, const T *vk, const T *vkm1, T *vout,
                           double delta, double gam, double gam1, double beta_k, double beta_k1, double inv_b,
                           T *xs, const double *pal_s, double &s0, double &s1, double &s2, int npsi = 0,
                           T *const *psi = nullptr, const double *cpsi = nullptr)
{
    const int64_t dup = H.dup, ddn = H.ddn;
    const uint32_t *ell = H.up.ell;
    const double *ellv = H.up.ell_val;
    const int K = H.up.ell_k;
    const double *dnv = H.dn.val;
    const double *upd = H.up.diag;
    const double *dnd = H.dn.diag;
    const double *icoef = H.int_coef;
    const double *jj = H.jj;
    const int nc = H.nc;
    for (int64_t g0 = 0; g0 < ddn; g0 += R) {
        int row[R];
#pragma unroll
        for (int r = 0; r < R; ++r) row[r] = g0 + r < ddn ? (int)(g0 + r) : -1;
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (row[r] >= 0)
                for (int64_t i = threadIdx.x; i < dup; i += blockDim.x) xs[r * dup + i] = ldcg(x + row[r] * dup + i);
        __syncthreads();
        for (int64_t c = threadIdx.x; c < dup; c += blockDim.x) {
            const int cu = H.up.imp[c];
            const double du = upd[c];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (row[r] < 0) continue;
                const T xo = xs[r * dup + c];
                const int cd = H.dn.imp[row[r]];
                const int cfg = cu * H.ncfg + cd;
                double acc = 0.0;
                for (int o = H.int_off[cfg]; o < H.int_off[cfg + 1]; ++o) acc = hmadd<T>(acc, icoef[o], xo);
                acc = hmadd<T>(acc, fadd(du, dnd[row[r]]), xo);
                for (int k = 0; k < K; ++k) {
                    const uint32_t ent = ell[(int64_t)k * dup + c];
                    const int64_t j = H.up.packed ? (int64_t)(ent & 0xFFFFFFu) : (int64_t)(int32_t)ent;
                    const double h = H.up.packed ? pal_s[ent >> 24] : ellv[(int64_t)k * dup + c];
                    acc = hmadd<T>(acc, h, xs[r * dup + j]);
                }
                for (int f = H.dn.ptr[row[r]]; f < H.dn.ptr[row[r] + 1]; ++f)
                    acc = hmadd<T>(acc, dnv[f], ldcg(x + (int64_t)H.dn.tgt[f] * dup + c));
                if (H.hund) {
                    // Hund spin flip and pair hopping (HAIMupdo.f90:1017-1129), gathers from x
                    for (int s1 = 0; s1 < nc; ++s1) {
                        const int b1u = (cu >> s1) & 1, b1d = (cd >> s1) & 1;
                        if (b1u + b1d != 1) continue;
                        for (int s2 = s1 + 1; s2 < nc; ++s2) {
                            if (!H.umask[s1 * nc + s2]) continue;
                            const int b2u = (cu >> s2) & 1, b2d = (cd >> s2) & 1;
                            if (b2u + b2d != 1) continue;
                            int mu = -1, md = -1;
                            if (b1u && b2d) { mu = s1 * (nc - 1) + (s2 < s1 ? s2 : s2 - 1); md = s2 * (nc - 1) + (s1 < s2 ? s1 : s1 - 1); }
                            else if (b1d && b2u) { mu = s2 * (nc - 1) + (s1 < s2 ? s1 : s1 - 1); md = s1 * (nc - 1) + (s2 < s1 ? s2 : s2 - 1); }
                            if (mu < 0) continue;
                            const int32_t pu = H.up.move[c * H.nmove + mu], pd = H.dn.move[(int64_t)row[r] * H.nmove + md];
                            if (pu == 0 || pd == 0) continue;
                            const int64_t ju = (pu > 0 ? pu : -pu) - 1, jdn = (pd > 0 ? pd : -pd) - 1;
                            const double t = fmul((double)ldcg(x + ju + jdn * dup), jj[s1 * nc + s2]);
                            acc = ((pu > 0) == (pd > 0)) ? fadd(acc, t) : fsub(acc, t);
                        }
                    }
                    for (int s1 = 0; s1 < nc; ++s1) {
                        if (!(((cu >> s1) & 1) && ((cd >> s1) & 1))) continue;
                        for (int s2 = 0; s2 < nc; ++s2) {
                            if (s2 == s1 || !H.umask[s1 * nc + s2]) continue;
                            if (((cu >> s2) & 1) || ((cd >> s2) & 1)) continue;
                            const int mi = s1 * (nc - 1) + (s2 < s1 ? s2 : s2 - 1);
                            const int32_t pu = H.up.move[c * H.nmove + mi], pd = H.dn.move[(int64_t)row[r] * H.nmove + mi];
                            if (pu == 0 || pd == 0) continue;
                            const int64_t ju = (pu > 0 ? pu : -pu) - 1, jdn = (pd > 0 ? pd : -pd) - 1;
                            const double t = fmul((double)ldcg(x + ju + jdn * dup), jj[s1 * nc + s2]);
                            acc = ((pu > 0) == (pd > 0)) ? fadd(acc, t) : fsub(acc, t);
                        }
                    }
                }
                const int64_t i = (int64_t)row[r] * dup + c;
                if (mode == kModeFirst) {
                    const double v = (double)xo;
                    const T st = (T)((double)acc - gam1 * v);
                    y[i] = st;
                    const double sd = (double)st;
                    s0 += sd * sd; s1 += sd * v; s2 += v * v;
                } else {
                    const double sv = (double)xo, vkk = (double)ldcg(vk + i);
                    const double vm = vkm1 ? (double)ldcg(vkm1 + i) : 0.0;
                    const T vt = (T)((sv - delta * vkk) * inv_b);
                    const double hv1 = ((double)acc - delta * (sv + gam * vkk + beta_k * vm)) * inv_b;
                    const double w = hv1 - beta_k1 * vkk;
                    const T wt = (T)(w - gam1 * (double)vt);
                    y[i] = wt;
                    vout[i] = vt;
                    for (int j = 0; j < npsi; ++j) psi[j][i] = (T)((double)psi[j][i] + cpsi[j] * (double)vt);
                    const double wd = (double)wt, vd = (double)vt;
                    s0 += wd * wd; s1 += wd * vd; s2 += vd * vd;
                }
            }
        }
    }
}

template <int NQ>
__device__ __forceinline__ void block_allreduce(double (&v)[NQ], double (*red)[32], double *out)
{
    block_sum<NQ>(v, red);
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < NQ; ++q) out[q] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = out[q];
    __syncthreads();
}

template <typename T, int R>
__global__ void __launch_bounds__(512, 1) batch_kernel(const HamDev *hams, const BatchItem *items, int nitems,
                                                    int *queue, T *work, int64_t maxdim, double cutoff)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *xs = reinterpret_cast<T *>(smem_raw);
    __shared__ double pal_s[256];
    __shared__ double red[3][32];
    __shared__ double bc[4];
    __shared__ int item_id;
    T *vA = work + (size_t)blockIdx.x * 4 * maxdim;
    T *vB = vA + maxdim, *sA = vB + maxdim, *sB = sA + maxdim;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) item_id = atomicAdd(queue, 1);
        __syncthreads();
        const int it = item_id;
        if (it >= nitems) return;
        const BatchItem &b = items[it];
        const HamDev &H = hams[b.ham];
        const T *start = static_cast<const T *>(b.start);
        if (H.up.packed)
            for (int i = threadIdx.x; i < H.up.npal; i += blockDim.x) pal_s[i] = H.up.pal[i];
        // |start|^2 and v1 = start / |start|
        double nv[3] = {0.0, 0.0, 0.0};
        for (int64_t i = threadIdx.x; i < b.dim; i += blockDim.x) {
            const double t = (double)start[i];
            nv[0] += t * t;
        }
        block_allreduce<3>(nv, red, bc);
        const double nrm = sqrt(nv[0]);
        if (!(nv[0] >= b.cutoff_dynamic) || !(nrm >= cutoff)) {
            if (threadIdx.x == 0) *b.done = 0;
            continue;
        }
        const double inv = 1.0 / nrm;
        for (int64_t i = threadIdx.x; i < b.dim; i += blockDim.x) vB[i] = (T)((double)start[i] * inv);
        if (threadIdx.x == 0) b.beta[0] = nrm;
        __syncthreads();
        T *vk = vB, *vkm1 = vA, *s = sA, *sn = sB;
        double alpha_prev = 0.0, gam_prev = b.gamma1, beta_prev = 0.0;
        int n = 0;
        for (int k = 0; k < b.niter; ++k) {
            double acc[3] = {0.0, 0.0, 0.0};
            double gam1;
            if (k == 0) {
                gam1 = b.gamma1;
                block_rows<T, R>(H, kModeFirst, vk, s, nullptr, nullptr, nullptr, 0, 0, gam1, 0, 0, 0, xs, pal_s,
                                 acc[0], acc[1], acc[2]);
            } else {
                const double beta_k1 = b.beta[k];
                if (!(beta_k1 >= cutoff)) break;
                const double delta = alpha_prev - gam_prev;
                gam1 = alpha_prev;
                block_rows<T, R>(H, kModeStep, s, sn, vk, k >= 2 ? vkm1 : nullptr, vkm1, delta, gam_prev, gam1,
                                 beta_prev, beta_k1, 1.0 / beta_k1, xs, pal_s, acc[0], acc[1], acc[2]);
                T *t1 = vk; vk = vkm1; vkm1 = t1;        // v_{k+1} was written over v_{k-1}
                T *t2 = s; s = sn; sn = t2;
            }
            __threadfence_block();
            block_allreduce<3>(acc, red, bc);
            // coefficients of this iteration (same formulas as lanczos_finalize)
            const double g = gam1;
            const double al = acc[1] + g * acc[2];
            const double de = al - g;
            const double b2 = acc[0] - 2.0 * de * acc[1] + de * de * acc[2];
            const double ww = acc[0] + 2.0 * g * acc[1] + g * g * acc[2];
            double be = (b2 > 0.0 && b2 > 1e-28 * ww && isfinite(b2)) ? sqrt(b2) : 0.0;
            if (threadIdx.x == 0) {
                b.alpha[k] = isfinite(al) ? al : 0.0;
                b.beta[k + 1] = be;
            }
            if (k >= 1) beta_prev = b.beta[k];
            gam_prev = (k == 0) ? b.gamma1 : alpha_prev;
            alpha_prev = al;
            n = k + 1;
            __syncthreads();
        }
        if (threadIdx.x == 0) *b.done = n;
    }
}

// ---------------------------------------------------------------------------
// Ground states of many small sectors (the sector scan of get_eigen_energies,
// solver.h:128-232): pass 1 of Lanczos_fast_diagonalize
// (Lanczos_plain.f90:33-154) for every sector in one persistent launch, one
// block per sector, with the convergence test of the per-sector driver run on
// the device; then pass 2 (Lanczos_get_GS_sector, Lanczos_plain.f90:156-229)
// for the kept states of every sector in a second launch.  The start vector
// is the library's table start (ran_tab, create_fix_initial_vector).
// ---------------------------------------------------------------------------

// number of eigenvalues below x of the tridiagonal with diagonal d[0..n) and
// squared couplings e2[0..n-1) (e2[i] couples i and i+1): the LDL^T count of
// the host solver (edk_tridiag.cpp)
__device__ int sturm_count_dev(int n, const double *d, const double *e2, double x, double pivmin)
{
    int cnt = 0;
    double q = d[0] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    if (q < 0) ++cnt;
    for (int i = 1; i < n; ++i) {
        q = d[i] - x - e2[i - 1] / q;
        if (fabs(q) < pivmin) q = -pivmin;
        if (q < 0) ++cnt;
    }
    return cnt;
}

// Lowest m eigenvalues of that tridiagonal into w (shared memory), by every
// thread of the block: multisection with blockDim.x points per round, down
// to the stopping width of the host's bisection.  sh: 4 doubles, ish: 1 int
// of shared scratch.
__device__ void block_tridiag_lowest(int n, const double *d, const double *e2, int m, double *w, double *sh, int *ish)
{
    const double eps = 2.220446049250313e-16, dmin = 2.2250738585072014e-308;
    if (threadIdx.x == 0) {
        double lo = d[0], hi = d[0], emax2 = 0.0;
        for (int i = 0; i < n; ++i) {
            const double r = (i > 0 ? sqrt(e2[i - 1]) : 0.0) + (i < n - 1 ? sqrt(e2[i]) : 0.0);
            lo = fmin(lo, d[i] - r);
            hi = fmax(hi, d[i] + r);
            if (i < n - 1) emax2 = fmax(emax2, e2[i]);
        }
        const double scale = fmax(fabs(lo), fabs(hi));
        const double pivmin = fmax(dmin, dmin * emax2) * 4.0;
        sh[0] = lo - (2.0 * eps * scale + pivmin);
        sh[1] = hi + 2.0 * eps * scale + pivmin;
        sh[2] = pivmin;
        sh[3] = scale;
    }
    __syncthreads();
    const double lo = sh[0], hi = sh[1], pivmin = sh[2], scale = sh[3];
    const int NT = blockDim.x;
    for (int k = 0; k < m; ++k) {
        double a = k > 0 ? w[k - 1] - 2.0 * eps * scale : lo, b = hi;
        if (a < lo) a = lo;
        for (int round = 0; round < 24; ++round) {
            if (b - a <= 2.0 * eps * fmax(fabs(a), fabs(b)) + pivmin) break;
            const double x = a + (b - a) * (double)(threadIdx.x + 1) / (double)(NT + 1);
            const bool above = sturm_count_dev(n, d, e2, x, pivmin) > k;
            if (threadIdx.x == 0) *ish = NT;
            __syncthreads();
            if (above) atomicMin(ish, (int)threadIdx.x);
            __syncthreads();
            const int f = *ish;
            __syncthreads();
            const double na = f > 0 ? a + (b - a) * (double)f / (double)(NT + 1) : a;
            const double nb = f < NT ? a + (b - a) * (double)(f + 1) / (double)(NT + 1) : b;
            if (!(na > a || nb < b)) break;   // the points collapsed onto the ends
            a = na;
            b = nb;
        }
        if (threadIdx.x == 0) w[k] = 0.5 * (a + b);
        __syncthreads();
    }
}

template <typename T, int R>
__global__ void __launch_bounds__(512, 1) gs_batch_kernel(const HamDev *hams, const GsItem *items, int nitems,
                                                       int *queue, T *work, int64_t maxdim, int maxdup, int nmax,
                                                       const double *tab, double cutoff, int every, int pass)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *xs = reinterpret_cast<T *>(smem_raw);
    double *td = reinterpret_cast<double *>(smem_raw + (((size_t)R * maxdup * sizeof(T) + 15) & ~(size_t)15));
    double *te2 = td + nmax;             // squared couplings
    __shared__ double pal_s[256];
    __shared__ double red[3][32];
    __shared__ double bc[4];
    __shared__ double wnow[kGsMaxNe], wprev[kGsMaxNe], sh[4];
    __shared__ int ish, item_id, stop;
    T *vA = work + (size_t)blockIdx.x * 4 * maxdim;
    T *V[2] = {vA, vA + maxdim};
    T *S[2] = {vA + 2 * maxdim, vA + 3 * maxdim};
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) item_id = atomicAdd(queue, 1);
        __syncthreads();
        const int it = item_id;
        if (it >= nitems) return;
        const GsItem &b = items[it];
        const HamDev &H = hams[b.ham];
        const int64_t dim = b.dim;
        if (H.up.packed)
            for (int i = threadIdx.x; i < H.up.npal; i += blockDim.x) pal_s[i] = H.up.pal[i];
        // start vector (start_kernel + scale_kernel): v1 = table start / |table start|
        double nv[3] = {0.0, 0.0, 0.0};
        for (int64_t i = threadIdx.x; i < dim; i += blockDim.x) {
            const T t = (T)tab[(i % 10000) + 1];
            nv[0] += (double)t * (double)t;
        }
        block_allreduce<3>(nv, red, bc);
        const double nrm = sqrt(nv[0]);
        if (!(nrm >= cutoff)) {
            if (threadIdx.x == 0) { b.result[0] = 0; b.result[1] = 2; }
            continue;
        }
        const double inv = 1.0 / nrm;
        const int npsi = pass == 2 ? b.ne : 0;
        T *psi[kGsMaxNe];
        double cps[kGsMaxNe];
        for (int j = 0; j < kGsMaxNe; ++j) psi[j] = j < npsi ? static_cast<T *>(b.psi[j]) : nullptr;
        for (int64_t i = threadIdx.x; i < dim; i += blockDim.x) {
            const T t = (T)((double)(T)tab[(i % 10000) + 1] * inv);
            V[0][i] = t;
            for (int j = 0; j < npsi; ++j) psi[j][i] = (T)(b.coef[(size_t)j * b.niter_max] * (double)t);
        }
        if (pass == 1 && threadIdx.x == 0) b.beta[0] = nrm;
        if (threadIdx.x == 0) stop = 0;
        __syncthreads();
        // pass 1: up to niter_max steps; pass 2: niter_max = the steps pass 1 took
        double alpha_prev = 0.0, gam_prev = 0.0, beta_prev = 0.0;
        int n = 0;
        for (int k = 0; k < b.niter_max; ++k) {
            double acc[3] = {0.0, 0.0, 0.0};
            double gam1;
            if (k == 0) {
                gam1 = 0.0;
                block_rows<T, R>(H, kModeFirst, V[0], S[0], nullptr, nullptr, nullptr, 0, 0, gam1, 0, 0, 0, xs,
                                 pal_s, acc[0], acc[1], acc[2]);
            } else {
                const double beta_k1 = b.beta[k];
                const double delta = alpha_prev - gam_prev;
                gam1 = alpha_prev;
                for (int j = 0; j < npsi; ++j) cps[j] = b.coef[(size_t)j * b.niter_max + k];
                block_rows<T, R>(H, kModeStep, S[(k - 1) & 1], S[k & 1], V[(k - 1) & 1], k >= 2 ? V[k & 1] : nullptr,
                                 V[k & 1], delta, gam_prev, gam1, beta_prev, beta_k1, 1.0 / beta_k1, xs, pal_s, acc[0],
                                 acc[1], acc[2], npsi, psi, cps);
            }
            __threadfence_block();
            block_allreduce<3>(acc, red, bc);
            const double g = gam1;
            const double al = acc[1] + g * acc[2];
            const double de = al - g;
            const double b2 = acc[0] - 2.0 * de * acc[1] + de * de * acc[2];
            const double ww = acc[0] + 2.0 * g * acc[1] + g * g * acc[2];
            const double be = (b2 > 0.0 && b2 > 1e-28 * ww && isfinite(b2)) ? sqrt(b2) : 0.0;
            if (pass == 1 && threadIdx.x == 0) {
                b.alpha[k] = isfinite(al) ? al : 0.0;
                b.beta[k + 1] = be;
            }
            if (k >= 1) beta_prev = b.beta[k];
            gam_prev = (k == 0) ? 0.0 : alpha_prev;
            alpha_prev = pass == 1 ? al : b.alpha[k];
            n = k + 1;
            __syncthreads();
            if (pass == 2) continue;
            // convergence (the per-sector driver's test, at every `every`-th
            // step): the lowest min(ne, n) eigenvalues of T_n against those of
            // T_{n-1}; breakdown ends the sector at once
            const bool broke = !(b.beta[n] >= cutoff);
            if (broke || n == b.niter_max || (n % every == 0 && n > 2 && n > b.ne)) {
                bool all = false;
                if (!broke && n < b.niter_max) {
                    for (int i = threadIdx.x; i < n; i += blockDim.x) {
                        td[i] = b.alpha[i];
                        te2[i] = b.beta[i + 1] * b.beta[i + 1];
                    }
                    __syncthreads();
                    const int m = b.ne < n ? b.ne : n;
                    block_tridiag_lowest(n, td, te2, m, wnow, sh, &ish);
                    block_tridiag_lowest(n - 1, td, te2, m < n - 1 ? m : n - 1, wprev, sh, &ish);
                    all = m == b.ne;
                    for (int j = 0; j < m; ++j)
                        if (!(fabs(wnow[j] - wprev[j]) < b.tolerance)) all = false;
                }
                if (threadIdx.x == 0 && (all || broke || n == b.niter_max)) {
                    stop = 1;
                    b.result[0] = n;
                    b.result[1] = (broke && !all && n < b.niter_max) ? 1 : 0;
                }
                __syncthreads();
                if (stop) break;
            }
        }
        if (pass == 2) {
            // normalise each state
            for (int j = 0; j < npsi; ++j) {
                double q[3] = {0.0, 0.0, 0.0};
                for (int64_t i = threadIdx.x; i < dim; i += blockDim.x) q[0] += (double)psi[j][i] * (double)psi[j][i];
                block_allreduce<3>(q, red, bc);
                const double pinv = 1.0 / sqrt(q[0]);
                for (int64_t i = threadIdx.x; i < dim; i += blockDim.x) psi[j][i] = (T)((double)psi[j][i] * pinv);
                __syncthreads();
            }
        } else if (threadIdx.x == 0 && !stop) {
            b.result[0] = n;
            b.result[1] = 0;
        }
    }
}

template <typename T, int R>
static cudaError_t launch_gs_batch_t(const HamDev *hams, const GsItem *items, int nitems, int *queue, void *work,
                                     int64_t maxdim, int64_t maxdup, int nmax, const double *tab, double cutoff,
                                     int every, int pass, int grid, cudaStream_t st)
{
    auto k = gs_batch_kernel<T, R>;
    const size_t smem = (((size_t)R * maxdup * sizeof(T) + 15) & ~(size_t)15) + (size_t)2 * nmax * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, 512, smem, st>>>(hams, items, nitems, queue, static_cast<T *>(work), maxdim, (int)maxdup, nmax, tab,
                               cutoff, every, pass);
    return cudaGetLastError();
}

cudaError_t launch_gs_batch(int R, const HamDev *hams, const GsItem *items, int nitems, int *queue, void *work,
                            int64_t maxdim, int64_t maxdup, int nmax, const double *tab, double cutoff, int every,
                            int pass, int grid, cudaStream_t st)
{
    if (R == 2)
        return launch_gs_batch_t<double, 2>(hams, items, nitems, queue, work, maxdim, maxdup, nmax, tab, cutoff, every,
                                            pass, grid, st);
    return launch_gs_batch_t<double, 1>(hams, items, nitems, queue, work, maxdim, maxdup, nmax, tab, cutoff, every,
                                        pass, grid, st);
}

// ---------------------------------------------------------------------------

template <typename T, int R>
static cudaError_t launch_batch_t(const HamDev *hams, const BatchItem *items, int nitems, int *queue, void *work,
                                  int64_t maxdim, int64_t maxdup, double cutoff, int grid, int block, cudaStream_t st)
{
    auto k = batch_kernel<T, R>;
    const size_t smem = (size_t)R * maxdup * sizeof(T);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(smem ? smem : 16));
    if (e != cudaSuccess) return e;
    k<<<grid, block, smem, st>>>(hams, items, nitems, queue, static_cast<T *>(work), maxdim, cutoff);
    return cudaGetLastError();
}

cudaError_t launch_batch(int dtype, int R, const HamDev *hams, const BatchItem *items, int nitems, int *queue,
                         void *work, int64_t maxdim, int64_t maxdup, double cutoff, int grid, int block,
                         cudaStream_t st)
{
    if (dtype == EDK_F64) {
        if (R == 4) return launch_batch_t<double, 4>(hams, items, nitems, queue, work, maxdim, maxdup, cutoff, grid, block, st);
        if (R == 2) return launch_batch_t<double, 2>(hams, items, nitems, queue, work, maxdim, maxdup, cutoff, grid, block, st);
        return launch_batch_t<double, 1>(hams, items, nitems, queue, work, maxdim, maxdup, cutoff, grid, block, st);
    }
    if (R == 4) return launch_batch_t<float, 4>(hams, items, nitems, queue, work, maxdim, maxdup, cutoff, grid, block, st);
    if (R == 2) return launch_batch_t<float, 2>(hams, items, nitems, queue, work, maxdim, maxdup, cutoff, grid, block, st);
    return launch_batch_t<float, 1>(hams, items, nitems, queue, work, maxdim, maxdup, cutoff, grid, block, st);
}

int batch_max_blocks_per_sm(int dtype, int R, int block, int64_t maxdup)
{
    int n = 0;
    const size_t smem = (size_t)R * maxdup * (dtype == EDK_F64 ? 8 : 4);
    cudaError_t e;
    if (dtype == EDK_F64)
        e = R == 4 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<double, 4>, block, smem)
          : R == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<double, 2>, block, smem)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<double, 1>, block, smem);
    else
        e = R == 4 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<float, 4>, block, smem)
          : R == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<float, 2>, block, smem)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<float, 1>, block, smem);
    return e == cudaSuccess ? n : 0;
}

}  // namespace edk
