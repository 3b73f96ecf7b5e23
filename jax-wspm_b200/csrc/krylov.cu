// SELL-32 SpMV and fused Krylov kernels.
//
// Algorithms (restated from the published methods, with the stopping rules of
// jax.scipy.sparse.linalg, which the reference calls at
// src/solvers/jax_linear_solver.py:349-397):
//   CG        preconditioned Hestenes-Stiefel; stop when r.r <= max(tol^2 b.b, atol^2)
//             (gamma = r.z instead of r.r when unpreconditioned) or k == maxiter.
//   BiCGSTAB  van der Vorst (1992), right preconditioned, r_hat = r0,
//             rho0 = alpha0 = omega0 = 1, p0 = q0 = r0; early exit on s.s < atol2;
//             breakdown exit when rho, alpha or omega is exactly zero.
//   GMRES(m)  Saad-Schultz, left preconditioned, classical Gram-Schmidt with one
//             re-orthogonalisation pass; maxiter counts restart cycles; the test is
//             ||M(b - A x)|| <= ||M b|| min(1, max(tol ||b||, atol) / ||b||).
//
// Kernel structure.  Every iteration is a short sequence of grid-wide kernels;
// kernels that need a global scalar read it from KrylovState, kernels that
// produce one reduce deterministically (common.cuh).  The kernel that tests
// convergence sets a CUDA-graph conditional handle, so a WHILE node can run
// the loop entirely on the device; every kernel returns immediately once
// `done` is set, so iteration bodies may be unrolled.
//
// CG fuses the p-update into the SpMV: q = A (z + beta p_old) gathers z and
// p_old at the neighbours and writes p_new for its own rows (p ping-pongs
// between two buffers), so one CG iteration is two kernels:
//   K1: p_new = z + beta p_old ; q = A p_new ; pq = p_new.q  -> alpha
//   K2: x += alpha p ; r -= alpha q ; z = M r ; r.z, r.r    -> beta, test
#include <float.h>
#include "krylov.cuh"

namespace wspm {

__device__ __forceinline__ void set_cond(cudaGraphConditionalHandle h, int use, unsigned v) {
    if (use) cudaGraphSetConditional(h, v);
}

template <typename T, int MW, typename XF>
__device__ __forceinline__ T sell_row(const Sell &A, const T *__restrict__ vals, int i, XF xf) {
    return sell_row_dot<T, MW>(A, vals, i, xf);
}

// ---------------------------------------------------------------- SpMV
template <typename T, int MW>
__global__ void __launch_bounds__(kBlock) spmv_kernel(Sell A, const T *__restrict__ vals, const T *__restrict__ x,
                                                      T *__restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n_rows) return;
    y[i] = sell_row<T, MW>(A, vals, i, [&](int c) { return __ldg(x + c); });
}

void spmv_f64(const Sell &A, const double *vals, const double *x, double *y, cudaStream_t st) {
    WSPM_WIDTH_DISPATCH(A.max_width,
                        spmv_kernel<double, MW><<<(A.n_rows + kBlock - 1) / kBlock, kBlock, 0, st>>>(A, vals, x, y));
}
void spmv_f32(const Sell &A, const float *vals, const float *x, float *y, cudaStream_t st) {
    WSPM_WIDTH_DISPATCH(A.max_width,
                        spmv_kernel<float, MW><<<(A.n_rows + kBlock - 1) / kBlock, kBlock, 0, st>>>(A, vals, x, y));
}

// ---------------------------------------------------------------- CG
template <typename T, int MW>
__global__ void __launch_bounds__(kBlock) cg_init_kernel(Sell A, const T *__restrict__ vals, const T *__restrict__ b,
                                                         const double *__restrict__ b64, const T *x0, T *x,
                                                         const T *__restrict__ dinv, T *r, T *z, T *p0,
                                                         T *partials, KrylovState *st, double tol, double atol,
                                                         int maxiter, int zero_x0, const double *tol_dev,
                                                         cudaGraphConditionalHandle cond, int use_cond) {
    T v[3] = {T(0), T(0), T(0)};
    const int n = A.n_rows;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const T bi = b64 ? (T)b64[i] : b[i];
        T ri;
        if (zero_x0) {
            x[i] = T(0);
            ri = bi;
        } else {
            const T ax = sell_row<T, MW>(A, vals, i, [&](int c) { return x0[c]; });
            ri = bi - ax;
        }
        const T zi = dinv ? dinv[i] * ri : ri;
        r[i] = ri;
        z[i] = zi;
        p0[i] = T(0);
        v[0] += ri * zi;
        v[1] += ri * ri;
        v[2] += bi * bi;
    }
    if (publish_partials<T, 3>(v, partials, &st->ticket[2])) {
        T tot[3];
        final_sum<T, 3>(partials, tot, &st->ticket[2]);
        if (threadIdx.x == 0) {
            const double gamma = tot[0], rr = tot[1], bs = tot[2];
            st->gamma = gamma; st->rr = rr; st->bs = bs;
            const double tl = tol_dev ? *tol_dev : tol;
            st->atol2 = fmax(tl * tl * bs, atol * atol);
            st->beta = 0.0; st->alpha = 0.0;
            st->k = 0; st->status = WSPM_OK;
            const double rs = dinv ? rr : gamma;
            int done = !(rs > st->atol2 && 0 < maxiter);
            if (!isfinite(rs)) { st->status = WSPM_NAN; done = 1; }
            st->done = done;
            set_cond(cond, use_cond, done ? 0u : 1u);
        }
    }
}

// Copy x0 into x when they are different buffers (separate from the init
// kernel so that the init SpMV never reads a partially written x).
template <typename T>
__global__ void copy_kernel(const T *__restrict__ src, T *__restrict__ dst, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i];
}

void copy_kernel_d(const double *src, double *dst, int n, cudaStream_t st) {
    copy_kernel<double><<<reduction_blocks(n), kBlock, 0, st>>>(src, dst, n);
}

template <typename T, int MW>
__global__ void __launch_bounds__(kBlock) cg_k1_kernel(Sell A, const T *__restrict__ vals, const T *__restrict__ z,
                                                       const T *__restrict__ p_old, T *__restrict__ p_new,
                                                       T *__restrict__ q, T *partials, KrylovState *st) {
    if (st->done) return;
    const T beta = (T)st->beta;
    T v[1] = {T(0)};
    const int n = A.n_rows;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const T qi = sell_row<T, MW>(A, vals, i, [&](int c) { return fma(beta, __ldg(p_old + c), __ldg(z + c)); });
        const T pi = fma(beta, p_old[i], z[i]);
        p_new[i] = pi;
        q[i] = qi;
        v[0] += pi * qi;
    }
    if (publish_partials<T, 1>(v, partials, &st->ticket[0])) {
        T tot[1];
        final_sum<T, 1>(partials, tot, &st->ticket[0]);
        if (threadIdx.x == 0) {
            st->pq = tot[0];
            st->alpha = (double)((T)st->gamma / tot[0]);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kBlock) cg_k2_kernel(int n, T *__restrict__ x, T *__restrict__ r, T *__restrict__ z,
                                                       const T *__restrict__ dinv, const T *__restrict__ p,
                                                       const T *__restrict__ q, T *partials, KrylovState *st,
                                                       int maxiter, cudaGraphConditionalHandle cond, int use_cond) {
    if (st->done) return;
    const T alpha = (T)st->alpha;
    T v[2] = {T(0), T(0)};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = fma(alpha, p[i], x[i]);
        const T ri = fma(-alpha, q[i], r[i]);
        r[i] = ri;
        const T zi = dinv ? dinv[i] * ri : ri;
        z[i] = zi;
        v[0] += ri * zi;
        v[1] += ri * ri;
    }
    if (publish_partials<T, 2>(v, partials, &st->ticket[1])) {
        T tot[2];
        final_sum<T, 2>(partials, tot, &st->ticket[1]);
        if (threadIdx.x == 0) {
            const T gamma_new = tot[0];
            st->beta = (double)(gamma_new / (T)st->gamma);
            st->gamma = (double)gamma_new;
            st->rr = (double)tot[1];
            st->k += 1;
            const double rs = dinv ? st->rr : st->gamma;
            int done = 0;
            if (!(rs > st->atol2)) done = 1;
            else if (st->k >= maxiter) { done = 1; st->status = WSPM_MAXITER; }
            if (!isfinite(rs) || !isfinite(st->alpha)) { done = 1; st->status = WSPM_NAN; }
            st->done = done;
            set_cond(cond, use_cond, done ? 0u : 1u);
        }
    }
}

template <typename T>
void cg_enqueue_init(const Sell &A, const T *vals, const T *b, const double *b64, const T *x0, T *x,
                     const T *dinv, const CgBuffers<T> &w, double tol, double atol, int maxiter, bool zero_x0,
                     cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st, const double *tol_dev) {
    const int nb = reduction_blocks(A.n_rows);
    if (!zero_x0 && x != x0) copy_kernel<T><<<nb, kBlock, 0, st>>>(x0, x, A.n_rows);
    WSPM_WIDTH_DISPATCH(A.max_width,
                        cg_init_kernel<T, MW><<<nb, kBlock, 0, st>>>(A, vals, b, b64, zero_x0 ? x : x0, x, dinv, w.r,
                                                                     w.z, w.p0, w.partials, w.st, tol, atol, maxiter,
                                                                     zero_x0 ? 1 : 0, tol_dev, cond, use_cond));
}

template <typename T>
void cg_enqueue_body(const Sell &A, const T *vals, T *x, const T *dinv, const CgBuffers<T> &w, int maxiter,
                     cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st) {
    const int nb = reduction_blocks(A.n_rows);
    WSPM_WIDTH_DISPATCH(A.max_width,
                        cg_k1_kernel<T, MW><<<nb, kBlock, 0, st>>>(A, vals, w.z, w.p0, w.p1, w.q, w.partials, w.st));
    cg_k2_kernel<T><<<nb, kBlock, 0, st>>>(A.n_rows, x, w.r, w.z, dinv, w.p1, w.q, w.partials, w.st, maxiter,
                                           cond, use_cond);
    WSPM_WIDTH_DISPATCH(A.max_width,
                        cg_k1_kernel<T, MW><<<nb, kBlock, 0, st>>>(A, vals, w.z, w.p1, w.p0, w.q, w.partials, w.st));
    cg_k2_kernel<T><<<nb, kBlock, 0, st>>>(A.n_rows, x, w.r, w.z, dinv, w.p0, w.q, w.partials, w.st, maxiter,
                                           cond, use_cond);
}

template void cg_enqueue_init<double>(const Sell &, const double *, const double *, const double *,
                                      const double *, double *, const double *, const CgBuffers<double> &, double,
                                      double, int, bool, cudaGraphConditionalHandle, int, cudaStream_t,
                                      const double *);
template void cg_enqueue_init<float>(const Sell &, const float *, const float *, const double *, const float *,
                                     float *, const float *, const CgBuffers<float> &, double, double, int, bool,
                                     cudaGraphConditionalHandle, int, cudaStream_t, const double *);
template void cg_enqueue_body<double>(const Sell &, const double *, double *, const double *,
                                      const CgBuffers<double> &, int, cudaGraphConditionalHandle, int, cudaStream_t);
template void cg_enqueue_body<float>(const Sell &, const float *, float *, const float *, const CgBuffers<float> &,
                                     int, cudaGraphConditionalHandle, int, cudaStream_t);

// ---------------------------------------------------------------- persistent CG
// One cooperative launch runs the whole (preconditioned) CG solve.  Block b owns
// a contiguous range of rows; each iteration is two phases separated by grid
// barriers:
//   phase 1: p_new = z + beta p_old ; q = A p_new (gathers z, p_old) ; partial p.q
//   phase 2: x += alpha p ; r -= alpha q ; z = M r ; partials r.z, r.r
// After a barrier every block sums all blocks' partials in the same fixed order,
// so every block holds bitwise identical alpha/beta and takes the same
// convergence decision (no broadcast, no atomics on the scalars).  Vectors that
// other blocks write during the kernel are gathered with ld.global.cg (L2) so
// that no stale L1 line is ever read.  Barrier waits are bounded: on timeout the
// block records an error and every block leaves the loop at its next check.
struct GridBarrier {
    unsigned int count;
    unsigned int gen;
    int error;
    int pad;
};

constexpr long long kBarrierSpinLimit = 20000000LL;   // ~ seconds; a legitimate wait is microseconds

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Returns false when the barrier failed (timeout anywhere in the grid).
__device__ __forceinline__ bool grid_barrier(GridBarrier *gb, unsigned int nblocks, unsigned int &gen_local) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int g = gen_local;
        __threadfence();
        const unsigned int arrived = atomicAdd(&gb->count, 1u);
        if (arrived == nblocks - 1) {
            gb->count = 0u;
            __threadfence();
            atomicExch(&gb->gen, g + 1u);
        } else {
            long long spins = 0;
            while (ld_acquire_u32(&gb->gen) == g) {
                if (++spins > kBarrierSpinLimit) {
                    atomicExch(&gb->error, 1);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        gen_local = g + 1u;
        ok = (*(volatile int *)&gb->error) == 0;
    }
    __syncthreads();
    return ok != 0;
}

// Fixed-order sum of nb partials (layout [NV][nb]) by the whole block; result broadcast to all threads.
template <typename T, int NV>
__device__ __forceinline__ void block_reduce_partials(const T *partials, int nb, T (&out)[NV]) {
    __shared__ T bc[NV];
    T acc[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        T a = T(0);
        for (int b = threadIdx.x; b < nb; b += blockDim.x) a += __ldcg(partials + (int64_t)j * nb + b);
        acc[j] = a;
    }
    block_sum<T, NV>(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) bc[j] = acc[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NV; ++j) out[j] = bc[j];
    __syncthreads();
}

template <typename T>
struct PcgArgs {
    Sell A;
    const T *vals;
    const T *b;            // right-hand side (or NULL with b64)
    const double *b64;     // FP64 right-hand side converted on the fly (refinement loop)
    T *x;                  // x0 on entry unless zero_x0, solution on exit
    const T *dinv;         // Jacobi 1/diag, NULL = none
    T *r, *z, *p0, *p1, *q;
    T *part;               // [2 phases][4][gridDim]
    KrylovState *st;
    GridBarrier *bar;
    double tol, atol;
    const double *tol_dev; // when set, the relative tolerance is read here
    int maxiter, zero_x0;
};

// One large block per SM (fewer barrier arrivals and partials): 1024 threads in
// FP32 (64 registers), 768 in FP64 (up to 85 registers), no spills.
template <typename T>
constexpr int pcg_block() { return sizeof(T) == 4 ? 1024 : 768; }

template <typename T, int MW>
__global__ void __launch_bounds__(pcg_block<T>(), 1) cg_persistent_kernel(PcgArgs<T> a) {
    const int n = a.A.n_rows;
    const int nb = gridDim.x;
    const int chunk = (((n + nb - 1) / nb) + kSlice - 1) & ~(kSlice - 1);
    const int r0 = blockIdx.x * chunk;
    const int r1 = min(n, r0 + chunk);
    // barrier generation at entry (the barrier words persist across solves; count is 0 between kernels)
    unsigned int gen = threadIdx.x == 0 ? ld_acquire_u32(&a.bar->gen) : 0u;
    T *P1 = a.part;                       // phase-1 partials [4][nb]
    T *P2 = a.part + 4 * (int64_t)nb;     // phase-2 partials [4][nb]
    const T *dinv = a.dinv;
    // ---- init: r = b - A x0, z = M r, p0 = 0
    {
        T v[3] = {T(0), T(0), T(0)};
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
            const T bi = a.b64 ? (T)a.b64[i] : a.b[i];
            T ri;
            if (a.zero_x0) {
                a.x[i] = T(0);
                ri = bi;
            } else {
                const T *x = a.x;
                ri = bi - sell_row_dot<T, MW>(a.A, a.vals, i, [&](int c) { return x[c]; });
            }
            const T zi = dinv ? dinv[i] * ri : ri;
            a.r[i] = ri;
            a.z[i] = zi;
            a.p0[i] = T(0);
            v[0] += ri * zi;
            v[1] += ri * ri;
            v[2] += bi * bi;
        }
        block_sum<T, 3>(v);
        if (threadIdx.x == 0) {
            P1[blockIdx.x] = v[0];
            P1[nb + blockIdx.x] = v[1];
            P1[2 * nb + blockIdx.x] = v[2];
        }
    }
    bool ok = grid_barrier(a.bar, nb, gen);
    T tot3[3];
    block_reduce_partials<T, 3>(P1, nb, tot3);
    double gamma = (double)tot3[0], rr = (double)tot3[1];
    const double bs = (double)tot3[2];
    const double tl = a.tol_dev ? *a.tol_dev : a.tol;
    const double atol2 = fmax(tl * tl * bs, a.atol * a.atol);
    double beta = 0.0, alpha = 0.0;
    int k = 0, status = WSPM_OK;
    double rs = dinv ? rr : gamma;
    bool done = !(rs > atol2 && 0 < a.maxiter);
    if (!isfinite(rs)) { done = true; status = WSPM_NAN; }
    T *po = a.p0, *pn = a.p1;
    while (!done && ok) {
        // ---- phase 1
        {
            const T bt = (T)beta;
            const T *z = a.z;
            const T *pold = po;
            T v[1] = {T(0)};
            for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                const T qi = sell_row_dot<T, MW>(a.A, a.vals, i, [&](int c) {
                    return fma(bt, __ldcg(pold + c), __ldcg(z + c));
                });
                const T pi = fma(bt, pold[i], z[i]);
                pn[i] = pi;
                a.q[i] = qi;
                v[0] += pi * qi;
            }
            block_sum<T, 1>(v);
            if (threadIdx.x == 0) P1[blockIdx.x] = v[0];
        }
        ok = grid_barrier(a.bar, nb, gen);
        if (!ok) break;
        T pq[1];
        block_reduce_partials<T, 1>(P1, nb, pq);
        alpha = (double)((T)gamma / pq[0]);
        // ---- phase 2
        {
            const T al = (T)alpha;
            T v[2] = {T(0), T(0)};
            for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                a.x[i] = fma(al, pn[i], a.x[i]);
                const T ri = fma(-al, a.q[i], a.r[i]);
                a.r[i] = ri;
                const T zi = dinv ? dinv[i] * ri : ri;
                a.z[i] = zi;
                v[0] += ri * zi;
                v[1] += ri * ri;
            }
            block_sum<T, 2>(v);
            if (threadIdx.x == 0) {
                P2[blockIdx.x] = v[0];
                P2[nb + blockIdx.x] = v[1];
            }
        }
        ok = grid_barrier(a.bar, nb, gen);
        if (!ok) break;
        T t2[2];
        block_reduce_partials<T, 2>(P2, nb, t2);
        const double gamma_new = (double)t2[0];
        beta = (double)(t2[0] / (T)gamma);
        gamma = gamma_new;
        rr = (double)t2[1];
        ++k;
        rs = dinv ? rr : gamma;
        if (!(rs > atol2)) done = true;
        else if (k >= a.maxiter) { done = true; status = WSPM_MAXITER; }
        if (!isfinite(rs) || !isfinite(alpha)) { done = true; status = WSPM_NAN; }
        T *t = po; po = pn; pn = t;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        KrylovState *st = a.st;
        st->gamma = gamma; st->rr = rr; st->bs = bs; st->atol2 = atol2;
        st->alpha = alpha; st->beta = beta;
        st->k = k;
        st->status = ok ? status : WSPM_CUDA_ERROR;
        st->done = 1;
    }
}

// Grid size for the persistent kernel: every block must be resident at once.
template <typename T, int MW>
static int pcg_grid(int n) {
    static int cached[2] = {0, 0};
    int &c = cached[sizeof(T) == 8 ? 1 : 0];
    if (c == 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, cg_persistent_kernel<T, MW>, pcg_block<T>(), 0);
        c = sms * (per > 0 ? per : 1);
    }
    const int need = (n + pcg_block<T>() - 1) / pcg_block<T>();
    int g = need < c ? need : c;
    if (g > kMaxPartials) g = kMaxPartials;
    return g < 1 ? 1 : g;
}

template <typename T>
int cg_persistent_enqueue(const Sell &A, const T *vals, const T *b, const double *b64, T *x, const T *dinv,
                          const CgBuffers<T> &w, double tol, double atol, int maxiter, bool zero_x0,
                          const double *tol_dev, cudaStream_t st) {
    PcgArgs<T> a;
    a.A = A; a.vals = vals; a.b = b; a.b64 = b64; a.x = x; a.dinv = dinv;
    a.r = w.r; a.z = w.z; a.p0 = w.p0; a.p1 = w.p1; a.q = w.q; a.part = w.partials; a.st = w.st;
    a.bar = (GridBarrier *)&w.st->ticket[0];
    a.tol = tol; a.atol = atol; a.tol_dev = tol_dev; a.maxiter = maxiter; a.zero_x0 = zero_x0 ? 1 : 0;
    cudaError_t e = cudaSuccess;
    WSPM_WIDTH_DISPATCH(A.max_width, {
        const int grid = pcg_grid<T, MW>(A.n_rows);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(pcg_block<T>());
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelEx(&cfg, cg_persistent_kernel<T, MW>, a);
    });
    return e == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

template int cg_persistent_enqueue<double>(const Sell &, const double *, const double *, const double *, double *,
                                           const double *, const CgBuffers<double> &, double, double, int, bool,
                                           const double *, cudaStream_t);
template int cg_persistent_enqueue<float>(const Sell &, const float *, const float *, const double *, float *,
                                          const float *, const CgBuffers<float> &, double, double, int, bool,
                                          const double *, cudaStream_t);

// ---------------------------------------------------------------- BiCGSTAB (FP64)
template <int MW>
__global__ void __launch_bounds__(kBlock) bicg_init_kernel(Sell A, const double *__restrict__ vals,
                                                           const double *__restrict__ b, const double *x0,
                                                           double *r, double *rhat, double *p, double *q,
                                                           double *partials, KrylovState *st, double tol,
                                                           double atol, int maxiter,
                                                           cudaGraphConditionalHandle cond, int use_cond) {
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_rows; i += gridDim.x * blockDim.x) {
        const double ri = b[i] - sell_row<double, MW>(A, vals, i, [&](int c) { return x0[c]; });
        r[i] = ri; rhat[i] = ri; p[i] = ri; q[i] = ri;
        v[0] += ri * ri;
        v[1] += b[i] * b[i];
    }
    if (publish_partials<double, 2>(v, partials, &st->ticket[2])) {
        double tot[2];
        final_sum<double, 2>(partials, tot, &st->ticket[2]);
        if (threadIdx.x == 0) {
            st->rr = tot[0]; st->bs = tot[1];
            st->atol2 = fmax(tol * tol * tot[1], atol * atol);
            st->rho = st->alpha = st->omega = 1.0;
            st->rho_next = tot[0];
            st->k = 0; st->status = WSPM_OK; st->exit_early = 0;
            int done = !(tot[0] > st->atol2 && 0 < maxiter);
            if (!isfinite(tot[0])) { done = 1; st->status = WSPM_NAN; }
            st->done = done;
            set_cond(cond, use_cond, done ? 0u : 1u);
        }
    }
}

__global__ void bicg_p_kernel(int n, const double *__restrict__ r, double *p, const double *__restrict__ q,
                              double *phat, const double *__restrict__ dinv, const KrylovState *st) {
    if (st->done) return;
    const double beta = st->rho_next / st->rho * st->alpha / st->omega;
    const double om = st->omega;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double pi = r[i] + beta * (p[i] - om * q[i]);
        p[i] = pi;
        phat[i] = dinv ? dinv[i] * pi : pi;
    }
}

template <int MW>
__global__ void __launch_bounds__(kBlock) bicg_q_kernel(Sell A, const double *__restrict__ vals,
                                                        const double *__restrict__ phat,
                                                        const double *__restrict__ rhat, double *q,
                                                        double *partials, KrylovState *st) {
    if (st->done) return;
    double v[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_rows; i += gridDim.x * blockDim.x) {
        const double qi = sell_row<double, MW>(A, vals, i, [&](int c) { return __ldg(phat + c); });
        q[i] = qi;
        v[0] += rhat[i] * qi;
    }
    if (publish_partials<double, 1>(v, partials, &st->ticket[0])) {
        double tot[1];
        final_sum<double, 1>(partials, tot, &st->ticket[0]);
        if (threadIdx.x == 0) {
            st->sigma = tot[0];
            st->rho = st->rho_next;               // rho of this iteration
            st->alpha = st->rho_next / tot[0];    // alpha of this iteration
        }
    }
}

template <int MW>
__global__ void __launch_bounds__(kBlock) bicg_t_kernel(Sell A, const double *__restrict__ vals,
                                                        const double *__restrict__ r, const double *__restrict__ q,
                                                        const double *__restrict__ dinv, double *t,
                                                        double *partials, KrylovState *st) {
    if (st->done) return;
    const double alpha = st->alpha;
    double v[3] = {0.0, 0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_rows; i += gridDim.x * blockDim.x) {
        const double ti = sell_row<double, MW>(A, vals, i, [&](int c) {
            const double sc = __ldg(r + c) - alpha * __ldg(q + c);
            return dinv ? __ldg(dinv + c) * sc : sc;
        });
        const double si = r[i] - alpha * q[i];
        t[i] = ti;
        v[0] += si * si;
        v[1] += ti * si;
        v[2] += ti * ti;
    }
    if (publish_partials<double, 3>(v, partials, &st->ticket[1])) {
        double tot[3];
        final_sum<double, 3>(partials, tot, &st->ticket[1]);
        if (threadIdx.x == 0) {
            st->ss = tot[0]; st->ts = tot[1]; st->tt = tot[2];
            st->omega = tot[1] / tot[2];
            st->exit_early = tot[0] < st->atol2;
        }
    }
}

__global__ void __launch_bounds__(kBlock) bicg_x_kernel(int n, double *x, double *r, const double *__restrict__ rhat,
                                                        const double *__restrict__ p, const double *__restrict__ q,
                                                        const double *__restrict__ t,
                                                        const double *__restrict__ dinv, double *partials,
                                                        KrylovState *st, int maxiter,
                                                        cudaGraphConditionalHandle cond, int use_cond) {
    if (st->done) return;
    const double alpha = st->alpha, omega = st->omega;
    const int early = st->exit_early;
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double si = r[i] - alpha * q[i];
        const double di = dinv ? dinv[i] : 1.0;
        const double phat = dinv ? di * p[i] : p[i];
        const double shat = dinv ? di * si : si;
        double ri;
        if (early) {
            x[i] = x[i] + alpha * phat;
            ri = si;
        } else {
            x[i] = x[i] + (alpha * phat + omega * shat);
            ri = si - omega * t[i];
        }
        r[i] = ri;
        v[0] += ri * ri;
        v[1] += rhat[i] * ri;
    }
    if (publish_partials<double, 2>(v, partials, &st->ticket[2])) {
        double tot[2];
        final_sum<double, 2>(partials, tot, &st->ticket[2]);
        if (threadIdx.x == 0) {
            st->rr = tot[0];
            st->rho_next = tot[1];
            int k = (st->omega == 0.0 || st->alpha == 0.0) ? -11 : st->k + 1;
            if (st->rho == 0.0) k = -10;
            st->k = k;
            int done = !(tot[0] > st->atol2 && k < maxiter && k >= 0);
            if (k < 0) st->status = WSPM_BREAKDOWN;
            else if (done && tot[0] > st->atol2) st->status = WSPM_MAXITER;
            if (!isfinite(tot[0])) { done = 1; st->status = WSPM_NAN; }
            st->done = done;
            set_cond(cond, use_cond, done ? 0u : 1u);
        }
    }
}

void bicgstab_enqueue_init(const Sell &A, const double *vals, const double *b, const double *x0, double *x,
                           const BicgBuffers &w, double tol, double atol, int maxiter,
                           cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st) {
    const int nb = reduction_blocks(A.n_rows);
    if (x != x0) copy_kernel<double><<<nb, kBlock, 0, st>>>(x0, x, A.n_rows);
    WSPM_WIDTH_DISPATCH(A.max_width,
                        bicg_init_kernel<MW><<<nb, kBlock, 0, st>>>(A, vals, b, x0, w.r, w.rhat, w.p, w.q, w.partials,
                                                                    w.st, tol, atol, maxiter, cond, use_cond));
}

void bicgstab_enqueue_body(const Sell &A, const double *vals, const double *b, double *x, const double *dinv,
                           const BicgBuffers &w, int maxiter, cudaGraphConditionalHandle cond, int use_cond,
                           cudaStream_t st) {
    (void)b;
    const int nb = reduction_blocks(A.n_rows);
    bicg_p_kernel<<<nb, kBlock, 0, st>>>(A.n_rows, w.r, w.p, w.q, w.phat, dinv, w.st);
    WSPM_WIDTH_DISPATCH(A.max_width,
                        bicg_q_kernel<MW><<<nb, kBlock, 0, st>>>(A, vals, w.phat, w.rhat, w.q, w.partials, w.st));
    WSPM_WIDTH_DISPATCH(A.max_width,
                        bicg_t_kernel<MW><<<nb, kBlock, 0, st>>>(A, vals, w.r, w.q, dinv, w.t, w.partials, w.st));
    bicg_x_kernel<<<nb, kBlock, 0, st>>>(A.n_rows, x, w.r, w.rhat, w.p, w.q, w.t, dinv, w.partials, w.st, maxiter,
                                         cond, use_cond);
}

// ---------------------------------------------------------------- GMRES(m) (FP64)
constexpr int kMaxRestart = 32;
constexpr int kMaxDots = kMaxRestart + 2;

// r = M (b - A x) into dst; ||r||^2 (and, at init, ||b||^2, ||M b||^2).
template <int MW>
__global__ void __launch_bounds__(kBlock) gm_residual_kernel(Sell A, const double *__restrict__ vals,
                                                             const double *__restrict__ b, const double *x,
                                                             const double *__restrict__ dinv, double *dst,
                                                             double *partials, KrylovState *st, int is_init,
                                                             double tol, double atol, int maxiter,
                                                             cudaGraphConditionalHandle cond, int use_cond) {
    if (!is_init && st->done) return;
    double v[3] = {0.0, 0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_rows; i += gridDim.x * blockDim.x) {
        const double d = dinv ? dinv[i] : 1.0;
        const double ri = d * (b[i] - sell_row<double, MW>(A, vals, i, [&](int c) { return x[c]; }));
        dst[i] = ri;
        v[0] += ri * ri;
        v[1] += b[i] * b[i];
        v[2] += (d * b[i]) * (d * b[i]);
    }
    if (publish_partials<double, 3>(v, partials, &st->ticket[2])) {
        double tot[3];
        final_sum<double, 3>(partials, tot, &st->ticket[2]);
        if (threadIdx.x == 0) {
            double rn = sqrt(tot[0]);
            if (!(rn > DBL_EPSILON)) rn = 0.0;
            st->rnorm = rn;
            st->inv_wn = rn > 0.0 ? 1.0 / rn : 0.0;
            if (is_init) {
                const double bn = sqrt(tot[1]);
                st->b_norm = bn;
                st->mb_norm = sqrt(tot[2]);
                const double at = fmax(tol * bn, atol);
                // jnp.minimum propagates NaN: with b == 0 the tolerance is NaN and the loop does not run
                st->ptol = bn > 0.0 ? st->mb_norm * fmin(1.0, at / bn) : __longlong_as_double(0x7ff8000000000000ULL);
                st->k = 0;
                st->status = WSPM_OK;
            } else {
                st->k += 1;
            }
            st->broken = 0;
            st->steps = 0;
            int done = !(st->k < maxiter && rn > st->ptol);
            if (done && st->k >= maxiter && rn > st->ptol) st->status = WSPM_MAXITER;
            if (!isfinite(tot[0])) { done = 1; st->status = WSPM_NAN; }
            st->done = done;
            set_cond(cond, use_cond, done ? 0u : 1u);
        }
    }
}

__global__ void gm_scale_kernel(int n, double *v, const KrylovState *st) {
    if (st->done || st->broken) return;
    const double s = st->inv_wn;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] *= s;
}

// phase 0: w = M A V_j, dots V_k.w (k <= j) and ||w||^2
// phase 1: w -= V h1 ; dots V_k.w
// phase 2: w -= V h2 ; ||w||^2, then H column j and breakdown test
template <int MW>
__global__ void __launch_bounds__(kBlock) gm_arnoldi_kernel(Sell A, const double *__restrict__ vals,
                                                            const double *__restrict__ dinv, const double *V,
                                                            double *w, double *H, double *hbuf, double *partials,
                                                            KrylovState *st, int j, int m, int phase, int64_t ld) {
    if (st->done || st->broken) return;
    const int n = A.n_rows;
    const int nd = j + 1;
    double v[kMaxDots];
#pragma unroll
    for (int k = 0; k < kMaxDots; ++k) v[k] = 0.0;
    double h[kMaxRestart + 1];
    if (phase > 0) {
        const double *src = hbuf + (phase - 1) * (kMaxRestart + 1);
#pragma unroll
        for (int k = 0; k <= kMaxRestart; ++k) h[k] = k < nd ? src[k] : 0.0;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double wi;
        if (phase == 0) {
            const double *vj = V + (int64_t)j * ld;
            wi = sell_row<double, MW>(A, vals, i, [&](int c) { return __ldg(vj + c); });
            if (dinv) wi *= dinv[i];
        } else {
            wi = w[i];
#pragma unroll
            for (int k = 0; k <= kMaxRestart; ++k)
                if (k < nd) wi -= h[k] * V[(int64_t)k * ld + i];
        }
        w[i] = wi;
        if (phase < 2) {
#pragma unroll
            for (int k = 0; k <= kMaxRestart; ++k)
                if (k < nd) v[k] += V[(int64_t)k * ld + i] * wi;
        }
        v[kMaxDots - 1] += wi * wi;
    }
    if (publish_partials<double, kMaxDots>(v, partials, &st->ticket[phase == 2 ? 1 : 0])) {
        double tot[kMaxDots];
        final_sum<double, kMaxDots>(partials, tot, &st->ticket[phase == 2 ? 1 : 0]);
        if (threadIdx.x == 0) {
            if (phase == 0) {
                st->wn0 = sqrt(tot[kMaxDots - 1]);
                for (int k = 0; k < nd; ++k) hbuf[k] = tot[k];
            } else if (phase == 1) {
                for (int k = 0; k < nd; ++k) hbuf[(kMaxRestart + 1) + k] = tot[k];
            } else {
                double *col = H + (int64_t)j * (m + 1);
                for (int k = 0; k < nd; ++k) col[k] = hbuf[k] + hbuf[(kMaxRestart + 1) + k];
                double wn = sqrt(tot[kMaxDots - 1]);
                const double thresh = DBL_EPSILON * st->wn0;
                if (!(wn > thresh)) wn = 0.0;
                col[j + 1] = wn;
                st->wn = wn;
                st->inv_wn = wn > 0.0 ? 1.0 / wn : 0.0;
                st->steps = j + 1;
                if (wn == 0.0) st->broken = 1;
            }
        }
    }
}

// V_{j+1} = w / ||w|| (zero after a breakdown); runs even on the breakdown step.
__global__ void gm_next_kernel(int n, double *V, const double *__restrict__ w, const KrylovState *st, int j,
                               int64_t ld) {
    if (st->done || st->steps != j + 1) return;
    const double s = st->inv_wn;
    double *dst = V + (int64_t)(j + 1) * ld;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = w[i] * s;
}

// Least squares min || rnorm e1 - H y || over the first `steps` columns
// (Givens QR of the upper-Hessenberg matrix; one thread, m <= 32).
__global__ void gm_lsq_kernel(const double *H, double *y, KrylovState *st, int m) {
    if (st->done || threadIdx.x != 0 || blockIdx.x != 0) return;
    const int ns = st->steps;
    double R[kMaxRestart + 1][kMaxRestart];
    double g[kMaxRestart + 1];
    for (int j = 0; j < ns; ++j)
        for (int i = 0; i <= ns; ++i) R[i][j] = (i <= j + 1) ? H[(int64_t)j * (m + 1) + i] : 0.0;
    for (int i = 0; i <= ns; ++i) g[i] = 0.0;
    g[0] = st->rnorm;
    for (int j = 0; j < ns; ++j) {
        const double a = R[j][j], bb = R[j + 1][j];
        const double rr = hypot(a, bb);
        const double c = rr > 0.0 ? a / rr : 1.0, s = rr > 0.0 ? bb / rr : 0.0;
        for (int k = j; k < ns; ++k) {
            const double t1 = R[j][k], t2 = R[j + 1][k];
            R[j][k] = c * t1 + s * t2;
            R[j + 1][k] = -s * t1 + c * t2;
        }
        const double g1 = g[j], g2 = g[j + 1];
        g[j] = c * g1 + s * g2;
        g[j + 1] = -s * g1 + c * g2;
    }
    for (int j = ns - 1; j >= 0; --j) {
        double acc = g[j];
        for (int k = j + 1; k < ns; ++k) acc -= R[j][k] * y[k];
        y[j] = R[j][j] != 0.0 ? acc / R[j][j] : 0.0;
    }
}

__global__ void gm_update_kernel(int n, double *x, const double *V, const double *__restrict__ y,
                                 const KrylovState *st, int64_t ld) {
    if (st->done) return;
    const int ns = st->steps;
    double yl[kMaxRestart];
#pragma unroll
    for (int k = 0; k < kMaxRestart; ++k) yl[k] = k < ns ? y[k] : 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < kMaxRestart; ++k)
            if (k < ns) acc += yl[k] * V[(int64_t)k * ld + i];
        x[i] += acc;
    }
}

void gmres_enqueue_init(const Sell &A, const double *vals, const double *b, const double *x0, double *x,
                        const double *dinv, const GmresBuffers &w, double tol, double atol, int maxiter,
                        cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st) {
    const int nb = reduction_blocks(A.n_rows);
    if (x != x0) copy_kernel<double><<<nb, kBlock, 0, st>>>(x0, x, A.n_rows);
    WSPM_WIDTH_DISPATCH(A.max_width,
                        gm_residual_kernel<MW><<<nb, kBlock, 0, st>>>(A, vals, b, x0, dinv, w.V, w.partials, w.st, 1,
                                                                      tol, atol, maxiter, cond, use_cond));
    gm_scale_kernel<<<nb, kBlock, 0, st>>>(A.n_rows, w.V, w.st);
}

void gmres_enqueue_body(const Sell &A, const double *vals, const double *b, double *x, const double *dinv,
                        const GmresBuffers &w, int maxiter, cudaGraphConditionalHandle cond, int use_cond,
                        cudaStream_t st) {
    const int nb = reduction_blocks(A.n_rows);
    for (int j = 0; j < w.m; ++j) {
        for (int ph = 0; ph < 3; ++ph)
            WSPM_WIDTH_DISPATCH(A.max_width,
                                gm_arnoldi_kernel<MW><<<nb, kBlock, 0, st>>>(A, vals, dinv, w.V, w.w, w.H, w.hbuf,
                                                                             w.partials, w.st, j, w.m, ph, w.ld));
        gm_next_kernel<<<nb, kBlock, 0, st>>>(A.n_rows, w.V, w.w, w.st, j, w.ld);
    }
    gm_lsq_kernel<<<1, 32, 0, st>>>(w.H, w.y, w.st, w.m);
    gm_update_kernel<<<nb, kBlock, 0, st>>>(A.n_rows, x, w.V, w.y, w.st, w.ld);
    WSPM_WIDTH_DISPATCH(A.max_width,
                        gm_residual_kernel<MW><<<nb, kBlock, 0, st>>>(A, vals, b, x, dinv, w.V, w.partials, w.st, 0,
                                                                      0.0, 0.0, maxiter, cond, use_cond));
    gm_scale_kernel<<<nb, kBlock, 0, st>>>(A.n_rows, w.V, w.st);
}

// ---------------------------------------------------------------- workspaces
static inline int64_t align32(int64_t n) { return (n + 31) & ~int64_t(31); }

int64_t cg_workspace_doubles(int n, int bytes) {
    const int64_t vec = align32(((int64_t)n * bytes + 7) / 8);
    return 5 * vec + align32(4 * kMaxPartials) + align32(sizeof(KrylovState) / 8 + 1);
}
int64_t bicgstab_workspace_doubles(int n) {
    return 6 * align32(n) + align32(4 * kMaxPartials) + align32(sizeof(KrylovState) / 8 + 1);
}
int64_t gmres_workspace_doubles(int n, int m) {
    return (m + 2) * align32(n) + align32((int64_t)(m + 1) * m) + align32(m) + align32(2 * (kMaxRestart + 1)) +
           align32((int64_t)kMaxDots * kMaxPartials) + align32(sizeof(KrylovState) / 8 + 1);
}

template <typename T>
CgBuffers<T> carve_cg(double *work, int n, int64_t *used) {
    const int64_t vec = align32(((int64_t)n * sizeof(T) + 7) / 8);
    CgBuffers<T> b;
    double *p = work;
    b.r = (T *)p; p += vec;
    b.z = (T *)p; p += vec;
    b.p0 = (T *)p; p += vec;
    b.p1 = (T *)p; p += vec;
    b.q = (T *)p; p += vec;
    b.partials = (T *)p; p += align32(4 * kMaxPartials);
    b.st = (KrylovState *)p; p += align32(sizeof(KrylovState) / 8 + 1);
    *used = p - work;
    return b;
}
template CgBuffers<double> carve_cg<double>(double *, int, int64_t *);
template CgBuffers<float> carve_cg<float>(double *, int, int64_t *);

BicgBuffers carve_bicgstab(double *work, int n, int64_t *used) {
    const int64_t vec = align32(n);
    BicgBuffers b;
    double *p = work;
    b.r = p; p += vec; b.rhat = p; p += vec; b.p = p; p += vec;
    b.phat = p; p += vec; b.q = p; p += vec; b.t = p; p += vec;
    b.partials = p; p += align32(4 * kMaxPartials);
    b.st = (KrylovState *)p; p += align32(sizeof(KrylovState) / 8 + 1);
    *used = p - work;
    return b;
}

GmresBuffers carve_gmres(double *work, int n, int m, int64_t *used) {
    const int64_t vec = align32(n);
    GmresBuffers b;
    double *p = work;
    b.m = m;
    b.ld = vec;
    b.V = p; p += (int64_t)(m + 1) * vec;
    b.w = p; p += vec;
    b.H = p; p += align32((int64_t)(m + 1) * m);
    b.y = p; p += align32(m);
    b.hbuf = p; p += align32(2 * (kMaxRestart + 1));
    b.partials = p; p += align32((int64_t)kMaxDots * kMaxPartials);
    b.st = (KrylovState *)p; p += align32(sizeof(KrylovState) / 8 + 1);
    *used = p - work;
    return b;
}

}  // namespace wspm
