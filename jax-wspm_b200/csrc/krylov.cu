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

// 16-byte vectors: a thread owns NV consecutive rows (4 in FP32, 2 in FP64) so
// every matrix diagonal and every per-row vector moves as one 16-byte access.
template <typename T> struct Vec16;
template <> struct Vec16<float> {
    using V = float4;
    static constexpr int N = 4;
    __device__ static __forceinline__ void split(const float4 &v, float (&o)[4]) {
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    }
    __device__ static __forceinline__ float4 join(const float (&o)[4]) { return make_float4(o[0], o[1], o[2], o[3]); }
};
template <> struct Vec16<double> {
    using V = double2;
    static constexpr int N = 2;
    __device__ static __forceinline__ void split(const double2 &v, double (&o)[2]) { o[0] = v.x; o[1] = v.y; }
    __device__ static __forceinline__ double2 join(const double (&o)[2]) { return make_double2(o[0], o[1]); }
};

// DIA SpMV: a thread owns 16 bytes of rows (2 in FP64, 4 in FP32); the live diagonals' offsets sit in shared
// memory, and every value load and gather of the thread's rows is issued before the first product (the generic
// kernel reads each offset from global memory before the gather that needs it).  Products in diagonal order,
// like sell_row.
template <typename T, int MW>
__global__ void __launch_bounds__(kBlock) spmv_dia_kernel(Sell A, const T *__restrict__ vals, const T *__restrict__ x,
                                                          T *__restrict__ y) {
    using VT = Vec16<T>;
    constexpr int N = VT::N;
    __shared__ int s_off[MW];
    __shared__ int64_t s_vo[MW];
    __shared__ int s_nd;
    if (threadIdx.x == 0) {
        int nd = 0;
        for (int k = 0; k < A.n_diags; ++k) {
            if (!dia_live(A, k)) continue;
            s_off[nd] = __ldg(A.diag_off + k);
            s_vo[nd] = (int64_t)k * A.ld;
            ++nd;
        }
        s_nd = nd;
    }
    __syncthreads();
    const int nd = s_nd;
    const int n = A.n_rows, last = n - 1;
    const int i = N * (blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= n) return;
    T e[MW][N], xv[MW][N];
#pragma unroll
    for (int k = 0; k < MW; ++k) {
        if (k < nd) {
            VT::split(__ldg(reinterpret_cast<const typename VT::V *>(vals + s_vo[k] + i)), e[k]);
#pragma unroll
            for (int q = 0; q < N; ++q) {
                int c = i + q + s_off[k];
                c = c < 0 ? 0 : (c > last ? last : c);
                xv[k][q] = __ldg(x + c);
            }
        }
    }
    T w[N];
#pragma unroll
    for (int q = 0; q < N; ++q) w[q] = T(0);
#pragma unroll
    for (int k = 0; k < MW; ++k)
        if (k < nd)
#pragma unroll
            for (int q = 0; q < N; ++q) w[q] = fma(e[k][q], xv[k][q], w[q]);
    if (i + N <= n) {
        *reinterpret_cast<typename VT::V *>(y + i) = VT::join(w);
    } else {
        for (int q = 0; q < N && i + q < n; ++q) y[i + q] = w[q];
    }
}

template <typename T>
static void spmv_launch(const Sell &A, const T *vals, const T *x, T *y, cudaStream_t st) {
    // the DIA form needs 16-byte aligned values and output (ld and every diagonal start are multiples of 32 rows)
    const bool aligned = ((((uintptr_t)vals) | ((uintptr_t)y)) % 16) == 0;
    if (A.n_diags > 0 && A.n_diags <= 16 && aligned) {
        const int threads = (A.n_rows + Vec16<T>::N - 1) / Vec16<T>::N;
        const int blocks = (threads + kBlock - 1) / kBlock;
        if (A.n_diags <= 8) spmv_dia_kernel<T, 8><<<blocks, kBlock, 0, st>>>(A, vals, x, y);
        else spmv_dia_kernel<T, 16><<<blocks, kBlock, 0, st>>>(A, vals, x, y);
        return;
    }
    WSPM_WIDTH_DISPATCH(A.max_width,
                        spmv_kernel<T, MW><<<(A.n_rows + kBlock - 1) / kBlock, kBlock, 0, st>>>(A, vals, x, y));
}

void spmv_f64(const Sell &A, const double *vals, const double *x, double *y, cudaStream_t st) {
    spmv_launch<double>(A, vals, x, y, st);
}
void spmv_f32(const Sell &A, const float *vals, const float *x, float *y, cudaStream_t st) {
    spmv_launch<float>(A, vals, x, y, st);
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
// Grid barrier of the cooperative CG kernel.  The words live in the solver's
// KrylovState (count returns to 0 at every barrier; gen only grows).  Waits are
// bounded: on timeout the block records an error and every block leaves its
// loop at the next check, so a failed launch ends with WSPM_CUDA_ERROR instead
// of hanging.
struct GridBarrier {
    unsigned int count;
    unsigned int gen;
    int error;
    unsigned int mono;     // arrivals at counting barriers since the kernel's first grid barrier
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

// Per-block vectors of the resident CG kernel, in the order in which they are
// given shared memory (the rest live in the global workspace).
enum RcgVec { kVR = 0, kVP, kVS, kVW, kVX, kVD, kNumRcgVec };

template <typename T>
struct RcgArgs {
    Sell A;
    const T *vals;
    const T *b;            // right-hand side (or NULL with b64)
    const double *b64;     // FP64 right-hand side converted on the fly (refinement loop)
    T *x;                  // x0 on entry unless zero_x0, solution on exit
    const T *dinv;         // Jacobi 1/diag, NULL = none
    T *z;                  // preconditioned residual, the only vector other blocks read
    T *gvec[kNumRcgVec];   // global homes of the vectors kept out of shared memory (row-indexed)
    int chunk;             // rows per block (multiple of 32)
    T *part;               // [2 parities][4][gridDim] partial sums, then [3][gridDim] for the init
    unsigned int *zflag;   // [gridDim] per-block z epoch
    KrylovState *st;
    GridBarrier *bar;
    double tol, atol;
    const double *tol_dev; // when set, the relative tolerance is read here
    const int *skip;       // when set and nonzero at launch: no iteration, k = 0 (refinement already done)
    int maxiter, zero_x0;
};

// Early exit of a resident CG launch whose refinement loop has already met its
// tolerance: every block reads the same word (written before the launch) and
// returns before touching any barrier; block 0 records an empty solve.
__device__ __forceinline__ bool resident_skip(const int *skip, KrylovState *st) {
    if (!skip || *(volatile const int *)skip == 0) return false;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->k = 0;
        st->status = WSPM_OK;
        st->done = 1;
        st->ns = 0ull;
    }
    return true;
}

constexpr int kRcgBlock = 512;    // 128 registers: the 2D instances run without spills

__device__ __forceinline__ void st_release_u32(unsigned int *p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_u32(unsigned int *p, unsigned int v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Counting barrier: every block adds one arrival; a block passes once the count
// reaches `target` (= gridDim * barriers passed so far).  One atomic per block
// and one polled word; bounded like grid_barrier.
__device__ __forceinline__ bool count_barrier(GridBarrier *gb, unsigned int target) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&gb->mono, 1u);
        int ok = 1;
        long long spins = 0;
        while (ld_acquire_u32(&gb->mono) < target) {
            if (++spins > kBarrierSpinLimit) { atomicExch(&gb->error, 1); ok = 0; break; }
            if ((spins & 1023) == 0 && *(volatile int *)&gb->error) { ok = 0; break; }
            __nanosleep(20);
        }
        ok_s = ok && (*(volatile int *)&gb->error) == 0;
    }
    __syncthreads();
    return ok_s != 0;
}

// Wait until blocks [lo, hi] (except this one) have published z epoch `epoch`;
// thread t polls block lo + t (strided), the verdict is OR-reduced by the block.
__device__ __forceinline__ bool wait_zflags(const unsigned int *zflag, int lo, int hi, unsigned int epoch,
                                            GridBarrier *gb) {
    int fail = 0;
    for (int c = lo + (int)threadIdx.x; c <= hi && !fail; c += blockDim.x) {
        if (c == (int)blockIdx.x) continue;
        long long spins = 0;
        while (ld_acquire_u32(zflag + c) < epoch) {
            if (++spins > kBarrierSpinLimit) { atomicExch(&gb->error, 1); fail = 1; break; }
            if ((spins & 1023) == 0 && *(volatile int *)&gb->error) { fail = 1; break; }
            __nanosleep(20);
        }
    }
    return __syncthreads_or(fail) == 0;
}

// Fixed-order sum of nb partials (layout [NV][nb]): warp j sums row j with all
// of a lane's loads in flight at once (one L2 round trip for nb <= 256),
// broadcast through shared memory with a single block barrier.  Every block
// runs the identical sequence, so all blocks hold bitwise identical sums.
template <typename T, int NV>
__device__ __forceinline__ void reduce_partials_rows(const T *partials, int nb, T (&out)[NV]) {
    __shared__ T bc[NV];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (wid < NV) {
        const T *pj = partials + (int64_t)wid * nb;
        T acc = T(0);
        for (int b0 = 0; b0 < nb; b0 += 256) {
            T x[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int b = b0 + lane + 32 * u;
                x[u] = b < nb ? __ldcg(pj + b) : T(0);
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) acc += x[u];
        }
        acc = warp_sum(acc);
        if (lane == 0) bc[wid] = acc;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NV; ++j) out[j] = bc[j];
}


// Row i of A times z with the values and gathers of a group of diagonals in
// flight at once, accumulated in diagonal order like sell_row_dot (used for
// the ragged rows that do not fill a 16-byte group).  z is read with plain
// loads: inside a phase no block writes z, and the acquire that ends the
// preceding wait (flag or barrier) followed by the block barrier orders every
// earlier z store before these loads.
//
// The resident kernels keep only the diagonals that can hold nonzeros: entry k
// of their lists has column offset s_off[k] and its values at s_vo[k] + row
// (s_vo[k] = (index of the diagonal) * ld).  A skipped diagonal is exactly zero,
// and fma(0, x, acc) == acc, so the products are those of the full row.
template <typename T, int MW>
__device__ __forceinline__ T dia_row_z(const T *__restrict__ vals, const int64_t *s_vo, int i, int last, int nd,
                                       const int *s_off, const T *z) {
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < MW; ++k) {
        if (k < nd) {
            int c = i + s_off[k];
            c = c < 0 ? 0 : (c > last ? last : c);
            acc = fma(__ldg(vals + s_vo[k] + i), z[c], acc);
        }
    }
    return acc;
}

// Rows i .. i+N-1 (i a multiple of N) of a DIA matrix times z: one 16-byte load
// per diagonal, issued G diagonals at a time before their first use, then the
// gathers diagonal by diagonal.  Each row accumulates in diagonal order.
//
// FP32: the four values z[i+o .. i+o+3] of a diagonal come from one or two
// aligned 16-byte loads (the window's misalignment (i+o) mod 4 is the same for
// every thread, so the selection below is a uniform branch).  With the lanes of
// a warp 16 bytes apart, a scalar gather moves 512 bytes through L1 for 128
// used; the windows move each byte once.  Groups whose window leaves [0, n)
// (the first and last rows) and unaligned z take the scalar gathers with the
// clamped columns.  Same products in the same order either way.
template <typename T, int MW>
__device__ __forceinline__ void dia_group_z(const T *__restrict__ vals, const int64_t *s_vo, int i, int last, int nd,
                                            const int *s_off, const T *z, T (&w)[Vec16<T>::N]) {
    using VT = Vec16<T>;
    constexpr int N = VT::N;
    constexpr int G = MW < 4 ? MW : (N == 4 ? 2 : 4);
    const bool zal = (reinterpret_cast<uintptr_t>(z) & 15) == 0;
#pragma unroll
    for (int q = 0; q < N; ++q) w[q] = T(0);
#pragma unroll
    for (int k0 = 0; k0 < MW; k0 += G) {
        if (k0 >= nd) break;
        typename VT::V vv[G];
#pragma unroll
        for (int g = 0; g < G; ++g)
            if (k0 + g < nd) vv[g] = __ldg(reinterpret_cast<const typename VT::V *>(vals + s_vo[k0 + g] + i));
#pragma unroll
        for (int g = 0; g < G; ++g) {
            if (k0 + g < nd) {
                T e[N];
                VT::split(vv[g], e);
                const int o = s_off[k0 + g];
                if constexpr (N == 4) {
                    const int c0 = i + o;
                    const int mis = c0 & 3;
                    const int base = c0 - mis;
                    if (zal && base >= 0 && base + (mis ? 8 : 4) <= last + 1) {
                        const float4 lo = *reinterpret_cast<const float4 *>(z + base);
                        float4 hi = lo;
                        if (mis) hi = *reinterpret_cast<const float4 *>(z + base + 4);
                        switch (mis) {
                        case 0:
                            w[0] = fma(e[0], lo.x, w[0]); w[1] = fma(e[1], lo.y, w[1]);
                            w[2] = fma(e[2], lo.z, w[2]); w[3] = fma(e[3], lo.w, w[3]);
                            break;
                        case 1:
                            w[0] = fma(e[0], lo.y, w[0]); w[1] = fma(e[1], lo.z, w[1]);
                            w[2] = fma(e[2], lo.w, w[2]); w[3] = fma(e[3], hi.x, w[3]);
                            break;
                        case 2:
                            w[0] = fma(e[0], lo.z, w[0]); w[1] = fma(e[1], lo.w, w[1]);
                            w[2] = fma(e[2], hi.x, w[2]); w[3] = fma(e[3], hi.y, w[3]);
                            break;
                        default:
                            w[0] = fma(e[0], lo.w, w[0]); w[1] = fma(e[1], hi.x, w[1]);
                            w[2] = fma(e[2], hi.y, w[2]); w[3] = fma(e[3], hi.z, w[3]);
                            break;
                        }
                        continue;
                    }
                }
#pragma unroll
                for (int q = 0; q < N; ++q) {
                    int c = i + q + o;
                    c = c < 0 ? 0 : (c > last ? last : c);
                    w[q] = fma(e[q], z[c], w[q]);
                }
            }
        }
    }
}

// SpMV of z over local rows [l0, l1) of the block starting at row r0 (SELL
// rows, one per thread): w into wbase[l], partial (w, z) into acc.
template <typename T, int MW>
__device__ __forceinline__ void rcg_spmv_rows(int l0, int l1, T &acc, const Sell &A, const T *__restrict__ vals,
                                              int r0, const T *z, T *wbase) {
    for (int l = l0 + threadIdx.x; l < l1; l += blockDim.x) {
        const int i = r0 + l;
        const T wi = sell_row_dot<T, MW>(A, vals, i, [z](int c) { return z[c]; });
        wbase[l] = wi;
        acc = fma(wi, z[i], acc);
    }
}

// SpMV phase of a DIA matrix over the block's rows in 16-byte groups: w into
// wbase[l], partial (w, z) into acc.  The interior groups (columns inside the
// block's own chunk) come first in one list with the halo groups; thread t
// takes list entries t, t + T, ...  With poll, the block waits for its
// neighbours' z flags before the first round that holds a halo group, so the
// critical path is ceil(groups / T) rounds whatever the interior/halo split.
// Returns false when that wait gave up.
template <typename T, int MW>
__device__ __forceinline__ bool rcg_spmv_dia(int nl, int lo_i, int hi_i, T &acc, const T *__restrict__ vals,
                                             const int64_t *s_vo, int r0, int last, int nd, const int *s_off, const T *z,
                                             T *wbase, const unsigned int *zflag, int nbr_lo, int nbr_hi,
                                             unsigned int epoch, bool poll, GridBarrier *bar) {
    using VT = Vec16<T>;
    constexpr int N = VT::N;
    const int ng = (nl + N - 1) / N;
    const int gi0 = lo_i / N, gi1 = hi_i / N;
    const int nint = gi1 - gi0, nlow = gi0;
    const int TB = blockDim.x;
    const int rounds = (ng + TB - 1) / TB;
    const int m_wait = poll ? nint / TB : rounds;
    for (int m = 0; m < rounds; ++m) {
        if (m == m_wait && !wait_zflags(zflag, nbr_lo, nbr_hi, epoch, bar)) return false;
        const int j = (int)threadIdx.x + m * TB;
        if (j >= ng) continue;
        int g;
        if (j < nint) g = gi0 + j;
        else {
            const int h = j - nint;
            g = h < nlow ? h : gi1 + (h - nlow);
        }
        const int l = g * N, i = r0 + l;
        if (l + N <= nl) {
            T w[N];
            dia_group_z<T, MW>(vals, s_vo, i, last, nd, s_off, z, w);
            *reinterpret_cast<typename VT::V *>(wbase + l) = VT::join(w);
            T zo[N];
            VT::split(*reinterpret_cast<const typename VT::V *>(z + i), zo);
#pragma unroll
            for (int q = 0; q < N; ++q) acc = fma(w[q], zo[q], acc);
        } else {
            for (int q = 0; l + q < nl; ++q) {
                const T wi = dia_row_z<T, MW>(vals, s_vo, i + q, last, nd, s_off, z);
                wbase[l + q] = wi;
                acc = fma(wi, z[i + q], acc);
            }
        }
    }
    if (m_wait >= rounds && poll && !wait_zflags(zflag, nbr_lo, nbr_hi, epoch, bar)) return false;
    return true;
}

// Whole preconditioned CG solve in one cooperative launch, single-reduction
// form (Chronopoulos & Gear, J. Comput. Appl. Math. 25 (1989) 153-168):
//   beta = g/g_old ; alpha = g/(d - beta g/alpha_old)
//   p = z + beta p ; s = w + beta s ; x += alpha p ; r -= alpha s ; z = M r
//   w = A z ; g = (r,z), d = (w,z), rho = (r,r)       (one grid reduction)
// Block b owns rows [b*chunk, (b+1)*chunk).  The first NS of its vectors
// r, p, s, w, x, M (NS = 6, 4 or 0, whatever fits in shared memory) stay on
// chip for the whole solve, the others live in the workspace (x: the caller's
// array).  z is the only vector that crosses blocks.  Per iteration the kernel
// streams the matrix once and moves z once through L2, instead of the 11
// vector passes of the textbook iteration.  A thread owns groups of N
// consecutive rows (16 bytes) in both phases.
//
// Synchronisation per iteration: after its z update a block publishes a z
// epoch flag; its SpMV first does the interior rows (DIA: rows whose columns
// all lie in its own chunk), then waits only for the flags of the blocks its
// halo rows read, then does the halo rows.  The partial sums go through one
// counting barrier and are summed by every block in the same fixed order, so
// all blocks hold bitwise identical scalars and take the same branch.  Partials
// alternate between two buffers: a block can only start writing reduction e+2
// after every block has arrived at reduction e+1, i.e. finished reading e.  z is
// overwritten only after the reduction that follows every block's SpMV.  The
// stopping rule is the textbook one on ||r_{k+1}||: the iteration count matches
// the two-reduction form up to rounding.  Every wait is bounded (error flag).
template <typename T, int MW, int NS>
__global__ void __launch_bounds__(kRcgBlock, 1) cg_resident_kernel(RcgArgs<T> a) {
    using VT = Vec16<T>;
    using V = typename VT::V;
    constexpr int N = VT::N;
    extern __shared__ __align__(16) unsigned char rcg_smem[];
    __shared__ int s_off[MW > 0 ? MW : 1];
    __shared__ int64_t s_vo[MW > 0 ? MW : 1];
    T *const sm = reinterpret_cast<T *>(rcg_smem);
    if (resident_skip(a.skip, a.st)) return;
    const unsigned long long t_entry = (blockIdx.x == 0 && threadIdx.x == 0) ? global_ns() : 0ull;
    const int n = a.A.n_rows;
    const int nb = gridDim.x;
    const int chunk = a.chunk;
    const int r0 = blockIdx.x * chunk;
    const int r1 = min(n, r0 + chunk);
    const int nl = max(0, r1 - r0);
    unsigned int gen = threadIdx.x == 0 ? ld_acquire_u32(&a.bar->gen) : 0u;
    if (threadIdx.x == 0) {
        a.zflag[blockIdx.x] = 0u;
        if (blockIdx.x == 0) a.bar->mono = 0u;
    }
    // every argument is copied to a local first: a lambda that captured the
    // parameter struct itself would force a copy of it into local memory
    const Sell A = a.A;
    T *const z = a.z;
    T *const xg = a.x;
    const T *const vals = a.vals;
    const T *const dg = a.dinv;
    T *const gvR = a.gvec[kVR] + r0, *const gvP = a.gvec[kVP] + r0;
    T *const gvS = a.gvec[kVS] + r0, *const gvW = a.gvec[kVW] + r0;
    T *const part = a.part;
    unsigned int *const zflag = a.zflag;
    GridBarrier *const bar = a.bar;
    // vector v at local row l: shared memory for v < NS, else its global home
#define RCG_G(v) ((v) == kVR ? gvR : (v) == kVP ? gvP : (v) == kVS ? gvS : gvW)
#define RCG_P(v, l) ((v) < NS ? (sm + (v) * chunk + (l)) : (RCG_G(v) + (l)))
#define RCG(v, l) (*RCG_P(v, l))
    const bool dia = MW > 0 && A.n_diags > 0 && A.n_diags <= MW;
    int nd = 0;                // diagonals that can hold nonzeros (A.live)
    int lo_i = 0, hi_i = 0, nbr_lo = 0, nbr_hi = nb - 1;
    if (dia) {
        int mn = 0, mx = 0;
        for (int k = 0; k < A.n_diags; ++k) {
            if (!dia_live(A, k)) continue;
            const int o = __ldg(A.diag_off + k);
            if (threadIdx.x == 0) {
                s_off[nd] = o;
                s_vo[nd] = (int64_t)k * A.ld;
            }
            ++nd;
            mn = min(mn, o);
            mx = max(mx, o);
        }
        // interior rows [lo_i, hi_i), rounded inwards to whole 16-byte groups
        lo_i = min(nl, (-mn + N - 1) / N * N);
        hi_i = max(lo_i, (nl - mx) / N * N);
        const int rlo = max(0, r0 + mn), rhi = min(n - 1, r1 - 1 + mx);
        nbr_lo = min(nb - 1, rlo / chunk);
        nbr_hi = min(nb - 1, rhi / chunk);
        if (nl == 0) { nbr_lo = 1; nbr_hi = 0; }
    }
    const int last = n - 1;
    T *const wbase = kVW < NS ? sm + kVW * chunk : gvW;
    // ---- init: x, M into place; r = b - A x0 ; z = M r.  On DIA patterns A x0
    // comes from the same row-group SpMV as the iterations (into w, which is
    // free until w0 = A z0); then a thread's rows l = tid + j T are handled
    // kBatch at a time, their loads issued before any store, the per-thread sums
    // in row order.
    {
        constexpr int kBatch = sizeof(T) == 4 ? 8 : 4;
        const bool ax_dia = !a.zero_x0 && dia;
        if (ax_dia) {
            __syncthreads();       // s_off (written by thread 0 above) is read by every thread
            T unused = T(0);
            rcg_spmv_dia<T, (MW > 0 ? MW : 1)>(nl, lo_i, hi_i, unused, vals, s_vo, r0, last, nd, s_off, xg, wbase,
                                                zflag, nbr_lo, nbr_hi, 0u, false, bar);
            __syncthreads();
        }
        T v[3] = {T(0), T(0), T(0)};
        for (int l0 = threadIdx.x; l0 < nl; l0 += kBatch * (int)blockDim.x) {
            T bq[kBatch], xq[kBatch], dq[kBatch], aq[kBatch];
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                const int l = l0 + q * (int)blockDim.x;
                bq[q] = xq[q] = aq[q] = T(0);
                dq[q] = T(1);
                if (l < nl) {
                    const int i = r0 + l;
                    bq[q] = a.b64 ? (T)a.b64[i] : a.b[i];
                    if (dg) dq[q] = dg[i];
                    if (!a.zero_x0) xq[q] = xg[i];
                    if (ax_dia) aq[q] = wbase[l];
                }
            }
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                const int l = l0 + q * (int)blockDim.x;
                if (l >= nl) continue;
                const int i = r0 + l;
                const T bi = bq[q];
                T ri;
                if (a.zero_x0) {
                    xg[i] = T(0);
                    if (kVX < NS) RCG(kVX, l) = T(0);
                    ri = bi;
                } else {
                    if (kVX < NS) RCG(kVX, l) = xq[q];
                    ri = bi - (ax_dia ? aq[q] : sell_row_dot<T, MW>(A, vals, i, [xg](int c) { return xg[c]; }));
                }
                const T di = dq[q];
                if (kVD < NS) RCG(kVD, l) = di;
                const T zi = di * ri;
                RCG(kVR, l) = ri;
                RCG(kVP, l) = T(0);
                RCG(kVS, l) = T(0);
                z[i] = zi;
                v[0] += ri * zi;
                v[1] += ri * ri;
                v[2] += bi * bi;
            }
        }
        block_sum<T, 3>(v);
        if (threadIdx.x == 0) {
            T *p0 = part + 8 * (int64_t)nb;   // third region: the two parities are reused below
            p0[blockIdx.x] = v[0];
            p0[nb + blockIdx.x] = v[1];
            p0[2 * nb + blockIdx.x] = v[2];
        }
    }
    bool ok = grid_barrier(bar, nb, gen);     // z0 complete everywhere; zflags and mono reset
    T init3[3];
    reduce_partials_rows<T, 3>(part + 8 * (int64_t)nb, nb, init3);
    const double bs = (double)init3[2];
    const double tl = a.tol_dev ? *a.tol_dev : a.tol;
    const double atol2 = fmax(tl * tl * bs, a.atol * a.atol);
    double gamma = (double)init3[0], rr = (double)init3[1];
    double beta = 0.0, alpha = 0.0, gamma_old = 1.0, delta = 0.0;
    int k = 0, status = WSPM_OK;
    double rs = dg ? rr : gamma;
    bool done = !(rs > atol2 && 0 < a.maxiter);
    if (!isfinite(rs)) { done = true; status = WSPM_NAN; }
    unsigned int red = 0;      // counting barriers passed
#define RCG_SPMV_DIA(acc, epoch, poll)                                                                       \
    rcg_spmv_dia<T, (MW > 0 ? MW : 1)>(nl, lo_i, hi_i, (acc), vals, s_vo, r0, last, nd, s_off, z, wbase, zflag, \
                                       nbr_lo, nbr_hi, (epoch), (poll), bar)
    // w0 = A z0 and d0 = (w0, z0) when iterating
    if (!done && ok) {
        T v[1] = {T(0)};
        if (dia) ok = RCG_SPMV_DIA(v[0], 0u, false);
        else rcg_spmv_rows<T, MW>(0, nl, v[0], A, vals, r0, z, wbase);
        block_sum<T, 1>(v);
        T *pp = part + (int64_t)(red & 1) * 4 * nb;
        if (threadIdx.x == 0) pp[blockIdx.x] = v[0];
        ++red;
        ok = count_barrier(bar, red * (unsigned)nb);
        T d1[1];
        reduce_partials_rows<T, 1>(pp, nb, d1);
        delta = (double)d1[0];
    }
    while (!done && ok) {
        if (k == 0) {
            beta = 0.0;
            alpha = (double)((T)gamma / (T)delta);
        } else {
            beta = (double)((T)gamma / (T)gamma_old);
            alpha = (double)((T)gamma / ((T)delta - (T)beta * (T)gamma / (T)alpha));
        }
        if (!isfinite(alpha)) { status = WSPM_NAN; break; }
        T *pp = part + (int64_t)(red & 1) * 4 * nb;
        // ---- update phase (own rows only), 16-byte row groups
        {
            const T al = (T)alpha, bt = (T)beta;
            T v[2] = {T(0), T(0)};
            for (int l = N * (int)threadIdx.x; l < nl; l += N * (int)blockDim.x) {
                if (l + N <= nl) {
                    T zz[N], pv[N], sv[N], wv[N], xv[N], rv[N], dv[N];
                    VT::split(*reinterpret_cast<const V *>(z + r0 + l), zz);
                    VT::split(*reinterpret_cast<const V *>(RCG_P(kVP, l)), pv);
                    VT::split(*reinterpret_cast<const V *>(RCG_P(kVS, l)), sv);
                    VT::split(*reinterpret_cast<const V *>(RCG_P(kVW, l)), wv);
                    VT::split(*reinterpret_cast<const V *>(RCG_P(kVR, l)), rv);
                    VT::split(*reinterpret_cast<const V *>(kVX < NS ? RCG_P(kVX, l) : xg + r0 + l), xv);
                    if (kVD < NS) VT::split(*reinterpret_cast<const V *>(RCG_P(kVD, l)), dv);
                    else if (dg) VT::split(__ldg(reinterpret_cast<const V *>(dg + r0 + l)), dv);
                    else {
#pragma unroll
                        for (int q = 0; q < N; ++q) dv[q] = T(1);
                    }
#pragma unroll
                    for (int q = 0; q < N; ++q) {
                        pv[q] = fma(bt, pv[q], zz[q]);
                        sv[q] = fma(bt, sv[q], wv[q]);
                        xv[q] = fma(al, pv[q], xv[q]);
                        rv[q] = fma(-al, sv[q], rv[q]);
                        zz[q] = dv[q] * rv[q];
                        v[0] += rv[q] * zz[q];
                        v[1] += rv[q] * rv[q];
                    }
                    *reinterpret_cast<V *>(RCG_P(kVP, l)) = VT::join(pv);
                    *reinterpret_cast<V *>(RCG_P(kVS, l)) = VT::join(sv);
                    *reinterpret_cast<V *>(RCG_P(kVR, l)) = VT::join(rv);
                    *reinterpret_cast<V *>(kVX < NS ? RCG_P(kVX, l) : xg + r0 + l) = VT::join(xv);
                    *reinterpret_cast<V *>(z + r0 + l) = VT::join(zz);
                } else {
                    for (int q = 0; l + q < nl; ++q) {
                        const int lq = l + q;
                        const T pi = fma(bt, RCG(kVP, lq), z[r0 + lq]);
                        const T si = fma(bt, RCG(kVS, lq), RCG(kVW, lq));
                        RCG(kVP, lq) = pi;
                        RCG(kVS, lq) = si;
                        T *xp = kVX < NS ? RCG_P(kVX, lq) : xg + r0 + lq;
                        *xp = fma(al, pi, *xp);
                        const T ri = fma(-al, si, RCG(kVR, lq));
                        RCG(kVR, lq) = ri;
                        const T di = kVD < NS ? RCG(kVD, lq) : (dg ? dg[r0 + lq] : T(1));
                        const T zi = di * ri;
                        z[r0 + lq] = zi;
                        v[0] += ri * zi;
                        v[1] += ri * ri;
                    }
                }
            }
            block_sum<T, 2>(v);        // ends with a block barrier: every z store of this block is done
            if (threadIdx.x == 0) {
                pp[nb + blockIdx.x] = v[0];
                pp[2 * nb + blockIdx.x] = v[1];
                __threadfence();
                st_release_u32(zflag + blockIdx.x, (unsigned)(k + 1));
            }
        }
        // ---- SpMV phase: interior rows, then halo rows once the neighbours' z is published
        {
            T v[1] = {T(0)};
            if (dia) {
                ok = RCG_SPMV_DIA(v[0], (unsigned)(k + 1), true);
                if (!ok) break;
            } else {
                ok = wait_zflags(zflag, 0, nb - 1, (unsigned)(k + 1), bar);
                if (!ok) break;
                rcg_spmv_rows<T, MW>(0, nl, v[0], A, vals, r0, z, wbase);
            }
            block_sum<T, 1>(v);
            if (threadIdx.x == 0) pp[blockIdx.x] = v[0];
        }
        ++red;
        ok = count_barrier(bar, red * (unsigned)nb);
        if (!ok) break;
        T t3[3];
        reduce_partials_rows<T, 3>(pp, nb, t3);
        gamma_old = gamma;
        delta = (double)t3[0];
        gamma = (double)t3[1];
        rr = (double)t3[2];
        ++k;
        rs = dg ? rr : gamma;
        if (!(rs > atol2)) done = true;
        else if (k >= a.maxiter) { done = true; status = WSPM_MAXITER; }
        if (!isfinite(rs)) { done = true; status = WSPM_NAN; }
    }
    if (kVX < NS) {
        for (int l = threadIdx.x; l < nl; l += blockDim.x) xg[r0 + l] = RCG(kVX, l);
    }
#undef RCG
#undef RCG_P
#undef RCG_G
#undef RCG_SPMV_DIA
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        KrylovState *st = a.st;
        st->gamma = gamma; st->rr = rr; st->bs = bs; st->atol2 = atol2;
        st->alpha = alpha; st->beta = beta;
        st->k = k;
        st->status = ok ? status : WSPM_CUDA_ERROR;
        st->done = 1;
        st->ns = global_ns() - t_entry;
    }
}

// Launch geometry of the resident kernel: one block per SM, rows split in
// contiguous chunks, 6, 4 or 0 per-block vectors in shared memory.
struct RcgPlan {
    int grid, chunk, ns;
    size_t smem_bytes;
};

template <typename T>
static RcgPlan rcg_plan(int n) {
    static int sms = 0, optin = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    }
    RcgPlan pl;
    int g = sms > 0 ? sms : 1;
    const int need = (n + kSlice - 1) / kSlice;            // never more blocks than 32-row groups
    if (g > need) g = need;
    if (g > 1024) g = 1024;                                // partials [2][4][g] + [3][g] + flags fit the slot area
    if (g < 1) g = 1;
    pl.grid = g;
    pl.chunk = (((n + g - 1) / g) + kSlice - 1) & ~(kSlice - 1);
    const int64_t per_vec = (int64_t)pl.chunk * sizeof(T);
    const int64_t room = (int64_t)optin - 4096;            // static shared memory of the kernel < 4 KB
    pl.ns = room >= 6 * per_vec ? 6 : (room >= 4 * per_vec ? 4 : 0);
    pl.smem_bytes = (size_t)(pl.ns * per_vec);
    return pl;
}

template <typename T, int MW, int NS>
static cudaError_t rcg_launch(const RcgPlan &pl, const RcgArgs<T> &a, cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(cg_resident_kernel<T, MW, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)pl.smem_bytes);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(pl.grid);
    cfg.blockDim = dim3(kRcgBlock);
    cfg.dynamicSmemBytes = pl.smem_bytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, cg_resident_kernel<T, MW, NS>, a);
}

template <typename T>
int cg_persistent_enqueue(const Sell &A, const T *vals, const T *b, const double *b64, T *x, const T *dinv,
                          const CgBuffers<T> &w, double tol, double atol, int maxiter, bool zero_x0,
                          const double *tol_dev, cudaStream_t st, const int *skip) {
    // the 16-byte row groups need 16-byte aligned arrays
    const uintptr_t al = (uintptr_t)vals | (uintptr_t)x | (uintptr_t)w.z | (uintptr_t)w.r | (uintptr_t)w.p0 |
                         (uintptr_t)w.p1 | (uintptr_t)w.q | (uintptr_t)(dinv ? dinv : vals);
    if (al % 16) return WSPM_BAD_ARG;
    RcgArgs<T> a;
    a.A = A; a.vals = vals; a.b = b; a.b64 = b64; a.x = x; a.dinv = dinv;
    a.z = w.z;
    a.part = w.partials; a.st = w.st;
    a.bar = (GridBarrier *)&w.st->ticket[0];
    a.zflag = reinterpret_cast<unsigned int *>(w.partials + 16 * 1024);    // after 11 * grid <= 11264 slots
    a.tol = tol; a.atol = atol; a.tol_dev = tol_dev; a.maxiter = maxiter; a.zero_x0 = zero_x0 ? 1 : 0;
    a.skip = skip;
    // global homes of the vectors that stay off chip (x: the caller's array; M: read in place)
    a.gvec[kVR] = w.r; a.gvec[kVP] = w.p0; a.gvec[kVS] = w.p1; a.gvec[kVW] = w.q;
    a.gvec[kVX] = x;
    a.gvec[kVD] = nullptr;
    const RcgPlan pl = rcg_plan<T>(A.n_rows);
    a.chunk = pl.chunk;
    cudaError_t e = cudaSuccess;
    WSPM_WIDTH_DISPATCH(A.max_width, {
        if (pl.ns == 6) e = rcg_launch<T, MW, 6>(pl, a, st);
        else if (pl.ns == 4) e = rcg_launch<T, MW, 4>(pl, a, st);
        else e = rcg_launch<T, MW, 0>(pl, a, st);
    });
    return e == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

template int cg_persistent_enqueue<double>(const Sell &, const double *, const double *, const double *, double *,
                                           const double *, const CgBuffers<double> &, double, double, int, bool,
                                           const double *, cudaStream_t, const int *);
template int cg_persistent_enqueue<float>(const Sell &, const float *, const float *, const double *, float *,
                                          const float *, const CgBuffers<float> &, double, double, int, bool,
                                          const double *, cudaStream_t, const int *);

// ---------------------------------------------------------------- pipelined CG
// Pipelined Jacobi-CG (Ghysels & Vanroose, Parallel Computing 40 (2014)
// 224-238, Alg. 4) as one resident cooperative launch.  With M diagonal the
// recurrences of u = M r, q = M s and m = M w collapse into products with
// 1/diag taken on the fly, leaving
//   gamma = (r, u), delta = (w, u), rho = (r, r)     (reduction i, in flight)
//   n = A m,  m = M w                                (SpMV i, overlapping it)
//   beta = gamma/gamma_old, alpha = gamma/(delta - beta gamma/alpha_old)
//   z = n + beta z ; s = w + beta s ; p = M r + beta p
//   x += alpha p ; r -= alpha s ; w -= alpha z
// so the grid-wide reduction of iteration i travels while the block computes
// its SpMV: the scalars are read after the SpMV, not before it.  The iterates
// equal those of CG in exact arithmetic; the recurrence for w (w = A M r is
// never recomputed) lets the recursive residual drift from the true one by
// rounding, which is why this form serves the FP32 inner solve of the mixed
// path, where the outer FP64 refinement measures the true residual.
//
// Block b owns rows [b*chunk, (b+1)*chunk); r, w, s, p, z, n (and x when it
// fits) stay in shared memory.  m crosses blocks through two alternating
// global vectors: m_{i+1} is written into the vector that held m_{i-1}, which
// every block finished reading before it arrived at reduction i (a block
// writes only after passing that reduction).  Partial sums alternate between
// two buffers for the same reason.  One warp of each block waits for the
// reduction and sums the partials while the other warps run the SpMV (named
// barrier 1 among them), so the reduction latency leaves the critical path.
// Every wait is bounded like the other resident kernels.
enum PcgVec { kPR = 0, kPW, kPS, kPP, kPZ, kPN, kPX, kNumPcgVec };

template <typename T>
struct PcgArgs {
    Sell A;
    const T *vals;
    const T *b;
    const double *b64;
    T *x;
    const T *dinv;
    T *ex[2];              // exchange vectors: u0 in ex[0], then m_i in ex[(i + 1) & 1]
    int chunk;
    T *part;               // [2 parities][3][grid], then [1][grid] for the init
    unsigned int *flag;    // [grid] per-block exchange epoch
    KrylovState *st;
    GridBarrier *bar;
    double tol, atol;
    const double *tol_dev;
    const int *skip;       // as RcgArgs::skip
    int maxiter, zero_x0;
};

// OR of `pred` over the nthreads threads that use named barrier `id`.
__device__ __forceinline__ int bar_red_or(int id, int nthreads, int pred) {
    int r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.s32 p, %1, 0;\n\tbar.red.or.pred q, %2, %3, p;\n\t"
        "selp.s32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"(pred), "r"(id), "r"(nthreads)
        : "memory");
    return r;
}

// wait_zflags for a group of threads [0, nthr) of the block: the block-wide
// barrier (named = false) or named barrier 1 (named = true).
__device__ __forceinline__ bool wait_flags_group(const unsigned int *flag, int lo, int hi, unsigned int epoch,
                                                 GridBarrier *gb, int tid, int nthr, bool named) {
    int fail = 0;
    for (int c = lo + tid; c <= hi && !fail; c += nthr) {
        if (c == (int)blockIdx.x) continue;
        long long spins = 0;
        while (ld_acquire_u32(flag + c) < epoch) {
            if (++spins > kBarrierSpinLimit) { atomicExch(&gb->error, 1); fail = 1; break; }
            if ((spins & 1023) == 0 && *(volatile int *)&gb->error) { fail = 1; break; }
            __nanosleep(20);
        }
    }
    if (named) return bar_red_or(1, nthr, fail) == 0;
    return __syncthreads_or(fail) == 0;
}

// Bounded wait until the counting barrier has seen `target` arrivals (one thread).
__device__ __forceinline__ bool count_wait(GridBarrier *gb, unsigned int target) {
    long long spins = 0;
    while (ld_acquire_u32(&gb->mono) < target) {
        if (++spins > kBarrierSpinLimit) { atomicExch(&gb->error, 1); return false; }
        if ((spins & 1023) == 0 && *(volatile int *)&gb->error) return false;
        __nanosleep(20);
    }
    return (*(volatile int *)&gb->error) == 0;
}

// reduce_partials_rows done by a single warp (the same arithmetic in every
// block, so every block gets bitwise identical sums).  The loads of all NV rows
// are issued together: one L2 round trip per 256 blocks instead of one per row
// (with a round trip per row the reduction, not the SpMV, was the longer of the
// two at 148 blocks: partial sums ready 4.8 us into the iteration, 3.1 us now).
template <typename T, int NV>
__device__ __forceinline__ void warp_partials(const T *partials, int nb, T (&out)[NV]) {
    const int lane = threadIdx.x & 31;
    T acc[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) acc[j] = T(0);
    for (int b0 = 0; b0 < nb; b0 += 256) {
        T x[NV][8];
#pragma unroll
        for (int j = 0; j < NV; ++j)
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int b = b0 + lane + 32 * u;
                x[j][u] = b < nb ? __ldcg(partials + (int64_t)j * nb + b) : T(0);
            }
#pragma unroll
        for (int j = 0; j < NV; ++j)
#pragma unroll
            for (int u = 0; u < 8; ++u) acc[j] += x[j][u];
    }
#pragma unroll
    for (int j = 0; j < NV; ++j) out[j] = warp_sum(acc[j]);
}

// dst[l] = (A src)[r0 + l] over the block's rows, 16-byte groups, threads
// [0, nthr) of the block (round-robin like rcg_spmv_dia: interior groups
// first, the wait for the neighbours' flags before the first round with a
// halo group).  Returns false when that wait gave up.
template <typename T, int MW>
__device__ __forceinline__ bool pcg_spmv_dia(int nl, int lo_i, int hi_i, const T *__restrict__ vals,
                                             const int64_t *s_vo, int r0, int last, int nd, const int *s_off,
                                             const T *src, T *dst,
                                             const unsigned int *flag, int nbr_lo, int nbr_hi, unsigned int epoch,
                                             bool poll, GridBarrier *bar, int tid, int nthr, bool named) {
    using VT = Vec16<T>;
    constexpr int N = VT::N;
    const int ng = (nl + N - 1) / N;
    const int gi0 = lo_i / N, gi1 = hi_i / N;
    const int nint = gi1 - gi0, nlow = gi0;
    const int rounds = (ng + nthr - 1) / nthr;
    const int m_wait = poll ? nint / nthr : rounds;
    for (int m = 0; m < rounds; ++m) {
        if (m == m_wait && !wait_flags_group(flag, nbr_lo, nbr_hi, epoch, bar, tid, nthr, named)) return false;
        const int j = tid + m * nthr;
        if (j >= ng) continue;
        int g;
        if (j < nint) g = gi0 + j;
        else {
            const int h = j - nint;
            g = h < nlow ? h : gi1 + (h - nlow);
        }
        const int l = g * N, i = r0 + l;
        if (l + N <= nl) {
            T w[N];
            dia_group_z<T, MW>(vals, s_vo, i, last, nd, s_off, src, w);
            *reinterpret_cast<typename VT::V *>(dst + l) = VT::join(w);
        } else {
            for (int q = 0; l + q < nl; ++q) dst[l + q] = dia_row_z<T, MW>(vals, s_vo, i + q, last, nd, s_off, src);
        }
    }
    if (m_wait >= rounds && poll && !wait_flags_group(flag, nbr_lo, nbr_hi, epoch, bar, tid, nthr, named))
        return false;
    return true;
}

constexpr int kInitBatch = 8;   // rows per thread whose loads the start-up loops issue together
// Threads per block of the pipelined kernel: for FP32 systems of at most 8 diagonals 32 warps per SM hide more
// of the SpMV's gather latency than 16 (the compiler fits that instance in 64 registers without spills: 9.7 vs
// 10.3 us per FP32 iteration at 1024^2); the other instances would spill at 64 registers and keep 512.
template <typename T, int MW>
constexpr int pcg_block() { return (sizeof(T) == 4 && MW <= 8) ? 1024 : kRcgBlock; }

template <typename T, int MW, bool XS, bool WS>
__global__ void __launch_bounds__(pcg_block<T, MW>(), 1) pcg_resident_kernel(PcgArgs<T> a) {
    using VT = Vec16<T>;
    using V = typename VT::V;
    constexpr int N = VT::N;
    extern __shared__ __align__(16) unsigned char rcg_smem[];
    __shared__ int s_off[MW];
    __shared__ int64_t s_vo[MW];
    __shared__ T s_scal[3];
    __shared__ int s_ok;
    T *const sm = reinterpret_cast<T *>(rcg_smem);
    if (resident_skip(a.skip, a.st)) return;
    const unsigned long long t_entry = (blockIdx.x == 0 && threadIdx.x == 0) ? global_ns() : 0ull;
    const int n = a.A.n_rows;
    const int nb = gridDim.x;
    const int chunk = a.chunk;
    const int r0 = blockIdx.x * chunk;
    const int r1 = min(n, r0 + chunk);
    const int nl = max(0, r1 - r0);
    const int TB = blockDim.x;
    const int tid = threadIdx.x;
    unsigned int gen = tid == 0 ? ld_acquire_u32(&a.bar->gen) : 0u;
    if (tid == 0) {
        a.flag[blockIdx.x] = 0u;
        if (blockIdx.x == 0) a.bar->mono = 0u;
    }
    const T *const vals = a.vals;
    const T *const dg = a.dinv;
    T *const xg = a.x;
    T *const ex0 = a.ex[0];
    T *const ex1 = a.ex[1];
    T *const part = a.part;
    unsigned int *const flag = a.flag;
    GridBarrier *const bar = a.bar;
    T *const vR = sm + kPR * chunk, *const vW = sm + kPW * chunk, *const vS = sm + kPS * chunk;
    T *const vP = sm + kPP * chunk, *const vZ = sm + kPZ * chunk, *const vN = sm + kPN * chunk;
    T *const vX = XS ? sm + kPX * chunk : xg + r0;   // x: on chip when it fits, else the caller's array
    const int last = n - 1;
    int nd = 0;                // diagonals that can hold nonzeros (A.live)
    int mn = 0, mx = 0;
    for (int k = 0; k < a.A.n_diags; ++k) {
        if (!dia_live(a.A, k)) continue;
        const int o = __ldg(a.A.diag_off + k);
        if (tid == 0) {
            s_off[nd] = o;
            s_vo[nd] = (int64_t)k * a.A.ld;
        }
        ++nd;
        mn = min(mn, o);
        mx = max(mx, o);
    }
    const int lo_i = min(nl, (-mn + N - 1) / N * N);
    const int hi_i = max(lo_i, (nl - mx) / N * N);
    int nbr_lo = min(nb - 1, max(0, r0 + mn) / chunk);
    int nbr_hi = min(nb - 1, min(n - 1, r1 - 1 + mx) / chunk);
    if (nl == 0) { nbr_lo = 1; nbr_hi = 0; }
    __syncthreads();
    // ---- init: r = b - A x0, p = s = z = 0, u0 = M r -> ex0.  A thread's rows are
    // l = tid + j TB; with x0 = 0 the loads of kInitBatch of them are issued before
    // any store (one memory latency per batch instead of one per row), and the
    // per-thread sum keeps the row order.
    {
        T v[1] = {T(0)};
        if (a.zero_x0) {
            for (int l0 = tid; l0 < nl; l0 += kInitBatch * TB) {
                T bq[kInitBatch], dq[kInitBatch];
#pragma unroll
                for (int q = 0; q < kInitBatch; ++q) {
                    const int l = l0 + q * TB;
                    bq[q] = T(0);
                    dq[q] = T(1);
                    if (l < nl) {
                        bq[q] = a.b64 ? (T)a.b64[r0 + l] : a.b[r0 + l];
                        if (dg) dq[q] = dg[r0 + l];
                    }
                }
#pragma unroll
                for (int q = 0; q < kInitBatch; ++q) {
                    const int l = l0 + q * TB;
                    if (l < nl) {
                        vX[l] = T(0);      // on chip, copied to x at the end; else x itself
                        vR[l] = bq[q];
                        vS[l] = T(0);
                        vP[l] = T(0);
                        vZ[l] = T(0);
                        ex0[r0 + l] = dq[q] * bq[q];
                        v[0] += bq[q] * bq[q];
                    }
                }
            }
        } else {
            for (int l = tid; l < nl; l += TB) {
                const int i = r0 + l;
                const T bi = a.b64 ? (T)a.b64[i] : a.b[i];
                if (XS) vX[l] = xg[i];
                const T ri = bi - dia_row_z<T, MW>(vals, s_vo, i, last, nd, s_off, xg);
                const T di = dg ? dg[i] : T(1);
                vR[l] = ri;
                vS[l] = T(0);
                vP[l] = T(0);
                vZ[l] = T(0);
                ex0[i] = di * ri;
                v[0] += bi * bi;
            }
        }
        block_sum<T, 1>(v);
        if (tid == 0) part[6 * (int64_t)nb + blockIdx.x] = v[0];
    }
    bool ok = grid_barrier(bar, nb, gen);     // u0 complete everywhere; flags and mono reset
    T binit[1];
    reduce_partials_rows<T, 1>(part + 6 * (int64_t)nb, nb, binit);
    const double bs = (double)binit[0];
    const double tl = a.tol_dev ? *a.tol_dev : a.tol;
    const double atol2 = fmax(tl * tl * bs, a.atol * a.atol);
    // publish the partials (r, Mr), (w, Mr), (r, r) of the block's rows, arrive, raise the exchange flag
    auto publish = [&](T *pp, unsigned int epoch, T (&v)[3]) {
        block_sum<T, 3>(v);        // ends with a block barrier: every m store of this block is done
        if (tid == 0) {
            pp[blockIdx.x] = v[0];
            pp[nb + blockIdx.x] = v[1];
            pp[2 * nb + blockIdx.x] = v[2];
            // one release fence orders the partials and (after the block barrier) every m store of
            // the block before both the arrival and the flag, which readers load with acquire
            fence_acq_rel_gpu();
            atomicAdd(&bar->mono, 1u);
            st_relaxed_u32(flag + blockIdx.x, epoch);
        }
    };
    // w0 = A u0 (the grid barrier published u0), then m0 = M w0 and reduction 0
    if (ok) {
        ok = pcg_spmv_dia<T, MW>(nl, lo_i, hi_i, vals, s_vo, r0, last, nd, s_off, ex0, vW, flag, nbr_lo, nbr_hi, 0u,
                                 false, bar, tid, TB, false);
        __syncthreads();
        T v[3] = {T(0), T(0), T(0)};
        for (int l0 = tid; l0 < nl; l0 += kInitBatch * TB) {
            T dq[kInitBatch];
#pragma unroll
            for (int q = 0; q < kInitBatch; ++q) {
                const int l = l0 + q * TB;
                dq[q] = (dg && l < nl) ? dg[r0 + l] : T(1);
            }
#pragma unroll
            for (int q = 0; q < kInitBatch; ++q) {
                const int l = l0 + q * TB;
                if (l < nl) {
                    const T ri = vR[l], wi = vW[l];
                    const T ui = dq[q] * ri;
                    ex1[r0 + l] = dq[q] * wi;
                    v[0] += ri * ui;
                    v[1] += wi * ui;
                    v[2] += ri * ri;
                }
            }
        }
        publish(part, 2u, v);
    }
    double gamma = 0.0, delta = 0.0, rho = 0.0, gamma_old = 1.0, alpha = 0.0, beta = 0.0;
    int k = 0, status = WSPM_OK;
    const int nthr = WS ? TB - 32 : TB;
    const bool red_warp = WS && tid >= TB - 32;
    while (ok) {
        // ---- SpMV n_k = A m_k (m_k in ex[(k + 1) & 1]) while reduction k travels
        const T *msrc = (k & 1) ? ex0 : ex1;
        const T *pp = part + (int64_t)(k & 1) * 3 * nb;
        const unsigned int target = (unsigned)(k + 1) * (unsigned)nb;
        // 1/diag of the thread's first update group, loaded after its SpMV share so that the loads are in
        // flight during the block barrier
        V dreg0 = V();
        auto load_dreg = [&]() {
            if (dg && N * tid + N <= nl) dreg0 = __ldg(reinterpret_cast<const V *>(dg + r0 + N * tid));
        };
        if (WS) {
            if (!red_warp) {
                const bool o = pcg_spmv_dia<T, MW>(nl, lo_i, hi_i, vals, s_vo, r0, last, nd, s_off, msrc, vN, flag,
                                                   nbr_lo, nbr_hi, (unsigned)(k + 2), true, bar, tid, nthr, true);
                if (tid == 0) s_ok = o ? 1 : 0;
            } else {
                int w_ok = 1;
                if ((tid & 31) == 0) w_ok = count_wait(bar, target) ? 1 : 0;
                w_ok = __shfl_sync(0xffffffffu, w_ok, 0);
                __syncwarp();
                T t3[3];
                warp_partials<T, 3>(pp, nb, t3);
                if ((tid & 31) == 0) {
                    s_scal[0] = t3[0];
                    s_scal[1] = t3[1];
                    s_scal[2] = t3[2];
                    if (!w_ok) atomicExch(&bar->error, 1);
                }
            }
            load_dreg();
            __syncthreads();
            ok = s_ok != 0 && (*(volatile int *)&bar->error) == 0;
            __syncthreads();       // every thread has read s_ok before it is written again
        } else {
            ok = pcg_spmv_dia<T, MW>(nl, lo_i, hi_i, vals, s_vo, r0, last, nd, s_off, msrc, vN, flag, nbr_lo, nbr_hi,
                                     (unsigned)(k + 2), true, bar, tid, TB, false);
            load_dreg();
            if (tid == 0) s_ok = count_wait(bar, target) ? 1 : 0;
            __syncthreads();
            ok = ok && s_ok != 0;
            T t3[3];
            reduce_partials_rows<T, 3>(pp, nb, t3);
            if (tid == 0) {
                s_scal[0] = t3[0];
                s_scal[1] = t3[1];
                s_scal[2] = t3[2];
            }
            __syncthreads();
        }
        if (!ok) break;
        gamma = (double)s_scal[0];
        delta = (double)s_scal[1];
        rho = (double)s_scal[2];
        const double rs = dg ? rho : gamma;
        if (!isfinite(rs)) { status = WSPM_NAN; break; }
        if (!(rs > atol2)) break;
        if (k >= a.maxiter) { status = WSPM_MAXITER; break; }
        if (k == 0) {
            beta = 0.0;
            alpha = (double)((T)gamma / (T)delta);
        } else {
            beta = (double)((T)gamma / (T)gamma_old);
            alpha = (double)((T)gamma / ((T)delta - (T)beta * (T)gamma / (T)alpha));
        }
        if (!isfinite(alpha)) { status = WSPM_NAN; break; }
        // ---- update: x_{k+1}, r, w, s, p, z; m_{k+1} = M w_{k+1} -> ex[k & 1]; reduction k + 1
        T *mdst = (k & 1) ? ex1 : ex0;
        T *pn = part + (int64_t)((k + 1) & 1) * 3 * nb;
        {
            const T al = (T)alpha, bt = (T)beta;
            T v[3] = {T(0), T(0), T(0)};
            int rnd = 0;
            for (int l = N * tid; l < nl; l += N * TB, ++rnd) {
                if (l + N <= nl) {
                    T nv[N], zv[N], sv[N], pv[N], xv[N], rv[N], wv[N], dv[N];
                    VT::split(*reinterpret_cast<const V *>(vN + l), nv);
                    VT::split(*reinterpret_cast<const V *>(vZ + l), zv);
                    VT::split(*reinterpret_cast<const V *>(vS + l), sv);
                    VT::split(*reinterpret_cast<const V *>(vP + l), pv);
                    VT::split(*reinterpret_cast<const V *>(vX + l), xv);
                    VT::split(*reinterpret_cast<const V *>(vR + l), rv);
                    VT::split(*reinterpret_cast<const V *>(vW + l), wv);
                    if (dg) VT::split(rnd == 0 ? dreg0 : __ldg(reinterpret_cast<const V *>(dg + r0 + l)), dv);
                    else {
#pragma unroll
                        for (int q = 0; q < N; ++q) dv[q] = T(1);
                    }
                    T mv[N];
#pragma unroll
                    for (int q = 0; q < N; ++q) {
                        zv[q] = fma(bt, zv[q], nv[q]);
                        sv[q] = fma(bt, sv[q], wv[q]);
                        pv[q] = fma(bt, pv[q], dv[q] * rv[q]);
                        xv[q] = fma(al, pv[q], xv[q]);
                        rv[q] = fma(-al, sv[q], rv[q]);
                        wv[q] = fma(-al, zv[q], wv[q]);
                        const T u = dv[q] * rv[q];
                        mv[q] = dv[q] * wv[q];
                        v[0] += rv[q] * u;
                        v[1] += wv[q] * u;
                        v[2] += rv[q] * rv[q];
                    }
                    *reinterpret_cast<V *>(vZ + l) = VT::join(zv);
                    *reinterpret_cast<V *>(vS + l) = VT::join(sv);
                    *reinterpret_cast<V *>(vP + l) = VT::join(pv);
                    *reinterpret_cast<V *>(vX + l) = VT::join(xv);
                    *reinterpret_cast<V *>(vR + l) = VT::join(rv);
                    *reinterpret_cast<V *>(vW + l) = VT::join(wv);
                    *reinterpret_cast<V *>(mdst + r0 + l) = VT::join(mv);
                } else {
                    for (int q = 0; l + q < nl; ++q) {
                        const int lq = l + q;
                        const T di = dg ? dg[r0 + lq] : T(1);
                        const T zi = fma(bt, vZ[lq], vN[lq]);
                        const T si = fma(bt, vS[lq], vW[lq]);
                        const T pi = fma(bt, vP[lq], di * vR[lq]);
                        const T xi = fma(al, pi, vX[lq]);
                        const T ri = fma(-al, si, vR[lq]);
                        const T wi = fma(-al, zi, vW[lq]);
                        const T u = di * ri;
                        vZ[lq] = zi; vS[lq] = si; vP[lq] = pi; vX[lq] = xi; vR[lq] = ri; vW[lq] = wi;
                        mdst[r0 + lq] = di * wi;
                        v[0] += ri * u;
                        v[1] += wi * u;
                        v[2] += ri * ri;
                    }
                }
            }
            publish(pn, (unsigned)(k + 3), v);
        }
        gamma_old = gamma;
        ++k;
    }
    if (XS) {
        __syncthreads();
        for (int l = tid; l < nl; l += TB) xg[r0 + l] = vX[l];
    }
    if (blockIdx.x == 0 && tid == 0) {
        KrylovState *st = a.st;
        st->gamma = gamma; st->rr = rho; st->bs = bs; st->atol2 = atol2;
        st->alpha = alpha; st->beta = beta;
        st->k = k;
        st->status = ok ? status : WSPM_CUDA_ERROR;
        st->done = 1;
        st->ns = global_ns() - t_entry;
    }
}

template <typename T, int MW, bool XS, bool WS>
static cudaError_t pcg_launch(int grid, size_t smem, const PcgArgs<T> &a, cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(pcg_resident_kernel<T, MW, XS, WS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(pcg_block<T, MW>());
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, pcg_resident_kernel<T, MW, XS, WS>, a);
}

template <typename T>
int pcg_persistent_enqueue(const Sell &A, const T *vals, const T *b, const double *b64, T *x, const T *dinv,
                           const CgBuffers<T> &w, double tol, double atol, int maxiter, bool zero_x0,
                           const double *tol_dev, cudaStream_t st, bool warp_specialized, const int *skip) {
    if (A.n_diags <= 0 || A.n_diags > 16) return WSPM_UNSUPPORTED;       // DIA patterns only
    const uintptr_t al = (uintptr_t)vals | (uintptr_t)x | (uintptr_t)w.z | (uintptr_t)w.q |
                         (uintptr_t)(dinv ? dinv : vals);
    if (al % 16) return WSPM_BAD_ARG;
    const RcgPlan pl = rcg_plan<T>(A.n_rows);
    static int optin = 0;
    if (optin == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    }
    const int64_t per_vec = (int64_t)pl.chunk * sizeof(T);
    const int64_t room = (int64_t)optin - 4096;
    int nsv;
    if (room >= kNumPcgVec * per_vec) nsv = kNumPcgVec;
    else if (room >= (kNumPcgVec - 1) * per_vec) nsv = kNumPcgVec - 1;
    else return WSPM_UNSUPPORTED;                                        // too many rows per block
    PcgArgs<T> a;
    a.A = A; a.vals = vals; a.b = b; a.b64 = b64; a.x = x; a.dinv = dinv;
    a.ex[0] = w.z; a.ex[1] = w.q;
    a.chunk = pl.chunk;
    a.part = w.partials; a.st = w.st;
    a.bar = (GridBarrier *)&w.st->ticket[0];
    a.flag = reinterpret_cast<unsigned int *>(w.partials + 16 * 1024);   // after 7 * grid <= 7168 slots
    a.tol = tol; a.atol = atol; a.tol_dev = tol_dev; a.maxiter = maxiter; a.zero_x0 = zero_x0 ? 1 : 0;
    a.skip = skip;
    const size_t smem = (size_t)(nsv * per_vec);
    cudaError_t e = cudaSuccess;
    const bool xs = nsv == kNumPcgVec;
#define WSPM_PCG(MW_)                                                                              \
    do {                                                                                           \
        if (xs) e = warp_specialized ? pcg_launch<T, MW_, true, true>(pl.grid, smem, a, st)        \
                                     : pcg_launch<T, MW_, true, false>(pl.grid, smem, a, st);      \
        else e = warp_specialized ? pcg_launch<T, MW_, false, true>(pl.grid, smem, a, st)          \
                                  : pcg_launch<T, MW_, false, false>(pl.grid, smem, a, st);        \
    } while (0)
    if (A.n_diags <= 8) WSPM_PCG(8);
    else WSPM_PCG(16);
#undef WSPM_PCG
    return e == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

template <typename T>
bool pcg_eligible(const Sell &A) {
    if (A.n_diags <= 0 || A.n_diags > 16) return false;
    const RcgPlan pl = rcg_plan<T>(A.n_rows);
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return (int64_t)optin - 4096 >= (kNumPcgVec - 1) * (int64_t)pl.chunk * (int64_t)sizeof(T);
}
template bool pcg_eligible<float>(const Sell &);
template bool pcg_eligible<double>(const Sell &);

template int pcg_persistent_enqueue<double>(const Sell &, const double *, const double *, const double *, double *,
                                            const double *, const CgBuffers<double> &, double, double, int, bool,
                                            const double *, cudaStream_t, bool, const int *);
template int pcg_persistent_enqueue<float>(const Sell &, const float *, const float *, const double *, float *,
                                           const float *, const CgBuffers<float> &, double, double, int, bool,
                                           const double *, cudaStream_t, bool, const int *);

// ---------------------------------------------------------------- BiCGSTAB
// Templated on the vector/matrix type T: FP64 for the plain path, FP32 for the
// mixed path's inner corrections (FP32 vectors and FP32 accumulation; the
// solver scalars are kept in the FP64 KrylovState).  Inner-solve options:
// b64 (the FP64 residual of the refinement loop, converted on the fly), x0 ==
// NULL (start from zero), tol_dev (relative tolerance read on the device).
template <typename T>
__device__ __forceinline__ T rhs_at(const T *b, const double *b64, int i) {
    return b64 ? (T)b64[i] : b[i];
}

template <typename T, int MW>
__global__ void __launch_bounds__(kBlock) bicg_init_kernel(Sell A, const T *__restrict__ vals,
                                                           const T *__restrict__ b, const double *__restrict__ b64,
                                                           const T *x0, T *x, T *r, T *rhat, T *p, T *q, T *partials,
                                                           KrylovState *st, double tol, double atol,
                                                           const double *tol_dev, int maxiter,
                                                           cudaGraphConditionalHandle cond, int use_cond) {
    T v[2] = {T(0), T(0)};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_rows; i += gridDim.x * blockDim.x) {
        const T bi = rhs_at(b, b64, i);
        T ri = bi;
        if (x0) ri = bi - sell_row<T, MW>(A, vals, i, [&](int c) { return x0[c]; });
        else x[i] = T(0);
        r[i] = ri; rhat[i] = ri; p[i] = ri; q[i] = ri;
        v[0] += ri * ri;
        v[1] += bi * bi;
    }
    if (publish_partials<T, 2>(v, partials, &st->ticket[2])) {
        T tot[2];
        final_sum<T, 2>(partials, tot, &st->ticket[2]);
        if (threadIdx.x == 0) {
            const double rr = (double)tot[0], bs = (double)tot[1];
            const double tl = tol_dev ? *tol_dev : tol;
            st->rr = rr; st->bs = bs;
            st->atol2 = fmax(tl * tl * bs, atol * atol);
            st->rho = st->alpha = st->omega = 1.0;
            st->rho_next = rr;
            st->k = 0; st->status = WSPM_OK; st->exit_early = 0;
            int done = !(rr > st->atol2 && 0 < maxiter);
            if (!isfinite(rr)) { done = 1; st->status = WSPM_NAN; }
            st->done = done;
            set_cond(cond, use_cond, done ? 0u : 1u);
        }
    }
}

template <typename T>
__global__ void bicg_p_kernel(int n, const T *__restrict__ r, T *p, const T *__restrict__ q, T *phat,
                              const T *__restrict__ dinv, const KrylovState *st) {
    if (st->done) return;
    const T beta = (T)(st->rho_next / st->rho * st->alpha / st->omega);
    const T om = (T)st->omega;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const T pi = r[i] + beta * (p[i] - om * q[i]);
        p[i] = pi;
        phat[i] = dinv ? dinv[i] * pi : pi;
    }
}

template <typename T, int MW>
__global__ void __launch_bounds__(kBlock) bicg_q_kernel(Sell A, const T *__restrict__ vals, const T *__restrict__ phat,
                                                        const T *__restrict__ rhat, T *q, T *partials,
                                                        KrylovState *st) {
    if (st->done) return;
    T v[1] = {T(0)};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_rows; i += gridDim.x * blockDim.x) {
        const T qi = sell_row<T, MW>(A, vals, i, [&](int c) { return __ldg(phat + c); });
        q[i] = qi;
        v[0] += rhat[i] * qi;
    }
    if (publish_partials<T, 1>(v, partials, &st->ticket[0])) {
        T tot[1];
        final_sum<T, 1>(partials, tot, &st->ticket[0]);
        if (threadIdx.x == 0) {
            st->sigma = (double)tot[0];
            st->rho = st->rho_next;                       // rho of this iteration
            st->alpha = st->rho_next / (double)tot[0];    // alpha of this iteration
        }
    }
}

template <typename T, int MW>
__global__ void __launch_bounds__(kBlock) bicg_t_kernel(Sell A, const T *__restrict__ vals, const T *__restrict__ r,
                                                        const T *__restrict__ q, const T *__restrict__ dinv, T *t,
                                                        T *partials, KrylovState *st) {
    if (st->done) return;
    const T alpha = (T)st->alpha;
    T v[3] = {T(0), T(0), T(0)};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_rows; i += gridDim.x * blockDim.x) {
        const T ti = sell_row<T, MW>(A, vals, i, [&](int c) {
            const T sc = __ldg(r + c) - alpha * __ldg(q + c);
            return dinv ? __ldg(dinv + c) * sc : sc;
        });
        const T si = r[i] - alpha * q[i];
        t[i] = ti;
        v[0] += si * si;
        v[1] += ti * si;
        v[2] += ti * ti;
    }
    if (publish_partials<T, 3>(v, partials, &st->ticket[1])) {
        T tot[3];
        final_sum<T, 3>(partials, tot, &st->ticket[1]);
        if (threadIdx.x == 0) {
            st->ss = (double)tot[0]; st->ts = (double)tot[1]; st->tt = (double)tot[2];
            st->omega = st->ts / st->tt;
            st->exit_early = st->ss < st->atol2;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kBlock) bicg_x_kernel(int n, T *x, T *r, const T *__restrict__ rhat,
                                                        const T *__restrict__ p, const T *__restrict__ q,
                                                        const T *__restrict__ t, const T *__restrict__ dinv,
                                                        T *partials, KrylovState *st, int maxiter,
                                                        cudaGraphConditionalHandle cond, int use_cond) {
    if (st->done) return;
    const T alpha = (T)st->alpha, omega = (T)st->omega;
    const int early = st->exit_early;
    T v[2] = {T(0), T(0)};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const T si = r[i] - alpha * q[i];
        const T di = dinv ? dinv[i] : T(1);
        const T phat = dinv ? di * p[i] : p[i];
        const T shat = dinv ? di * si : si;
        T ri;
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
    if (publish_partials<T, 2>(v, partials, &st->ticket[2])) {
        T tot[2];
        final_sum<T, 2>(partials, tot, &st->ticket[2]);
        if (threadIdx.x == 0) {
            const double rr = (double)tot[0];
            st->rr = rr;
            st->rho_next = (double)tot[1];
            int k = (st->omega == 0.0 || st->alpha == 0.0) ? -11 : st->k + 1;
            if (st->rho == 0.0) k = -10;
            st->k = k;
            int done = !(rr > st->atol2 && k < maxiter && k >= 0);
            if (k < 0) st->status = WSPM_BREAKDOWN;
            else if (done && rr > st->atol2) st->status = WSPM_MAXITER;
            if (!isfinite(rr)) { done = 1; st->status = WSPM_NAN; }
            st->done = done;
            set_cond(cond, use_cond, done ? 0u : 1u);
        }
    }
}

template <typename T>
void bicgstab_enqueue_init(const Sell &A, const T *vals, const T *b, const double *b64, const T *x0, T *x,
                           const BicgBuffers<T> &w, double tol, double atol, const double *tol_dev, int maxiter,
                           cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st) {
    const int nb = reduction_blocks(A.n_rows);
    if (x0 && x != x0) copy_kernel<T><<<nb, kBlock, 0, st>>>(x0, x, A.n_rows);
    WSPM_WIDTH_DISPATCH(A.max_width,
                        bicg_init_kernel<T, MW><<<nb, kBlock, 0, st>>>(A, vals, b, b64, x0, x, w.r, w.rhat, w.p, w.q,
                                                                       w.partials, w.st, tol, atol, tol_dev, maxiter,
                                                                       cond, use_cond));
}

template <typename T>
void bicgstab_enqueue_body(const Sell &A, const T *vals, T *x, const T *dinv, const BicgBuffers<T> &w, int maxiter,
                           cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st) {
    const int nb = reduction_blocks(A.n_rows);
    bicg_p_kernel<T><<<nb, kBlock, 0, st>>>(A.n_rows, w.r, w.p, w.q, w.phat, dinv, w.st);
    WSPM_WIDTH_DISPATCH(A.max_width,
                        bicg_q_kernel<T, MW><<<nb, kBlock, 0, st>>>(A, vals, w.phat, w.rhat, w.q, w.partials, w.st));
    WSPM_WIDTH_DISPATCH(A.max_width,
                        bicg_t_kernel<T, MW><<<nb, kBlock, 0, st>>>(A, vals, w.r, w.q, dinv, w.t, w.partials, w.st));
    bicg_x_kernel<T><<<nb, kBlock, 0, st>>>(A.n_rows, x, w.r, w.rhat, w.p, w.q, w.t, dinv, w.partials, w.st, maxiter,
                                            cond, use_cond);
}

template void bicgstab_enqueue_init<double>(const Sell &, const double *, const double *, const double *,
                                            const double *, double *, const BicgBuffers<double> &, double, double,
                                            const double *, int, cudaGraphConditionalHandle, int, cudaStream_t);
template void bicgstab_enqueue_init<float>(const Sell &, const float *, const float *, const double *, const float *,
                                           float *, const BicgBuffers<float> &, double, double, const double *, int,
                                           cudaGraphConditionalHandle, int, cudaStream_t);
template void bicgstab_enqueue_body<double>(const Sell &, const double *, double *, const double *,
                                            const BicgBuffers<double> &, int, cudaGraphConditionalHandle, int,
                                            cudaStream_t);
template void bicgstab_enqueue_body<float>(const Sell &, const float *, float *, const float *,
                                           const BicgBuffers<float> &, int, cudaGraphConditionalHandle, int,
                                           cudaStream_t);

// ---------------------------------------------------------------- GMRES(m)
constexpr int kMaxRestart = 32;
constexpr int kMaxDots = kMaxRestart + 2;

// Templated like BiCGSTAB: basis V, w and the reductions in T; the small
// Hessenberg matrix, the least-squares solve and the scalars in FP64.
template <typename T>
__device__ __forceinline__ double type_eps() { return sizeof(T) == 4 ? (double)FLT_EPSILON : DBL_EPSILON; }

// r = M (b - A x) into dst; ||r||^2 (and, at init, ||b||^2, ||M b||^2).
// x == NULL at init: x starts from zero (xz is then cleared).
template <typename T, int MW>
__global__ void __launch_bounds__(kBlock) gm_residual_kernel(Sell A, const T *__restrict__ vals,
                                                             const T *__restrict__ b, const double *__restrict__ b64,
                                                             const T *x, T *xz, const T *__restrict__ dinv, T *dst,
                                                             T *partials, KrylovState *st, int is_init, double tol,
                                                             double atol, const double *tol_dev, int maxiter,
                                                             cudaGraphConditionalHandle cond, int use_cond) {
    if (!is_init && st->done) return;
    T v[3] = {T(0), T(0), T(0)};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_rows; i += gridDim.x * blockDim.x) {
        const T d = dinv ? dinv[i] : T(1);
        const T bi = rhs_at(b, b64, i);
        T ri;
        if (x) {
            ri = d * (bi - sell_row<T, MW>(A, vals, i, [&](int c) { return x[c]; }));
        } else {
            ri = d * bi;
            xz[i] = T(0);
        }
        dst[i] = ri;
        v[0] += ri * ri;
        v[1] += bi * bi;
        v[2] += (d * bi) * (d * bi);
    }
    if (publish_partials<T, 3>(v, partials, &st->ticket[2])) {
        T tot[3];
        final_sum<T, 3>(partials, tot, &st->ticket[2]);
        if (threadIdx.x == 0) {
            double rn = sqrt((double)tot[0]);
            if (!(rn > type_eps<T>())) rn = 0.0;
            st->rnorm = rn;
            st->inv_wn = rn > 0.0 ? 1.0 / rn : 0.0;
            if (is_init) {
                const double bn = sqrt((double)tot[1]);
                const double tl = tol_dev ? *tol_dev : tol;
                st->b_norm = bn;
                st->mb_norm = sqrt((double)tot[2]);
                const double at = fmax(tl * bn, atol);
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
            if (!isfinite((double)tot[0])) { done = 1; st->status = WSPM_NAN; }
            st->done = done;
            set_cond(cond, use_cond, done ? 0u : 1u);
        }
    }
}

template <typename T>
__global__ void gm_scale_kernel(int n, T *v, const KrylovState *st) {
    if (st->done || st->broken) return;
    const T s = (T)st->inv_wn;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] *= s;
}

// phase 0: w = M A V_j, dots V_k.w (k <= j) and ||w||^2
// phase 1: w -= V h1 ; dots V_k.w
// phase 2: w -= V h2 ; ||w||^2, then H column j and breakdown test
template <typename T, int MW>
__global__ void __launch_bounds__(kBlock) gm_arnoldi_kernel(Sell A, const T *__restrict__ vals,
                                                            const T *__restrict__ dinv, const T *V, T *w, double *H,
                                                            double *hbuf, T *partials, KrylovState *st, int j, int m,
                                                            int phase, int64_t ld) {
    if (st->done || st->broken) return;
    const int n = A.n_rows;
    const int nd = j + 1;
    T v[kMaxDots];
#pragma unroll
    for (int k = 0; k < kMaxDots; ++k) v[k] = T(0);
    T h[kMaxRestart + 1];
    if (phase > 0) {
        const double *src = hbuf + (phase - 1) * (kMaxRestart + 1);
#pragma unroll
        for (int k = 0; k <= kMaxRestart; ++k) h[k] = k < nd ? (T)src[k] : T(0);
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        T wi;
        if (phase == 0) {
            const T *vj = V + (int64_t)j * ld;
            wi = sell_row<T, MW>(A, vals, i, [&](int c) { return __ldg(vj + c); });
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
    if (publish_partials<T, kMaxDots>(v, partials, &st->ticket[phase == 2 ? 1 : 0])) {
        T tot[kMaxDots];
        final_sum<T, kMaxDots>(partials, tot, &st->ticket[phase == 2 ? 1 : 0]);
        if (threadIdx.x == 0) {
            if (phase == 0) {
                st->wn0 = sqrt((double)tot[kMaxDots - 1]);
                for (int k = 0; k < nd; ++k) hbuf[k] = (double)tot[k];
            } else if (phase == 1) {
                for (int k = 0; k < nd; ++k) hbuf[(kMaxRestart + 1) + k] = (double)tot[k];
            } else {
                double *col = H + (int64_t)j * (m + 1);
                for (int k = 0; k < nd; ++k) col[k] = hbuf[k] + hbuf[(kMaxRestart + 1) + k];
                double wn = sqrt((double)tot[kMaxDots - 1]);
                const double thresh = type_eps<T>() * st->wn0;
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
template <typename T>
__global__ void gm_next_kernel(int n, T *V, const T *__restrict__ w, const KrylovState *st, int j, int64_t ld) {
    if (st->done || st->steps != j + 1) return;
    const T s = (T)st->inv_wn;
    T *dst = V + (int64_t)(j + 1) * ld;
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

template <typename T>
__global__ void gm_update_kernel(int n, T *x, const T *V, const double *__restrict__ y, const KrylovState *st,
                                 int64_t ld) {
    if (st->done) return;
    const int ns = st->steps;
    T yl[kMaxRestart];
#pragma unroll
    for (int k = 0; k < kMaxRestart; ++k) yl[k] = k < ns ? (T)y[k] : T(0);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        T acc = T(0);
#pragma unroll
        for (int k = 0; k < kMaxRestart; ++k)
            if (k < ns) acc += yl[k] * V[(int64_t)k * ld + i];
        x[i] += acc;
    }
}

template <typename T>
void gmres_enqueue_init(const Sell &A, const T *vals, const T *b, const double *b64, const T *x0, T *x,
                        const T *dinv, const GmresBuffers<T> &w, double tol, double atol, const double *tol_dev,
                        int maxiter, cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st) {
    const int nb = reduction_blocks(A.n_rows);
    if (x0 && x != x0) copy_kernel<T><<<nb, kBlock, 0, st>>>(x0, x, A.n_rows);
    WSPM_WIDTH_DISPATCH(A.max_width,
                        gm_residual_kernel<T, MW><<<nb, kBlock, 0, st>>>(A, vals, b, b64, x0, x, dinv, w.V,
                                                                         w.partials, w.st, 1, tol, atol, tol_dev,
                                                                         maxiter, cond, use_cond));
    gm_scale_kernel<T><<<nb, kBlock, 0, st>>>(A.n_rows, w.V, w.st);
}

template <typename T>
void gmres_enqueue_body(const Sell &A, const T *vals, const T *b, const double *b64, T *x, const T *dinv,
                        const GmresBuffers<T> &w, int maxiter, cudaGraphConditionalHandle cond, int use_cond,
                        cudaStream_t st) {
    const int nb = reduction_blocks(A.n_rows);
    for (int j = 0; j < w.m; ++j) {
        for (int ph = 0; ph < 3; ++ph)
            WSPM_WIDTH_DISPATCH(A.max_width,
                                gm_arnoldi_kernel<T, MW><<<nb, kBlock, 0, st>>>(A, vals, dinv, w.V, w.w, w.H, w.hbuf,
                                                                                w.partials, w.st, j, w.m, ph, w.ld));
        gm_next_kernel<T><<<nb, kBlock, 0, st>>>(A.n_rows, w.V, w.w, w.st, j, w.ld);
    }
    gm_lsq_kernel<<<1, 32, 0, st>>>(w.H, w.y, w.st, w.m);
    gm_update_kernel<T><<<nb, kBlock, 0, st>>>(A.n_rows, x, w.V, w.y, w.st, w.ld);
    WSPM_WIDTH_DISPATCH(A.max_width,
                        gm_residual_kernel<T, MW><<<nb, kBlock, 0, st>>>(A, vals, b, b64, x, x, dinv, w.V,
                                                                         w.partials, w.st, 0, 0.0, 0.0, nullptr,
                                                                         maxiter, cond, use_cond));
    gm_scale_kernel<T><<<nb, kBlock, 0, st>>>(A.n_rows, w.V, w.st);
}

template void gmres_enqueue_init<double>(const Sell &, const double *, const double *, const double *,
                                         const double *, double *, const double *, const GmresBuffers<double> &,
                                         double, double, const double *, int, cudaGraphConditionalHandle, int,
                                         cudaStream_t);
template void gmres_enqueue_init<float>(const Sell &, const float *, const float *, const double *, const float *,
                                        float *, const float *, const GmresBuffers<float> &, double, double,
                                        const double *, int, cudaGraphConditionalHandle, int, cudaStream_t);
template void gmres_enqueue_body<double>(const Sell &, const double *, const double *, const double *, double *,
                                         const double *, const GmresBuffers<double> &, int,
                                         cudaGraphConditionalHandle, int, cudaStream_t);
template void gmres_enqueue_body<float>(const Sell &, const float *, const float *, const double *, float *,
                                        const float *, const GmresBuffers<float> &, int, cudaGraphConditionalHandle,
                                        int, cudaStream_t);

// ---------------------------------------------------------------- workspaces
static inline int64_t align32(int64_t n) { return (n + 31) & ~int64_t(31); }

int64_t cg_workspace_doubles(int n, int bytes) {
    const int64_t vec = align32(((int64_t)n * bytes + 7) / 8);
    return 5 * vec + align32(4 * kMaxPartials) + align32(sizeof(KrylovState) / 8 + 1);
}
int64_t bicgstab_workspace_doubles(int n, int bytes) {
    const int64_t vec = align32(((int64_t)n * bytes + 7) / 8);
    return 6 * vec + align32(4 * kMaxPartials) + align32(sizeof(KrylovState) / 8 + 1);
}
int64_t gmres_workspace_doubles(int n, int m, int bytes) {
    const int64_t vec = align32(((int64_t)n * bytes + 7) / 8);
    return (m + 2) * vec + align32((int64_t)(m + 1) * m) + align32(m) + align32(2 * (kMaxRestart + 1)) +
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

template <typename T>
BicgBuffers<T> carve_bicgstab(double *work, int n, int64_t *used) {
    const int64_t vec = align32(((int64_t)n * sizeof(T) + 7) / 8);
    BicgBuffers<T> b;
    double *p = work;
    b.r = (T *)p; p += vec; b.rhat = (T *)p; p += vec; b.p = (T *)p; p += vec;
    b.phat = (T *)p; p += vec; b.q = (T *)p; p += vec; b.t = (T *)p; p += vec;
    b.partials = (T *)p; p += align32(4 * kMaxPartials);
    b.st = (KrylovState *)p; p += align32(sizeof(KrylovState) / 8 + 1);
    *used = p - work;
    return b;
}
template BicgBuffers<double> carve_bicgstab<double>(double *, int, int64_t *);
template BicgBuffers<float> carve_bicgstab<float>(double *, int, int64_t *);

template <typename T>
GmresBuffers<T> carve_gmres(double *work, int n, int m, int64_t *used) {
    const int64_t vec = align32(((int64_t)n * sizeof(T) + 7) / 8);   // in doubles
    GmresBuffers<T> b;
    double *p = work;
    b.m = m;
    b.ld = vec * (int64_t)(8 / sizeof(T));                          // in elements of T
    b.V = (T *)p; p += (int64_t)(m + 1) * vec;
    b.w = (T *)p; p += vec;
    b.H = p; p += align32((int64_t)(m + 1) * m);
    b.y = p; p += align32(m);
    b.hbuf = p; p += align32(2 * (kMaxRestart + 1));
    b.partials = (T *)p; p += align32((int64_t)kMaxDots * kMaxPartials);
    b.st = (KrylovState *)p; p += align32(sizeof(KrylovState) / 8 + 1);
    *used = p - work;
    return b;
}
template GmresBuffers<double> carve_gmres<double>(double *, int, int, int64_t *);
template GmresBuffers<float> carve_gmres<float>(double *, int, int, int64_t *);

}  // namespace wspm
