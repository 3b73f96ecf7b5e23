// Shared device helpers for libwspm (sm_100a).
//
// Reductions are deterministic: every block writes its partial sums to a
// fixed slot, the last block to arrive (atomic ticket, no spinning) sums the
// slots in slot order and publishes the scalar.  The grid size of every
// reducing kernel is a fixed function of the problem size, so results are
// bitwise repeatable run to run.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "wspm.h"

namespace wspm {

constexpr int kSlice = 32;          // SELL slice height == warp size
constexpr int kBlock = 256;         // threads per block for vector kernels
constexpr int kMaxPartials = 16384; // partial-sum slots: one block per 256 rows up to 4M rows

// Host-side consistency check of a pattern's storage description (everything
// the sparse kernels index with, except the diagonal positions, which only the
// entry points that read the diagonal need): slices cover the rows, DIA
// patterns have one width, widths fit the unrolled row loops.
inline bool pattern_layout_ok(const wspm_pattern *p) {
    return p && p->n_rows > 0 && p->n_slices == (p->n_rows + 31) / 32 && p->slice_ptr && p->slice_width &&
           p->cols && p->max_width > 0 && p->max_width <= 63 && p->nnz_padded > 0 &&
           (p->n_diags == 0 || (p->n_diags == p->max_width && p->diag_offsets));
}

// Grid of a reducing kernel: one thread per row (or element) up to 8 blocks
// per SM, grid-stride beyond.  Every block publishes one partial through an
// atomic ticket on a single word, so the cap bounds that serialised tail
// (4,000+ blocks at 10^6 rows would queue 4,000+ atomics); the grid stays a
// fixed function of n, so the summation order is fixed.
inline int reduction_blocks(int64_t n) {
    static int cap = 0;
    if (cap == 0) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cap = sms > 0 ? 8 * sms : 1024;
        if (cap > kMaxPartials) cap = kMaxPartials;
    }
    int64_t b = (n + kBlock - 1) / kBlock;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (int)b;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of NV values per thread; result valid in thread 0.
template <typename T, int NV>
__device__ __forceinline__ void block_sum(T (&v)[NV]) {
    __shared__ T sh[NV][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = warp_sum(v[j]);
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) sh[j][wid] = v[j];
    }
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    if (wid == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            T t = lane < nw ? sh[j][lane] : T(0);
            v[j] = warp_sum(t);
        }
    }
    __syncthreads();
}

// Publish per-block partials; returns true in exactly one block (the last to
// finish), whose threads can then read all partials.  `partials` is laid out
// [NV][gridDim.x].  The ticket is reset by the last block.
template <typename T, int NV>
__device__ __forceinline__ bool publish_partials(T (&v)[NV], T *partials, unsigned int *ticket) {
    __shared__ bool is_last;
    block_sum<T, NV>(v);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) partials[j * gridDim.x + blockIdx.x] = v[j];
        __threadfence();
        unsigned int t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

// In the last block: fixed-order sum of the partials; result in thread 0.
// Loads go through L2 (ld.global.cg: the other blocks' stores are visible
// there after their __threadfence) and are unrolled so many are in flight.
template <typename T, int NV>
__device__ __forceinline__ void final_sum(const T *partials, T (&out)[NV], unsigned int *ticket) {
    const int nb = (int)gridDim.x;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        const T *pj = partials + (int64_t)j * nb;
        T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
        int b = threadIdx.x;
        const int step = blockDim.x;
        for (; b + 3 * step < nb; b += 4 * step) {
            const T x0 = __ldcg(pj + b), x1 = __ldcg(pj + b + step);
            const T x2 = __ldcg(pj + b + 2 * step), x3 = __ldcg(pj + b + 3 * step);
            a0 += x0; a1 += x1; a2 += x2; a3 += x3;
        }
        for (; b < nb; b += step) a0 += __ldcg(pj + b);
        out[j] = (a0 + a1) + (a2 + a3);
    }
    block_sum<T, NV>(out);
    if (threadIdx.x == 0) *ticket = 0u;
}

__device__ __forceinline__ bool finite_d(double v) { return isfinite(v); }

// Matrix layout shared by every sparse kernel.
//   SELL-32: entry k of row i at slice_ptr[i/32] + 32k + i%32, column cols[...].
//   DIA (n_diags > 0): entry k of row i at k*ld + i, column i + diag_off[k]
//   (out-of-range columns hold value 0 and are clamped for the gather).
struct Sell {
    int n_rows;
    int n_slices;
    int max_width;
    const int64_t *slice_ptr;
    const int32_t *slice_width;
    const int32_t *cols;
    int n_diags;
    const int32_t *diag_off;
    int64_t ld;
    // DIA: bit k clear = diagonal k holds exact zeros in every row (a structural
    // zero of the discretisation, e.g. the edge opposite a right angle of P1
    // triangles); the sparse kernels then skip its loads.  fma(0, x, acc) == acc
    // for finite x, so skipping changes no result bit.  All ones by default.
    unsigned long long live;
};

__host__ __device__ __forceinline__ bool dia_live(const Sell &A, int k) { return (A.live >> k) & 1ull; }

__device__ __forceinline__ int64_t entry_pos(const Sell &A, int i, int k) {
    return A.n_diags > 0 ? (int64_t)k * A.ld + i : __ldg(A.slice_ptr + (i >> 5)) + (int64_t)kSlice * k + (i & 31);
}

__device__ __forceinline__ int row_width(const Sell &A, int i) {
    return A.n_diags > 0 ? A.n_diags : __ldg(A.slice_width + (i >> 5));
}

// Row i of A times x, with x supplied by the functor xf(col).  MW > 0: the
// row's entries are processed in groups of 4 whose column/value loads and
// gathers are issued together (memory-level parallelism with a bounded
// register footprint); requires row width <= MW.
template <typename T, int MW, typename XF>
__device__ __forceinline__ T sell_row_dot(const Sell &A, const T *__restrict__ vals, int i, XF xf) {
    constexpr int G = 4;
    T acc = T(0);
    if (A.n_diags > 0) {
        const int nd = A.n_diags;
        const int last = A.n_rows - 1;
        if constexpr (MW > 0) {
#pragma unroll 1
            for (int k0 = 0; k0 < MW; k0 += G) {
                if (k0 >= nd) break;
                T v[G];
                int c[G];
#pragma unroll
                for (int g = 0; g < G; ++g) {
                    const int k = k0 + g;
                    if (k < nd && dia_live(A, k)) {
                        v[g] = __ldg(vals + (int64_t)k * A.ld + i);
                        const int cc = i + __ldg(A.diag_off + k);
                        c[g] = cc < 0 ? 0 : (cc > last ? last : cc);
                    }
                }
#pragma unroll
                for (int g = 0; g < G; ++g)
                    if (k0 + g < nd && dia_live(A, k0 + g)) acc = fma(v[g], xf(c[g]), acc);
            }
        } else {
            for (int k = 0; k < nd; ++k) {
                if (!dia_live(A, k)) continue;
                int cc = i + __ldg(A.diag_off + k);
                cc = cc < 0 ? 0 : (cc > last ? last : cc);
                acc = fma(__ldg(vals + (int64_t)k * A.ld + i), xf(cc), acc);
            }
        }
        return acc;
    }
    const int s = i >> 5, lane = i & 31;
    const int w = __ldg(A.slice_width + s);
    const int64_t base = __ldg(A.slice_ptr + s) + lane;
    if constexpr (MW > 0) {
#pragma unroll 1
        for (int k0 = 0; k0 < MW; k0 += G) {
            if (k0 >= w) break;
            T v[G];
            int c[G];
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int k = k0 + g;
                if (k < w) {
                    c[g] = __ldg(A.cols + base + (int64_t)kSlice * k);
                    v[g] = __ldg(vals + base + (int64_t)kSlice * k);
                }
            }
#pragma unroll
            for (int g = 0; g < G; ++g)
                if (k0 + g < w) acc = fma(v[g], xf(c[g]), acc);
        }
    } else {
        for (int k = 0; k < w; ++k) {
            const int64_t o = base + (int64_t)kSlice * k;
            acc = fma(__ldg(vals + o), xf(__ldg(A.cols + o)), acc);
        }
    }
    return acc;
}

}  // namespace wspm

#define WSPM_CUDA_TRY(expr)                                   \
    do {                                                      \
        cudaError_t _e = (expr);                              \
        if (_e != cudaSuccess) return WSPM_CUDA_ERROR;        \
    } while (0)
