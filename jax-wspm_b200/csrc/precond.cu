// The reference's ILU / SSOR / block-Jacobi preconditioners
// (src/solvers/jax_linear_solver.py:38-252) on the GPU.
//
// What the reference's code computes (d = diag(A), L / U strict parts of A):
//   create_ilu0:  forward  y_i = x_i - sum_{j<i} (A_ij / d'_j) y_j      (d' = d, zeros -> 1)
//                 backward z_i = (y_i - sum_{j>i} A_ij z_j) / d'_i
//   create_ssor:  forward  y_i = (x_i - sum_{j<i} A_ij y_j) / (d_i / omega); its backward sweep
//                 reads entries of z not yet computed (zeros), so z = omega y
//   create_block_jacobi: z_b = (A_bb + 1e-12 I)^-1 x_b on diagonal blocks of block_size rows.
// Triangular sweeps are level scheduled: the host groups the rows so that a
// row only depends on rows of earlier levels; one CTA walks the levels with a
// block barrier between them (the sweep is inherently sequential across
// levels; every row of a level runs in parallel).
#include "common.cuh"
#include "krylov.cuh"

namespace wspm {

__device__ __forceinline__ int entry_col(const Sell &A, int i, int k) {
    if (A.n_diags > 0) return i + __ldg(A.diag_off + k);
    return __ldg(A.cols + entry_pos(A, i, k));
}

__device__ __forceinline__ double diag_of(const Sell &A, const double *vals, const int32_t *diag_pos, int j) {
    return vals[entry_pos(A, j, diag_pos[j])];
}

// mode 0: ILU forward, 1: ILU backward, 2: SSOR forward (then scaled by omega)
template <int MODE>
__global__ void __launch_bounds__(1024) tri_sweep_kernel(Sell A, const double *__restrict__ vals,
                                                         const int32_t *__restrict__ diag_pos,
                                                         const int32_t *__restrict__ level_ptr,
                                                         const int32_t *__restrict__ rows, int n_levels,
                                                         const double *__restrict__ x, double *y, double omega) {
    const int n = A.n_rows;
    for (int lv = 0; lv < n_levels; ++lv) {
        const int k1 = level_ptr[lv + 1];
        for (int k = level_ptr[lv] + threadIdx.x; k < k1; k += blockDim.x) {
            const int i = rows[k];
            const int w = row_width(A, i);
            double s = x[i];
            for (int q = 0; q < w; ++q) {
                const int j = entry_col(A, i, q);
                if (j < 0 || j >= n) continue;
                if (MODE == 1 ? !(j > i) : !(j < i)) continue;
                const double a = vals[entry_pos(A, i, q)];
                if (a == 0.0) continue;
                if (MODE == 0) {
                    const double dj = diag_of(A, vals, diag_pos, j);
                    s -= (a / (dj == 0.0 ? 1.0 : dj)) * y[j];
                } else {
                    s -= a * y[j];
                }
            }
            if (MODE == 0) {
                y[i] = s;
            } else if (MODE == 1) {
                const double di = diag_of(A, vals, diag_pos, i);
                y[i] = s / (di == 0.0 ? 1.0 : di);
            } else {
                y[i] = s / (diag_of(A, vals, diag_pos, i) / omega);
            }
        }
        __syncthreads();
    }
    if (MODE == 2) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = omega * y[i];
    }
}

// ---- true ILU(0) -------------------------------------------------------------
// Incomplete LU with zero fill on A's own pattern (Saad, Iterative Methods for
// Sparse Linear Systems, 2nd ed., Alg. 10.4, IKJ form): for each row i, for its
// entries k < i in ascending column order, l_ik = a_ik / u_kk, then
// a_ij -= l_ik u_kj for every later entry j of row i that row k also holds.  Row i
// reads only rows k < i, all of earlier levels of the lower sweep's schedule, so
// the rows of one level factor in parallel.  Result in `lu` (same layout as
// `vals`): the strict lower part holds L (unit diagonal implied), the rest U.  A
// zero pivot u_kk is taken as 1 (the reference's convention for zero diagonals).
// Not the reference's `ilu` (which never updates a pivot, see create_ilu0
// above): this is the textbook incomplete LU with zero fill.

// position q of column j in row i, -1 when the row does not hold it
__device__ __forceinline__ int entry_index(const Sell &A, int i, int j) {
    const int w = row_width(A, i);
    for (int q = 0; q < w; ++q)
        if (entry_col(A, i, q) == j) return q;
    return -1;
}

__global__ void __launch_bounds__(1024) ilu0_factor_kernel(Sell A, const int32_t *__restrict__ diag_pos,
                                                           const int32_t *__restrict__ level_ptr,
                                                           const int32_t *__restrict__ rows, int n_levels,
                                                           double *lu) {
    const int n = A.n_rows;
    for (int lv = 0; lv < n_levels; ++lv) {
        const int k1 = level_ptr[lv + 1];
        for (int kk = level_ptr[lv] + threadIdx.x; kk < k1; kk += blockDim.x) {
            const int i = rows[kk];
            const int w = row_width(A, i);
            const int dpi = diag_pos[i];     // SELL padding slots also name column i: only this one is the diagonal
            // entries in ascending column order: SELL rows are sorted; DIA offsets ascend
            for (int q = 0; q < w; ++q) {
                const int k = entry_col(A, i, q);
                if (k < 0 || k >= n || k >= i) continue;
                const int64_t pik = entry_pos(A, i, q);
                const double aik = lu[pik];
                if (aik == 0.0) continue;
                const double ukk = lu[entry_pos(A, k, diag_pos[k])];
                const double l = aik / (ukk != 0.0 ? ukk : 1.0);
                lu[pik] = l;
                for (int q2 = q + 1; q2 < w; ++q2) {
                    const int j = entry_col(A, i, q2);
                    if (j <= k || j < 0 || j >= n || (j == i && q2 != dpi)) continue;
                    const int qk = entry_index(A, k, j);
                    if (qk < 0) continue;
                    lu[entry_pos(A, i, q2)] -= l * lu[entry_pos(A, k, qk)];
                }
            }
        }
        __syncthreads();
    }
}

// y = (LU)^-1 x with the factors above: forward sweep with unit-lower L, backward with U.
template <int MODE>
__global__ void __launch_bounds__(1024) ilu0_sweep_kernel(Sell A, const double *__restrict__ lu,
                                                          const int32_t *__restrict__ diag_pos,
                                                          const int32_t *__restrict__ level_ptr,
                                                          const int32_t *__restrict__ rows, int n_levels,
                                                          const double *__restrict__ x, double *y) {
    const int n = A.n_rows;
    for (int lv = 0; lv < n_levels; ++lv) {
        const int k1 = level_ptr[lv + 1];
        for (int kk = level_ptr[lv] + threadIdx.x; kk < k1; kk += blockDim.x) {
            const int i = rows[kk];
            const int w = row_width(A, i);
            double s = x[i];
            for (int q = 0; q < w; ++q) {
                const int j = entry_col(A, i, q);
                if (j < 0 || j >= n) continue;
                if (MODE == 1 ? !(j > i) : !(j < i)) continue;
                const double a = lu[entry_pos(A, i, q)];
                if (a != 0.0) s -= a * y[j];
            }
            if (MODE == 0) {
                y[i] = s;
            } else {
                const double d = lu[entry_pos(A, i, diag_pos[i])];
                y[i] = s / (d != 0.0 ? d : 1.0);
            }
        }
        __syncthreads();
    }
}

// value of A(i, j) in row i (0 when absent)
__device__ __forceinline__ double entry_value(const Sell &A, const double *vals, int i, int j) {
    const int w = row_width(A, i);
    for (int q = 0; q < w; ++q)
        if (entry_col(A, i, q) == j) return vals[entry_pos(A, i, q)];
    return 0.0;
}

__global__ void block_jacobi_kernel(Sell A, const double *__restrict__ vals, int bs, const double *__restrict__ x,
                                    double *__restrict__ y) {
    const int n = A.n_rows;
    const int nb = (n + bs - 1) / bs;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int i0 = b * bs;
        if (bs == 1 || i0 + 1 >= n) {
            y[i0] = x[i0] / (entry_value(A, vals, i0, i0) + 1e-12);
            continue;
        }
        const double a = entry_value(A, vals, i0, i0) + 1e-12, bb = entry_value(A, vals, i0, i0 + 1);
        const double c = entry_value(A, vals, i0 + 1, i0), d = entry_value(A, vals, i0 + 1, i0 + 1) + 1e-12;
        const double det = a * d - bb * c;
        y[i0] = (d * x[i0] - bb * x[i0 + 1]) / det;
        y[i0 + 1] = (-c * x[i0] + a * x[i0 + 1]) / det;
    }
}

}  // namespace wspm

using namespace wspm;

extern "C" int wspm_precond_apply(const wspm_pattern *pat, const double *vals, int32_t kind, double omega,
                                  int32_t block_size, const wspm_levels *lower, const wspm_levels *upper,
                                  const double *x, double *y, double *tmp, void *stream) {
    if (!pat || !vals || !x || !y || pat->n_rows <= 0) return WSPM_BAD_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const Sell A = make_sell(pat);
    if (kind == WSPM_PRECOND_BLOCK_JACOBI) {
        if (block_size != 1 && block_size != 2) return WSPM_UNSUPPORTED;
        const int nb = (pat->n_rows + block_size - 1) / block_size;
        block_jacobi_kernel<<<(nb + 255) / 256, 256, 0, st>>>(A, vals, block_size, x, y);
    } else if (kind == WSPM_PRECOND_ILU) {
        if (!lower || !upper || !tmp || !lower->level_ptr || !lower->rows || !upper->level_ptr || !upper->rows)
            return WSPM_BAD_ARG;
        tri_sweep_kernel<0><<<1, 1024, 0, st>>>(A, vals, pat->diag_pos, lower->level_ptr, lower->rows,
                                                lower->n_levels, x, tmp, omega);
        tri_sweep_kernel<1><<<1, 1024, 0, st>>>(A, vals, pat->diag_pos, upper->level_ptr, upper->rows,
                                                upper->n_levels, tmp, y, omega);
    } else if (kind == WSPM_PRECOND_ILU0) {
        // vals holds the factors of wspm_ilu0_factor
        if (!lower || !upper || !tmp || !lower->level_ptr || !lower->rows || !upper->level_ptr || !upper->rows)
            return WSPM_BAD_ARG;
        ilu0_sweep_kernel<0><<<1, 1024, 0, st>>>(A, vals, pat->diag_pos, lower->level_ptr, lower->rows,
                                                 lower->n_levels, x, tmp);
        ilu0_sweep_kernel<1><<<1, 1024, 0, st>>>(A, vals, pat->diag_pos, upper->level_ptr, upper->rows,
                                                 upper->n_levels, tmp, y);
    } else if (kind == WSPM_PRECOND_SSOR) {
        if (!lower || !lower->level_ptr || !lower->rows || !(omega != 0.0)) return WSPM_BAD_ARG;
        tri_sweep_kernel<2><<<1, 1024, 0, st>>>(A, vals, pat->diag_pos, lower->level_ptr, lower->rows,
                                                lower->n_levels, x, y, omega);
    } else {
        return WSPM_UNSUPPORTED;
    }
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

extern "C" int wspm_ilu0_factor(const wspm_pattern *pat, const double *vals, const wspm_levels *lower, double *lu,
                                void *stream) {
    if (!pat || !vals || !lu || !lower || !lower->level_ptr || !lower->rows || pat->n_rows <= 0 || !pat->diag_pos)
        return WSPM_BAD_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    WSPM_CUDA_TRY(cudaMemcpyAsync(lu, vals, (size_t)pat->nnz_padded * sizeof(double), cudaMemcpyDeviceToDevice, st));
    ilu0_factor_kernel<<<1, 1024, 0, st>>>(make_sell(pat), pat->diag_pos, lower->level_ptr, lower->rows,
                                           lower->n_levels, lu);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}
