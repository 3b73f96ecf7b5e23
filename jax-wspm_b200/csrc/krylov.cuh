// Krylov solvers on SELL-32 matrices: declarations shared by krylov.cu,
// picard.cu and capi.cu.
#pragma once
#include "common.cuh"

namespace wspm {

inline Sell make_sell(const wspm_pattern *p) {
    Sell s;
    s.n_rows = p->n_rows; s.n_slices = p->n_slices; s.max_width = p->max_width;
    s.slice_ptr = p->slice_ptr; s.slice_width = p->slice_width; s.cols = p->cols;
    s.n_diags = p->n_diags; s.diag_off = p->diag_offsets; s.ld = (int64_t)p->n_slices * kSlice;
    s.live = ~0ull;
    return s;
}

// Device-resident solver scalars (one cache line per group).
struct KrylovState {
    double gamma, alpha, beta, atol2, bs, rr, pq, rz;      // CG
    double rho, omega, sigma, ss, ts, tt, rho_next;        // BiCGSTAB
    double rnorm, ptol, wn0, wn, inv_wn, b_norm, mb_norm;  // GMRES
    double inner_tol;                                      // refinement: tolerance of the next inner solve
    int k, done, status, exit_early, broken, steps, pad0, pad1;
    unsigned int ticket[4];
    // resident CG kernels: %globaltimer ns from block 0's entry to its exit of the
    // last launch; refinement state: the sum over the loop's inner solves
    unsigned long long ns;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Reduction tail of the refinement steps (the start, fused into the assembly or
// as ir_residual_kernel, and ir_update_kernel): tot = (r.r, b.b); sets
// the next inner tolerance, the continue flag and the graph condition.
// inner_launches: kernels the inner solve just finished launched (launch accounting).
__device__ __forceinline__ void ir_decide(const double (&tot)[2], KrylovState *irs, const KrylovState *inner,
                                          int is_init, double tol, double inner_floor, int maxit,
                                          cudaGraphConditionalHandle cond, int use_cond, int inner_launches = 1) {
    if (is_init) {
        irs->bs = tot[1];
        irs->atol2 = tol * tol * tot[1];
        irs->k = 0;
        irs->steps = 0;
        irs->pad0 = 0;
        irs->ns = 0ull;
        irs->status = WSPM_OK;
    } else {
        irs->k += 1;
        irs->steps += inner->k > 0 ? inner->k : 0;      // a BiCGSTAB breakdown reports k < 0
        irs->pad0 += inner_launches;
        irs->ns += inner->ns;
    }
    irs->rr = tot[0];
    // the next FP32 solve aims at the reduction the FP64 residual still needs,
    // never tighter than the floor FP32 can reach (a margin below it measured
    // slower: the inner iterations it adds cost more than the corrections it
    // saves; the FP64 residual decides when the loop ends)
    const double need = sqrt(irs->atol2 / fmax(tot[0], 1e-300));
    irs->inner_tol = fmin(0.5, fmax(inner_floor, need));
    int cont = tot[0] > irs->atol2 && irs->k < maxit;
    if (!cont && tot[0] > irs->atol2) irs->status = WSPM_MAXITER;
    if (!isfinite(tot[0])) { cont = 0; irs->status = WSPM_NAN; }
    irs->done = !cont;
    if (use_cond) cudaGraphSetConditional(cond, cont ? 1u : 0u);
}

// Start of the FP64 refinement loop fused into the assembly: with this set, the
// row kernel also writes r = b - A x0, x = x0 and the FP32 1/diag of its row
// and ends with the (r.r, b.b) reduction and ir_decide.
struct RefineStart {
    const double *x0;
    double *x, *r;
    float *dinv32;             // may be null
    double *partials;          // 2 x (assembly blocks)
    KrylovState *irs;
    double tol, inner_floor;
    int maxit;
    cudaGraphConditionalHandle cond;
    int use_cond;
};

// Precision-generic CG over one matrix.  Buffers are carved from a workspace.
template <typename T>
struct CgBuffers {
    T *r, *z, *p0, *p1, *q;
    T *partials;      // [4 * kMaxPartials]
    KrylovState *st;
};

// Launch helpers.  `cond`/`use_cond`: CUDA-graph conditional handle set by the
// last block of the convergence-testing kernel (while-loop continue flag).
// Rows are processed with their column/value loads issued up front, unrolled
// to a compile-time width MW (8 for triangle meshes, 16 for tetrahedra, 0 =
// generic loop); the launch helpers pick MW from the pattern's max width.
#define WSPM_WIDTH_DISPATCH(maxw, ...)             \
    do {                                            \
        if ((maxw) <= 8) {                          \
            constexpr int MW = 8;                   \
            __VA_ARGS__;                            \
        } else if ((maxw) <= 16) {                  \
            constexpr int MW = 16;                  \
            __VA_ARGS__;                            \
        } else {                                    \
            constexpr int MW = 0;                   \
            __VA_ARGS__;                            \
        }                                           \
    } while (0)

template <typename T>
void cg_enqueue_init(const Sell &A, const T *vals, const T *b, const double *b64_source,
                     const T *x0, T *x, const T *dinv, const CgBuffers<T> &w, double tol, double atol,
                     int maxiter, bool zero_x0, cudaGraphConditionalHandle cond, int use_cond,
                     cudaStream_t st, const double *tol_dev = nullptr);
template <typename T>
void cg_enqueue_body(const Sell &A, const T *vals, T *x, const T *dinv, const CgBuffers<T> &w,
                     int maxiter, cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st);

// Whole CG solve in one cooperative launch (x0 in x unless zero_x0); the final
// scalars, iteration count and status are written to w.st.  The barrier words
// live in w.st->ticket and must be zero before the launch (state reset).
// skip: optional device word; nonzero when the launch starts means "no solve"
// (k = 0), for the first refinement of a loop whose start already met its
// tolerance (the launch is a plain graph node, not inside the loop's WHILE node).
template <typename T>
int cg_persistent_enqueue(const Sell &A, const T *vals, const T *b, const double *b64, T *x, const T *dinv,
                          const CgBuffers<T> &w, double tol, double atol, int maxiter, bool zero_x0,
                          const double *tol_dev, cudaStream_t st, const int *skip = nullptr);

// Pipelined Jacobi-CG (one reduction per iteration, overlapped with the SpMV)
// in one cooperative launch, same buffers and state as cg_persistent_enqueue.
// DIA patterns whose per-block vectors fit in shared memory only; returns
// WSPM_UNSUPPORTED (nothing launched) otherwise.
template <typename T>
int pcg_persistent_enqueue(const Sell &A, const T *vals, const T *b, const double *b64, T *x, const T *dinv,
                           const CgBuffers<T> &w, double tol, double atol, int maxiter, bool zero_x0,
                           const double *tol_dev, cudaStream_t st, bool warp_specialized = true,
                           const int *skip = nullptr);
// Whether pcg_persistent_enqueue accepts the pattern for element type T (DIA
// with at most 16 diagonals, at least six per-block vectors on chip).
template <typename T>
bool pcg_eligible(const Sell &A);

// BiCGSTAB and GMRES(m) buffers, templated on the vector type (double for the
// plain path, float for the mixed path's inner corrections).
template <typename T>
struct BicgBuffers {
    T *r, *rhat, *p, *phat, *q, *t;
    T *partials;
    KrylovState *st;
};
// b64: optional FP64 right-hand side read in place of b (converted on the fly);
// x0 == NULL: start from zero; tol_dev: optional device-side relative tolerance.
template <typename T>
void bicgstab_enqueue_init(const Sell &A, const T *vals, const T *b, const double *b64, const T *x0, T *x,
                           const BicgBuffers<T> &w, double tol, double atol, const double *tol_dev, int maxiter,
                           cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st);
template <typename T>
void bicgstab_enqueue_body(const Sell &A, const T *vals, T *x, const T *dinv, const BicgBuffers<T> &w, int maxiter,
                           cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st);

template <typename T>
struct GmresBuffers {
    T *V;             // [(m+1) * ld]
    T *w;             // [n]
    double *H;        // [(m+1) * m], column-major by Arnoldi step: H[j*(m+1) + i]
    double *y;        // [m]
    double *hbuf;     // [2 * (m+1)]
    T *partials;      // [(m+2) * kMaxPartials]
    KrylovState *st;
    int m;
    int64_t ld;       // leading dimension of V in elements (padded n)
};
template <typename T>
void gmres_enqueue_init(const Sell &A, const T *vals, const T *b, const double *b64, const T *x0, T *x,
                        const T *dinv, const GmresBuffers<T> &w, double tol, double atol, const double *tol_dev,
                        int maxiter, cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st);
template <typename T>
void gmres_enqueue_body(const Sell &A, const T *vals, const T *b, const double *b64, T *x, const T *dinv,
                        const GmresBuffers<T> &w, int maxiter, cudaGraphConditionalHandle cond, int use_cond,
                        cudaStream_t st);

// Workspace sizing / carving (in doubles).
int64_t cg_workspace_doubles(int n, int bytes_per_elem);
int64_t bicgstab_workspace_doubles(int n, int bytes_per_elem = 8);
int64_t gmres_workspace_doubles(int n, int m, int bytes_per_elem = 8);
template <typename T>
CgBuffers<T> carve_cg(double *work, int n, int64_t *used);
template <typename T>
BicgBuffers<T> carve_bicgstab(double *work, int n, int64_t *used);
template <typename T>
GmresBuffers<T> carve_gmres(double *work, int n, int m, int64_t *used);

void copy_kernel_d(const double *src, double *dst, int n, cudaStream_t st);
void spmv_f64(const Sell &A, const double *vals, const double *x, double *y, cudaStream_t st);
void spmv_f32(const Sell &A, const float *vals, const float *x, float *y, cudaStream_t st);

}  // namespace wspm
