// One implicit Richards time step as a single CUDA graph.
//
//   step_init:  theta_n = theta(h_n); h_m = h_n; C, K, theta_m at h_m; Picard counters reset
//   WHILE picard (err >= tol && it < maxit):                richards_solver_v2.py:160-165
//     assembly:   A, b, Dirichlet rows, Jacobi 1/diag        :118-146
//     Krylov:     FP64 CG | BiCGSTAB | GMRES(m), x0 = h_m    :148-153
//                 or FP32 CG inside FP64 iterative refinement on the true residual
//     update:     err = ||x - h_m|| (/ ||x||); h_m = x; it++ :155
//                 and the soil fields C, K, theta_m at the new h_m (:114-115 of the next iteration)
//   step_finish: h_n = h_m, counters to the caller's result words
//
// Every loop is a conditional WHILE node whose handle is cleared by the
// kernel that tests convergence, and every loop has an iteration cap, so
// the graph always terminates.  The host launches the graph once per time
// step and never synchronises inside it.
#include <cstring>
#include <mutex>
#include <new>
#include <vector>
#include "krylov.cuh"
#include "graph.cuh"
#include "soil.cuh"

namespace wspm {

int launch_soil(const SoilParams &sp, const double *h, int64_t n, double *C, double *K, double *theta,
                cudaStream_t st);
void quadrature_constants(int dim, const double *Q, const double *W, int nq, double s[4], double m[4]);
int launch_edge_terms(const wspm_pattern *pat, const wspm_edges *e, int mode, double flux, double c_in,
                      const double *K, const double *theta, double *vals, double *rhs, cudaStream_t st);
int launch_richards_assembly_dev_dt(const wspm_mesh *mesh, const wspm_pattern *pat, const double *theta_m,
                                    const double *theta_n, const double *h_m, const double *K, const double *C,
                                    const double *Ks_elem, const double *Ks_inc, const double s[4],
                                    const double mc[4], const double *dt_dev, const double *bc_val, double *vals,
                                    float *vals32, double *rhs, double *dinv, const RefineStart *res,
                                    const uint32_t *shape_words, const double *shape_tab, int n_shapes,
                                    int shape_mode, cudaStream_t st);
int richards_assembly_blocks(const wspm_mesh *mesh, const wspm_pattern *pat);
int64_t richards_shape_bytes(const wspm_mesh *mesh, const wspm_pattern *pat);
int richards_build_shapes(const wspm_mesh *mesh, const wspm_pattern *pat, void *buf, const uint32_t **words,
                          const double **table, int *mode);
unsigned long long richards_dia_live_mask(const wspm_mesh *mesh, const wspm_pattern *pat, unsigned long long *word);
int launch_incidence_gather(const wspm_pattern *pat, const double *elem, double *out, cudaStream_t st);

struct PicardState {
    double err, tol;
    int it, maxit, relative, status;
    int krylov_total, refine_total, krylov_maxiter_hits, last_krylov_status;
    int bodies;        // Krylov loop bodies executed (launch accounting)
    int solver;        // WSPM_SOLVER_*
    int cont;          // 1 while the Picard loop continues (read by the host-driven mode)
    int restart_m;     // GMRES restart length (launch accounting)
    unsigned int ticket[4];
    unsigned long long krylov_ns;   // resident CG kernels: summed %globaltimer duration of this step's launches
};

__global__ void state_reset_kernel(unsigned int *words, int n_words) {
    for (int i = threadIdx.x; i < n_words; i += blockDim.x) words[i] = 0u;
}

// theta_n = theta(h_n), h_m = h_n, and the soil fields of the first Picard
// iteration (C, K, theta_m at h_m = h_n: theta_m = theta_n).
__global__ void step_init_kernel(SoilParams sp, int n, const double *__restrict__ h_n, double *theta_n, double *h_m,
                                 double *C, double *K, double *theta_m, PicardState *ps, double tol, int maxit,
                                 int relative, int solver, int restart_m, cudaGraphConditionalHandle cond,
                                 int use_cond) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double c, k, t;
        const double h = h_n[i];
        soil_eval(sp, h, c, k, t);
        theta_n[i] = t;
        h_m[i] = h;
        C[i] = c;
        K[i] = k;
        theta_m[i] = t;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ps->err = __longlong_as_double(0x7ff0000000000000ULL);  // +inf, like the reference's carry
        ps->tol = tol; ps->it = 0; ps->maxit = maxit; ps->relative = relative; ps->status = WSPM_OK;
        ps->krylov_total = 0; ps->refine_total = 0; ps->krylov_maxiter_hits = 0; ps->last_krylov_status = 0;
        ps->bodies = 0;
        ps->krylov_ns = 0ull;
        ps->solver = solver;
        ps->cont = maxit > 0 ? 1 : 0;
        ps->restart_m = restart_m;
        for (int j = 0; j < 4; ++j) ps->ticket[j] = 0u;
        if (use_cond) cudaGraphSetConditional(cond, maxit > 0 ? 1u : 0u);
    }
}

// Picard norm and test; h_m = x, and the soil fields of the next Picard
// iteration at the new h_m (C, K, theta_m; unused after the last iteration).
__global__ void __launch_bounds__(kBlock) picard_update_kernel(int n, const double *__restrict__ x, double *h_m,
                                                               SoilParams sp, double *C, double *K, double *theta_m,
                                                               double *partials, PicardState *ps,
                                                               const KrylovState *ks, const KrylovState *irs,
                                                               cudaGraphConditionalHandle cond, int use_cond) {
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double xi = x[i];
        const double d = xi - h_m[i];
        v[0] += d * d;
        v[1] += xi * xi;
        h_m[i] = xi;
        double c, k, t;
        soil_eval(sp, xi, c, k, t);
        C[i] = c;
        K[i] = k;
        theta_m[i] = t;
    }
    if (publish_partials<double, 2>(v, partials, &ps->ticket[0])) {
        double tot[2];
        final_sum<double, 2>(partials, tot, &ps->ticket[0]);
        if (threadIdx.x == 0) {
            const double dn = sqrt(tot[0]);
            const double err = ps->relative ? dn / sqrt(tot[1]) : dn;
            ps->err = err;
            ps->it += 1;
            if (irs) {
                ps->krylov_ns += irs->ns;
                ps->refine_total += irs->k;
                ps->krylov_total += irs->steps;   // inner iterations accumulated by the refinement loop
                ps->bodies += irs->pad0;          // inner CG launches accumulated by the refinement loop
                ps->last_krylov_status = irs->status;
            } else {
                const int kk = ks->k > 0 ? ks->k : 0;
                ps->krylov_total += kk;
                if (ps->solver == WSPM_SOLVER_CG) ps->krylov_ns += ks->ns;
                // Krylov-loop launches: CG is one persistent kernel; BiCGSTAB 4 kernels per
                // iteration; GMRES 4 m + 4 kernels per restart cycle
                if (ps->solver == WSPM_SOLVER_CG) ps->bodies += 1;
                else if (ps->solver == WSPM_SOLVER_BICGSTAB) ps->bodies += 4 * (ks->k < 0 ? 1 : kk);
                else ps->bodies += (4 * ps->restart_m + 4) * kk;
                ps->last_krylov_status = ks->status;
            }
            if (ps->last_krylov_status == WSPM_MAXITER) ps->krylov_maxiter_hits += 1;
            int cont = (err >= ps->tol) && (ps->it < ps->maxit);
            if (!isfinite(err)) { cont = 0; ps->status = WSPM_NAN; }
            else if (!cont && err >= ps->tol) ps->status = WSPM_MAXITER;
            ps->cont = cont;
            if (use_cond) cudaGraphSetConditional(cond, cont ? 1u : 0u);
        }
    }
}

__global__ void step_finish_kernel(int n, const double *__restrict__ h_m, double *h_n, const PicardState *ps,
                                   int32_t *result, double *result_f64) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) h_n[i] = h_m[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        result[0] = ps->status;
        result[1] = ps->it;
        result[2] = ps->krylov_total;
        result[3] = ps->refine_total;
        result[4] = ps->krylov_maxiter_hits;
        result[5] = ps->last_krylov_status;
        result[6] = ps->bodies;
        result_f64[0] = ps->err;
        result_f64[1] = 1e-9 * (double)ps->krylov_ns;
    }
}

// ---- mixed precision: FP32 Krylov corrections inside FP64 refinement --------
// ir state (KrylovState): bs, atol2, rr, k (refinement iterations), steps (inner
// iterations summed), pad0 (inner-solve kernel launches), status.

// The FP32 inner solver: Jacobi-CG (pipelined or single-reduction resident
// kernel), BiCGSTAB or GMRES(m), the same method as the FP64 path's solver.
struct InnerSolver {
    int solver = WSPM_SOLVER_CG;
    CgBuffers<float> cg;
    BicgBuffers<float> bicg;
    GmresBuffers<float> gm;
    KrylovState *st() const {
        return solver == WSPM_SOLVER_BICGSTAB ? bicg.st : solver == WSPM_SOLVER_GMRES ? gm.st : cg.st;
    }
};

static int64_t inner_workspace_doubles(int n, int solver, int restart) {
    if (solver == WSPM_SOLVER_BICGSTAB) return bicgstab_workspace_doubles(n, 4);
    if (solver == WSPM_SOLVER_GMRES) return gmres_workspace_doubles(n, restart, 4);
    return cg_workspace_doubles(n, 4);
}

static InnerSolver carve_inner(double *p, int n, int solver, int restart, int64_t *used) {
    InnerSolver in;
    in.solver = solver;
    if (solver == WSPM_SOLVER_BICGSTAB) in.bicg = carve_bicgstab<float>(p, n, used);
    else if (solver == WSPM_SOLVER_GMRES) in.gm = carve_gmres<float>(p, n, restart, used);
    else in.cg = carve_cg<float>(p, n, used);
    return in;
}

// Kernels launched by one inner solve of k iterations: CG one resident launch;
// BiCGSTAB init + 4 per iteration; GMRES(m) 2 + (4m + 4) per restart cycle.
__device__ __forceinline__ int inner_launches(int solver, int m, int k) {
    if (k < 0) k = -k;
    if (solver == WSPM_SOLVER_BICGSTAB) return 1 + 4 * k;
    if (solver == WSPM_SOLVER_GMRES) return 2 + (4 * m + 4) * k;
    return 1;
}


// Start of the refinement loop: x = x0, r = b - A x0 (FP64), the FP32 copy of
// 1/diag, and the loop state.
template <int MW>
__global__ void __launch_bounds__(kBlock) ir_residual_kernel(Sell A, const double *__restrict__ vals,
                                                             const double *__restrict__ b,
                                                             const double *__restrict__ x0, double *x, double *r,
                                                             const double *__restrict__ dinv, float *dinv32,
                                                             double *partials, KrylovState *irs, double tol,
                                                             double inner_floor, int maxit,
                                                             cudaGraphConditionalHandle cond, int use_cond) {
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_rows; i += gridDim.x * blockDim.x) {
        const double ri = b[i] - sell_row_dot<double, MW>(A, vals, i, [&](int c) { return x0[c]; });
        r[i] = ri;
        x[i] = x0[i];
        if (dinv32) dinv32[i] = (float)dinv[i];
        v[0] += ri * ri;
        v[1] += b[i] * b[i];
    }
    if (publish_partials<double, 2>(v, partials, &irs->ticket[0])) {
        double tot[2];
        final_sum<double, 2>(partials, tot, &irs->ticket[0]);
        if (threadIdx.x == 0) ir_decide(tot, irs, nullptr, 1, tol, inner_floor, maxit, cond, use_cond);
    }
}

// After an FP32 correction d: x += d and r -= A d (FP64; equal to b - A x up to
// FP64 rounding, without re-reading b and the previous x).  skip: as for the
// resident CG launch before it (the first refinement, outside the WHILE node):
// nonzero at launch = the loop is already done, nothing to apply.
template <int MW>
__global__ void __launch_bounds__(kBlock) ir_update_kernel(Sell A, const double *__restrict__ vals,
                                                           const float *__restrict__ d, double *x, double *r,
                                                           double *partials, KrylovState *irs,
                                                           const KrylovState *inner, int inner_solver, int inner_m,
                                                           double tol, double inner_floor, int maxit, const int *skip,
                                                           cudaGraphConditionalHandle cond, int use_cond) {
    // every block reads the word before any block can reach the reduction tail that rewrites it
    if (skip && *(volatile const int *)skip) return;
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_rows; i += gridDim.x * blockDim.x) {
        const double ri = r[i] - sell_row_dot<double, MW>(A, vals, i, [&](int c) { return (double)d[c]; });
        r[i] = ri;
        x[i] += (double)d[i];
        v[0] += ri * ri;
    }
    if (publish_partials<double, 2>(v, partials, &irs->ticket[0])) {
        double tot[2];
        final_sum<double, 2>(partials, tot, &irs->ticket[0]);
        if (threadIdx.x == 0)
            ir_decide(tot, irs, inner, 0, tol, inner_floor, maxit, cond, use_cond,
                      inner_launches(inner_solver, inner_m, inner->k));
    }
}

static int read_flag(const int *dev_word, cudaStream_t st, int *out, int *pinned);

// One FP32 solve of A d = r64 from d = 0 to the relative tolerance the
// refinement loop left in *tol_dev.  use_cond = 1 (graph capture): BiCGSTAB and
// GMRES loop in a nested WHILE node; use_cond = 0 (host-driven mode): bounded
// chunks of loop bodies between host reads of the solver's done word.  `skip`
// (CG only): the resident launch returns at once when the word is set.
static int inner_enqueue(const Sell &A, const float *vals32, const double *r64, float *x32, const float *dv32,
                         const InnerSolver &in, double inner_tol, int inner_maxiter, const double *tol_dev,
                         cudaStream_t s, int use_cond, const int *skip, int *pinned) {
    if (in.solver == WSPM_SOLVER_CG) {
        const int rc = pcg_persistent_enqueue<float>(A, vals32, nullptr, r64, x32, dv32, in.cg, inner_tol, 0.0,
                                                     inner_maxiter, true, tol_dev, s, true, skip);
        if (rc == WSPM_UNSUPPORTED)
            return cg_persistent_enqueue<float>(A, vals32, nullptr, r64, x32, dv32, in.cg, inner_tol, 0.0,
                                                inner_maxiter, true, tol_dev, s, skip);
        return rc;
    }
    constexpr int kChunk = 8;
    cudaGraphConditionalHandle hk = cudaGraphConditionalHandle();
    if (use_cond && make_cond_handle(s, &hk) != cudaSuccess) return WSPM_CUDA_ERROR;
    auto body = [&](cudaStream_t b) {
        if (in.solver == WSPM_SOLVER_BICGSTAB)
            bicgstab_enqueue_body<float>(A, vals32, x32, dv32, in.bicg, inner_maxiter, hk, use_cond, b);
        else
            gmres_enqueue_body<float>(A, vals32, nullptr, r64, x32, dv32, in.gm, inner_maxiter, hk, use_cond, b);
    };
    if (in.solver == WSPM_SOLVER_BICGSTAB)
        bicgstab_enqueue_init<float>(A, vals32, nullptr, r64, nullptr, x32, in.bicg, inner_tol, 0.0, tol_dev,
                                     inner_maxiter, hk, use_cond, s);
    else
        gmres_enqueue_init<float>(A, vals32, nullptr, r64, nullptr, x32, dv32, in.gm, inner_tol, 0.0, tol_dev,
                                  inner_maxiter, hk, use_cond, s);
    if (use_cond) return capture_while(s, hk, body) == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
    int flag = 0, rc = WSPM_OK;
    for (int b = 0; b < inner_maxiter + 1 && rc == WSPM_OK; b += kChunk) {
        if ((rc = read_flag(&in.st()->done, s, &flag, pinned)) != WSPM_OK || flag) break;
        for (int c = 0; c < kChunk; ++c) body(s);
    }
    return rc;
}

struct PicardPlan {
    wspm_mesh mesh;
    wspm_pattern pat;
    wspm_picard_desc d;
    wspm_edges neumann, drainage;   // copies (n_bnodes == 0: unused)
    SoilParams sp_field;   // soil law of the step (theta_n, and C, K, theta_m for the assembly)
    double s[4], mc[4];
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    PicardState *ps = nullptr;
    double *partials = nullptr;
    CgBuffers<double> cg64;
    InnerSolver inner;              // mixed path: the FP32 corrections
    BicgBuffers<double> bicg;
    GmresBuffers<double> gm;
    KrylovState *irs = nullptr;
    double *r64 = nullptr;
    float *x32 = nullptr, *dinv32 = nullptr;
    double *Ks_inc = nullptr;   // Ks_elem in incidence order (caller's buffer), refreshed at every step start
    unsigned long long live = ~0ull;   // DIA diagonals that can hold nonzeros (structural zeros skipped)
    // element shapes (caller's buffer): incidence words tagged with shape ids and the shapes' geometric
    // factors; n_shapes == 0 when the mesh has too many distinct Jacobians or no buffer was given
    const uint32_t *shape_words = nullptr;
    const double *shape_tab = nullptr;
    int n_shapes = 0;
    int shape_mode = 0;   // 1: table in shared memory, 2: global table (4-bit row positions in the words)
};

// The plan's matrix descriptor: the pattern with its structural-zero diagonals marked.
static Sell plan_sell(const PicardPlan *P) {
    Sell A = make_sell(&P->pat);
    A.live = P->live;
    return A;
}

// The mixed path starts each refinement loop inside the assembly launch (r = b - A h_m
// from the rows just built) when nothing is added to the rows after it (no Neumann or
// drainage edges) and its partial sums fit the plan's slots.
static bool fuse_refine_start(const PicardPlan *P) {
    return P->d.mixed && P->neumann.n_bnodes <= 0 && P->drainage.n_bnodes <= 0 &&
           richards_assembly_blocks(&P->mesh, &P->pat) <= kMaxPartials;
}

static RefineStart refine_start(const PicardPlan *P, cudaGraphConditionalHandle cond, int use_cond) {
    RefineStart r;
    r.x0 = P->d.h_m; r.x = P->d.x; r.r = P->r64; r.dinv32 = P->dinv32;
    r.partials = P->partials; r.irs = P->irs;
    r.tol = P->d.krylov_tol; r.inner_floor = P->d.inner_tol; r.maxit = P->d.refine_maxiter;
    r.cond = cond; r.use_cond = use_cond;
    return r;
}

int64_t picard_workspace_doubles(int n, int mixed, int solver, int restart) {
    const int64_t vec = (n + 31) & ~int64_t(31);
    int64_t t = 64 + ((sizeof(PicardState) + 7) / 8) + 2 * kMaxPartials + 64;
    if (mixed) {
        t += inner_workspace_doubles(n, solver, restart) + 64 + vec /* r64 */ + vec /* x32 + dinv32 as floats */ + 64;
        t += 64 + ((sizeof(KrylovState) + 7) / 8);
    } else if (solver == WSPM_SOLVER_BICGSTAB) {
        t += bicgstab_workspace_doubles(n);
    } else if (solver == WSPM_SOLVER_GMRES) {
        t += gmres_workspace_doubles(n, restart);
    } else {
        t += cg_workspace_doubles(n, 8);
    }
    return t;
}

static int build_picard_graph(PicardPlan *P) {
    const wspm_picard_desc &d = P->d;
    const int n = P->mesh.n_nodes;
    const Sell A = plan_sell(P);
    const int nb = reduction_blocks(n);
    const double *dinv = d.precond == WSPM_PRECOND_JACOBI ? d.dinv : nullptr;
    cudaStream_t cs;
    WSPM_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    WSPM_CUDA_TRY(cudaGraphCreate(&g, 0));
    cudaError_t e = cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) { cudaGraphDestroy(g); cudaStreamDestroy(cs); return WSPM_CUDA_ERROR; }

    cudaGraphConditionalHandle hp;
    e = make_cond_handle(cs, &hp);
    state_reset_kernel<<<1, 32, 0, cs>>>((unsigned int *)P->ps->ticket, 4);
    {
        KrylovState *sts[4] = {P->cg64.st, d.mixed ? P->inner.st() : nullptr, P->bicg.st, P->gm.st};
        for (KrylovState *k : sts)
            if (k) state_reset_kernel<<<1, 32, 0, cs>>>((unsigned int *)k, (int)(sizeof(KrylovState) / 4));
        if (P->irs) state_reset_kernel<<<1, 32, 0, cs>>>((unsigned int *)P->irs, (int)(sizeof(KrylovState) / 4));
    }
    if (P->Ks_inc) launch_incidence_gather(&P->pat, d.Ks_elem, P->Ks_inc, cs);
    step_init_kernel<<<nb, kBlock, 0, cs>>>(P->sp_field, n, d.h_n, d.theta_n, d.h_m, d.C, d.K, d.theta_m, P->ps,
                                            d.picard_tol, d.picard_maxiter, d.picard_relative, d.solver, P->gm.m, hp,
                                            1);
    if (e == cudaSuccess) e = capture_while(cs, hp, [&](cudaStream_t bs) {
        cudaGraphConditionalHandle hir = cudaGraphConditionalHandle();
        if (d.mixed) make_cond_handle(bs, &hir);
        const RefineStart rs = refine_start(P, hir, 1);
        const bool fused = fuse_refine_start(P);
        launch_richards_assembly_dev_dt(&P->mesh, &P->pat, d.theta_m, d.theta_n, d.h_m, d.K, d.C, d.Ks_elem,
                                        P->Ks_inc, P->s, P->mc, d.dt_dev, d.bc_val, d.vals,
                                        d.mixed ? d.vals32 : nullptr, d.rhs, d.dinv, fused ? &rs : nullptr,
                                        P->shape_words, P->shape_tab, P->n_shapes,
                                        P->shape_mode, bs);
        launch_edge_terms(&P->pat, &P->neumann, WSPM_EDGE_NEUMANN, d.neumann_flux, 0.0, d.K, nullptr, d.vals, d.rhs,
                          bs);
        launch_edge_terms(&P->pat, &P->drainage, WSPM_EDGE_DRAINAGE_WATER, 0.0, 0.0, d.K, nullptr, d.vals, d.rhs,
                          bs);
        const KrylovState *ks = nullptr;
        const KrylovState *irs = nullptr;
        if (d.mixed) {
            if (!fused)
                WSPM_WIDTH_DISPATCH(A.max_width,
                                    ir_residual_kernel<MW><<<nb, kBlock, 0, bs>>>(A, d.vals, d.rhs, d.h_m, d.x,
                                                                                  P->r64, d.dinv, P->dinv32,
                                                                                  P->partials, P->irs, d.krylov_tol,
                                                                                  d.inner_tol, d.refine_maxiter, hir,
                                                                                  1));
            const float *dv32 = dinv ? P->dinv32 : nullptr;
            const InnerSolver &in = P->inner;
            auto correction = [&](cudaStream_t cb, const int *skip) {
                inner_enqueue(A, d.vals32, P->r64, P->x32, dv32, in, d.inner_tol, d.inner_maxiter,
                              &P->irs->inner_tol, cb, 1, skip, nullptr);
                WSPM_WIDTH_DISPATCH(A.max_width,
                                    ir_update_kernel<MW><<<nb, kBlock, 0, cb>>>(A, d.vals, P->x32, d.x, P->r64,
                                                                                P->partials, P->irs, in.st(),
                                                                                in.solver, in.gm.m, d.krylov_tol,
                                                                                d.inner_tol, d.refine_maxiter, skip,
                                                                                hir, 1));
            };
            // CG: the first correction as plain nodes (both kernels return at once when the start already met
            // the tolerance), the rest inside the WHILE node: one body launch fewer per Picard iteration
            if (in.solver == WSPM_SOLVER_CG) correction(bs, &P->irs->done);
            capture_while(bs, hir, [&](cudaStream_t ibs) { correction(ibs, nullptr); });
            irs = P->irs;
        } else if (d.solver == WSPM_SOLVER_BICGSTAB) {
            cudaGraphConditionalHandle hk;
            make_cond_handle(bs, &hk);
            bicgstab_enqueue_init<double>(A, d.vals, d.rhs, nullptr, d.h_m, d.x, P->bicg, d.krylov_tol, 0.0, nullptr,
                                          d.krylov_maxiter, hk, 1, bs);
            capture_while(bs, hk, [&](cudaStream_t kbs) {
                bicgstab_enqueue_body<double>(A, d.vals, d.x, dinv, P->bicg, d.krylov_maxiter, hk, 1, kbs);
            });
            ks = P->bicg.st;
        } else if (d.solver == WSPM_SOLVER_GMRES) {
            cudaGraphConditionalHandle hk;
            make_cond_handle(bs, &hk);
            gmres_enqueue_init<double>(A, d.vals, d.rhs, nullptr, d.h_m, d.x, dinv, P->gm, d.krylov_tol, 0.0, nullptr,
                                       d.krylov_maxiter, hk, 1, bs);
            capture_while(bs, hk, [&](cudaStream_t kbs) {
                gmres_enqueue_body<double>(A, d.vals, d.rhs, nullptr, d.x, dinv, P->gm, d.krylov_maxiter, hk, 1, kbs);
            });
            ks = P->gm.st;
        } else {
            copy_kernel_d(d.h_m, d.x, n, bs);
            cg_persistent_enqueue<double>(A, d.vals, d.rhs, nullptr, d.x, dinv, P->cg64, d.krylov_tol, 0.0,
                                          d.krylov_maxiter, false, nullptr, bs);
            ks = P->cg64.st;
        }
        picard_update_kernel<<<nb, kBlock, 0, bs>>>(n, d.x, d.h_m, P->sp_field, d.C, d.K, d.theta_m, P->partials,
                                                    P->ps, ks, irs, hp, 1);
    });
    step_finish_kernel<<<nb, kBlock, 0, cs>>>(n, d.h_m, d.h_n, P->ps, d.result, d.result_f64);
    cudaGraph_t out = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(cs, &out);
    cudaStreamDestroy(cs);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) { cudaGraphDestroy(g); return WSPM_CUDA_ERROR; }
    e = cudaGraphInstantiate(&P->exec, g, 0);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return WSPM_CUDA_ERROR; }
    P->graph = g;
    return WSPM_OK;
}

// Host-driven variant of the same step: identical kernels, loop control from
// the host (bounded loops that read the device's done/cont words).  Used when
// a tool cannot follow conditional graph nodes (ncu profiles no kernel node
// of such graphs) and as a fallback.
static int read_flag(const int *dev_word, cudaStream_t st, int *out, int *pinned) {
    WSPM_CUDA_TRY(cudaMemcpyAsync(pinned, dev_word, sizeof(int), cudaMemcpyDeviceToHost, st));
    WSPM_CUDA_TRY(cudaStreamSynchronize(st));
    *out = *pinned;
    return WSPM_OK;
}

static int picard_step_host(PicardPlan *P, cudaStream_t st) {
    const wspm_picard_desc &d = P->d;
    const int n = P->mesh.n_nodes;
    const Sell A = plan_sell(P);
    const int nb = reduction_blocks(n);
    const double *dinv = d.precond == WSPM_PRECOND_JACOBI ? d.dinv : nullptr;
    const cudaGraphConditionalHandle none = cudaGraphConditionalHandle();
    int *pinned = nullptr;
    WSPM_CUDA_TRY(cudaMallocHost(&pinned, sizeof(int)));
    int rc = WSPM_OK, flag = 0;
    constexpr int kChunk = 8;
    state_reset_kernel<<<1, 32, 0, st>>>((unsigned int *)P->ps->ticket, 4);
    KrylovState *sts[5] = {P->cg64.st, d.mixed ? P->inner.st() : nullptr, P->bicg.st, P->gm.st, P->irs};
    for (KrylovState *k : sts)
        if (k) state_reset_kernel<<<1, 32, 0, st>>>((unsigned int *)k, (int)(sizeof(KrylovState) / 4));
    if (P->Ks_inc) launch_incidence_gather(&P->pat, d.Ks_elem, P->Ks_inc, st);
    step_init_kernel<<<nb, kBlock, 0, st>>>(P->sp_field, n, d.h_n, d.theta_n, d.h_m, d.C, d.K, d.theta_m, P->ps,
                                            d.picard_tol, d.picard_maxiter, d.picard_relative, d.solver, P->gm.m,
                                            none, 0);
    for (int it = 0; it < d.picard_maxiter && rc == WSPM_OK; ++it) {
        const RefineStart rs = refine_start(P, none, 0);
        const bool fused = fuse_refine_start(P);
        launch_richards_assembly_dev_dt(&P->mesh, &P->pat, d.theta_m, d.theta_n, d.h_m, d.K, d.C, d.Ks_elem,
                                        P->Ks_inc, P->s, P->mc, d.dt_dev, d.bc_val, d.vals,
                                        d.mixed ? d.vals32 : nullptr, d.rhs, d.dinv, fused ? &rs : nullptr,
                                        P->shape_words, P->shape_tab, P->n_shapes,
                                        P->shape_mode, st);
        launch_edge_terms(&P->pat, &P->neumann, WSPM_EDGE_NEUMANN, d.neumann_flux, 0.0, d.K, nullptr, d.vals, d.rhs,
                          st);
        launch_edge_terms(&P->pat, &P->drainage, WSPM_EDGE_DRAINAGE_WATER, 0.0, 0.0, d.K, nullptr, d.vals, d.rhs,
                          st);
        const KrylovState *ks = nullptr, *irs = nullptr;
        if (d.mixed) {
            if (!fused)
                WSPM_WIDTH_DISPATCH(A.max_width,
                                    ir_residual_kernel<MW><<<nb, kBlock, 0, st>>>(A, d.vals, d.rhs, d.h_m, d.x,
                                                                                  P->r64, d.dinv, P->dinv32,
                                                                                  P->partials, P->irs, d.krylov_tol,
                                                                                  d.inner_tol, d.refine_maxiter, none,
                                                                                  0));
            const float *dv32 = dinv ? P->dinv32 : nullptr;
            const InnerSolver &in = P->inner;
            for (int r = 0; r <= d.refine_maxiter && rc == WSPM_OK; ++r) {
                if ((rc = read_flag(&P->irs->done, st, &flag, pinned)) != WSPM_OK || flag) break;
                rc = inner_enqueue(A, d.vals32, P->r64, P->x32, dv32, in, d.inner_tol, d.inner_maxiter,
                                   &P->irs->inner_tol, st, 0, nullptr, pinned);
                WSPM_WIDTH_DISPATCH(A.max_width,
                                    ir_update_kernel<MW><<<nb, kBlock, 0, st>>>(A, d.vals, P->x32, d.x, P->r64,
                                                                                P->partials, P->irs, in.st(),
                                                                                in.solver, in.gm.m, d.krylov_tol,
                                                                                d.inner_tol, d.refine_maxiter, nullptr,
                                                                                none, 0));
            }
            irs = P->irs;
        } else {
            KrylovState *kst = nullptr;
            int max_bodies = d.krylov_maxiter;
            if (d.solver == WSPM_SOLVER_BICGSTAB) {
                bicgstab_enqueue_init<double>(A, d.vals, d.rhs, nullptr, d.h_m, d.x, P->bicg, d.krylov_tol, 0.0,
                                              nullptr, d.krylov_maxiter, none, 0, st);
                kst = P->bicg.st;
            } else if (d.solver == WSPM_SOLVER_GMRES) {
                gmres_enqueue_init<double>(A, d.vals, d.rhs, nullptr, d.h_m, d.x, dinv, P->gm, d.krylov_tol, 0.0,
                                           nullptr, d.krylov_maxiter, none, 0, st);
                kst = P->gm.st;
            } else {
                copy_kernel_d(d.h_m, d.x, n, st);
                cg_persistent_enqueue<double>(A, d.vals, d.rhs, nullptr, d.x, dinv, P->cg64, d.krylov_tol, 0.0,
                                              d.krylov_maxiter, false, nullptr, st);
                kst = P->cg64.st;
                max_bodies = -1;     // the persistent kernel ran the whole solve
            }
            for (int b = 0; b < max_bodies + 1 && rc == WSPM_OK; b += kChunk) {
                if ((rc = read_flag(&kst->done, st, &flag, pinned)) != WSPM_OK || flag) break;
                for (int c = 0; c < kChunk; ++c) {
                    if (d.solver == WSPM_SOLVER_BICGSTAB)
                        bicgstab_enqueue_body<double>(A, d.vals, d.x, dinv, P->bicg, d.krylov_maxiter, none, 0, st);
                    else if (d.solver == WSPM_SOLVER_GMRES)
                        gmres_enqueue_body<double>(A, d.vals, d.rhs, nullptr, d.x, dinv, P->gm, d.krylov_maxiter, none,
                                                   0, st);
                    else
                        break;
                }
            }
            ks = kst;
        }
        picard_update_kernel<<<nb, kBlock, 0, st>>>(n, d.x, d.h_m, P->sp_field, d.C, d.K, d.theta_m, P->partials,
                                                    P->ps, ks, irs, none, 0);
        if (rc == WSPM_OK && (rc = read_flag(&P->ps->cont, st, &flag, pinned)) == WSPM_OK && !flag) break;
    }
    step_finish_kernel<<<nb, kBlock, 0, st>>>(n, d.h_m, d.h_n, P->ps, d.result, d.result_f64);
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFreeHost(pinned);
    if (rc == WSPM_OK && (e != cudaSuccess || cudaGetLastError() != cudaSuccess)) rc = WSPM_CUDA_ERROR;
    return rc;
}

}  // namespace wspm

using namespace wspm;

extern "C" int wspm_picard_step_host(void *plan, void *stream) {
    if (!plan) return WSPM_BAD_ARG;
    return picard_step_host((PicardPlan *)plan, (cudaStream_t)stream);
}

extern "C" int64_t wspm_picard_workspace_doubles(int32_t n_rows, int32_t mixed) {
    // sized for the largest solver choice so that one buffer fits any plan
    int64_t a = picard_workspace_doubles(n_rows, mixed, WSPM_SOLVER_GMRES, n_rows < 32 ? n_rows : 32);
    int64_t b = picard_workspace_doubles(n_rows, mixed, WSPM_SOLVER_BICGSTAB, 0);
    int64_t c = picard_workspace_doubles(n_rows, mixed, WSPM_SOLVER_CG, 0);
    return a > b ? (a > c ? a : c) : (b > c ? b : c);
}

extern "C" int64_t wspm_picard_shape_bytes(const wspm_mesh *mesh, const wspm_pattern *pat) {
    return richards_shape_bytes(mesh, pat);
}

extern "C" int64_t wspm_picard_ks_inc_doubles(const wspm_pattern *pat) {
    if (!pat || pat->n_slices <= 0) return -1;
    return (int64_t)pat->n_slices * kSlice * (int64_t)(pat->max_inc > 0 ? pat->max_inc : 1);
}

extern "C" int wspm_picard_create(const wspm_picard_desc *desc, void **plan_out) {
    if (!desc || !plan_out || !desc->mesh || !desc->pat) return WSPM_BAD_ARG;
    const wspm_picard_desc &d = *desc;
    const int n = d.mesh->n_nodes;
    if (n <= 0 || d.pat->n_rows != n || d.nq <= 0 || d.nq > 16) return WSPM_BAD_ARG;
    if (d.mesh->dim != 2 && d.mesh->dim != 3) return WSPM_BAD_ARG;
    if (!d.h_n || !d.theta_n || !d.h_m || !d.x || !d.K || !d.C || !d.theta_m || !d.vals || !d.rhs || !d.dinv ||
        !d.work || !d.dt_dev || !d.result || !d.result_f64)
        return WSPM_BAD_ARG;
    if (d.mixed && !d.vals32) return WSPM_BAD_ARG;
    if (d.Ks_elem && !d.Ks_inc) return WSPM_BAD_ARG;
    if (d.solver == WSPM_SOLVER_GMRES && (d.restart < 1 || d.restart > 32)) return WSPM_UNSUPPORTED;
    if (d.solver < WSPM_SOLVER_CG || d.solver > WSPM_SOLVER_GMRES) return WSPM_BAD_ARG;
    if (d.work_doubles < wspm_picard_workspace_doubles(n, d.mixed)) return WSPM_BAD_ARG;
    PicardPlan *P = new (std::nothrow) PicardPlan();
    if (!P) return WSPM_BAD_ARG;
    P->mesh = *d.mesh;
    P->pat = *d.pat;
    P->d = d;
    P->neumann = d.neumann ? *d.neumann : wspm_edges();
    P->drainage = d.drainage ? *d.drainage : wspm_edges();
    P->d.neumann = nullptr;
    P->d.drainage = nullptr;
    P->d.mesh = &P->mesh;
    P->d.pat = &P->pat;
    P->sp_field.model = d.soil_model;
    for (int j = 0; j < 6; ++j) P->sp_field.p[j] = d.phi[j];
    quadrature_constants(d.mesh->dim, d.quad_points, d.weights, d.nq, P->s, P->mc);
    // carve the workspace
    double *p = d.work;
    P->ps = (PicardState *)p; p += 64;
    P->partials = p; p += 2 * kMaxPartials + 64;
    int64_t used = 0;
    if (d.mixed) {
        const int m = d.restart < n ? d.restart : n;
        P->inner = carve_inner(p, n, d.solver, m, &used); p += used + 64;
        const int64_t vec = (n + 31) & ~int64_t(31);
        P->r64 = p; p += vec;
        P->x32 = (float *)p; P->dinv32 = (float *)p + vec; p += vec + 64;
        P->irs = (KrylovState *)p; p += 64 + ((sizeof(KrylovState) + 7) / 8);
    } else if (d.solver == WSPM_SOLVER_BICGSTAB) {
        P->bicg = carve_bicgstab<double>(p, n, &used); p += used;
    } else if (d.solver == WSPM_SOLVER_GMRES) {
        const int m = d.restart < n ? d.restart : n;
        P->gm = carve_gmres<double>(p, n, m, &used); p += used;
    } else {
        P->cg64 = carve_cg<double>(p, n, &used); p += used;
    }
    P->Ks_inc = d.Ks_elem ? d.Ks_inc : nullptr;
    // structural zeros of the DIA layout, found once from the geometry (the first
    // partial-sum slot of the workspace serves as the scratch word)
    P->live = richards_dia_live_mask(&P->mesh, &P->pat, reinterpret_cast<unsigned long long *>(P->partials));
    // element shapes, found once from the geometry (synchronous)
    if (d.shapes)
        P->n_shapes = richards_build_shapes(&P->mesh, &P->pat, d.shapes, &P->shape_words, &P->shape_tab,
                                            &P->shape_mode);
    // Ks in incidence order as of creation (every step refreshes it at its start)
    if (P->Ks_inc && (launch_incidence_gather(&P->pat, d.Ks_elem, P->Ks_inc, 0) != WSPM_OK ||
                      cudaDeviceSynchronize() != cudaSuccess)) {
        delete P;
        return WSPM_CUDA_ERROR;
    }
    int rc = build_picard_graph(P);
    if (rc != WSPM_OK) {
        delete P;
        return rc;
    }
    *plan_out = P;
    return WSPM_OK;
}

extern "C" int wspm_picard_assemble(void *plan, void *stream) {
    if (!plan) return WSPM_BAD_ARG;
    PicardPlan *P = (PicardPlan *)plan;
    const wspm_picard_desc &d = P->d;
    cudaStream_t st = (cudaStream_t)stream;
    return launch_richards_assembly_dev_dt(&P->mesh, &P->pat, d.theta_m, d.theta_n, d.h_m, d.K, d.C, d.Ks_elem,
                                           P->Ks_inc, P->s, P->mc, d.dt_dev, d.bc_val, d.vals,
                                           d.mixed ? d.vals32 : nullptr, d.rhs, d.dinv, nullptr, P->shape_words,
                                           P->shape_tab, P->n_shapes, P->shape_mode, st);
}

extern "C" int32_t wspm_picard_shapes(void *plan) {
    return plan ? ((const PicardPlan *)plan)->n_shapes : -1;
}

extern "C" int64_t wspm_picard_dia_live(void *plan) {
    if (!plan) return -1;
    const PicardPlan *P = (const PicardPlan *)plan;
    return P->pat.n_diags > 0 ? (int64_t)(P->live & ((1ull << P->pat.n_diags) - 1ull)) : -1;
}

extern "C" int wspm_picard_step(void *plan, void *stream) {
    if (!plan) return WSPM_BAD_ARG;
    PicardPlan *P = (PicardPlan *)plan;
    WSPM_CUDA_TRY(cudaGraphLaunch(P->exec, (cudaStream_t)stream));
    return WSPM_OK;
}

extern "C" int wspm_picard_destroy(void *plan) {
    if (!plan) return WSPM_OK;
    PicardPlan *P = (PicardPlan *)plan;
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->graph) cudaGraphDestroy(P->graph);
    delete P;
    return WSPM_OK;
}

// ---- one linear system in mixed precision ------------------------------------
// FP32 Jacobi-CG corrections inside FP64 iterative refinement, the refinement
// loop of the Picard graph without the Picard step around it: x = x0, r =
// b - A x (FP64); while ||r|| > tol ||b||: solve A d = r in FP32 (pipelined CG
// where the pattern allows it) to the reduction still needed (floor
// inner_tol), then x += d, r -= A d (FP64).  Captured once per argument set as
// a CUDA graph (WHILE node for the refinements) and replayed, like
// wspm_krylov_solve.
namespace {

__global__ void to_f32_kernel(const double *__restrict__ a, float *b, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

__global__ void mixed_result_kernel(const KrylovState *irs, int32_t *out) {
    if (threadIdx.x == 0) {
        out[0] = irs->status;
        out[1] = irs->steps;     // FP32 iterations (CG, BiCGSTAB) or restart cycles (GMRES), all refinements
        out[2] = irs->k;         // refinements (FP32 solves)
        out[3] = 0;
    }
}

// Everything a captured graph depends on: the arrays it reads and writes, the
// whole storage description of the pattern (a pattern rebuilt into reused
// buffers with another layout or width must not replay a graph captured for
// the old one) and the device.
struct MixedKey {
    const void *pat_cols, *pat_ptr, *pat_width, *pat_diag_off, *vals, *vals32, *b, *x, *dinv, *work, *result;
    int64_t nnz_padded;
    int n, n_slices, max_width, n_diags, device, inner_maxiter, refine_maxiter, solver, restart, pad_;
    double tol, inner_tol;
    bool operator==(const MixedKey &o) const { return std::memcmp(this, &o, sizeof(MixedKey)) == 0; }
};
struct MixedEntry {
    MixedKey key;
    cudaGraphExec_t exec;
    cudaGraph_t graph;
};
std::mutex g_mixed_mu;
std::vector<MixedEntry> g_mixed;
constexpr size_t kMixedCacheMax = 8;

int64_t mixed_vec(int n) { return (n + 31) & ~int64_t(31); }

int build_mixed_graph(const wspm_pattern *pat, const double *vals, const float *vals32, const double *b, double *x,
                      const double *dinv, int solver, int restart, double tol, double inner_tol, int inner_maxiter,
                      int refine_maxiter, double *work, int32_t *result, cudaGraphExec_t *exec_out,
                      cudaGraph_t *graph_out) {
    const Sell A = make_sell(pat);
    const int n = pat->n_rows;
    const int nb = reduction_blocks(n);
    const int64_t vec = mixed_vec(n);
    // workspace: partials | refinement state | FP32 solver buffers | r64 | x32, dinv32 | vals32 (when not given),
    // every part on a 256-byte boundary (the CG kernels move 16-byte row groups)
    auto align = [](double *q) { return (double *)(((uintptr_t)q + 255) & ~(uintptr_t)255); };
    double *p = align(work);
    double *partials = p; p = align(p + 2 * kMaxPartials + 64);
    KrylovState *irs = (KrylovState *)p; p = align(p + 64 + ((sizeof(KrylovState) + 7) / 8));
    int64_t used = 0;
    const InnerSolver in = carve_inner(p, n, solver, restart < n ? restart : n, &used);
    p = align(p + used + 64);
    double *r64 = p; p = align(p + vec);
    float *x32 = (float *)p, *dinv32 = (float *)p + vec; p = align(p + vec + 64);
    float *v32 = vals32 ? const_cast<float *>(vals32) : (float *)p;
    cudaStream_t cs;
    WSPM_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    WSPM_CUDA_TRY(cudaGraphCreate(&g, 0));
    cudaError_t e = cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e == cudaSuccess) {
        state_reset_kernel<<<1, 32, 0, cs>>>((unsigned int *)irs, (int)(sizeof(KrylovState) / 4));
        state_reset_kernel<<<1, 32, 0, cs>>>((unsigned int *)in.st(), (int)(sizeof(KrylovState) / 4));
        if (!vals32) to_f32_kernel<<<reduction_blocks(pat->nnz_padded), kBlock, 0, cs>>>(vals, v32, pat->nnz_padded);
        cudaGraphConditionalHandle h;
        e = make_cond_handle(cs, &h);
        float *dv32 = dinv ? dinv32 : nullptr;
        WSPM_WIDTH_DISPATCH(A.max_width,
                            ir_residual_kernel<MW><<<nb, kBlock, 0, cs>>>(A, vals, b, x, x, r64, dinv, dv32, partials,
                                                                          irs, tol, inner_tol, refine_maxiter, h, 1));
        // one correction: the FP32 solve (CG: skipped when `skip` is set at launch) and x += d, r -= A d
        auto correction = [&](cudaStream_t bs, const int *skip) {
            if (inner_enqueue(A, v32, r64, x32, dv32, in, inner_tol, inner_maxiter, &irs->inner_tol, bs, 1, skip,
                              nullptr) != WSPM_OK)
                e = cudaErrorLaunchFailure;
            WSPM_WIDTH_DISPATCH(A.max_width,
                                ir_update_kernel<MW><<<nb, kBlock, 0, bs>>>(A, vals, x32, x, r64, partials, irs,
                                                                            in.st(), in.solver, in.gm.m, tol,
                                                                            inner_tol, refine_maxiter, skip, h, 1));
        };
        // CG: the first correction as plain nodes, the rest inside the WHILE node
        if (e == cudaSuccess && solver == WSPM_SOLVER_CG) correction(cs, &irs->done);
        if (e == cudaSuccess) e = capture_while(cs, h, [&](cudaStream_t bs) { correction(bs, nullptr); });
        mixed_result_kernel<<<1, 32, 0, cs>>>(irs, result);
        cudaGraph_t out = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(cs, &out);
        if (e == cudaSuccess) e = e2;
    }
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return WSPM_CUDA_ERROR; }
    e = cudaGraphInstantiate(exec_out, g, 0);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return WSPM_CUDA_ERROR; }
    *graph_out = g;
    return WSPM_OK;
}

}  // namespace

extern "C" int64_t wspm_krylov_mixed_workspace_doubles(int32_t n_rows, int64_t nnz_padded, int32_t solver,
                                                       int32_t restart) {
    if (n_rows <= 0 || nnz_padded <= 0 || solver < WSPM_SOLVER_CG || solver > WSPM_SOLVER_GMRES) return 0;
    if (solver == WSPM_SOLVER_GMRES && (restart < 1 || restart > 32)) return 0;
    const int64_t vec = mixed_vec(n_rows);
    const int m = restart < n_rows ? restart : n_rows;
    return 2 * kMaxPartials + 64 + 64 + ((sizeof(KrylovState) + 7) / 8) + inner_workspace_doubles(n_rows, solver, m) +
           64 + vec + vec + 64 + (nnz_padded + 1) / 2 + 64 + 6 * 32;   // + alignment slack of six parts
}

extern "C" int wspm_krylov_solve_mixed(const wspm_pattern *pat, const double *vals, const float *vals32,
                                       const double *b, double *x, const double *dinv, int32_t solver,
                                       int32_t restart, double tol, double inner_tol, int32_t inner_maxiter,
                                       int32_t refine_maxiter, double *work, int64_t work_doubles, int32_t *result,
                                       void *stream) {
    if (!pattern_layout_ok(pat)) return WSPM_BAD_ARG;
    if (!vals || !b || !x || !work || !result) return WSPM_BAD_ARG;
    if (solver < WSPM_SOLVER_CG || solver > WSPM_SOLVER_GMRES) return WSPM_BAD_ARG;
    if (solver == WSPM_SOLVER_GMRES && (restart < 1 || restart > 32)) return WSPM_UNSUPPORTED;
    if (solver != WSPM_SOLVER_GMRES) restart = 0;
    if (!(tol > 0.0) || !(inner_tol > 0.0) || inner_tol >= 1.0 || inner_maxiter < 1 || refine_maxiter < 1)
        return WSPM_BAD_ARG;
    const int64_t need = wspm_krylov_mixed_workspace_doubles(pat->n_rows, pat->nnz_padded, solver, restart > 0 ? restart : 1);
    if (need <= 0 || work_doubles < need) return WSPM_BAD_ARG;
    MixedKey key;
    std::memset(&key, 0, sizeof(key));
    key.pat_cols = pat->cols; key.pat_ptr = pat->slice_ptr; key.pat_width = pat->slice_width;
    key.pat_diag_off = pat->n_diags > 0 ? pat->diag_offsets : nullptr;
    key.vals = vals; key.vals32 = vals32; key.b = b;
    key.x = x; key.dinv = dinv; key.work = work; key.result = result; key.nnz_padded = pat->nnz_padded;
    key.n = pat->n_rows; key.n_slices = pat->n_slices; key.max_width = pat->max_width; key.n_diags = pat->n_diags;
    WSPM_CUDA_TRY(cudaGetDevice(&key.device));
    key.inner_maxiter = inner_maxiter; key.refine_maxiter = refine_maxiter; key.tol = tol;
    key.solver = solver; key.restart = restart;
    key.inner_tol = inner_tol;
    cudaGraphExec_t exec = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mixed_mu);
        for (auto &en : g_mixed)
            if (en.key == key) { exec = en.exec; break; }
        if (!exec) {
            cudaGraph_t graph = nullptr;
            const int rc = build_mixed_graph(pat, vals, vals32, b, x, dinv, solver, restart, tol, inner_tol,
                                             inner_maxiter, refine_maxiter, work, result, &exec, &graph);
            if (rc != WSPM_OK) return rc;
            if (g_mixed.size() >= kMixedCacheMax) {
                cudaGraphExecDestroy(g_mixed.front().exec);
                cudaGraphDestroy(g_mixed.front().graph);
                g_mixed.erase(g_mixed.begin());
            }
            g_mixed.push_back({key, exec, graph});
        }
    }
    WSPM_CUDA_TRY(cudaGraphLaunch(exec, (cudaStream_t)stream));
    return WSPM_OK;
}
