// extern "C" entry points of libwspm.so (declared in include/wspm.h).
#include <mutex>
#include <vector>
#include <cstring>
#include "krylov.cuh"
#include "graph.cuh"
#include "soil.cuh"

namespace wspm {
int launch_soil(const SoilParams &sp, const double *h, int64_t n, double *C, double *K, double *theta,
                cudaStream_t st);
void quadrature_constants(int dim, const double *Q, const double *W, int nq, double s[4], double m[4]);
int launch_richards_assembly(const wspm_mesh *mesh, const wspm_pattern *pat, const double *theta_m,
                             const double *theta_n, const double *h_m, const double *K, const double *C,
                             const double *Ks_elem, const double s[4], const double mc[4], double dt,
                             const double *bc_val, double *vals, float *vals32, double *rhs, double *dinv,
                             cudaStream_t st);

int launch_flux_dispersion(const wspm_mesh *mesh, const wspm_pattern *pat, const double *h, const SoilParams &sp,
                           double DL, double DT, double Dm, double *qx, double *qz, double *aq, double *Dxx,
                           double *Dxz, double *Dzz, double *theta, cudaStream_t st);
int launch_adr(const wspm_mesh *mesh, const wspm_pattern *pat, const double *theta, const double *qx,
               const double *qz, const double *Dxx, const double *Dxz, const double *Dzz, const double *c_n,
               const double *c_up, double mu, double sorption, double mu_up, int lumped, const double *Q,
               const double *W, int nq, double dt, double *vals, double *rhs, double *dinv, cudaStream_t st);
int launch_edge_terms(const wspm_pattern *pat, const wspm_edges *e, int mode, double flux, double c_in,
                      const double *K, const double *theta, double *vals, double *rhs, cudaStream_t st);

__global__ void dirichlet_rows_kernel(Sell A, const int32_t *__restrict__ diag_pos, const int32_t *__restrict__ nodes,
                                      const double *__restrict__ values, int n_bc, double *vals, double *rhs) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_bc) return;
    const int i = nodes[t];
    if (i < 0 || i >= A.n_rows) return;
    const int w = row_width(A, i);
    const int dp = diag_pos[i];
    for (int k = 0; k < w; ++k) vals[entry_pos(A, i, k)] = (k == dp) ? 1.0 : 0.0;
    rhs[i] = values[t];
}

__global__ void jacobi_kernel(Sell A, const int32_t *__restrict__ diag_pos, const double *__restrict__ vals,
                              double *dinv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n_rows) return;
    const double d = vals[entry_pos(A, i, diag_pos[i])];
    dinv[i] = 1.0 / (d != 0.0 ? d : 1.0);
}

__global__ void write_result_kernel(const KrylovState *st, int32_t *result) {
    if (threadIdx.x == 0) {
        result[0] = st->status;
        result[1] = st->k;
        result[2] = 0;
        result[3] = 0;
    }
}

// ---- cache of instantiated stand-alone solve graphs ------------------------
// Everything a captured solve graph depends on, the pattern's whole storage
// description and the device included.
struct SolveKey {
    const void *pat_cols, *pat_ptr, *pat_width, *pat_diag_off, *vals, *b, *x, *dinv, *work, *result;
    int64_t nnz_padded;
    int n, n_slices, max_width, n_diags, device, solver, maxiter, restart;
    double tol, atol;
    bool operator==(const SolveKey &o) const { return std::memcmp(this, &o, sizeof(SolveKey)) == 0; }
};
struct SolveEntry {
    SolveKey key;
    cudaGraphExec_t exec;
    cudaGraph_t graph;
};
static std::mutex g_cache_mu;
static std::vector<SolveEntry> g_cache;
constexpr size_t kCacheMax = 16;

static int build_solve_graph(const wspm_pattern *pat, const double *vals, const double *b, double *x,
                             const double *dinv, int solver, double tol, double atol, int maxiter, int restart,
                             double *work, int32_t *result, cudaGraphExec_t *exec_out, cudaGraph_t *graph_out) {
    const Sell A = make_sell(pat);
    const int n = pat->n_rows;
    int64_t used = 0;
    cudaStream_t cs;
    WSPM_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    WSPM_CUDA_TRY(cudaGraphCreate(&g, 0));
    cudaError_t e = cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e == cudaSuccess) {
        cudaGraphConditionalHandle h = cudaGraphConditionalHandle();
        // CG is one persistent kernel (no loop node); the other solvers loop in a WHILE node
        if (solver != WSPM_SOLVER_CG) e = make_cond_handle(cs, &h);
        KrylovState *kst = nullptr;
        if (solver == WSPM_SOLVER_CG) {
            CgBuffers<double> w = carve_cg<double>(work, n, &used);
            kst = w.st;
            state_reset_kernel<<<1, 32, 0, cs>>>((unsigned int *)kst, (int)(sizeof(KrylovState) / 4));
            if (cg_persistent_enqueue<double>(A, vals, b, nullptr, x, dinv, w, tol, atol, maxiter, false, nullptr,
                                              cs) != WSPM_OK && e == cudaSuccess)
                e = cudaErrorLaunchFailure;
        } else if (solver == WSPM_SOLVER_BICGSTAB) {
            BicgBuffers<double> w = carve_bicgstab<double>(work, n, &used);
            kst = w.st;
            state_reset_kernel<<<1, 32, 0, cs>>>((unsigned int *)kst, (int)(sizeof(KrylovState) / 4));
            bicgstab_enqueue_init<double>(A, vals, b, nullptr, x, x, w, tol, atol, nullptr, maxiter, h, 1, cs);
            if (e == cudaSuccess)
                e = capture_while(cs, h, [&](cudaStream_t bs) {
                    bicgstab_enqueue_body<double>(A, vals, x, dinv, w, maxiter, h, 1, bs);
                });
        } else {
            const int m = restart < n ? restart : n;
            GmresBuffers<double> w = carve_gmres<double>(work, n, m, &used);
            kst = w.st;
            state_reset_kernel<<<1, 32, 0, cs>>>((unsigned int *)kst, (int)(sizeof(KrylovState) / 4));
            gmres_enqueue_init<double>(A, vals, b, nullptr, x, x, dinv, w, tol, atol, nullptr, maxiter, h, 1, cs);
            if (e == cudaSuccess)
                e = capture_while(cs, h, [&](cudaStream_t bs) {
                    gmres_enqueue_body<double>(A, vals, b, nullptr, x, dinv, w, maxiter, h, 1, bs);
                });
        }
        write_result_kernel<<<1, 32, 0, cs>>>(kst, result);
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

}  // namespace wspm

using namespace wspm;

static int soil_entry(int model, const double *h, int64_t n, const double *phi, int nphi, double *C, double *K,
                      double *theta, void *stream) {
    if (n < 0 || !phi || (n > 0 && !h)) return WSPM_BAD_ARG;
    SoilParams sp;
    sp.model = model;
    for (int j = 0; j < 6; ++j) sp.p[j] = j < nphi ? phi[j] : 0.0;
    return launch_soil(sp, h, n, C, K, theta, (cudaStream_t)stream);
}

extern "C" int wspm_soil_van_genuchten(const double *h, int64_t n, const double *phi, double *C, double *K,
                                       double *theta, void *stream) {
    return soil_entry(WSPM_SOIL_VAN_GENUCHTEN, h, n, phi, 6, C, K, theta, stream);
}

extern "C" int wspm_soil_exponential(const double *h, int64_t n, const double *phi, double *C, double *K,
                                     double *theta, void *stream) {
    return soil_entry(WSPM_SOIL_EXPONENTIAL, h, n, phi, 4, C, K, theta, stream);
}

static bool pattern_ok(const wspm_pattern *p) { return pattern_layout_ok(p) && p->diag_pos; }

extern "C" int wspm_assemble_richards(const wspm_mesh *mesh, const wspm_pattern *pat, const double *theta_m,
                                      const double *theta_n, const double *h_m, const double *K, const double *C,
                                      const double *Ks_elem, const double *quad_points, const double *weights,
                                      int32_t nq, double dt, const double *bc_val, double *vals, float *vals32,
                                      double *rhs, double *dinv, void *stream) {
    if (!mesh || !pattern_ok(pat) || !pat->inc_ptr || !pat->inc_width || !pat->inc_elem || !pat->inc_slots)
        return WSPM_BAD_ARG;
    if ((mesh->dim != 2 && mesh->dim != 3) || mesh->nv != mesh->dim + 1 || mesh->n_nodes != pat->n_rows)
        return WSPM_BAD_ARG;
    if (!mesh->conn || !mesh->coords || !theta_m || !theta_n || !h_m || !K || !C || !vals || !rhs)
        return WSPM_BAD_ARG;
    if (!quad_points || !weights || nq <= 0 || !(dt > 0.0) || !isfinite(dt)) return WSPM_BAD_ARG;
    double s[4], mc[4];
    quadrature_constants(mesh->dim, quad_points, weights, nq, s, mc);
    return launch_richards_assembly(mesh, pat, theta_m, theta_n, h_m, K, C, Ks_elem, s, mc, dt, bc_val, vals, vals32,
                                    rhs, dinv, (cudaStream_t)stream);
}

static bool incidence_ok(const wspm_pattern *p) {
    return p->inc_ptr && p->inc_width && p->inc_elem && p->inc_slots;
}

extern "C" int wspm_flux_dispersion_2d(const wspm_mesh *mesh, const wspm_pattern *pat, const double *h,
                                       const double *phi, double DL, double DT, double Dm, double *qx, double *qz,
                                       double *aq, double *Dxx, double *Dxz, double *Dzz, double *theta,
                                       void *stream) {
    if (!mesh || !pattern_ok(pat) || !incidence_ok(pat) || mesh->dim != 2 || mesh->nv != 3 ||
        mesh->n_nodes != pat->n_rows || !mesh->conn || !mesh->coords || !h || !phi)
        return WSPM_BAD_ARG;
    if (!qx || !qz || !aq || !Dxx || !Dxz || !Dzz || !theta) return WSPM_BAD_ARG;
    SoilParams sp;
    sp.model = WSPM_SOIL_VAN_GENUCHTEN;
    for (int j = 0; j < 6; ++j) sp.p[j] = phi[j];
    return launch_flux_dispersion(mesh, pat, h, sp, DL, DT, Dm, qx, qz, aq, Dxx, Dxz, Dzz, theta,
                                  (cudaStream_t)stream);
}

extern "C" int wspm_assemble_adr_2d(const wspm_mesh *mesh, const wspm_pattern *pat, const double *theta,
                                    const double *qx, const double *qz, const double *Dxx, const double *Dxz,
                                    const double *Dzz, const double *c_n, const double *c_up, double mu,
                                    double sorption, double mu_up, int32_t lumped, const double *quad_points,
                                    const double *weights, int32_t nq, double dt, double *vals, double *rhs,
                                    double *dinv, void *stream) {
    if (!mesh || !pattern_ok(pat) || !incidence_ok(pat) || mesh->dim != 2 || mesh->nv != 3 ||
        mesh->n_nodes != pat->n_rows || !mesh->conn || !mesh->coords)
        return WSPM_BAD_ARG;
    if (!theta || !qx || !qz || !Dxx || !Dxz || !Dzz || !c_n || !vals || !rhs) return WSPM_BAD_ARG;
    if (!quad_points || !weights || nq <= 0 || nq > 16 || !(dt > 0.0) || !isfinite(dt)) return WSPM_BAD_ARG;
    return launch_adr(mesh, pat, theta, qx, qz, Dxx, Dxz, Dzz, c_n, c_up, mu, sorption, mu_up, lumped, quad_points,
                      weights, nq, dt, vals, rhs, dinv, (cudaStream_t)stream);
}

extern "C" int wspm_apply_edge_terms(const wspm_pattern *pat, const wspm_edges *edges, int32_t mode, double flux,
                                     double c_in, const double *K, const double *theta, double *vals, double *rhs,
                                     void *stream) {
    if (!pattern_ok(pat) || !edges || !rhs || mode < 0 || mode > 3) return WSPM_BAD_ARG;
    if (edges->n_bnodes < 0) return WSPM_BAD_ARG;
    if (edges->n_bnodes > 0 && (!edges->node || !edges->e_cnt || !edges->e_local || !edges->e_other ||
                                !edges->e_kother || !edges->e_jac))
        return WSPM_BAD_ARG;
    if ((mode == WSPM_EDGE_DRAINAGE_WATER || mode == WSPM_EDGE_DRAINAGE_SOLUTE) && !K) return WSPM_BAD_ARG;
    if (mode == WSPM_EDGE_DRAINAGE_SOLUTE && !theta) return WSPM_BAD_ARG;
    if (mode >= WSPM_EDGE_CAUCHY && !vals) return WSPM_BAD_ARG;
    return launch_edge_terms(pat, edges, mode, flux, c_in, K, theta, vals, rhs, (cudaStream_t)stream);
}

extern "C" int wspm_spmv_f64(const wspm_pattern *pat, const double *vals, const double *x, double *y,
                             void *stream) {
    if (!pattern_ok(pat) || !vals || !x || !y) return WSPM_BAD_ARG;
    spmv_f64(make_sell(pat), vals, x, y, (cudaStream_t)stream);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

extern "C" int wspm_spmv_f32(const wspm_pattern *pat, const float *vals, const float *x, float *y, void *stream) {
    if (!pattern_ok(pat) || !vals || !x || !y) return WSPM_BAD_ARG;
    spmv_f32(make_sell(pat), vals, x, y, (cudaStream_t)stream);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

extern "C" int wspm_apply_dirichlet(const wspm_pattern *pat, const int32_t *nodes, const double *values,
                                    int32_t n_bc, double *vals, double *rhs, void *stream) {
    if (!pattern_ok(pat) || n_bc < 0 || (n_bc > 0 && (!nodes || !values)) || !vals || !rhs) return WSPM_BAD_ARG;
    if (n_bc == 0) return WSPM_OK;
    dirichlet_rows_kernel<<<(n_bc + 127) / 128, 128, 0, (cudaStream_t)stream>>>(make_sell(pat), pat->diag_pos, nodes,
                                                                               values, n_bc, vals, rhs);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

extern "C" int wspm_jacobi_dinv(const wspm_pattern *pat, const double *vals, double *dinv, void *stream) {
    if (!pattern_ok(pat) || !vals || !dinv) return WSPM_BAD_ARG;
    jacobi_kernel<<<(pat->n_rows + 255) / 256, 256, 0, (cudaStream_t)stream>>>(make_sell(pat), pat->diag_pos, vals,
                                                                              dinv);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

extern "C" int64_t wspm_krylov_workspace_doubles(int32_t n_rows, int32_t solver, int32_t restart) {
    if (n_rows <= 0) return -1;
    if (solver == WSPM_SOLVER_CG) return cg_workspace_doubles(n_rows, 8);
    if (solver == WSPM_SOLVER_BICGSTAB) return bicgstab_workspace_doubles(n_rows);
    if (solver == WSPM_SOLVER_GMRES) {
        if (restart < 1 || restart > 32) return -1;
        return gmres_workspace_doubles(n_rows, restart < n_rows ? restart : n_rows);
    }
    return -1;
}

extern "C" int wspm_krylov_solve(const wspm_pattern *pat, const double *vals, const double *b, double *x,
                                 const double *dinv, int32_t solver, double tol, double atol, int32_t maxiter,
                                 int32_t restart, double *work, int64_t work_doubles, int32_t *result,
                                 void *stream) {
    if (!pattern_ok(pat) || !vals || !b || !x || !work || !result) return WSPM_BAD_ARG;
    if (solver < WSPM_SOLVER_CG || solver > WSPM_SOLVER_GMRES) return WSPM_BAD_ARG;
    if (solver == WSPM_SOLVER_GMRES && (restart < 1 || restart > 32)) return WSPM_UNSUPPORTED;
    if (maxiter < 0 || !(tol >= 0.0) || !(atol >= 0.0)) return WSPM_BAD_ARG;
    const int64_t need = wspm_krylov_workspace_doubles(pat->n_rows, solver, restart);
    if (need < 0 || work_doubles < need) return WSPM_BAD_ARG;
    SolveKey key;
    std::memset(&key, 0, sizeof(key));
    key.pat_cols = pat->cols; key.pat_ptr = pat->slice_ptr; key.pat_width = pat->slice_width;
    key.pat_diag_off = pat->n_diags > 0 ? pat->diag_offsets : nullptr;
    key.vals = vals; key.b = b; key.x = x; key.dinv = dinv; key.work = work;
    key.result = result; key.nnz_padded = pat->nnz_padded; key.n = pat->n_rows; key.n_slices = pat->n_slices;
    key.max_width = pat->max_width; key.n_diags = pat->n_diags;
    WSPM_CUDA_TRY(cudaGetDevice(&key.device));
    key.solver = solver; key.maxiter = maxiter;
    key.restart = solver == WSPM_SOLVER_GMRES ? restart : 0; key.tol = tol; key.atol = atol;
    cudaGraphExec_t exec = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        for (auto &en : g_cache)
            if (en.key == key) { exec = en.exec; break; }
        if (!exec) {
            cudaGraph_t graph = nullptr;
            int rc = build_solve_graph(pat, vals, b, x, dinv, solver, tol, atol, maxiter, restart, work, result,
                                       &exec, &graph);
            if (rc != WSPM_OK) return rc;
            if (g_cache.size() >= kCacheMax) {
                cudaGraphExecDestroy(g_cache.front().exec);
                cudaGraphDestroy(g_cache.front().graph);
                g_cache.erase(g_cache.begin());
            }
            g_cache.push_back({key, exec, graph});
        }
    }
    WSPM_CUDA_TRY(cudaGraphLaunch(exec, (cudaStream_t)stream));
    return WSPM_OK;
}

__global__ void copy_k_kernel(const KrylovState *st, int32_t *out) { *out = st->k; }

extern "C" int wspm_cg_iterations(const wspm_pattern *pat, int32_t mode, const void *vals, const void *b, void *x,
                                  const void *dinv, int32_t iters, double *work, int64_t work_doubles,
                                  int32_t *iters_done, void *stream) {
    if (!pattern_ok(pat) || !vals || !b || !x || !work || iters < 0 || mode < 0 || mode > 7) return WSPM_BAD_ARG;
    const bool fp32 = (mode & WSPM_CGIT_FP32) != 0;
    const bool pipelined = (mode & WSPM_CGIT_PIPELINED) != 0;
    const bool ws = (mode & WSPM_CGIT_NO_WARP_SPECIALIZATION) == 0;
    if (work_doubles < cg_workspace_doubles(pat->n_rows, fp32 ? 4 : 8)) return WSPM_BAD_ARG;
    const Sell A = make_sell(pat);
    cudaStream_t st = (cudaStream_t)stream;
    int64_t used = 0;
    int rc;
    KrylovState *state;
    // tolerance 0: the solve runs `iters` iterations unless the residual is exactly 0 or non-finite
    if (fp32) {
        CgBuffers<float> w = carve_cg<float>(work, pat->n_rows, &used);
        state = w.st;
        state_reset_kernel<<<1, 32, 0, st>>>((unsigned int *)w.st, (int)(sizeof(KrylovState) / 4));
        if (pipelined)
            rc = pcg_persistent_enqueue<float>(A, (const float *)vals, (const float *)b, nullptr, (float *)x,
                                               (const float *)dinv, w, 0.0, 0.0, iters, false, nullptr, st, ws);
        else
            rc = cg_persistent_enqueue<float>(A, (const float *)vals, (const float *)b, nullptr, (float *)x,
                                              (const float *)dinv, w, 0.0, 0.0, iters, false, nullptr, st);
    } else {
        CgBuffers<double> w = carve_cg<double>(work, pat->n_rows, &used);
        state = w.st;
        state_reset_kernel<<<1, 32, 0, st>>>((unsigned int *)w.st, (int)(sizeof(KrylovState) / 4));
        if (pipelined)
            rc = pcg_persistent_enqueue<double>(A, (const double *)vals, (const double *)b, nullptr, (double *)x,
                                                (const double *)dinv, w, 0.0, 0.0, iters, false, nullptr, st, ws);
        else
            rc = cg_persistent_enqueue<double>(A, (const double *)vals, (const double *)b, nullptr, (double *)x,
                                               (const double *)dinv, w, 0.0, 0.0, iters, false, nullptr, st);
    }
    if (rc == WSPM_OK && iters_done) copy_k_kernel<<<1, 1, 0, st>>>(state, iters_done);
    return rc;
}

extern "C" const char *wspm_version(void) { return "wspm-b200 0.1 (sm_100a)"; }

extern "C" const char *wspm_status_string(int status) {
    switch (status) {
        case WSPM_OK: return "ok";
        case WSPM_MAXITER: return "iteration cap reached";
        case WSPM_NAN: return "non-finite value";
        case WSPM_BREAKDOWN: return "Krylov breakdown";
        case WSPM_BAD_ARG: return "invalid argument";
        case WSPM_CUDA_ERROR: return "CUDA error";
        case WSPM_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}
