// Batched ensemble of independent 2D Richards domains in one persistent launch.
//
// The domains are the diagonal blocks of one mesh: node ranges
// [node_off[d], node_off[d+1]), elements never cross domains, so the union
// pattern is block diagonal.  A CTA owns a whole domain at a time and runs
// that domain's complete implicit step -- soil law with the domain's van
// Genuchten parameters, row-gather assembly with fused Dirichlet rows, Jacobi
// preconditioned CG with block-level reductions, the Picard norm and test --
// then adapts the domain's dt and advances its time (richards_solver_v2.py:
// 91-168 per domain).  Domains are taken from a device work queue in the
// given order (largest first), so CTAs that draw small domains go on to the
// next one: no CTA ever waits for another, and every loop has an iteration
// cap.  The assembly walks each row's incident elements in ascending element
// id, as the single-domain row kernel does, so a domain's matrix is bitwise
// the matrix the single-domain path assembles for it.
//
// With a cluster size CS > 1 a domain is taken by a thread-block cluster of CS
// CTAs (one per SM): CTA rank c owns the c-th slice of the domain's rows, the
// phases that read other slices (soil -> assembly, p -> SpMV, h_m -> residual)
// are separated by hardware cluster barriers, and every reduction sums the
// CTAs' partials through distributed shared memory in rank order, so all CTAs
// of the cluster hold bitwise identical scalars and take the same branches.
// This spreads the largest domains, which bound the step, over CS SMs.
#include <cooperative_groups.h>

#include "common.cuh"
#include "soil.cuh"
#include "krylov.cuh"
#include "graph.cuh"

namespace wspm {

void quadrature_constants(int dim, const double *Q, const double *W, int nq, double s[4], double m[4]);

struct EnsArgs {
    Sell A;
    const int32_t *diag_pos;
    const int64_t *inc_ptr;
    const int32_t *inc_width;
    const int32_t *inc_elem;
    const uint32_t *inc_slots;
    const int32_t *conn;
    const double *coords;
    const int64_t *node_off;
    const int32_t *order;
    const double *phi;
    const double *Ks_elem;
    const double *bc_val;
    double s[3], mc[3];
    double krylov_tol, picard_tol, tmax, lambda_amp, lambda_red;
    int krylov_maxiter, picard_maxiter, picard_relative, m_it, M_it, n_domains;
    double *h_n, *h_m, *theta_n, *C, *K, *theta_m, *rhs, *dinv, *x, *r, *z, *p, *q, *vals;
    double *dt, *t, *err;
    int32_t *its, *kits, *status;
    unsigned int *queue;
};

// Barrier over the CTAs that share a domain (the block, or the cluster).
template <int CS>
__device__ __forceinline__ void domain_sync() {
    if constexpr (CS == 1) __syncthreads();
    else cooperative_groups::this_cluster().sync();
}

// Sums of NV values over the domain's CTAs, broadcast to every thread.  CS > 1:
// each CTA publishes its block sum in shared memory, one cluster barrier, then
// thread j of every CTA adds component j over the ranks in rank order.  The
// published slots alternate between two buffers: a CTA rewrites a buffer only
// two sums later, after a cluster barrier that every CTA reaches once it has
// read that buffer.
template <int CS, int NV>
__device__ __forceinline__ void domain_allsum(double (&v)[NV], int &parity) {
    __shared__ double bc[NV];
    __shared__ double cpart[2][NV];
    block_sum<double, NV>(v);
    if constexpr (CS == 1) {
        if (threadIdx.x == 0) {
#pragma unroll
            for (int j = 0; j < NV; ++j) bc[j] = v[j];
        }
    } else {
        cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int j = 0; j < NV; ++j) cpart[parity][j] = v[j];
        }
        cl.sync();
        if (threadIdx.x < NV) {
            double t = 0.0;
            for (int r = 0; r < CS; ++r) t += *cl.map_shared_rank(&cpart[parity][threadIdx.x], r);
            bc[threadIdx.x] = t;
        }
        parity ^= 1;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = bc[j];
    __syncthreads();
}

// Row i of the Richards system (P1 triangles), elements in ascending id.
template <int MW>
__device__ __forceinline__ void ens_assemble_row(const EnsArgs &a, const Sell &A, int i, double inv_dt, double *acc,
                                                 int TB) {
    const int s = i >> 5, lane = i & 31;
    const int width = row_width(A, i);
    for (int k = 0; k < width; ++k) acc[k * TB] = 0.0;
    const int dpos = a.diag_pos[i];
    const double bcv = a.bc_val ? a.bc_val[i] : __longlong_as_double(0x7ff8000000000000ULL);
    double rhs_i, diag;
    if (!isnan(bcv)) {
        acc[dpos * TB] = 1.0;
        rhs_i = bcv;
        diag = 1.0;
    } else {
        const double Ci = a.C[i];
        const double storage = a.theta_m[i] - a.theta_n[i] - Ci * a.h_m[i];
        double bsum = 0.0;
        const int deg = a.inc_width[s];
        const int64_t ib = a.inc_ptr[s] + lane;
        for (int k = 0; k < deg; ++k) {
            const int e = a.inc_elem[ib + (int64_t)kSlice * k];
            if (e < 0) continue;
            const uint32_t packed = a.inc_slots[ib + (int64_t)kSlice * k];
            const int li = packed & 3;
            int nd[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) nd[j] = a.conn[3 * (int64_t)e + j];
            const double x0 = a.coords[2 * nd[0]], y0 = a.coords[2 * nd[0] + 1];
            const double J00 = a.coords[2 * nd[1]] - x0, J01 = a.coords[2 * nd[1] + 1] - y0;
            const double J10 = a.coords[2 * nd[2]] - x0, J11 = a.coords[2 * nd[2] + 1] - y0;
            const double detJ = J00 * J11 - J01 * J10;
            const double id = 1.0 / detJ;
            double G[2][3];
            G[0][1] = J11 * id;  G[1][1] = -J10 * id;
            G[0][2] = -J01 * id; G[1][2] = J00 * id;
            G[0][0] = -(G[0][1] + G[0][2]);
            G[1][0] = -(G[1][1] + G[1][2]);
            double Kbar = 0.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) Kbar = fma(a.s[j], a.K[nd[j]], Kbar);
            if (a.Ks_elem) Kbar *= a.Ks_elem[e];
            const double kd = Kbar * detJ;
            const double Ml = a.mc[li] * detJ;
            // column li of G by selects (an indexed register array would live in local memory)
            const double g0 = li == 0 ? G[0][0] : (li == 1 ? G[0][1] : G[0][2]);
            const double g1 = li == 0 ? G[1][0] : (li == 1 ? G[1][1] : G[1][2]);
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double gg = fma(g0, G[0][j], 0.0);
                gg = fma(g1, G[1][j], gg);
                double v = kd * gg;
                if (j == li) v += inv_dt * (Ml * Ci);
                const int kpos = (packed >> (2 + 6 * j)) & 63;
                acc[kpos * TB] += v;
            }
            bsum += -kd * g1 - inv_dt * (Ml * storage);
        }
        rhs_i = bsum;
        diag = acc[dpos * TB];
    }
    a.rhs[i] = rhs_i;
    a.dinv[i] = 1.0 / (diag != 0.0 ? diag : 1.0);
    for (int k = 0; k < width; ++k) a.vals[entry_pos(A, i, k)] = acc[k * TB];
}

// Row i of the (SELL) matrix times the vector given by xf.  The values are
// written by this kernel (every Picard iteration re-assembles the domain), so
// they are read with plain coherent loads, never through the read-only path;
// only the pattern arrays use it.  Entries accumulate in row order, as in
// sell_row_dot.
template <int MW, typename XF>
__device__ __forceinline__ double ens_row_dot(const Sell &A, const double *vals, int i, XF xf) {
    const int s = i >> 5, lane = i & 31;
    const int w = __ldg(A.slice_width + s);
    const int64_t base = __ldg(A.slice_ptr + s) + lane;
    double acc = 0.0;
#pragma unroll 8
    for (int k = 0; k < w; ++k) {
        const int64_t o = base + (int64_t)kSlice * k;
        acc = fma(vals[o], xf(__ldg(A.cols + o)), acc);
    }
    return acc;
}

template <int MW, int CS>
__global__ void __launch_bounds__(512, 1) ensemble_step_kernel(EnsArgs a) {
    extern __shared__ double acc_sm[];   // [MW][blockDim.x]
    __shared__ int s_j;
    int par = 0;                         // buffer parity of domain_allsum
    const int rank = CS == 1 ? 0 : (int)cooperative_groups::this_cluster().block_rank();
    const int TB = blockDim.x;
    const Sell A = a.A;
    double *acc = acc_sm + threadIdx.x;
    double *const hn = a.h_n, *const hm = a.h_m, *const x = a.x, *const r = a.r, *const z = a.z;
    double *const p = a.p, *const q = a.q;
    const double *const vals = a.vals, *const dinv = a.dinv, *const rhs = a.rhs;
    for (;;) {
        if (rank == 0 && threadIdx.x == 0) s_j = (int)atomicAdd(a.queue, 1u);
        domain_sync<CS>();
        int j;
        if constexpr (CS == 1) j = s_j;
        else j = *cooperative_groups::this_cluster().map_shared_rank(&s_j, 0);
        domain_sync<CS>();                                // rank 0 rewrites s_j only after every rank read it
        if (j >= a.n_domains) break;
        const int d = a.order[j];
        if (!(a.t[d] < a.tmax)) continue;                 // finished domain: masked out
        // this CTA's slice [n0, n1) of the domain's rows
        const int d0 = (int)a.node_off[d], d1 = (int)a.node_off[d + 1];
        const int slice = (d1 - d0 + CS - 1) / CS;
        const int n0 = min(d1, d0 + rank * slice), n1 = min(d1, n0 + slice);
        SoilParams sp;
        sp.model = WSPM_SOIL_VAN_GENUCHTEN;
        for (int k = 0; k < 6; ++k) sp.p[k] = a.phi[6 * d + k];
        const double dtd = a.dt[d];
        const double inv_dt = 1.0 / dtd;
        for (int i = n0 + threadIdx.x; i < n1; i += TB) {
            double c, k, th;
            soil_eval(sp, hn[i], c, k, th);
            a.theta_n[i] = th;
            hm[i] = hn[i];
        }
        domain_sync<CS>();
        int it = 0, kits = 0, status = WSPM_OK;
        double err = __longlong_as_double(0x7ff0000000000000LL);   // +inf
        while (it < a.picard_maxiter && !(err < a.picard_tol)) {
            for (int i = n0 + threadIdx.x; i < n1; i += TB) {
                double c, k, th;
                soil_eval(sp, hm[i], c, k, th);
                a.C[i] = c;
                a.K[i] = k;
                a.theta_m[i] = th;
            }
            domain_sync<CS>();                            // K of the slice's neighbours
            for (int i = n0 + threadIdx.x; i < n1; i += TB) ens_assemble_row<MW>(a, A, i, inv_dt, acc, TB);
            __syncthreads();
            // ---- Jacobi-CG from x0 = h_m (textbook recurrences, stop on ||r|| <= tol ||b||)
            double v3[3] = {0.0, 0.0, 0.0};
            for (int i = n0 + threadIdx.x; i < n1; i += TB) {
                x[i] = hm[i];
                const double ri = rhs[i] - ens_row_dot<MW>(A, vals, i, [hm](int c) { return hm[c]; });
                const double zi = dinv[i] * ri;
                r[i] = ri;
                z[i] = zi;
                p[i] = zi;
                v3[0] += ri * zi;
                v3[1] += ri * ri;
                v3[2] += rhs[i] * rhs[i];
            }
            domain_allsum<CS, 3>(v3, par);
            double gamma = v3[0], rr = v3[1];
            const double atol2 = a.krylov_tol * a.krylov_tol * v3[2];
            int k = 0;
            while (rr > atol2 && k < a.krylov_maxiter) {
                double v1[1] = {0.0};
                for (int i = n0 + threadIdx.x; i < n1; i += TB) {
                    const double qi = ens_row_dot<MW>(A, vals, i, [p](int c) { return p[c]; });
                    q[i] = qi;
                    v1[0] += p[i] * qi;
                }
                domain_allsum<CS, 1>(v1, par);
                const double alpha = gamma / v1[0];
                double v2[2] = {0.0, 0.0};
                for (int i = n0 + threadIdx.x; i < n1; i += TB) {
                    x[i] = fma(alpha, p[i], x[i]);
                    const double ri = fma(-alpha, q[i], r[i]);
                    r[i] = ri;
                    const double zi = dinv[i] * ri;
                    z[i] = zi;
                    v2[0] += ri * zi;
                    v2[1] += ri * ri;
                }
                domain_allsum<CS, 2>(v2, par);
                const double beta = v2[0] / gamma;
                gamma = v2[0];
                rr = v2[1];
                for (int i = n0 + threadIdx.x; i < n1; i += TB) p[i] = fma(beta, p[i], z[i]);
                domain_sync<CS>();                        // p of the neighbouring slices for the next SpMV
                ++k;
                if (!isfinite(rr) || !isfinite(alpha)) break;
            }
            kits += k;
            // ---- Picard error and update
            double ve[2] = {0.0, 0.0};
            for (int i = n0 + threadIdx.x; i < n1; i += TB) {
                const double dx = x[i] - hm[i];
                ve[0] += dx * dx;
                ve[1] += x[i] * x[i];
            }
            domain_allsum<CS, 2>(ve, par);
            err = a.picard_relative ? sqrt(ve[0]) / sqrt(ve[1]) : sqrt(ve[0]);
            for (int i = n0 + threadIdx.x; i < n1; i += TB) hm[i] = x[i];
            domain_sync<CS>();
            ++it;
            if (!isfinite(err)) { status = WSPM_NAN; break; }
        }
        if (status == WSPM_OK && !(err < a.picard_tol)) status = WSPM_MAXITER;
        for (int i = n0 + threadIdx.x; i < n1; i += TB) hn[i] = hm[i];
        if (rank == 0 && threadIdx.x == 0) {
            a.its[d] = it;
            a.kits[d] = kits;
            a.status[d] = status;
            a.err[d] = err;
            // adapt_time_step (richards_solver_v2.py:91-105); time advances by the new dt (:352)
            const double dt_new = it <= a.m_it ? a.lambda_amp * dtd : (it <= a.M_it ? dtd : a.lambda_red * dtd);
            a.t[d] += dt_new;
            a.dt[d] = dt_new;
        }
        __syncthreads();
    }
}

// One CTA (CS = 1) or one cluster of CS CTAs per domain at a time, as many
// CTAs (whole clusters) as can be resident at once, at most one per domain.
template <int MW, int CS>
static cudaError_t ensemble_launch(const EnsArgs &a, int TB, int sms, int n_domains, cudaStream_t st) {
    const int mw = MW > 0 ? MW : 64;
    const size_t smem = (size_t)mw * TB * sizeof(double);
    cudaError_t e = cudaSuccess;
    if (smem > 48 * 1024)
        e = cudaFuncSetAttribute(ensemble_step_kernel<MW, CS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per = 0;
    if (e == cudaSuccess && CS > 8)   // above the portable cluster size: opt in (the launch fails where unsupported)
        e = cudaFuncSetAttribute(ensemble_step_kernel<MW, CS>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, ensemble_step_kernel<MW, CS>, TB, smem);
    if (e != cudaSuccess) return e;
    int clusters = sms * (per > 0 ? per : 1) / CS;
    if (clusters > n_domains) clusters = n_domains;
    if (clusters < 1) clusters = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(clusters * CS);
    cfg.blockDim = dim3(TB);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (CS > 1) {
        // no more clusters than can be resident together: GPCs whose SM count is not a multiple of CS hold
        // fewer, and a cluster that could only start after another finished would run its domain last
        int fit = 0;
        if (cudaOccupancyMaxActiveClusters(&fit, ensemble_step_kernel<MW, CS>, &cfg) == cudaSuccess && fit > 0 &&
            clusters > fit) {
            clusters = fit;
            cfg.gridDim = dim3(clusters * CS);
        }
        cudaGetLastError();   // a failed query leaves the grid as it was
    }
    e = cudaLaunchKernelEx(&cfg, ensemble_step_kernel<MW, CS>, a);
    if (e != cudaSuccess) cudaGetLastError();   // a refused launch (e.g. a cluster size this GPU lacks) is not sticky
    return e;
}

}  // namespace wspm

using namespace wspm;

extern "C" int64_t wspm_ensemble_workspace_doubles(int32_t n_rows, int64_t nnz_padded) {
    if (n_rows <= 0 || nnz_padded <= 0) return 0;
    return 12 * (int64_t)n_rows + nnz_padded + 64;
}

static int ensemble_enqueue(const wspm_mesh *mesh, const wspm_pattern *pat, const wspm_ensemble *ens,
                            int32_t block_threads, cudaStream_t st);

extern "C" int wspm_ensemble_step(const wspm_mesh *mesh, const wspm_pattern *pat, const wspm_ensemble *ens,
                                  int32_t block_threads, void *stream) {
    return ensemble_enqueue(mesh, pat, ens, block_threads, (cudaStream_t)stream);
}

// ---- several steps on the device: WHILE(any domain below tmax && steps < max){ step; tail }
namespace {

// active[d] = t[d] < tmax; its_total = 0; run[0] = steps = 0, run[1] = active domains.
__global__ void ens_run_init_kernel(int D, const double *t, double tmax, int32_t *active, int64_t *its_total,
                                    int32_t *run, int max_steps, cudaGraphConditionalHandle cond) {
    __shared__ int s_n;
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    int n = 0;
    for (int d = threadIdx.x; d < D; d += blockDim.x) {
        const int a = t[d] < tmax;
        active[d] = a;
        its_total[d] = 0;
        n += a;
    }
    atomicAdd(&s_n, n);
    __syncthreads();
    if (threadIdx.x == 0) {
        run[0] = 0;
        run[1] = s_n;
        cudaGraphSetConditional(cond, (s_n > 0 && max_steps > 0) ? 1u : 0u);
    }
}

// After a step: the Picard iterations of the domains that were active are added up, the
// step is counted, the active set is recomputed and the loop continues while a domain is
// below tmax and fewer than max_steps steps ran.
__global__ void ens_run_tail_kernel(int D, const double *t, double tmax, const int32_t *its, int32_t *active,
                                    int64_t *its_total, int32_t *run, int max_steps,
                                    cudaGraphConditionalHandle cond) {
    __shared__ int s_n;
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    int n = 0;
    for (int d = threadIdx.x; d < D; d += blockDim.x) {
        if (active[d]) its_total[d] += its[d];
        const int a = t[d] < tmax;
        active[d] = a;
        n += a;
    }
    atomicAdd(&s_n, n);
    __syncthreads();
    if (threadIdx.x == 0) {
        const int steps = run[0] + 1;
        run[0] = steps;
        run[1] = s_n;
        cudaGraphSetConditional(cond, (s_n > 0 && steps < max_steps) ? 1u : 0u);
    }
}

}  // namespace

extern "C" int wspm_ensemble_run(const wspm_mesh *mesh, const wspm_pattern *pat, const wspm_ensemble *ens,
                                 int32_t block_threads, int32_t max_steps, int32_t *active, int64_t *its_total,
                                 int32_t *run, void *stream) {
    if (!ens || !active || !its_total || !run || max_steps < 0) return WSPM_BAD_ARG;
    cudaStream_t cs;
    WSPM_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    if (cudaGraphCreate(&g, 0) != cudaSuccess) { cudaStreamDestroy(cs); return WSPM_CUDA_ERROR; }
    int rc = WSPM_OK;
    cudaError_t e = cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e == cudaSuccess) {
        cudaGraphConditionalHandle h;
        e = make_cond_handle(cs, &h);
        const int D = ens->n_domains;
        if (e == cudaSuccess) {
            ens_run_init_kernel<<<1, 256, 0, cs>>>(D, ens->t, ens->tmax, active, its_total, run, max_steps, h);
            e = capture_while(cs, h, [&](cudaStream_t bs) {
                rc = ensemble_enqueue(mesh, pat, ens, block_threads, bs);
                ens_run_tail_kernel<<<1, 256, 0, bs>>>(D, ens->t, ens->tmax, ens->its, active, its_total, run,
                                                       max_steps, h);
            });
        }
        cudaGraph_t out = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(cs, &out);
        if (e == cudaSuccess) e = e2;
    }
    cudaStreamDestroy(cs);
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess && rc == WSPM_OK) e = cudaGraphInstantiate(&exec, g, 0);
    if (e == cudaSuccess && rc == WSPM_OK) e = cudaGraphLaunch(exec, (cudaStream_t)stream);
    // the executable graph is released once the launch completes (freed asynchronously)
    if (exec) cudaGraphExecDestroy(exec);
    cudaGraphDestroy(g);
    if (rc != WSPM_OK) return rc;
    return e == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

static int ensemble_enqueue(const wspm_mesh *mesh, const wspm_pattern *pat, const wspm_ensemble *ens,
                            int32_t block_threads, cudaStream_t st) {
    if (!mesh || !pat || !ens || mesh->dim != 2 || !ens->node_off || !ens->order || !ens->phi || !ens->h_n ||
        !ens->work || !ens->dt || !ens->t || !ens->its || !ens->kits || !ens->status || !ens->err || !ens->queue ||
        ens->n_domains <= 0 || ens->nq <= 0 || ens->nq > 16 || pat->n_rows != mesh->n_nodes)
        return WSPM_BAD_ARG;
    if (pat->n_diags > 0) return WSPM_UNSUPPORTED;        // domains of different size do not share diagonals
    const int64_t n = pat->n_rows;
    if (ens->work_doubles < wspm_ensemble_workspace_doubles(pat->n_rows, pat->nnz_padded)) return WSPM_BAD_ARG;
    const int TB = block_threads == 0 ? 512 : block_threads;
    if (TB != 128 && TB != 256 && TB != 512) return WSPM_BAD_ARG;
    if (ens->cluster_size != 0 && ens->cluster_size != 1 && ens->cluster_size != 2 && ens->cluster_size != 4 &&
        ens->cluster_size != 8 && ens->cluster_size != 16)
        return WSPM_BAD_ARG;
    EnsArgs a;
    a.A = make_sell(pat);
    a.diag_pos = pat->diag_pos;
    a.inc_ptr = pat->inc_ptr; a.inc_width = pat->inc_width; a.inc_elem = pat->inc_elem; a.inc_slots = pat->inc_slots;
    a.conn = mesh->conn; a.coords = mesh->coords;
    a.node_off = ens->node_off; a.order = ens->order; a.phi = ens->phi; a.Ks_elem = ens->Ks_elem;
    a.bc_val = ens->bc_val;
    double s4[4], m4[4];
    quadrature_constants(2, ens->quad_points, ens->weights, ens->nq, s4, m4);
    for (int j = 0; j < 3; ++j) { a.s[j] = s4[j]; a.mc[j] = m4[j]; }
    a.krylov_tol = ens->krylov_tol; a.krylov_maxiter = ens->krylov_maxiter;
    a.picard_tol = ens->picard_tol; a.picard_maxiter = ens->picard_maxiter; a.picard_relative = ens->picard_relative;
    a.tmax = ens->tmax; a.m_it = ens->m_it; a.M_it = ens->M_it;
    a.lambda_amp = ens->lambda_amp; a.lambda_red = ens->lambda_red;
    a.n_domains = ens->n_domains;
    double *w = ens->work;
    double **vecs[12] = {&a.h_m, &a.theta_n, &a.C, &a.K, &a.theta_m, &a.rhs, &a.dinv, &a.x, &a.r, &a.z, &a.p, &a.q};
    for (int v = 0; v < 12; ++v) { *vecs[v] = w; w += n; }
    a.vals = w;
    a.h_n = ens->h_n;
    a.dt = ens->dt; a.t = ens->t; a.err = ens->err;
    a.its = ens->its; a.kits = ens->kits; a.status = ens->status;
    a.queue = ens->queue;
    if (cudaMemsetAsync(ens->queue, 0, sizeof(uint32_t), st) != cudaSuccess) return WSPM_CUDA_ERROR;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int cs = ens->cluster_size == 0 ? 1 : ens->cluster_size;
    cudaError_t e = cudaSuccess;
    WSPM_WIDTH_DISPATCH(pat->max_width, {
        if (cs == 1) e = ensemble_launch<MW, 1>(a, TB, sms, ens->n_domains, st);
        else if (cs == 2) e = ensemble_launch<MW, 2>(a, TB, sms, ens->n_domains, st);
        else if (cs == 4) e = ensemble_launch<MW, 4>(a, TB, sms, ens->n_domains, st);
        else if (cs == 8) e = ensemble_launch<MW, 8>(a, TB, sms, ens->n_domains, st);
        else e = ensemble_launch<MW, 16>(a, TB, sms, ens->n_domains, st);
    });
    return e == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}
