/*
 * wspm.h -- C ABI of libwspm.so, the B200 (sm_100a) implementation of the
 * JAX-WSPM implicit P1-FEM Picard step.
 *
 * Conventions
 *  - Every array argument is a DEVICE pointer (caller-allocated; the library
 *    never allocates device memory).  Sizes are explicit.  `stream` is a
 *    cudaStream_t passed as void*; NULL means the legacy default stream.
 *  - Every entry point returns an int status (WSPM_OK = 0).  Launch and
 *    argument errors are reported synchronously; numerical outcomes
 *    (iteration caps, NaN, breakdown) are written to device status words
 *    so that no call has to synchronise with the host.
 *  - Sparse matrices use the SELL-32 layout described by wspm_pattern: rows
 *    are grouped in slices of 32; entry k of row i lives at
 *    slice_ptr[i/32] + 32*k + i%32.  Padding entries have column = own row
 *    and value 0.  Structured meshes may use the DIA variant (see
 *    wspm_pattern.n_diags).
 *  - Meshes: conn is element-major int32 [E*nv] (0-based), coords is
 *    node-major float64 [N*dim].
 *
 * The reference (JAX-WSPM) is pure Python + JAX; each entry point below names
 * the reference function whose behaviour it implements (file:line within the
 * reference project).  Python shims with the reference's own signatures live
 * in jax-wspm_b200/src/.
 */
#ifndef WSPM_H
#define WSPM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define WSPM_OK            0
#define WSPM_MAXITER       1   /* Krylov or Picard iteration cap reached      */
#define WSPM_NAN           2   /* non-finite residual / iterate               */
#define WSPM_BREAKDOWN     3   /* Krylov breakdown (rho, alpha or omega = 0)  */
#define WSPM_BAD_ARG      10   /* invalid argument (null pointer, size, ...)  */
#define WSPM_CUDA_ERROR   11   /* a CUDA runtime call failed                  */
#define WSPM_UNSUPPORTED  12   /* feature/combination not implemented         */

/* ---- solver / model ids ------------------------------------------------ */
#define WSPM_SOLVER_CG        0
#define WSPM_SOLVER_BICGSTAB  1
#define WSPM_SOLVER_GMRES     2
#define WSPM_PRECOND_NONE     0
#define WSPM_PRECOND_JACOBI   1
#define WSPM_PRECOND_ILU      2   /* the reference's create_ilu0 (symmetric Gauss-Seidel form) */
#define WSPM_PRECOND_SSOR     3   /* the reference's create_ssor: omega (D/omega + L)^-1        */
#define WSPM_PRECOND_BLOCK_JACOBI 4
#define WSPM_PRECOND_ILU0     5   /* true ILU(0) on A's pattern (wspm_ilu0_factor), not the reference's ilu */
#define WSPM_SOIL_VAN_GENUCHTEN 0
#define WSPM_SOIL_EXPONENTIAL   1

/* ---- data descriptors -------------------------------------------------- */
typedef struct wspm_mesh {
    int32_t n_nodes;
    int32_t n_elems;
    int32_t dim;              /* 2 (triangles) or 3 (tetrahedra)             */
    int32_t nv;               /* vertices per element: dim + 1               */
    const int32_t *conn;      /* [n_elems * nv]                              */
    const double  *coords;    /* [n_nodes * dim]                             */
} wspm_mesh;

typedef struct wspm_pattern {
    int32_t n_rows;
    int32_t n_slices;         /* ceil(n_rows / 32)                           */
    int32_t max_width;        /* max over slices of slice_width              */
    int32_t max_inc;          /* max over slices of inc_width                */
    int64_t nnz_padded;       /* slice_ptr[n_slices]                         */
    const int64_t *slice_ptr; /* [n_slices + 1]                              */
    const int32_t *slice_width;/* [n_slices]                                 */
    const int32_t *cols;      /* [nnz_padded]                                */
    const int32_t *diag_pos;  /* [n_rows] position k of the diagonal entry   */
    /* node -> element incidence, same sliced layout (element ids ascending) */
    const int64_t *inc_ptr;   /* [n_slices + 1]                              */
    const int32_t *inc_width; /* [n_slices]                                  */
    const int32_t *inc_elem;  /* element id, -1 = padding                    */
    const uint32_t *inc_slots;/* bits 0-1: local vertex of the row's node;
                                 bits 2+6j..7+6j: row position of vertex j   */
    /* DIA layout (n_diags > 0): the matrix holds n_diags diagonals with column
     * offsets diag_offsets[k]; entry k of row i is at k*ld + i with
     * ld = 32*n_slices (slice_ptr/slice_width/cols then describe the same
     * layout: width n_diags everywhere).  Used when every row's column
     * offsets belong to one small set (structured meshes): no column-index
     * stream is read by the sparse kernels.                               */
    int32_t n_diags;
    int32_t pad_;
    const int32_t *diag_offsets;
} wspm_pattern;

/* Host-side pattern builder (replaces the reference's per-assembly COO fill +
 * BCOO.sum_duplicates, src/numerics/assembly_re_v2.py:114-152 and
 * assembly_re_3D.py:118-151, by a pattern built once per mesh).
 * elements: [n_elems * nv] 0-based vertex ids (nv = 3 triangles, 4 tetrahedra);
 * extra_pairs: [n_extra * 2] node pairs that need matrix slots although no
 * element holds both (boundary edges), added in both directions, or NULL.
 * layout: WSPM_LAYOUT_AUTO (DIA when every row's column offsets belong to one
 * set of at most 16, else SELL-32), _SELL or _DIA.  On success *out holds host
 * arrays (free with wspm_pattern_free) from which a wspm_pattern is made by
 * uploading them to the device.  WSPM_BAD_ARG for ids out of range or a node
 * in no element; WSPM_UNSUPPORTED for more than 63 diagonals (DIA) or rows
 * longer than 63 (SELL).  Single-threaded, O(E nv^2 log).                  */
#define WSPM_LAYOUT_AUTO 0
#define WSPM_LAYOUT_SELL 1
#define WSPM_LAYOUT_DIA  2
typedef struct wspm_pattern_host {
    int32_t n_rows, n_slices, max_width, max_inc, n_diags, layout;
    int64_t nnz;              /* unique (row, col) pairs                     */
    int64_t nnz_padded;       /* storage slots                               */
    int64_t n_inc;            /* incidence slots (inc_ptr[n_slices])         */
    int64_t ld;               /* DIA: 32 * n_slices; SELL: 0                 */
    int64_t *csr_indptr;      /* [n_rows + 1]                                */
    int32_t *csr_indices;     /* [nnz], ascending per row                    */
    int64_t *sell_index;      /* [nnz] CSR entry -> storage slot             */
    int64_t *slice_ptr;       /* [n_slices + 1]                              */
    int32_t *slice_width;     /* [n_slices]                                  */
    int32_t *cols;            /* [nnz_padded]                                */
    int32_t *diag_pos;        /* [n_rows]                                    */
    int32_t *diag_offsets;    /* [n_diags]                                   */
    int64_t *inc_ptr;         /* [n_slices + 1]                              */
    int32_t *inc_width;       /* [n_slices]                                  */
    int32_t *inc_elem;        /* [n_inc], -1 = padding                       */
    uint32_t *inc_slots;      /* [n_inc], packed as in wspm_pattern          */
} wspm_pattern_host;
int wspm_pattern_build(const int64_t *elements, int64_t n_elems, int32_t nv, int32_t n_nodes,
                       const int64_t *extra_pairs, int64_t n_extra, int32_t layout, wspm_pattern_host **out);
void wspm_pattern_free(wspm_pattern_host *p);
/* Device-side pattern builder: the arrays of wspm_pattern_build (no extra
 * pairs), element for element, built on the GPU from the connectivity already
 * there (conn: int32 [n_elems * nv], device).  Same reference function as the
 * host builder.  Two phases, because the library allocates nothing:
 *   wspm_pattern_device_count: fills *sizes (host struct) and leaves its work in
 *     `scratch` (device, wspm_pattern_device_scratch_bytes bytes); synchronises
 *     with the host once to read the sizes;
 *   wspm_pattern_device_fill: writes the device arrays, sized from *sizes
 *     (csr_indptr [n_rows+1], csr_indices / sell_index [nnz], slice_ptr /
 *     inc_ptr [n_slices+1], slice_width / inc_width [n_slices], cols
 *     [nnz_padded], diag_pos [n_rows], diag_offsets [n_diags], inc_elem /
 *     inc_slots [n_inc]); the scratch must be the one count filled.
 * WSPM_BAD_ARG for ids out of range or a node in no element; WSPM_UNSUPPORTED
 * where the host builder returns it, for a row that gathers more than 128
 * element vertices, and beyond 2^33 rows (use the host builder then).       */
typedef struct wspm_pattern_sizes {
    int32_t n_rows, n_slices, max_width, max_inc, n_diags, layout;
    int64_t nnz, nnz_padded, n_inc, ld;
    int32_t diag_offsets[64];
} wspm_pattern_sizes;
int64_t wspm_pattern_device_scratch_bytes(int64_t n_elems, int32_t nv, int32_t n_nodes);
int wspm_pattern_device_count(const int32_t *conn, int64_t n_elems, int32_t nv, int32_t n_nodes, int32_t layout,
                              void *scratch, int64_t scratch_bytes, wspm_pattern_sizes *sizes, void *stream);
int wspm_pattern_device_fill(const int32_t *conn, int64_t n_elems, int32_t nv, int32_t n_nodes,
                             const wspm_pattern_sizes *sizes, void *scratch, int64_t scratch_bytes,
                             int64_t *csr_indptr, int32_t *csr_indices, int64_t *sell_index, int64_t *slice_ptr,
                             int32_t *slice_width, int32_t *cols, int32_t *diag_pos, int32_t *diag_offsets,
                             int64_t *inc_ptr, int32_t *inc_width, int32_t *inc_elem, uint32_t *inc_slots,
                             void *stream);
/* Level schedule of a triangular sweep over a CSR pattern (host): level[i] =
 * 1 + the highest level among the rows row i depends on (columns j < i when
 * lower != 0, j > i otherwise), 0 without dependencies; *n_levels = max + 1.
 * Used by the level-scheduled sweeps of wspm_precond_apply (the reference's
 * ilu / ssor, src/solvers/jax_linear_solver.py:91-252, sweeps row by row). */
int wspm_pattern_levels(const int64_t *indptr, const int32_t *indices, int32_t n_rows, int32_t lower,
                        int32_t *level, int32_t *n_levels);

/* ---- soil models -------------------------------------------------------- */
/* van_genuchten_model, src/models/van_genuchten.py:9-47 (vmapped over nodes).
 * phi = {alpha, theta_s, theta_r, n, m, Ks} (host array, 6 doubles).
 * Any of C, K, theta may be NULL.                                          */
int wspm_soil_van_genuchten(const double *h, int64_t n, const double *phi,
                            double *C, double *K, double *theta, void *stream);

/* exponential_model, src/models/exponential.py:10-41.
 * phi = {alpha0, theta_s, theta_r, Ks} (host array, 4 doubles).            */
int wspm_soil_exponential(const double *h, int64_t n, const double *phi,
                          double *C, double *K, double *theta, void *stream);

/* ---- assembly ----------------------------------------------------------- */
/* assemble_global_matrices_sparse_re, src/numerics/assembly_re_v2.py:62-166
 * (mesh->dim == 2) and assemble_global_matrices_sparse_3D,
 * src/numerics/assembly_re_3D.py:72-169 (mesh->dim == 3), fused with
 * apply_dirichlet_bcs (src/models/boundary.py:38-53) and the diagonal of
 * Preconditioner.create_jacobi (src/solvers/jax_linear_solver.py:11-36).
 *   quad_points [nq*dim], weights [nq]: host arrays (the reference's rule).
 *   Ks_elem: optional per-element factor multiplying K (NULL = 1).
 *   bc_val:  optional per-node Dirichlet value, NaN = free node (NULL = none).
 *   vals32, dinv: optional outputs (NULL = skip).                          */
int wspm_assemble_richards(const wspm_mesh *mesh, const wspm_pattern *pat,
                           const double *theta_m, const double *theta_n,
                           const double *h_m, const double *K, const double *C,
                           const double *Ks_elem,
                           const double *quad_points, const double *weights, int32_t nq,
                           double dt, const double *bc_val,
                           double *vals, float *vals32, double *rhs, double *dinv,
                           void *stream);

/* ---- transport ------------------------------------------------------------ */
/* calculate_fluxes_and_dispersion_FE, src/models/transport_utilities.py:118-192
 * (triangles): nodal Darcy flux from the mean element gradient of h over the
 * node's triangles, van Genuchten theta/K (phi as for wspm_soil_van_genuchten)
 * and the dispersion tensor.  Outputs [n_nodes] each.                      */
int wspm_flux_dispersion_2d(const wspm_mesh *mesh, const wspm_pattern *pat, const double *h,
                            const double *phi, double DL, double DT, double Dm,
                            double *qx, double *qz, double *aq, double *Dxx, double *Dxz,
                            double *Dzz, double *theta, void *stream);

/* Advection-dispersion-reaction system on triangles:
 *   lumped == 0: assemble_global_matrices_solute, src/numerics/assembly_solute.py:88-186,
 *                then A = M/dt + K and b = M c_n / dt (coupled_solver_v2.py:164-185);
 *   lumped == 1: assemble_nitrogen_species{1,2,3}_sparse, src/numerics/assembly_nitrogen.py:311-606,
 *                lump_sparse_mass_matrix and A = M/dt + K, b = M c_n/dt + F
 *                (src/solvers/nitrogen_solver.py:36-66, 151-235).
 * K = -dispersion - advection + mu*theta*N N^T, M = -(theta + sorption) N N^T,
 * F = -mu_up * theta * c_up * N (c_up may be NULL: no source).            */
int wspm_assemble_adr_2d(const wspm_mesh *mesh, const wspm_pattern *pat, const double *theta,
                         const double *qx, const double *qz, const double *Dxx, const double *Dxz,
                         const double *Dzz, const double *c_n, const double *c_up, double mu,
                         double sorption, double mu_up, int32_t lumped,
                         const double *quad_points, const double *weights, int32_t nq, double dt,
                         double *vals, double *rhs, double *dinv, void *stream);

/* Boundary edges (consecutive boundary nodes, 2-point Gauss rule), grouped per
 * boundary node so that each node sums its at most two edges in edge order.
 * Built on the host (wspm_b200.device.BoundaryEdges); device arrays.       */
typedef struct wspm_edges {
    int32_t n_bnodes;
    int32_t pad_;
    const int32_t *node;      /* [n_bnodes]                                   */
    const int32_t *e_cnt;     /* [n_bnodes] edges of this node (0..2)         */
    const int32_t *e_local;   /* [2 n_bnodes] 0 if the node is the edge's I   */
    const int32_t *e_other;   /* [2 n_bnodes] the edge's other node           */
    const int32_t *e_kother;  /* [2 n_bnodes] row position of the other node  */
    const double  *e_jac;     /* [2 n_bnodes] (x_J - x_I) / 2                 */
} wspm_edges;

#define WSPM_EDGE_NEUMANN          0  /* apply_neumann_bcs, boundary.py:108-128 (rhs)          */
#define WSPM_EDGE_DRAINAGE_WATER   1  /* apply_freedrainage_water_bcs, boundary.py:132-173     */
#define WSPM_EDGE_CAUCHY           2  /* apply_cauchy_bcs_sparse, boundary.py:217-277          */
#define WSPM_EDGE_DRAINAGE_SOLUTE  3  /* apply_freedrainage_nitrogen_bcs_sparse, :336-421     */
int wspm_apply_edge_terms(const wspm_pattern *pat, const wspm_edges *edges, int32_t mode,
                          double flux, double c_in, const double *K, const double *theta,
                          double *vals, double *rhs, void *stream);

/* ---- sparse kernels ----------------------------------------------------- */
/* y = A x (BCOO matvec inside jax.scipy.sparse.linalg, SELL-32 here).       */
int wspm_spmv_f64(const wspm_pattern *pat, const double *vals, const double *x,
                  double *y, void *stream);
int wspm_spmv_f32(const wspm_pattern *pat, const float *vals, const float *x,
                  float *y, void *stream);

/* apply_dirichlet_bcs, src/models/boundary.py:38-53: rows nodes[i] become
 * e_i and rhs[nodes[i]] = values[i].  nodes must be unique; callers that
 * apply several sets in sequence (top, then bottom) merge them first, later
 * sets overriding earlier ones.                                            */
int wspm_apply_dirichlet(const wspm_pattern *pat, const int32_t *nodes,
                         const double *values, int32_t n_bc, double *vals,
                         double *rhs, void *stream);

/* Preconditioner.create_jacobi, src/solvers/jax_linear_solver.py:11-36:
 * dinv = 1 / diag(A) with zero diagonals replaced by 1.                    */
int wspm_jacobi_dinv(const wspm_pattern *pat, const double *vals, double *dinv,
                     void *stream);

/* ---- Krylov solves -------------------------------------------------------- */
/* solve_system, src/solvers/solver_types.py:7-67 with JAXSparseSolver
 * (src/solvers/jax_linear_solver.py:255-329): x holds x0 on entry and the
 * solution on exit.  dinv == NULL means no preconditioner.  `work` is a
 * device buffer of wspm_krylov_workspace_doubles() doubles.  `result` is a
 * device int32[4]: {status, iterations, 0, 0}; iterations count Krylov
 * iterations (CG, BiCGSTAB) or restart cycles (GMRES) like JAX's maxiter.  */
int64_t wspm_krylov_workspace_doubles(int32_t n_rows, int32_t solver, int32_t restart);
int wspm_krylov_solve(const wspm_pattern *pat, const double *vals,
                      const double *b, double *x, const double *dinv,
                      int32_t solver, double tol, double atol, int32_t maxiter,
                      int32_t restart, double *work, int64_t work_doubles,
                      int32_t *result, void *stream);

/* One linear system in mixed precision (the reference's solve_system,
 * src/solvers/solver_types.py:7-67, with cg / bicgstab / gmres at a tolerance
 * FP32 alone cannot reach): FP32 Krylov corrections inside FP64 iterative
 * refinement.  x = x0 (in x), r = b - A x in FP64; while ||r|| > tol ||b||:
 * solve A d = r in FP32 from d = 0 with `solver` -- CG: the pipelined
 * resident kernel on DIA patterns whose vectors fit on chip, the
 * single-reduction one otherwise; BiCGSTAB; GMRES(restart) -- to the reduction
 * still needed (never tighter than inner_tol; at most inner_maxiter
 * iterations, restart cycles for GMRES), then x += d and r -= A d in FP64; at
 * most refine_maxiter corrections.  FP32 vectors, FP32 accumulation; the
 * residual and the decision are FP64.  vals32: the FP32 copy of vals in the
 * same layout, or NULL (made in the workspace on each call).  dinv: FP64
 * Jacobi 1/diag, or NULL for no preconditioner.  result (device int32[4]):
 * status, FP32 iterations (cycles for GMRES) over all corrections,
 * corrections, 0.  Captured once per argument set as a CUDA graph and
 * replayed on `stream`; no host sync.                                      */
int64_t wspm_krylov_mixed_workspace_doubles(int32_t n_rows, int64_t nnz_padded, int32_t solver, int32_t restart);
int wspm_krylov_solve_mixed(const wspm_pattern *pat, const double *vals, const float *vals32,
                            const double *b, double *x, const double *dinv, int32_t solver, int32_t restart,
                            double tol, double inner_tol, int32_t inner_maxiter, int32_t refine_maxiter,
                            double *work, int64_t work_doubles, int32_t *result, void *stream);

/* Measurement hook (no reference counterpart): runs up to `iters` Jacobi-CG
 * iterations of a persistent CG kernel with tolerance 0 from x on the given
 * system, as plain launches on `stream`, so the per-iteration time of the
 * dominant kernel can be taken with CUDA events.  The kernel still stops early
 * on an exactly zero residual or a non-finite value; `iters_done` (device
 * int32, may be NULL) receives the iterations actually run, so a timing can be
 * rejected when it is short.  `mode` is a bit set: WSPM_CGIT_FP32 selects the
 * FP32 kernel (vals, b, x, dinv are then float arrays); WSPM_CGIT_PIPELINED
 * the pipelined form used by the mixed path's inner solve (DIA patterns whose
 * per-block vectors fit on chip; WSPM_UNSUPPORTED otherwise), whose
 * reduction is waited for by one dedicated warp per block unless
 * WSPM_CGIT_NO_WARP_SPECIALIZATION is set.  `work` as for CG.              */
#define WSPM_CGIT_FP32 1
#define WSPM_CGIT_PIPELINED 2
#define WSPM_CGIT_NO_WARP_SPECIALIZATION 4
int wspm_cg_iterations(const wspm_pattern *pat, int32_t mode, const void *vals, const void *b, void *x,
                       const void *dinv, int32_t iters, double *work, int64_t work_doubles,
                       int32_t *iters_done, void *stream);

/* Measurement hook (no reference counterpart): `reps` streaming passes of 16-byte
 * reads over buf[0 .. n16) (buf 16-byte aligned), each of blocks_per_sm (1 or 2)
 * x SMs blocks of 1024 threads reading its own contiguous share with loads that
 * bypass L1; *out (device float, zeroed by the caller) receives a checksum.  With
 * a buffer that fits in L2 the passes after the first are L2 hits: bench.py times
 * two launches with CUDA events to obtain the L2 read bandwidth that bounds the
 * resident CG kernels (their matrix stays in L2 between iterations).          */
int wspm_read_probe(const void *buf, int64_t n16, int32_t reps, int32_t blocks_per_sm, float *out, void *stream);

/* Allocation-free Jacobi-CG solve.  No counterpart in the reference: it is
 * for callers that cannot allocate device memory -- typically code running
 * inside a JAX program (the reference's runtime), whose allocator reserves
 * most of the GPU's memory up front, or code where cudaMalloc is not allowed
 * (inside a stream capture) or too slow.  It runs the kernel that
 * wspm_krylov_solve runs for WSPM_SOLVER_CG, with the same arguments (x holds
 * x0 on entry, the solution on exit; dinv == NULL: no preconditioner; result =
 * {status, iterations, 0, 0}), so the iteration count and the iterate are
 * those of that call; but the Krylov vectors and solver state live in a
 * static device array inside the library instead of a caller-supplied
 * workspace, and nothing is allocated.  One kernel launch per call, whatever
 * maxiter is.  vals, x, dinv must start on 16-byte boundaries (WSPM_BAD_ARG
 * otherwise).  Limits: at most WSPM_NOALLOC_MAX_ROWS rows (larger systems
 * return WSPM_BAD_ARG before anything else is looked at); the scratch (about
 * 11 MB) is held by every GPU that loads the library until the process exits.
 * All calls on a device share that one array: calls that overlap on the GPU
 * (two streams, or two host threads on one device) race and corrupt each
 * other.  The first call on each device looks up the array's address and
 * caches it; make that first call before any stream capture.               */
#define WSPM_NOALLOC_MAX_ROWS 262144
int wspm_cg_solve_noalloc(const wspm_pattern *pat, const double *vals, const double *b, double *x,
                          const double *dinv, double tol, double atol, int32_t maxiter,
                          int32_t *result, void *stream);

/* ---- Picard time step (device-resident loop in a CUDA graph) ------------- */
/* RichardsSolver.solve_timestep, src/solvers/richards_solver_v2.py:107-168
 * (relative Picard error) and RichardsSolver3D.solve_timestep,
 * src/solvers/richards_solver_3D_v2.py:177-222 (absolute error).  One call
 * runs one implicit time step; the Picard loop, the Krylov loop and both
 * convergence tests run on the device inside one CUDA graph.              */
typedef struct wspm_picard_desc {
    const wspm_mesh *mesh;
    const wspm_pattern *pat;
    int32_t soil_model;        /* WSPM_SOIL_*                                */
    double  phi[6];            /* soil parameters (see wspm_soil_*)          */
    const double *Ks_elem;     /* optional per-element conductivity factor   */
    const double *bc_val;      /* optional Dirichlet values (NaN = free)     */
    double quad_points[16 * 3];/* reference quadrature rule (nq <= 16)       */
    double weights[16];
    int32_t nq;
    int32_t solver;            /* WSPM_SOLVER_*                              */
    int32_t precond;           /* WSPM_PRECOND_*                             */
    double  krylov_tol;        /* relative tolerance                         */
    int32_t krylov_maxiter;    /* iterations (CG, BiCGSTAB) or cycles (GMRES) */
    int32_t restart;           /* GMRES restart length m (1..32)             */
    int32_t mixed;             /* 1: FP32 Krylov (the same solver) inside FP64
                                  refinement on the true residual           */
    double  inner_tol;         /* mixed: relative tolerance of each FP32 solve */
    int32_t inner_maxiter;
    int32_t refine_maxiter;
    double  picard_tol;
    int32_t picard_maxiter;
    int32_t picard_relative;   /* 1: ||h-h_m||/||h||, 0: ||h-h_m||           */
    /* optional boundary-edge right-hand-side terms applied after assembly, in
     * this order (coupled_solver_v2.py:106-116, nitrogen_solver.py:116-127)  */
    const wspm_edges *neumann;  /* NULL = none                                */
    double  neumann_flux;
    const wspm_edges *drainage; /* free drainage of water, NULL = none        */
    /* state (device, caller-owned, n_nodes doubles unless noted) */
    double *h_n;               /* in: previous step; out: this step's head   */
    double *theta_n;           /* scratch: theta(h_n)                        */
    double *h_m, *x;           /* Picard iterate, Krylov iterate             */
    double *K, *C, *theta_m;   /* soil fields                                */
    double *vals;              /* [pat->nnz_padded]                          */
    float  *vals32;            /* [pat->nnz_padded], mixed only              */
    double *rhs, *dinv;
    double *work;              /* wspm_picard_workspace_doubles()            */
    int64_t work_doubles;
    double *dt_dev;            /* device double: the step's dt               */
    int32_t *result;           /* device int32[8]: status, picard its,
                                  total Krylov its, refinement its, ...     */
    double *result_f64;        /* device double[4]: picard error; seconds the
                                  resident CG kernels ran in this step (their
                                  %globaltimer, entry to exit of block 0) */
    double *Ks_inc;            /* with Ks_elem: wspm_picard_ks_inc_doubles(pat)
                                  doubles, Ks_elem gathered in incidence order
                                  at every step start; NULL without Ks_elem */
    void *shapes;              /* optional, wspm_picard_shape_bytes(mesh, pat)
                                  bytes of device memory: the plan records the
                                  mesh's distinct element Jacobians (bitwise)
                                  there at creation, and when they are few
                                  (up to 64 shapes, the table in shared
                                  memory; for patterns with at most 16 stored
                                  entries per row, up to 16,384 shapes and at
                                  least 8 elements per shape, a global table;
                                  wider rows: up to 256 triangle shapes in
                                  shared memory) its assembly
                                  reads each element-row's geometric factors
                                  from the per-shape table instead of
                                  recomputing them (same values bit for bit);
                                  NULL: always recompute                     */
} wspm_picard_desc;

int64_t wspm_picard_workspace_doubles(int32_t n_rows, int32_t mixed);
/* Size of wspm_picard_desc.Ks_inc: one double per incidence slot
 * (n_slices * 32 * max_inc).                                               */
int64_t wspm_picard_ks_inc_doubles(const wspm_pattern *pat);
/* Size in bytes of wspm_picard_desc.shapes for this mesh and pattern.      */
int64_t wspm_picard_shape_bytes(const wspm_mesh *mesh, const wspm_pattern *pat);
int wspm_picard_create(const wspm_picard_desc *desc, void **plan_out);
int wspm_picard_step(void *plan, void *stream);
/* The same step with the loops driven from the host (identical kernels; the
 * host reads the device's convergence words between bounded chunks of
 * Krylov iterations).  Synchronises with the host; for profiling tools that
 * cannot follow conditional graph nodes, and as a fallback.               */
int wspm_picard_step_host(void *plan, void *stream);
int wspm_picard_destroy(void *plan);
/* Structural zeros of a DIA plan: bit k set = diagonal k can hold nonzeros.  At
 * plan creation the element geometry is scanned once (the stiffness factor
 * (G^T G)[i][j] of every element pair, computed as the assembly computes it);
 * a diagonal on which every factor is exactly zero is exactly zero in every
 * assembly (the lumped mass and the Dirichlet rows touch only the main
 * diagonal), and the step's sparse kernels skip its loads -- fma(0, x, acc) ==
 * acc, so no result changes.  -1 for SELL patterns (nothing skipped).       */
int64_t wspm_picard_dia_live(void *plan);
/* Element shapes of a plan: the number of distinct element Jacobians its
 * assembly takes from the shape table (0: the assembly recomputes every
 * element's geometry -- no shape buffer, or too many shapes).  No
 * counterpart in the reference: an assembly-time lookup, results unchanged. */
int32_t wspm_picard_shapes(void *plan);
/* One assembly of the plan's system at its current state (theta_m, h_m, K, C
 * and dt as the step left them; Dirichlet rows, 1/diag, the FP32 copy on a
 * mixed plan) with the kernel the step runs, the shape path included; Ks
 * is taken in incidence order as gathered at plan creation or at the start
 * of the last step.
 * Replaces assemble_global_matrices_sparse_re (src/numerics/
 * assembly_re_v2.py:62-166) for a caller that holds a plan.               */
int wspm_picard_assemble(void *plan, void *stream);

/* ---- batched ensemble of independent domains -------------------------------
 * No single reference function: the reference solves one domain per
 * RichardsSolver (richards_solver_v2.py:107-168 per step, :272-352 time
 * loop); an ensemble there is a Python loop over solver instances.  Here the
 * domains are the diagonal blocks of one mesh (node ranges node_off[d] ..
 * node_off[d+1], elements never cross domains) and ONE persistent launch
 * advances every active domain by one implicit step: each CTA takes the next
 * domain from a device work queue (order[]: largest first), evaluates the VG
 * soil law with that domain's parameters, assembles its rows, runs Jacobi-CG
 * with block-level reductions, iterates Picard to the domain's own
 * tolerance, then adapts that domain's dt (richards_solver_v2.py:91-105) and
 * advances its time.  Domains with t >= tmax are skipped (the convergence
 * mask).  Per-domain outcomes are written to its[], kits[], status[], err[]. */
typedef struct wspm_ensemble {
    int32_t n_domains;
    const int64_t *node_off;   /* [n_domains + 1]                              */
    const int32_t *order;      /* [n_domains] processing order                 */
    const double  *phi;        /* [n_domains * 6] VG parameters per domain      */
    const double  *Ks_elem;    /* [n_elems] per-element conductivity factor or NULL */
    const double  *bc_val;     /* [n_nodes] Dirichlet values, NaN = free, or NULL */
    double quad_points[16 * 3];
    double weights[16];
    int32_t nq;
    double  krylov_tol;        /* relative residual of each CG solve           */
    int32_t krylov_maxiter;
    double  picard_tol;
    int32_t picard_maxiter;
    int32_t picard_relative;
    double  tmax;
    int32_t m_it, M_it;        /* dt rule: its <= m_it: dt *= lambda_amp ...  */
    double  lambda_amp, lambda_red;
    /* state (device) */
    double *h_n;               /* [n_nodes] in: previous step, out: new step */
    double *work;              /* wspm_ensemble_workspace_doubles()          */
    int64_t work_doubles;
    double *dt, *t;            /* [n_domains] current dt and time            */
    int32_t *its, *kits, *status;  /* [n_domains] last step's Picard its, Krylov its, status */
    double *err;               /* [n_domains] last step's Picard error       */
    uint32_t *queue;           /* device word, zeroed by the call            */
    int32_t cluster_size;      /* CTAs per domain (thread-block cluster): 0 or 1, 2, 4, 8, 16 (16: where the GPU allows non-portable clusters) */
} wspm_ensemble;

int64_t wspm_ensemble_workspace_doubles(int32_t n_rows, int64_t nnz_padded);
/* block_threads: CTA size (128, 256 or 512; 0 = 512); ens->cluster_size CTAs
 * (one thread-block cluster) share each domain.                                */
int wspm_ensemble_step(const wspm_mesh *mesh, const wspm_pattern *pat, const wspm_ensemble *ens,
                       int32_t block_threads, void *stream);
/* The time loop of the ensemble on the device (RichardsSolver.solve's loop,
 * richards_solver_v2.py:272-352, for every domain at once): one CUDA graph
 * whose WHILE node launches wspm_ensemble_step's kernel until every domain has
 * reached tmax or max_steps steps ran; no host round trip between steps.
 * Scratch/outputs (device): active[n_domains] (int32, domains below tmax
 * after the last step), its_total[n_domains] (int64, Picard iterations summed
 * over the steps each domain took), run[2] (int32: steps launched, domains
 * still active).  The graph is captured on every call and released when the
 * launch completes; `stream` orders it like any other call.                 */
int wspm_ensemble_run(const wspm_mesh *mesh, const wspm_pattern *pat, const wspm_ensemble *ens,
                      int32_t block_threads, int32_t max_steps, int32_t *active, int64_t *its_total,
                      int32_t *run, void *stream);

/* ---- per-element soil parameters and the discrete adjoint --------------------
 * No reference counterpart: the reference evaluates one van Genuchten
 * parameter set per run (van_genuchten.py:9-47) and differentiates with JAX.
 * Here every element e carries params[3e..3e+2] = (ln Ks, ln alpha, ln n),
 * m = 1 - 1/n, theta_r / theta_s shared; the soil law is evaluated per element
 * at its vertices, and the element matrices follow assembly_re_v2.py:13-60
 * with those element-wise values (2D P1 triangles).
 *   wspm_elem_assemble_richards: the Picard system A(h_m) h = b(h_m, h_n) with
 *     Dirichlet rows (bc_val, NaN = free) and Jacobi 1/diag (dinv may be NULL).
 *   wspm_elem_assemble_jt: J^T, J = dR/dh of the converged-step residual
 *     R(h) = sum_e Kbar_e detJ G.(grad h + e_z) + Ml (theta(h) - theta(h_old))/dt.
 *   wspm_elem_adjoint_rhs: rhs = g + lam_next * sum_e Ml C(h_old) / dt_next on free rows.
 *   wspm_elem_theta_node: theta_node = sum_e Ml theta_e / sum_e Ml, its d/dh, the lumped mass.
 *   wspm_elem_param_grad: grad[E][3] += -(dR/dp)^T lam + direct theta-sensor term (wl = dL/dtheta_node). */
int wspm_elem_assemble_richards(const wspm_mesh *mesh, const wspm_pattern *pat, const double *params,
                                double theta_r, double theta_s, const double *quad_points, const double *weights,
                                int32_t nq, double dt, const double *bc_val, const double *h_m, const double *h_n,
                                double *vals, double *rhs, double *dinv, void *stream);
int wspm_elem_assemble_jt(const wspm_mesh *mesh, const wspm_pattern *pat, const double *params, double theta_r,
                          double theta_s, const double *quad_points, const double *weights, int32_t nq, double dt,
                          const double *bc_val, const double *h, const double *h_old, double *vals, double *dinv,
                          void *stream);
int wspm_elem_adjoint_rhs(const wspm_mesh *mesh, const wspm_pattern *pat, const double *params, double theta_r,
                          double theta_s, const double *quad_points, const double *weights, int32_t nq,
                          double dt_next, const double *bc_val, const double *h_old, const double *lam_next,
                          const double *g, double *rhs, void *stream);
int wspm_elem_theta_node(const wspm_mesh *mesh, const wspm_pattern *pat, const double *params, double theta_r,
                         double theta_s, const double *quad_points, const double *weights, int32_t nq,
                         const double *h, double *theta_node, double *dtheta_dh, double *mass, void *stream);
int wspm_elem_param_grad(const wspm_mesh *mesh, const wspm_pattern *pat, const double *params, double theta_r,
                         double theta_s, const double *quad_points, const double *weights, int32_t nq, double dt,
                         const double *bc_val, const double *h, const double *h_old, const double *lam,
                         const double *wl, const double *mass, double *grad, void *stream);

/* ---- the reference's other preconditioners ---------------------------------
 * Preconditioner.create_ilu0 / create_ssor / create_block_jacobi,
 * src/solvers/jax_linear_solver.py:38-252, as their code computes them
 * (d = diag(A), L / U = strict lower / upper parts of A):
 *   WSPM_PRECOND_ILU:  y = (D' + U)^-1 (I + L D'^-1)^-1 x, D' = D with zeros -> 1;
 *   WSPM_PRECOND_SSOR: y = omega (D/omega + L)^-1 x;
 *   WSPM_PRECOND_BLOCK_JACOBI: y = blockdiag((A_bb + 1e-12 I)^-1) x, blocks of block_size (1 or 2).
 * The triangular sweeps run level by level: rows of one level depend only on
 * rows of earlier levels (lower: columns j < i, upper: j > i), listed by
 * wspm_levels (built on the host from the pattern).  One CTA walks the levels,
 * so a sweep costs one block barrier per level.  tmp: n_rows doubles.        */
typedef struct wspm_levels {
    int32_t n_levels;
    const int32_t *level_ptr;  /* [n_levels + 1] offsets into rows           */
    const int32_t *rows;       /* [n_rows] row ids grouped by level          */
} wspm_levels;

int wspm_precond_apply(const wspm_pattern *pat, const double *vals, int32_t kind, double omega,
                       int32_t block_size, const wspm_levels *lower, const wspm_levels *upper, const double *x,
                       double *y, double *tmp, void *stream);
/* True ILU(0): incomplete LU with zero fill on A's own pattern (IKJ form; the
 * rows of one level of the lower sweep's schedule factor in parallel).  No
 * reference counterpart: the reference's `ilu` never updates a pivot (see
 * WSPM_PRECOND_ILU); this is the factorization that name stands for.  lu: a
 * values array in the pattern's layout receiving L (strict lower part, unit
 * diagonal implied) and U; apply with wspm_precond_apply(kind =
 * WSPM_PRECOND_ILU0, vals = lu, lower and upper schedules).  Zero pivots are
 * taken as 1.                                                               */
int wspm_ilu0_factor(const wspm_pattern *pat, const double *vals, const wspm_levels *lower, double *lu,
                     void *stream);

/* ---- mass balance and transport stability numbers (2D) ---------------------
 * integrate_2d_domain, src/solvers/.ipynb_checkpoints/richards_mass_balance-checkpoint.py:25-69
 * (3-point rule, weights 1/3 times |det J|: twice the integral, as the
 * reference); calculate_peclet_courant, src/models/transport_utilities.py:193-242.
 * Results land in device memory (out: 1 double; out2: Pe, Cr); work holds
 * wspm_balance_workspace_doubles() doubles.  Fixed-order reductions.           */
int64_t wspm_balance_workspace_doubles(void);
int wspm_integrate_2d(const wspm_mesh *mesh, const double *f, double *out, double *work, void *stream);
int wspm_peclet_courant(const wspm_mesh *mesh, const double *qx, const double *qz, const double *theta,
                        const double *Dxx, const double *Dzz, double dt, double *out2, double *work, void *stream);

/* ---- misc ------------------------------------------------------------------ */
const char *wspm_version(void);
const char *wspm_status_string(int status);

#ifdef __cplusplus
}
#endif
#endif /* WSPM_H */
