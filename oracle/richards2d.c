/*
 * Oracle (test infrastructure, not the product): a C + OpenMP restatement of
 * the NumPy oracle's 2D Richards time loop with van Genuchten soil, fixed dt,
 * mass-lumped mixed-form P1 assembly, Dirichlet rows and Jacobi-CG, for the
 * workloads too large for the NumPy restatement to finish in seconds.  It is
 * the same algorithm as
 *   oracle/soil.py:van_genuchten_model      (src/models/van_genuchten.py:24-47)
 *   oracle/assembly.py:assemble_richards    (src/numerics/assembly_re_v2.py:13-166)
 *   oracle/assembly.py:apply_dirichlet_rows (src/models/boundary.py:38-53)
 *   oracle/krylov.py:cg with a Jacobi diagonal
 *                                           (src/solvers/jax_linear_solver.py:11-36, 262-283)
 *   oracle/picard.py:RichardsProblem.timestep (src/solvers/richards_solver_v2.py:107-168)
 * evaluated in the same order per element (quadrature points in rule order,
 * element contributions summed per row in ascending element order, like the
 * reference's fori_loop scatter) and checked against the NumPy oracle in
 * tests/test_oracle_c.py.  Parallel over rows and elements with OpenMP;
 * dot products are OpenMP reductions (the summation order depends on the
 * thread count, so results agree with the NumPy oracle to rounding, not
 * bitwise).  Nothing in the product path loads this library.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* 3-point triangle rule of the reference (src/numerics/gauss.py:31-37), literal decimals */
static const double QP[3][2] = {{0.166666666666667, 0.166666666666667},
                                {0.166666666666667, 0.666666666666667},
                                {0.666666666666667, 0.166666666666667}};
static const double QW[3] = {0.166666666666667, 0.166666666666667, 0.166666666666667};

typedef struct {
    int64_t n, e;
    const double *pts;
    const int64_t *tri;
    const double *Ks;        /* per element or NULL */
    double phi[6];           /* alpha, theta_s, theta_r, n, m, Ks */
    /* node -> element incidence (ascending element ids) */
    int64_t *inc_ptr;
    int64_t *inc_el;
    int8_t *inc_loc;         /* local vertex of the row's node */
    /* CSR pattern and, per incidence entry, the CSR slot of each element vertex */
    int64_t *indptr;
    int32_t *indices;
    int64_t *slot;           /* [3 * n_inc] */
    int64_t *diag;           /* [n] CSR position of the diagonal */
    /* per element geometry: G (2 x 3, row-major) and det J */
    double *G, *detJ;
    int8_t *is_bc;
    double *bc_val;
} Problem;

static int cmp_i32(const void *a, const void *b) {
    const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

static int build(Problem *P) {
    const int64_t n = P->n, E = P->e;
    P->inc_ptr = calloc((size_t)n + 1, sizeof(int64_t));
    if (!P->inc_ptr) return -1;
    for (int64_t e = 0; e < E; ++e)
        for (int a = 0; a < 3; ++a) {
            const int64_t v = P->tri[3 * e + a];
            if (v < 0 || v >= n) return -2;
            P->inc_ptr[v + 1]++;
        }
    for (int64_t i = 0; i < n; ++i) P->inc_ptr[i + 1] += P->inc_ptr[i];
    const int64_t ninc = P->inc_ptr[n];
    P->inc_el = malloc((size_t)ninc * sizeof(int64_t));
    P->inc_loc = malloc((size_t)ninc);
    int64_t *fill = malloc((size_t)n * sizeof(int64_t));
    if (!P->inc_el || !P->inc_loc || !fill) return -1;
    memcpy(fill, P->inc_ptr, (size_t)n * sizeof(int64_t));
    for (int64_t e = 0; e < E; ++e)        /* ascending e: each node's list is sorted */
        for (int a = 0; a < 3; ++a) {
            const int64_t v = P->tri[3 * e + a];
            P->inc_el[fill[v]] = e;
            P->inc_loc[fill[v]] = (int8_t)a;
            fill[v]++;
        }
    free(fill);
    /* CSR pattern: per row the sorted union of the incident elements' vertices */
    P->indptr = calloc((size_t)n + 1, sizeof(int64_t));
    if (!P->indptr) return -1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        int32_t buf[256];
        int m = 0;
        for (int64_t k = P->inc_ptr[i]; k < P->inc_ptr[i + 1] && m + 3 <= 256; ++k)
            for (int a = 0; a < 3; ++a) buf[m++] = (int32_t)P->tri[3 * P->inc_el[k] + a];
        qsort(buf, (size_t)m, sizeof(int32_t), cmp_i32);
        int u = 0;
        for (int j = 0; j < m; ++j)
            if (j == 0 || buf[j] != buf[j - 1]) ++u;
        P->indptr[i + 1] = u;
    }
    for (int64_t i = 0; i < n; ++i) P->indptr[i + 1] += P->indptr[i];
    const int64_t nnz = P->indptr[n];
    P->indices = malloc((size_t)nnz * sizeof(int32_t));
    P->slot = malloc((size_t)ninc * 3 * sizeof(int64_t));
    P->diag = malloc((size_t)n * sizeof(int64_t));
    if (!P->indices || !P->slot || !P->diag) return -1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        int32_t buf[256];
        int m = 0;
        for (int64_t k = P->inc_ptr[i]; k < P->inc_ptr[i + 1] && m + 3 <= 256; ++k)
            for (int a = 0; a < 3; ++a) buf[m++] = (int32_t)P->tri[3 * P->inc_el[k] + a];
        qsort(buf, (size_t)m, sizeof(int32_t), cmp_i32);
        int64_t q = P->indptr[i];
        for (int j = 0; j < m; ++j)
            if (j == 0 || buf[j] != buf[j - 1]) P->indices[q++] = buf[j];
        for (int64_t s = P->indptr[i]; s < P->indptr[i + 1]; ++s)
            if (P->indices[s] == i) P->diag[i] = s;
        for (int64_t k = P->inc_ptr[i]; k < P->inc_ptr[i + 1]; ++k)
            for (int b = 0; b < 3; ++b) {
                const int32_t c = (int32_t)P->tri[3 * P->inc_el[k] + b];
                int64_t lo = P->indptr[i], hi = P->indptr[i + 1] - 1;
                while (lo < hi) {
                    const int64_t mid = (lo + hi) / 2;
                    if (P->indices[mid] < c) lo = mid + 1; else hi = mid;
                }
                P->slot[3 * k + b] = lo;
            }
    }
    /* geometry: J = dref . X (2 x 2), G = J^-1 dref (2 x 3); dref = [[-1, 1, 0], [-1, 0, 1]] */
    P->G = malloc((size_t)E * 6 * sizeof(double));
    P->detJ = malloc((size_t)E * sizeof(double));
    if (!P->G || !P->detJ) return -1;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < E; ++e) {
        const double *p0 = P->pts + 2 * P->tri[3 * e], *p1 = P->pts + 2 * P->tri[3 * e + 1],
                     *p2 = P->pts + 2 * P->tri[3 * e + 2];
        const double j00 = p1[0] - p0[0], j01 = p1[1] - p0[1];
        const double j10 = p2[0] - p0[0], j11 = p2[1] - p0[1];
        const double det = j00 * j11 - j01 * j10;
        const double i00 = j11 / det, i01 = -j01 / det, i10 = -j10 / det, i11 = j00 / det;
        double *G = P->G + 6 * e;
        /* G = inv(J) @ dref */
        G[0] = -i00 - i01; G[1] = i00; G[2] = i01;
        G[3] = -i10 - i11; G[4] = i10; G[5] = i11;
        P->detJ[e] = det;
    }
    return 0;
}

/* van_genuchten_model (src/models/van_genuchten.py:24-47), literal formula */
static void soil(const double phi[6], double h, double *C, double *K, double *th) {
    const double alpha = phi[0], ts = phi[1], tr = phi[2], n = phi[3], m = phi[4], Ks = phi[5];
    if (h < 0) {
        const double ah = alpha * fabs(h);
        const double t = (ts - tr) * pow(1 + pow(ah, n), -m) + tr;
        const double Se = (t - tr) / (ts - tr);
        *th = t;
        *K = Ks * (pow(Se, 0.5) * pow(1 - pow(1 - pow(Se, 1 / m), m), 2));
        *C = (ts - tr) * alpha * m * n * pow(ah, n - 1) * pow(1 + pow(ah, n), -m - 1);
    } else {
        *th = ts; *K = Ks; *C = 0.0;
    }
}

/* Row i of A and b (assembly_re_v2.py:13-60 per element, summed in element order), then the
 * Dirichlet row replacement (boundary.py:38-53). */
static void assemble(const Problem *P, const double *h, const double *thn, const double *C, const double *Kn,
                     const double *thm, double dt, double *A, double *b) {
    const int64_t n = P->n;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t s = P->indptr[i]; s < P->indptr[i + 1]; ++s) A[s] = 0.0;
        double bi = 0.0;
        for (int64_t k = P->inc_ptr[i]; k < P->inc_ptr[i + 1]; ++k) {
            const int64_t e = P->inc_el[k];
            const int a = P->inc_loc[k];
            const int64_t *v = P->tri + 3 * e;
            const double *G = P->G + 6 * e;
            const double dj = P->detJ[e];
            const double ks = P->Ks ? P->Ks[e] : 1.0;
            double Ke[3];
            for (int c = 0; c < 3; ++c) Ke[c] = ks * Kn[v[c]];
            double stiff[3] = {0, 0, 0}, Ml = 0.0, src = 0.0;
            for (int q = 0; q < 3; ++q) {
                const double N[3] = {1 - QP[q][0] - QP[q][1], QP[q][0], QP[q][1]};
                const double w = QW[q];
                const double NK = Ke[0] * N[0] + Ke[1] * N[1] + Ke[2] * N[2];
                for (int c = 0; c < 3; ++c) {
                    const double gtg = G[a] * G[c] + G[3 + a] * G[3 + c];
                    stiff[c] += w * NK * gtg * dj;
                }
                for (int c = 0; c < 3; ++c) Ml += w * (N[a] * N[c]) * dj;
                src -= w * NK * G[3 + a] * dj;
            }
            const double Ca = C[i];
            for (int c = 0; c < 3; ++c) {
                double val = stiff[c];
                if (c == a) val = (1 / dt) * (Ml * Ca) + stiff[c];
                A[P->slot[3 * k + c]] += val;
            }
            bi += src - (1 / dt) * (Ml * (thm[i] - thn[i] - Ca * h[i]));
        }
        b[i] = bi;
        if (P->is_bc[i]) {
            for (int64_t s = P->indptr[i]; s < P->indptr[i + 1]; ++s) A[s] = 0.0;
            A[P->diag[i]] = 1.0;
            b[i] = P->bc_val[i];
        }
    }
}

static void spmv(const Problem *P, const double *A, const double *x, double *y) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < P->n; ++i) {
        double s = 0.0;
        for (int64_t q = P->indptr[i]; q < P->indptr[i + 1]; ++q) s += A[q] * x[P->indices[q]];
        y[i] = s;
    }
}

static double dot(int64_t n, const double *a, const double *b) {
    double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s)
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* oracle/krylov.py:cg with M = diag(dinv): stop when r.r <= tol^2 b.b or after maxiter. */
static int64_t cg(const Problem *P, const double *A, const double *b, double *x, double tol, int64_t maxiter,
                  double *r, double *z, double *p, double *q, double *dinv) {
    const int64_t n = P->n;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double d = A[P->diag[i]];
        dinv[i] = 1.0 / (d != 0.0 ? d : 1.0);
    }
    const double atol2 = tol * tol * dot(n, b, b);
    spmv(P, A, x, q);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        r[i] = b[i] - q[i];
        z[i] = dinv[i] * r[i];
        p[i] = z[i];
    }
    double gamma = dot(n, r, z);
    int64_t k = 0;
    while (dot(n, r, r) > atol2 && k < maxiter) {
        spmv(P, A, p, q);
        const double alpha = gamma / dot(n, p, q);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            x[i] = x[i] + alpha * p[i];
            r[i] = r[i] - alpha * q[i];
            z[i] = dinv[i] * r[i];
        }
        const double gamma_new = dot(n, r, z);
        const double beta = gamma_new / gamma;
        gamma = gamma_new;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        ++k;
    }
    return k;
}

static void free_problem(Problem *P) {
    free(P->inc_ptr); free(P->inc_el); free(P->inc_loc); free(P->indptr); free(P->indices); free(P->slot);
    free(P->diag); free(P->G); free(P->detJ); free(P->is_bc); free(P->bc_val);
}

/*
 * Fixed-dt time loop of the VG Dirichlet case (oracle/picard.py:run_time_loop with fixed_dt):
 * per step theta_n = theta(h_n), then the Picard loop of RichardsProblem.timestep
 * (err = ||h - h_m|| (/ ||h|| when relative), stop at err < picard_tol or picard_max
 * iterations), each linear system solved by Jacobi-CG from x0 = h_m.
 *   points [n*2], tri [e*3] (0-based), Ks [e] or NULL (then phi[5] is Ks), bc_nodes/bc_vals [n_bc].
 *   h_io [n]: h0 on entry, the last step's head on exit; h_steps [n_steps*n] or NULL.
 *   picard_its [n_steps], cg_its [n_steps]; *seconds: wall time of the time loop only;
 *   threads: OpenMP threads (<= 0: the runtime's default).
 * Returns 0, or < 0 on a bad mesh / allocation failure.
 */
int oracle_richards2d_vg_run(int64_t n, int64_t e, const double *points, const int64_t *tri, const double *Ks,
                             const double *phi, const int64_t *bc_nodes, const double *bc_vals, int64_t n_bc,
                             double dt, int32_t n_steps, double picard_tol, int32_t picard_max,
                             int32_t picard_relative, double cg_tol, int64_t cg_maxiter, int32_t threads,
                             double *h_io, double *h_steps, int32_t *picard_its, int64_t *cg_its, double *seconds) {
    if (threads > 0) omp_set_num_threads(threads);
    Problem P;
    memset(&P, 0, sizeof(P));
    P.n = n; P.e = e; P.pts = points; P.tri = tri; P.Ks = Ks;
    for (int j = 0; j < 6; ++j) P.phi[j] = phi[j];
    int rc = build(&P);
    P.is_bc = calloc((size_t)n, 1);
    P.bc_val = calloc((size_t)n, sizeof(double));
    if (rc != 0 || !P.is_bc || !P.bc_val) { free_problem(&P); return rc ? rc : -1; }
    for (int64_t j = 0; j < n_bc; ++j) {
        if (bc_nodes[j] < 0 || bc_nodes[j] >= n) { free_problem(&P); return -2; }
        P.is_bc[bc_nodes[j]] = 1;
        P.bc_val[bc_nodes[j]] = bc_vals[j];
    }
    const int64_t nnz = P.indptr[n];
    double *A = malloc((size_t)nnz * sizeof(double));
    double *vec = malloc((size_t)n * 11 * sizeof(double));
    if (!A || !vec) { free(A); free(vec); free_problem(&P); return -1; }
    double *hn = vec, *hm = vec + n, *thn = vec + 2 * n, *C = vec + 3 * n, *Kn = vec + 4 * n, *thm = vec + 5 * n,
           *b = vec + 6 * n, *r = vec + 7 * n, *z = vec + 8 * n, *p = vec + 9 * n, *q = vec + 10 * n;
    double *dinv = malloc((size_t)n * sizeof(double)), *x = malloc((size_t)n * sizeof(double));
    if (!dinv || !x) { free(A); free(vec); free(dinv); free(x); free_problem(&P); return -1; }
    memcpy(hn, h_io, (size_t)n * sizeof(double));
    const double t0 = omp_get_wtime();
    for (int s = 0; s < n_steps; ++s) {
        double dummy_c, dummy_k;
#pragma omp parallel for schedule(static) private(dummy_c, dummy_k)
        for (int64_t i = 0; i < n; ++i) {
            soil(P.phi, hn[i], &dummy_c, &dummy_k, &thn[i]);
            hm[i] = hn[i];
        }
        double err = INFINITY;
        int it = 0;
        int64_t kits = 0;
        while (err >= picard_tol && it < picard_max) {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) soil(P.phi, hm[i], &C[i], &Kn[i], &thm[i]);
            assemble(&P, hm, thn, C, Kn, thm, dt, A, b);
            memcpy(x, hm, (size_t)n * sizeof(double));
            kits += cg(&P, A, b, x, cg_tol, cg_maxiter, r, z, p, q, dinv);
            double dd = 0.0, xx = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : dd, xx)
            for (int64_t i = 0; i < n; ++i) {
                const double d = x[i] - hm[i];
                dd += d * d;
                xx += x[i] * x[i];
                hm[i] = x[i];
            }
            err = picard_relative ? sqrt(dd) / sqrt(xx) : sqrt(dd);
            ++it;
        }
        memcpy(hn, hm, (size_t)n * sizeof(double));
        if (h_steps) memcpy(h_steps + (int64_t)s * n, hn, (size_t)n * sizeof(double));
        picard_its[s] = it;
        cg_its[s] = kits;
    }
    *seconds = omp_get_wtime() - t0;
    memcpy(h_io, hn, (size_t)n * sizeof(double));
    free(A); free(vec); free(dinv); free(x);
    free_problem(&P);
    return 0;
}

int oracle_max_threads(void) { return omp_get_max_threads(); }
