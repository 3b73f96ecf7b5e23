// Richards with per-element van Genuchten parameters, and its discrete adjoint.
//
// Parameters per element e: p_e = (ln Ks_e, ln alpha_e, ln n_e), m_e = 1 - 1/n_e;
// theta_r, theta_s shared.  The soil law is evaluated per element at the
// element's vertices (theta_{e,j}, K_{e,j}, C_{e,j} = f(h_j; p_e)).  Forward
// Picard system of one implicit step, element e, own vertex i (as
// assembly_re_v2.py:13-60 with element-wise soil values):
//   A_e[i][j] = Kbar_e detJ G_i.G_j + [i=j] Ml_e,i C_e,i / dt,  Kbar_e = sum_j s_j K_{e,j}
//   b_e[i]    = -Kbar_e detJ G_i[z] - Ml_e,i (theta_e,i(h_m) - theta_e,i(h_n) - C_e,i h_m,i) / dt
// At the Picard fixed point h = h_m the C terms cancel and the step solves
//   R_i(h) = sum_e Kbar_e(h) detJ G_i.(grad h_e + e_z) + sum_e Ml_e,i (theta_e,i(h_i) - theta_e,i(h^n_i)) / dt = 0
// (Dirichlet rows: R_i = h_i - g_i).  The adjoint of the time stepper uses
//   J = dR/dh:  J_ij = sum_e [Kbar_e detJ G_i.G_j + s_j Ks_e Kr'_{e}(h_j) detJ G_i.(grad h_e + e_z)]
//                      + [i=j] sum_e Ml_e,i C_e,i(h_i) / dt
//   dR^{n+1}_i/dh^n_i = -sum_e Ml_e,i C_e,i(h^n_i) / dt
//   dR_i/dp_e  from dKbar_e/dp and dtheta_e,i/dp at h and h^n.
// J^T is assembled row by row (row i of J^T = column i of J), so the
// transpose solve runs on the ordinary sparse kernels.  Every kernel is a
// row gather over the node -> element incidence (ascending element id) or a
// thread per element, so no atomics and a fixed summation order.
#include "common.cuh"
#include "krylov.cuh"

namespace wspm {

void quadrature_constants(int dim, const double *Q, const double *W, int nq, double s[4], double m[4]);

// van Genuchten-Mualem at one head with its derivatives.  a = (alpha|h|)^n,
// Se = (1 + a)^-m, theta = thr + (ths - thr) Se, Kr = sqrt(Se) (1 - (a/(1+a))^m)^2.
// Directional derivatives use ra = (da)/a and dm:
//   d ln Se = -dm log1p(a) - m a ra / (1 + a),  d L = ra / (1 + a)  with L = log(a / (1 + a))
//   d ln w  = dm L + m dL,  w = exp(m L),  t = 1 - w
//   dtheta  = (ths - thr) Se d ln Se,  dKr = Kr d ln Se / 2 - 2 sqrt(Se) t w d ln w
// Directions: h (ra = -n/|h|, dm = 0; dtheta/dh = C), ln alpha (ra = n, dm = 0),
// ln n (ra = n ln(alpha|h|), dm = 1/n).
struct VgDer {
    double theta, Kr, C, dKr_dh;
    double dth_la, dth_ln, dKr_la, dKr_ln;
};

__device__ __forceinline__ VgDer vg_with_derivatives(double h, double alpha, double n, double thr, double ths) {
    VgDer o;
    if (!(h < 0.0)) {
        o.theta = ths; o.Kr = 1.0; o.C = 0.0; o.dKr_dh = 0.0;
        o.dth_la = o.dth_ln = o.dKr_la = o.dKr_ln = 0.0;
        return o;
    }
    const double m = 1.0 - 1.0 / n;
    const double ah = alpha * fabs(h);
    const double la = log(ah);
    const double ahn1 = pow(ah, n - 1.0);
    const double a = ahn1 * ah;
    const double onep = 1.0 + a;
    const double L1 = log1p(a);
    const double Se = exp(-m * L1);
    const double L = a >= 1.0 ? -log1p(1.0 / a) : log(a / onep);
    const double mL = m * L;
    const double w = exp(mL);
    const double t = -expm1(mL);
    const double sq = sqrt(Se);
    const double dth = ths - thr;
    o.theta = thr + dth * Se;
    o.Kr = sq * (t * t);
    o.C = dth * alpha * m * n * ahn1 * (Se / onep);
    auto dir = [&](double ra, double dm, double &dtheta, double &dKr) {
        const double dlnSe = -dm * L1 - m * a * ra / onep;
        const double dL = ra / onep;
        const double dlnw = dm * L + m * dL;
        dtheta = dth * Se * dlnSe;
        dKr = o.Kr * 0.5 * dlnSe - 2.0 * sq * t * w * dlnw;
    };
    double dummy;
    dir(-n / fabs(h), 0.0, dummy, o.dKr_dh);
    dir(n, 0.0, o.dth_la, o.dKr_la);
    dir(n * la, 1.0 / n, o.dth_ln, o.dKr_ln);
    return o;
}

struct ElemArgs {
    Sell A;
    const int32_t *diag_pos;
    const int64_t *inc_ptr;
    const int32_t *inc_width;
    const int32_t *inc_elem;
    const uint32_t *inc_slots;
    const int32_t *conn;
    const double *coords;
    int n_nodes, n_elems;
    const double *params;      // [E][3]: ln Ks, ln alpha, ln n
    double thr, ths;
    double s[3], mc[3];
    double inv_dt;
    const double *bc_val;      // NaN = free
    const double *h;           // forward: Picard iterate h_m; adjoint: converged h^{n+1}
    const double *h_old;       // h^n
    const double *lam;         // adjoint variable at this step (param gradient) / at step n+1 (rhs)
    const double *g;           // dL/dh at this step
    const double *wl;          // dL/dtheta_node at this step (direct parameter term), may be NULL
    const double *mass;        // lumped mass per node (sum_e Ml_e,i)
    double *vals, *rhs, *dinv;
    double *out1, *out2;       // theta_node, dtheta_node/dh
    double *grad;              // [E][3]
};

struct ElemGeo {
    int nd[3];
    double G[2][3], detJ;
};

__device__ __forceinline__ ElemGeo elem_geometry(const ElemArgs &a, int e) {
    ElemGeo g;
#pragma unroll
    for (int j = 0; j < 3; ++j) g.nd[j] = a.conn[3 * (int64_t)e + j];
    const double x0 = a.coords[2 * g.nd[0]], y0 = a.coords[2 * g.nd[0] + 1];
    const double J00 = a.coords[2 * g.nd[1]] - x0, J01 = a.coords[2 * g.nd[1] + 1] - y0;
    const double J10 = a.coords[2 * g.nd[2]] - x0, J11 = a.coords[2 * g.nd[2] + 1] - y0;
    g.detJ = J00 * J11 - J01 * J10;
    const double id = 1.0 / g.detJ;
    g.G[0][1] = J11 * id;  g.G[1][1] = -J10 * id;
    g.G[0][2] = -J01 * id; g.G[1][2] = J00 * id;
    g.G[0][0] = -(g.G[0][1] + g.G[0][2]);
    g.G[1][0] = -(g.G[1][1] + g.G[1][2]);
    return g;
}

__device__ __forceinline__ bool is_free(const double *bc_val, int i) { return !bc_val || isnan(bc_val[i]); }

// ---- forward Picard system (element-wise soil) ----------------------------------
template <int MW>
__global__ void __launch_bounds__(128) elem_forward_rows_kernel(ElemArgs a) {
    extern __shared__ double acc_sm[];
    const int TB = blockDim.x;
    const int i = blockIdx.x * TB + threadIdx.x;
    if (i >= a.n_nodes) return;
    double *acc = acc_sm + threadIdx.x;
    const Sell &A = a.A;
    const int width = row_width(A, i);
    for (int k = 0; k < width; ++k) acc[k * TB] = 0.0;
    const int dpos = a.diag_pos[i];
    double rhs_i = 0.0;
    if (!is_free(a.bc_val, i)) {
        acc[dpos * TB] = 1.0;
        rhs_i = a.bc_val[i];
    } else {
        const int s = i >> 5, lane = i & 31;
        const int deg = a.inc_width[s];
        const int64_t ib = a.inc_ptr[s] + lane;
        const double hi = a.h[i], hni = a.h_old[i];
        for (int k = 0; k < deg; ++k) {
            const int e = a.inc_elem[ib + (int64_t)kSlice * k];
            if (e < 0) continue;
            const uint32_t packed = a.inc_slots[ib + (int64_t)kSlice * k];
            const int li = packed & 3;
            const ElemGeo g = elem_geometry(a, e);
            const double Ks = exp(a.params[3 * (int64_t)e]);
            const double al = exp(a.params[3 * (int64_t)e + 1]), nn = exp(a.params[3 * (int64_t)e + 2]);
            double Kbar = 0.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const VgDer v = vg_with_derivatives(a.h[g.nd[j]], al, nn, a.thr, a.ths);
                Kbar = fma(a.s[j], Ks * v.Kr, Kbar);
            }
            const VgDer vi = vg_with_derivatives(hi, al, nn, a.thr, a.ths);
            const double thn = vg_with_derivatives(hni, al, nn, a.thr, a.ths).theta;
            const double kd = Kbar * g.detJ;
            const double Ml = a.mc[li] * g.detJ;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double v = kd * (g.G[0][li] * g.G[0][j] + g.G[1][li] * g.G[1][j]);
                if (j == li) v += a.inv_dt * (Ml * vi.C);
                acc[((packed >> (2 + 6 * j)) & 63) * TB] += v;
            }
            rhs_i += -kd * g.G[1][li] - a.inv_dt * (Ml * (vi.theta - thn - vi.C * hi));
        }
    }
    const double diag = acc[dpos * TB];
    a.rhs[i] = rhs_i;
    if (a.dinv) a.dinv[i] = 1.0 / (diag != 0.0 ? diag : 1.0);
    for (int k = 0; k < width; ++k) a.vals[entry_pos(A, i, k)] = acc[k * TB];
}

// ---- J^T at the converged state h (= h^{n+1}), previous state h_old ---------------
template <int MW>
__global__ void __launch_bounds__(128) elem_jt_rows_kernel(ElemArgs a) {
    extern __shared__ double acc_sm[];
    const int TB = blockDim.x;
    const int i = blockIdx.x * TB + threadIdx.x;
    if (i >= a.n_nodes) return;
    double *acc = acc_sm + threadIdx.x;
    const Sell &A = a.A;
    const int width = row_width(A, i);
    for (int k = 0; k < width; ++k) acc[k * TB] = 0.0;
    const int dpos = a.diag_pos[i];
    const bool free_i = is_free(a.bc_val, i);
    const int s = i >> 5, lane = i & 31;
    const int deg = a.inc_width[s];
    const int64_t ib = a.inc_ptr[s] + lane;
    const double hi = a.h[i];
    for (int k = 0; k < deg; ++k) {
        const int e = a.inc_elem[ib + (int64_t)kSlice * k];
        if (e < 0) continue;
        const uint32_t packed = a.inc_slots[ib + (int64_t)kSlice * k];
        const int li = packed & 3;
        const ElemGeo g = elem_geometry(a, e);
        const double Ks = exp(a.params[3 * (int64_t)e]);
        const double al = exp(a.params[3 * (int64_t)e + 1]), nn = exp(a.params[3 * (int64_t)e + 2]);
        double Kbar = 0.0, gx = 0.0, gz = 1.0;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double hj = a.h[g.nd[j]];
            Kbar = fma(a.s[j], Ks * vg_with_derivatives(hj, al, nn, a.thr, a.ths).Kr, Kbar);
            gx = fma(g.G[0][j], hj, gx);
            gz = fma(g.G[1][j], hj, gz);
        }
        const VgDer vi = vg_with_derivatives(hi, al, nn, a.thr, a.ths);
        // column i of J restricted to element e: rows j of e
        //   J_ji = Kbar detJ G_j.G_i + s_i Ks Kr'(h_i) detJ G_j.(grad h + e_z) + [j=i] Ml_i C_i / dt
        const double kd = Kbar * g.detJ;
        const double kp = a.s[li] * Ks * vi.dKr_dh * g.detJ;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int node_j = g.nd[j];
            if (j != li && !is_free(a.bc_val, node_j)) continue;     // a Dirichlet row of J has only its diagonal
            if (j == li && !free_i) continue;                          // (set below)
            double v = kd * (g.G[0][j] * g.G[0][li] + g.G[1][j] * g.G[1][li]) +
                       kp * (g.G[0][j] * gx + g.G[1][j] * gz);
            if (j == li) v += a.inv_dt * (a.mc[li] * g.detJ * vi.C);
            acc[((packed >> (2 + 6 * j)) & 63) * TB] += v;
        }
    }
    if (!free_i) acc[dpos * TB] = 1.0;
    const double diag = acc[dpos * TB];
    if (a.dinv) a.dinv[i] = 1.0 / (diag != 0.0 ? diag : 1.0);
    for (int k = 0; k < width; ++k) a.vals[entry_pos(A, i, k)] = acc[k * TB];
}

// ---- adjoint right-hand side: g^n + (-dR^{n+1}/dh^n)^T lam^{n+1} -----------------------
// out: rhs_i = g_i + [i free] lam_i sum_e Ml_e,i C_e,i(h_old_i) / dt  (h_old = h^n, lam = lam^{n+1})
__global__ void elem_adjoint_rhs_kernel(ElemArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_nodes) return;
    double r = a.g ? a.g[i] : 0.0;
    if (a.lam && is_free(a.bc_val, i)) {
        const int s = i >> 5, lane = i & 31;
        const int deg = a.inc_width[s];
        const int64_t ib = a.inc_ptr[s] + lane;
        double S = 0.0;
        for (int k = 0; k < deg; ++k) {
            const int e = a.inc_elem[ib + (int64_t)kSlice * k];
            if (e < 0) continue;
            const int li = a.inc_slots[ib + (int64_t)kSlice * k] & 3;
            const ElemGeo g = elem_geometry(a, e);
            const double al = exp(a.params[3 * (int64_t)e + 1]), nn = exp(a.params[3 * (int64_t)e + 2]);
            S += a.mc[li] * g.detJ * vg_with_derivatives(a.h_old[i], al, nn, a.thr, a.ths).C;
        }
        r += a.inv_dt * S * a.lam[i];
    }
    a.rhs[i] = r;
}

// ---- nodal water content theta_node_i = sum_e Ml_e,i theta_e,i / sum_e Ml_e,i and d/dh ---------
__global__ void elem_theta_node_kernel(ElemArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_nodes) return;
    const int s = i >> 5, lane = i & 31;
    const int deg = a.inc_width[s];
    const int64_t ib = a.inc_ptr[s] + lane;
    double M = 0.0, T = 0.0, D = 0.0;
    for (int k = 0; k < deg; ++k) {
        const int e = a.inc_elem[ib + (int64_t)kSlice * k];
        if (e < 0) continue;
        const int li = a.inc_slots[ib + (int64_t)kSlice * k] & 3;
        const ElemGeo g = elem_geometry(a, e);
        const double al = exp(a.params[3 * (int64_t)e + 1]), nn = exp(a.params[3 * (int64_t)e + 2]);
        const VgDer v = vg_with_derivatives(a.h[i], al, nn, a.thr, a.ths);
        const double Ml = a.mc[li] * g.detJ;
        M += Ml;
        T += Ml * v.theta;
        D += Ml * v.C;
    }
    if (a.out1) a.out1[i] = T / M;
    if (a.out2) a.out2[i] = D / M;
    if (a.rhs) a.rhs[i] = M;   // lumped mass per node (when asked for)
}

// ---- parameter gradient of one step: grad_e -= sum_{i in e, free} lam_i dR_i/dp_e
//      + sum_{i in e} wl_i Ml_e,i dtheta_e,i/dp_e / mass_i   (direct theta-sensor term)
__global__ void elem_param_grad_kernel(ElemArgs a) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.n_elems) return;
    const ElemGeo g = elem_geometry(a, e);
    const double lKs = a.params[3 * (int64_t)e];
    const double Ks = exp(lKs);
    const double al = exp(a.params[3 * (int64_t)e + 1]), nn = exp(a.params[3 * (int64_t)e + 2]);
    double Kbar = 0.0, dK_la = 0.0, dK_ln = 0.0, gx = 0.0, gz = 1.0;
    VgDer v[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const double hj = a.h[g.nd[j]];
        v[j] = vg_with_derivatives(hj, al, nn, a.thr, a.ths);
        Kbar = fma(a.s[j], Ks * v[j].Kr, Kbar);
        dK_la = fma(a.s[j], Ks * v[j].dKr_la, dK_la);
        dK_ln = fma(a.s[j], Ks * v[j].dKr_ln, dK_ln);
        gx = fma(g.G[0][j], hj, gx);
        gz = fma(g.G[1][j], hj, gz);
    }
    double d0 = 0.0, d1 = 0.0, d2 = 0.0;
#pragma unroll
    for (int li = 0; li < 3; ++li) {
        const int node = g.nd[li];
        const double Ml = a.mc[li] * g.detJ;
        if (a.lam && is_free(a.bc_val, node)) {
            const double lam = a.lam[node];
            const double flux = g.detJ * (g.G[0][li] * gx + g.G[1][li] * gz);
            const VgDer vo = vg_with_derivatives(a.h_old[node], al, nn, a.thr, a.ths);
            d0 -= lam * (Kbar * flux);
            d1 -= lam * (dK_la * flux + a.inv_dt * Ml * (v[li].dth_la - vo.dth_la));
            d2 -= lam * (dK_ln * flux + a.inv_dt * Ml * (v[li].dth_ln - vo.dth_ln));
        }
        if (a.wl) {
            const double w = a.wl[node];
            if (w != 0.0) {
                const double f = w * Ml / a.mass[node];
                d1 += f * v[li].dth_la;
                d2 += f * v[li].dth_ln;
            }
        }
    }
    a.grad[3 * (int64_t)e] += d0;
    a.grad[3 * (int64_t)e + 1] += d1;
    a.grad[3 * (int64_t)e + 2] += d2;
}

}  // namespace wspm

using namespace wspm;

static bool elem_args(const wspm_mesh *mesh, const wspm_pattern *pat, const double *params, double thr, double ths,
                      const double *quad_points, const double *weights, int nq, double dt, const double *bc_val,
                      ElemArgs &a) {
    if (!mesh || !pat || !params || mesh->dim != 2 || nq <= 0 || nq > 16 || pat->n_rows != mesh->n_nodes ||
        !(dt > 0.0))
        return false;
    a.A = make_sell(pat);
    a.diag_pos = pat->diag_pos;
    a.inc_ptr = pat->inc_ptr; a.inc_width = pat->inc_width; a.inc_elem = pat->inc_elem; a.inc_slots = pat->inc_slots;
    a.conn = mesh->conn; a.coords = mesh->coords;
    a.n_nodes = mesh->n_nodes; a.n_elems = mesh->n_elems;
    a.params = params; a.thr = thr; a.ths = ths;
    double s4[4], m4[4];
    quadrature_constants(2, quad_points, weights, nq, s4, m4);
    for (int j = 0; j < 3; ++j) { a.s[j] = s4[j]; a.mc[j] = m4[j]; }
    a.inv_dt = 1.0 / dt;
    a.bc_val = bc_val;
    a.h = a.h_old = a.lam = a.g = a.wl = a.mass = nullptr;
    a.vals = a.rhs = a.dinv = a.out1 = a.out2 = a.grad = nullptr;
    return true;
}

template <typename K>
static int launch_rows(K kernel8, K kernel16, const wspm_pattern *pat, const ElemArgs &a, cudaStream_t st) {
    const int threads = 128;
    const int blocks = (a.n_nodes + threads - 1) / threads;
    if (pat->max_width > 16) return WSPM_UNSUPPORTED;
    const int mw = pat->max_width <= 8 ? 8 : 16;
    const size_t smem = (size_t)mw * threads * sizeof(double);
    K k = mw == 8 ? kernel8 : kernel16;
    k<<<blocks, threads, smem, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

extern "C" int wspm_elem_assemble_richards(const wspm_mesh *mesh, const wspm_pattern *pat, const double *params,
                                           double theta_r, double theta_s, const double *quad_points,
                                           const double *weights, int32_t nq, double dt, const double *bc_val,
                                           const double *h_m, const double *h_n, double *vals, double *rhs,
                                           double *dinv, void *stream) {
    ElemArgs a;
    if (!elem_args(mesh, pat, params, theta_r, theta_s, quad_points, weights, nq, dt, bc_val, a) || !h_m || !h_n ||
        !vals || !rhs)
        return WSPM_BAD_ARG;
    a.h = h_m; a.h_old = h_n; a.vals = vals; a.rhs = rhs; a.dinv = dinv;
    return launch_rows(elem_forward_rows_kernel<8>, elem_forward_rows_kernel<16>, pat, a, (cudaStream_t)stream);
}

extern "C" int wspm_elem_assemble_jt(const wspm_mesh *mesh, const wspm_pattern *pat, const double *params,
                                     double theta_r, double theta_s, const double *quad_points, const double *weights,
                                     int32_t nq, double dt, const double *bc_val, const double *h,
                                     const double *h_old, double *vals, double *dinv, void *stream) {
    ElemArgs a;
    if (!elem_args(mesh, pat, params, theta_r, theta_s, quad_points, weights, nq, dt, bc_val, a) || !h || !h_old ||
        !vals)
        return WSPM_BAD_ARG;
    a.h = h; a.h_old = h_old; a.vals = vals; a.dinv = dinv;
    return launch_rows(elem_jt_rows_kernel<8>, elem_jt_rows_kernel<16>, pat, a, (cudaStream_t)stream);
}

extern "C" int wspm_elem_adjoint_rhs(const wspm_mesh *mesh, const wspm_pattern *pat, const double *params,
                                     double theta_r, double theta_s, const double *quad_points, const double *weights,
                                     int32_t nq, double dt_next, const double *bc_val, const double *h_old,
                                     const double *lam_next, const double *g, double *rhs, void *stream) {
    ElemArgs a;
    if (!elem_args(mesh, pat, params, theta_r, theta_s, quad_points, weights, nq, dt_next, bc_val, a) || !h_old ||
        !rhs)
        return WSPM_BAD_ARG;
    a.h_old = h_old; a.lam = lam_next; a.g = g; a.rhs = rhs;
    const int threads = 256;
    elem_adjoint_rhs_kernel<<<(a.n_nodes + threads - 1) / threads, threads, 0, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

extern "C" int wspm_elem_theta_node(const wspm_mesh *mesh, const wspm_pattern *pat, const double *params,
                                    double theta_r, double theta_s, const double *quad_points, const double *weights,
                                    int32_t nq, const double *h, double *theta_node, double *dtheta_dh,
                                    double *mass, void *stream) {
    ElemArgs a;
    if (!elem_args(mesh, pat, params, theta_r, theta_s, quad_points, weights, nq, 1.0, nullptr, a) || !h)
        return WSPM_BAD_ARG;
    a.h = h; a.out1 = theta_node; a.out2 = dtheta_dh; a.rhs = mass;
    const int threads = 256;
    elem_theta_node_kernel<<<(a.n_nodes + threads - 1) / threads, threads, 0, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

extern "C" int wspm_elem_param_grad(const wspm_mesh *mesh, const wspm_pattern *pat, const double *params,
                                    double theta_r, double theta_s, const double *quad_points, const double *weights,
                                    int32_t nq, double dt, const double *bc_val, const double *h,
                                    const double *h_old, const double *lam, const double *wl, const double *mass,
                                    double *grad, void *stream) {
    ElemArgs a;
    if (!elem_args(mesh, pat, params, theta_r, theta_s, quad_points, weights, nq, dt, bc_val, a) || !h || !h_old ||
        !grad || (wl && !mass))
        return WSPM_BAD_ARG;
    a.h = h; a.h_old = h_old; a.lam = lam; a.wl = wl; a.mass = mass; a.grad = grad;
    const int threads = 256;
    elem_param_grad_kernel<<<(a.n_elems + threads - 1) / threads, threads, 0, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}
