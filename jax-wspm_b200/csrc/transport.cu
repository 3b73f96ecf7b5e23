// Transport kernels: nodal Darcy flux + dispersion, advection-dispersion-reaction
// (ADR) assembly, and boundary-edge terms.
//
//  flux_dispersion_kernel  transport_utilities.py:118-192.  The reference
//      averages the constant P1 gradient of h over the triangles containing
//      each node by a masked sum over ALL elements (O(N*E)); here each node
//      walks its own incident elements (the incidence lists of the pattern).
//  adr_rows_kernel         assembly_solute.py:39-85 (consistent mass) and
//      assembly_nitrogen.py:67-133, 166-218, 250-302 (reaction, sorption,
//      upstream-species source, lumped mass).  Row-gather like the Richards
//      assembly: per row, per incident element, per quadrature point of the
//      reference's rule, the element row is accumulated in shared memory;
//      outputs A = M/dt + K and b = (M c_n)/dt + F directly.
//  edge_terms_kernel       boundary.py:108-173 (Neumann, free drainage of
//      water: right-hand side only), :217-277 (Cauchy: matrix + rhs),
//      :336-421 (free drainage of a solute: matrix).  Each boundary node sums
//      the contributions of its (at most two) boundary edges in edge order.
#include "common.cuh"
#include "soil.cuh"

namespace wspm {

struct FluxArgs {
    int n_rows;
    const int64_t *inc_ptr;
    const int32_t *inc_width;
    const int32_t *inc_elem;
    const int32_t *conn;
    const double *coords;
    const double *h;
    SoilParams sp;
    double DL, DT, Dm;
    double *qx, *qz, *aq, *Dxx, *Dxz, *Dzz, *theta;
};

__global__ void flux_dispersion_kernel(FluxArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_rows) return;
    const int s = i >> 5, lane = i & 31;
    const int deg = a.inc_width[s];
    const int64_t ib = a.inc_ptr[s] + lane;
    double sx = 0.0, sz = 0.0;
    int cnt = 0;
    for (int k = 0; k < deg; ++k) {
        const int e = a.inc_elem[ib + (int64_t)kSlice * k];
        if (e < 0) break;
        const int n0 = a.conn[3 * (int64_t)e], n1 = a.conn[3 * (int64_t)e + 1], n2 = a.conn[3 * (int64_t)e + 2];
        const double x0 = a.coords[2 * n0], y0 = a.coords[2 * n0 + 1];
        const double x1 = a.coords[2 * n1], y1 = a.coords[2 * n1 + 1];
        const double x2 = a.coords[2 * n2], y2 = a.coords[2 * n2 + 1];
        const double b1 = y1 - y2, b2 = y2 - y0, b3 = y0 - y1;
        const double c1 = x2 - x1, c2 = x0 - x2, c3 = x1 - x0;
        const double aire = fabs(c3 * b2 - c2 * b3) / 2;
        const double h0 = a.h[n0], h1 = a.h[n1], h2 = a.h[n2];
        sx += (b1 * h0 + b2 * h1 + b3 * h2) / (2 * aire);
        sz += (c1 * h0 + c2 * h1 + c3 * h2) / (2 * aire);
        ++cnt;
    }
    const double gx = sx / cnt, gz = sz / cnt;
    double C, K, th;
    soil_eval(a.sp, a.h[i], C, K, th);
    const double qx = -K * gx;
    const double qz = -K * (gz + 1);
    const double aq = sqrt(qx * qx + qz * qz);
    const double thS = a.sp.p[1];
    const double tau = pow(th, 7.0 / 3.0) / (thS * thS);
    a.qx[i] = qx;
    a.qz[i] = qz;
    a.aq[i] = aq;
    a.Dxx[i] = (a.DL * qx * qx + a.DT * qz * qz) / aq + th * a.Dm * tau;
    a.Dzz[i] = (a.DL * qz * qz + a.DT * qx * qx) / aq + th * a.Dm * tau;
    a.Dxz[i] = (a.DL - a.DT) * qx * qz / aq;
    a.theta[i] = th;
}

struct AdrArgs {
    int n_rows;
    const int64_t *slice_ptr;
    const int32_t *slice_width;
    const int32_t *diag_pos;
    const int64_t *inc_ptr;
    const int32_t *inc_width;
    const int32_t *inc_elem;
    const uint32_t *inc_slots;
    int n_diags;
    int max_width;      // block-uniform size of each accumulator block in shared memory
    int64_t ld;
    const int32_t *conn;
    const double *coords;
    const double *theta, *qx, *qz, *Dxx, *Dxz, *Dzz, *c_n, *c_up;
    double mu, sorption, mu_up, inv_dt;
    int lumped;
    int nq;
    double qN[16][3];   // shape functions at the quadrature points
    double qw[16];
    double *vals, *rhs, *dinv;
};

__global__ void __launch_bounds__(128) adr_rows_kernel(AdrArgs a) {
    extern __shared__ double sm[];          // [2][max_width][blockDim.x]: K and M accumulators
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = i >> 5, lane = i & 31;
    if (s >= ((a.n_rows + kSlice - 1) >> 5)) return;
    const bool dia = a.n_diags > 0;
    const int width = dia ? a.n_diags : a.slice_width[s];
    const int64_t vb = dia ? (int64_t)i : a.slice_ptr[s] + lane;
    const int64_t kstride = dia ? a.ld : (int64_t)kSlice;
    if (i >= a.n_rows) {
        for (int k = 0; k < width; ++k) a.vals[vb + kstride * k] = 0.0;
        return;
    }
    const int stride = blockDim.x;
    double *accK = sm + threadIdx.x;                                         // [max_width][blockDim]
    double *accM = sm + (size_t)blockDim.x * (size_t)a.max_width + threadIdx.x;  // [max_width][blockDim]
    for (int k = 0; k < width; ++k) { accK[k * stride] = 0.0; accM[k * stride] = 0.0; }
    double F = 0.0, Mc = 0.0, Ml = 0.0;
    const int deg = a.inc_width[s];
    const int64_t ib = a.inc_ptr[s] + lane;
    for (int kk = 0; kk < deg; ++kk) {
        const int e = a.inc_elem[ib + (int64_t)kSlice * kk];
        if (e < 0) break;
        const uint32_t packed = a.inc_slots[ib + (int64_t)kSlice * kk];
        const int li = packed & 3;
        int nd[3];
        for (int j = 0; j < 3; ++j) nd[j] = a.conn[3 * (int64_t)e + j];
        const double x0 = a.coords[2 * nd[0]], y0 = a.coords[2 * nd[0] + 1];
        const double J00 = a.coords[2 * nd[1]] - x0, J01 = a.coords[2 * nd[1] + 1] - y0;
        const double J10 = a.coords[2 * nd[2]] - x0, J11 = a.coords[2 * nd[2] + 1] - y0;
        const double detJ = J00 * J11 - J01 * J10;
        const double id = 1.0 / detJ;
        double G0[3], G1[3];
        G0[1] = J11 * id;  G1[1] = -J10 * id;
        G0[2] = -J01 * id; G1[2] = J00 * id;
        G0[0] = -(G0[1] + G0[2]);
        G1[0] = -(G1[1] + G1[2]);
        double f[7][3];
        for (int j = 0; j < 3; ++j) {
            f[0][j] = a.Dxx[nd[j]]; f[1][j] = a.Dxz[nd[j]]; f[2][j] = a.Dzz[nd[j]];
            f[3][j] = a.qx[nd[j]];  f[4][j] = a.qz[nd[j]];  f[5][j] = a.theta[nd[j]];
            f[6][j] = a.c_up ? a.c_up[nd[j]] : 0.0;
        }
        double rowK[3] = {0.0, 0.0, 0.0}, rowM[3] = {0.0, 0.0, 0.0};
        for (int q = 0; q < a.nq; ++q) {
            const double *N = a.qN[q];
            const double w = a.qw[q];
            double v[7];
            for (int c = 0; c < 7; ++c) v[c] = N[0] * f[c][0] + N[1] * f[c][1] + N[2] * f[c][2];
            const double g0 = G0[li], g1 = G1[li], nl = N[li];
            for (int j = 0; j < 3; ++j) {
                const double disp = -(v[0] * g0 * G0[j]) - v[1] * g0 * G1[j] - v[1] * g1 * G0[j] - v[2] * g1 * G1[j];
                const double adv = -(v[3] * nl * G0[j]) - v[4] * nl * G1[j];
                const double nn = nl * N[j];
                rowK[j] += w * disp * detJ + w * adv * detJ + (a.mu != 0.0 ? w * (a.mu * v[5]) * nn * detJ : 0.0);
                rowM[j] += w * (-v[5] - a.sorption) * nn * detJ;
            }
            if (a.c_up) F += -w * a.mu_up * v[5] * v[6] * nl * detJ;
        }
        for (int j = 0; j < 3; ++j) {
            const int kp = (packed >> (2 + 6 * j)) & 63;
            accK[kp * stride] += rowK[j];
            accM[kp * stride] += rowM[j];
            Mc += rowM[j] * a.c_n[nd[j]];
            Ml += rowM[j];
        }
    }
    const int dp = a.diag_pos[i];
    double diag = 0.0;
    for (int k = 0; k < width; ++k) {
        double v;
        if (a.lumped) v = accK[k * stride] + (k == dp ? a.inv_dt * Ml : 0.0);
        else v = a.inv_dt * accM[k * stride] + accK[k * stride];
        if (k == dp) diag = v;
        a.vals[vb + kstride * k] = v;
    }
    a.rhs[i] = a.lumped ? a.inv_dt * (Ml * a.c_n[i]) + F : a.inv_dt * Mc + F;
    if (a.dinv) a.dinv[i] = 1.0 / (diag != 0.0 ? diag : 1.0);
}

// Boundary edges, per boundary node t (node[t]); up to two edges per node
// listed in edge order: edge id, this node's local index (0 = I, 1 = J), the
// other node, and the row positions of the diagonal and of the other node.
struct EdgeArgs {
    int n_bnodes;
    const int32_t *node;       // [n_bnodes]
    const int32_t *e_cnt;      // [n_bnodes] 0..2
    const int32_t *e_local;    // [2*n_bnodes]
    const int32_t *e_other;    // [2*n_bnodes]
    const double *e_jac;       // [2*n_bnodes] edge Jacobian (x_J - x_I) / 2
    const int32_t *e_kother;   // [2*n_bnodes] row position of the other node's column
    int mode;                  // 0 Neumann rhs, 1 free-drainage water rhs, 2 Cauchy, 3 free-drainage solute
    double flux, c_in;
    const double *K, *theta;
    const int64_t *slice_ptr;
    const int32_t *diag_pos;
    int n_diags;
    int64_t ld;
    double *vals, *rhs;
};

__global__ void edge_terms_kernel(EdgeArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n_bnodes) return;
    const int I = a.node[t];
    // 2-point Gauss rule on [-1, 1], weights 1 (richards_solver_v2.py:65-66)
    const double xi[2] = {-1.0 / sqrt(3.0), 1.0 / sqrt(3.0)};
    double Nm[2][2];
    for (int j = 0; j < 2; ++j) { Nm[0][j] = (1 - xi[j]) / 2; Nm[1][j] = (1 + xi[j]) / 2; }
    const bool dia = a.n_diags > 0;
    auto pos = [&](int k) -> int64_t {
        return dia ? (int64_t)k * a.ld + I : a.slice_ptr[I >> 5] + (int64_t)kSlice * k + (I & 31);
    };
    double rhs_add = 0.0, d_add = 0.0;
    for (int c = 0; c < a.e_cnt[t]; ++c) {
        const int l = a.e_local[2 * t + c];
        const int O = a.e_other[2 * t + c];
        const double jac = a.e_jac[2 * t + c];
        const int nI = l == 0 ? I : O, nJ = l == 0 ? O : I;
        if (a.mode == 0) {
            double loc = 0.0;
            for (int j = 0; j < 2; ++j) loc = loc - jac * 1.0 * a.flux * Nm[l][j];
            rhs_add += loc;
        } else if (a.mode == 1) {
            double loc = 0.0;
            for (int j = 0; j < 2; ++j) {
                const double kav = Nm[0][j] * a.K[nI] + Nm[1][j] * a.K[nJ];
                loc = loc + (-jac * 1.0 * kav * Nm[l][j]);
            }
            rhs_add += loc;
        } else {
            double mll = 0.0, mlo = 0.0;
            for (int j = 0; j < 2; ++j) {
                double wgt;
                if (a.mode == 2) {
                    wgt = jac * 1.0 * a.flux;
                } else {
                    const double kav = Nm[0][j] * a.K[nI] + Nm[1][j] * a.K[nJ];
                    const double tav = Nm[0][j] * a.theta[nI] + Nm[1][j] * a.theta[nJ];
                    wgt = jac * 1.0 * (-kav / tav);
                }
                mll += wgt * Nm[l][j] * Nm[l][j];
                mlo += wgt * Nm[l][j] * Nm[1 - l][j];
            }
            d_add += mll;
            a.vals[pos(a.e_kother[2 * t + c])] += mlo;
            if (a.mode == 2)
                rhs_add += jac * a.c_in * a.flux * (1.0 * Nm[l][0] + 1.0 * Nm[l][1]);
        }
    }
    if (a.mode >= 2) a.vals[pos(a.diag_pos[I])] += d_add;
    a.rhs[I] += rhs_add;
}

}  // namespace wspm

namespace wspm {

void quadrature_constants(int dim, const double *Q, const double *W, int nq, double s[4], double m[4]);

int launch_flux_dispersion(const wspm_mesh *mesh, const wspm_pattern *pat, const double *h, const SoilParams &sp,
                           double DL, double DT, double Dm, double *qx, double *qz, double *aq, double *Dxx,
                           double *Dxz, double *Dzz, double *theta, cudaStream_t st) {
    FluxArgs a;
    a.n_rows = pat->n_rows;
    a.inc_ptr = pat->inc_ptr; a.inc_width = pat->inc_width; a.inc_elem = pat->inc_elem;
    a.conn = mesh->conn; a.coords = mesh->coords; a.h = h; a.sp = sp;
    a.DL = DL; a.DT = DT; a.Dm = Dm;
    a.qx = qx; a.qz = qz; a.aq = aq; a.Dxx = Dxx; a.Dxz = Dxz; a.Dzz = Dzz; a.theta = theta;
    flux_dispersion_kernel<<<(pat->n_rows + 127) / 128, 128, 0, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

int launch_adr(const wspm_mesh *mesh, const wspm_pattern *pat, const double *theta, const double *qx,
               const double *qz, const double *Dxx, const double *Dxz, const double *Dzz, const double *c_n,
               const double *c_up, double mu, double sorption, double mu_up, int lumped, const double *Q,
               const double *W, int nq, double dt, double *vals, double *rhs, double *dinv, cudaStream_t st) {
    AdrArgs a;
    a.n_rows = pat->n_rows;
    a.slice_ptr = pat->slice_ptr; a.slice_width = pat->slice_width; a.diag_pos = pat->diag_pos;
    a.inc_ptr = pat->inc_ptr; a.inc_width = pat->inc_width; a.inc_elem = pat->inc_elem; a.inc_slots = pat->inc_slots;
    a.n_diags = pat->n_diags; a.max_width = pat->max_width; a.ld = (int64_t)pat->n_slices * kSlice;
    a.conn = mesh->conn; a.coords = mesh->coords;
    a.theta = theta; a.qx = qx; a.qz = qz; a.Dxx = Dxx; a.Dxz = Dxz; a.Dzz = Dzz; a.c_n = c_n; a.c_up = c_up;
    a.mu = mu; a.sorption = sorption; a.mu_up = mu_up; a.inv_dt = 1.0 / dt; a.lumped = lumped;
    a.nq = nq;
    for (int q = 0; q < nq; ++q) {
        a.qN[q][0] = 1 - Q[2 * q] - Q[2 * q + 1];
        a.qN[q][1] = Q[2 * q];
        a.qN[q][2] = Q[2 * q + 1];
        a.qw[q] = W[q];
    }
    a.vals = vals; a.rhs = rhs; a.dinv = dinv;
    const int threads = 128;
    const size_t smem = 2 * (size_t)pat->max_width * threads * sizeof(double);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(adr_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    adr_rows_kernel<<<(pat->n_slices * kSlice + threads - 1) / threads, threads, smem, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

int launch_edge_terms(const wspm_pattern *pat, const wspm_edges *e, int mode, double flux, double c_in,
                      const double *K, const double *theta, double *vals, double *rhs, cudaStream_t st) {
    if (e->n_bnodes <= 0) return WSPM_OK;
    EdgeArgs a;
    a.n_bnodes = e->n_bnodes;
    a.node = e->node; a.e_cnt = e->e_cnt; a.e_local = e->e_local; a.e_other = e->e_other;
    a.e_jac = e->e_jac; a.e_kother = e->e_kother;
    a.mode = mode; a.flux = flux; a.c_in = c_in; a.K = K; a.theta = theta;
    a.slice_ptr = pat->slice_ptr; a.diag_pos = pat->diag_pos;
    a.n_diags = pat->n_diags; a.ld = (int64_t)pat->n_slices * kSlice;
    a.vals = vals; a.rhs = rhs;
    edge_terms_kernel<<<(e->n_bnodes + 127) / 128, 128, 0, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

}  // namespace wspm
