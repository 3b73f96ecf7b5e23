// Domain integral of a nodal field (mass balance) and the Peclet / Courant
// numbers of the transport step, 2D P1 triangles.
//
//  * wspm_integrate_2d: integrate_2d_domain of the reference's mass-balance
//    driver (src/solvers/.ipynb_checkpoints/richards_mass_balance-checkpoint.py:25-69):
//    sum over triangles of |det J| * sum_q (1/3) f(x_q) with the 3-point rule
//    (1/6,1/6), (2/3,1/6), (1/6,2/3).  The weights sum to 1 (not 1/2), as in
//    the reference, so the value is twice the integral; mass-balance ratios
//    are unaffected.
//  * wspm_peclet_courant: calculate_peclet_courant
//    (src/models/transport_utilities.py:193-242): per element h = shortest
//    edge, v = q / theta at its nodes, Pe = max |v| h / (2 D), Cr = max |v| dt / h
//    over nodes and both directions, then the maxima over elements.
// Both are two-pass reductions over a fixed grid (per-block partials, then one
// block in fixed order), so sums are bitwise repeatable.
#include "common.cuh"

namespace wspm {

constexpr int kBalBlocks = 592;   // 4 x 148: fixed grid, fixed summation order

__global__ void integrate_2d_kernel(const int32_t *__restrict__ conn, const double *__restrict__ coords, int E,
                                    const double *__restrict__ f, double *partials) {
    const double gp[3][2] = {{1.0 / 6.0, 1.0 / 6.0}, {2.0 / 3.0, 1.0 / 6.0}, {1.0 / 6.0, 2.0 / 3.0}};
    double v[1] = {0.0};
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        const int n0 = conn[3 * (int64_t)e], n1 = conn[3 * (int64_t)e + 1], n2 = conn[3 * (int64_t)e + 2];
        const double x0 = coords[2 * n0], y0 = coords[2 * n0 + 1];
        const double J00 = coords[2 * n1] - x0, J01 = coords[2 * n2] - x0;
        const double J10 = coords[2 * n1 + 1] - y0, J11 = coords[2 * n2 + 1] - y0;
        const double det = fabs(J00 * J11 - J01 * J10);
        const double f0 = f[n0], f1 = f[n1], f2 = f[n2];
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double a = gp[q][0], b = gp[q][1];
            s += (1.0 / 3.0) * (f0 * (1.0 - a - b) + f1 * a + f2 * b);
        }
        v[0] += s * det;
    }
    block_sum<double, 1>(v);
    if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

__global__ void peclet_courant_kernel(const int32_t *__restrict__ conn, const double *__restrict__ coords, int E,
                                      const double *__restrict__ qx, const double *__restrict__ qz,
                                      const double *__restrict__ theta, const double *__restrict__ Dxx,
                                      const double *__restrict__ Dzz, double dt, double *partials) {
    double pe = 0.0, cr = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        int nd[3];
        for (int j = 0; j < 3; ++j) nd[j] = conn[3 * (int64_t)e + j];
        double h = 1e300;
        for (int j = 0; j < 3; ++j) {
            const int a = nd[j], b = nd[(j + 2) % 3];
            const double dx = coords[2 * a] - coords[2 * b], dy = coords[2 * a + 1] - coords[2 * b + 1];
            h = fmin(h, sqrt(dx * dx + dy * dy));
        }
        for (int j = 0; j < 3; ++j) {
            const int i = nd[j];
            const double vx = fabs(qx[i] / theta[i]), vz = fabs(qz[i] / theta[i]);
            pe = fmax(pe, fmax(vx * h / (2.0 * Dxx[i]), vz * h / (2.0 * Dzz[i])));
            cr = fmax(cr, fmax(vx * dt / h, vz * dt / h));
        }
    }
    // block max (order-free)
    __shared__ double s_pe[32], s_cr[32];
    for (int o = 16; o > 0; o >>= 1) {
        pe = fmax(pe, __shfl_down_sync(0xffffffffu, pe, o));
        cr = fmax(cr, __shfl_down_sync(0xffffffffu, cr, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { s_pe[wid] = pe; s_cr[wid] = cr; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { pe = fmax(pe, s_pe[w]); cr = fmax(cr, s_cr[w]); }
        partials[2 * blockIdx.x] = pe;
        partials[2 * blockIdx.x + 1] = cr;
    }
}

// One block: fixed-order sum (mode 0) or max of pairs (mode 1) of the partials.
__global__ void finish_kernel(const double *partials, int nb, int mode, double *out) {
    if (mode == 0) {
        double v[1] = {0.0};
        for (int b = threadIdx.x; b < nb; b += blockDim.x) v[0] += partials[b];
        block_sum<double, 1>(v);
        if (threadIdx.x == 0) out[0] = v[0];
    } else if (threadIdx.x == 0) {
        double pe = 0.0, cr = 0.0;
        for (int b = 0; b < nb; ++b) { pe = fmax(pe, partials[2 * b]); cr = fmax(cr, partials[2 * b + 1]); }
        out[0] = pe;
        out[1] = cr;
    }
}

}  // namespace wspm

using namespace wspm;

extern "C" int64_t wspm_balance_workspace_doubles(void) { return 2 * kBalBlocks; }

extern "C" int wspm_integrate_2d(const wspm_mesh *mesh, const double *f, double *out, double *work, void *stream) {
    if (!mesh || mesh->dim != 2 || !mesh->conn || !mesh->coords || !f || !out || !work) return WSPM_BAD_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    integrate_2d_kernel<<<kBalBlocks, 256, 0, st>>>(mesh->conn, mesh->coords, mesh->n_elems, f, work);
    finish_kernel<<<1, 256, 0, st>>>(work, kBalBlocks, 0, out);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

extern "C" int wspm_peclet_courant(const wspm_mesh *mesh, const double *qx, const double *qz, const double *theta,
                                   const double *Dxx, const double *Dzz, double dt, double *out2, double *work,
                                   void *stream) {
    if (!mesh || mesh->dim != 2 || !qx || !qz || !theta || !Dxx || !Dzz || !out2 || !work) return WSPM_BAD_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    peclet_courant_kernel<<<kBalBlocks, 256, 0, st>>>(mesh->conn, mesh->coords, mesh->n_elems, qx, qz, theta, Dxx,
                                                      Dzz, dt, work);
    finish_kernel<<<1, 32, 0, st>>>(work, kBalBlocks, 1, out2);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}
