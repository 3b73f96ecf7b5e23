// Soil-model and Richards assembly kernels.
//
// Assembly is row-gather: thread i owns row i of the global matrix.  It walks
// the elements incident to node i (ascending element id, the order in which
// the reference's COO entries meet in BCOO.sum_duplicates and in which its
// fori_loop scatters the right-hand side, assembly_re_v2.py:145-164), computes
// row "local vertex of i" of each element matrix in registers, and
// accumulates into the row's SELL slots held in shared memory.  Each row is
// written exactly once, coalesced across the warp, with no atomics.
//
// Element math (P1, constant gradient): G = J^-1 dN/dref, detJ signed as
// jnp.linalg.det.  With the reference's quadrature rule (points Q, weights W)
//   Kbar   = sum_q w_q (N_q . K)            = sum_j s_j K_j,  s_j = sum_q w_q N_qj
//   Ml_i   = rowsum_j sum_q w_q N_qi N_qj * detJ = mcoef_i * detJ
//   A_e    = Kbar (G^T G) detJ + diag(Ml * C) / dt
//   b_e,i  = -Kbar G[dim-1, i] detJ - Ml_i (theta_m,i - theta_n,i - C_i h_i) / dt
// which is compute_local_matrices_mixed_form (assembly_re_v2.py:13-60) and its
// 3D twin (assembly_re_3D.py:12-70).
#include "common.cuh"
#include "krylov.cuh"
#include "soil.cuh"

namespace wspm {

__global__ void soil_kernel(SoilParams sp, const double *__restrict__ h, int64_t n,
                            double *C, double *K, double *theta) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double c, k, t;
        soil_eval(sp, h[i], c, k, t);
        if (C) C[i] = c;
        if (K) K[i] = k;
        if (theta) theta[i] = t;
    }
}

struct RichardsAsmArgs {
    int n_rows;
    const int64_t *slice_ptr;
    const int32_t *slice_width;
    const int32_t *diag_pos;
    const int64_t *inc_ptr;
    const int32_t *inc_width;
    const int32_t *inc_elem;
    const uint32_t *inc_slots;
    const int32_t *conn;
    const double *coords;
    const double *theta_m, *theta_n, *h_m, *K, *C, *Ks_elem, *bc_val;
    const double *Ks_inc;    // per-element factor in incidence order (pad marker on padding slots)
    double s[4];       // K-average weights per vertex
    double mcoef[4];   // lumped-mass coefficients per vertex
    double inv_dt;
    const double *dt_dev;   // when set, dt is read from device memory (graph replay)
    int n_diags;            // > 0: DIA layout, entry k of row i at k*ld + i
    int64_t ld;
    const int32_t *diag_off;   // DIA column offsets
    const int32_t *cols;       // SELL column indices
    double *vals;
    float *vals32;
    double *rhs, *dinv;
    RefineStart res;           // used by the RES instantiations only
    const double *shape_tab;   // CLS: per element shape, kShapeStride<DIM> doubles (shape_table_kernel)
    int n_shapes;
};

// Element shapes: elements whose Jacobians are bitwise equal have bitwise equal
// geometry, so a mesh with few distinct Jacobians (a grid whose coordinates are
// exact binary fractions has two triangle shapes, six Kuhn tetrahedra) can take
// the geometric factors of every element-row from a small table instead of
// recomputing them.  Entry of a shape: detJ, then gg[li][j] = G[:,li] . G[:,j]
// (NV x NV, the fma chain of the row kernel), then G[DIM-1][li] (NV values).
//
// Two forms of the tagged incidence words.  Mode 1: the words keep their 6-bit
// row positions, the shape id sits above them (12 bits in 2D, 6 in 3D) and the
// table (at most 256 triangle / 64 tetrahedron shapes) is copied into shared
// memory.  Mode 2, for patterns with at most 16 entries per row: the row
// positions are repacked into 4 bits each, the id takes the 18 (2D) or 14 (3D)
// bits above them, and the table (up to 16,384 shapes; 1.7 MB for the 10,368
// tetrahedra of a 96^3 grid with coordinates i/96) is read from global memory,
// where it stays in L2.
template <int DIM> constexpr int kShapeStride = 1 + (DIM + 1) * (DIM + 1) + (DIM + 1);
template <int DIM, int SHP> constexpr int kPosBits = SHP == 2 ? 4 : 6;
template <int DIM, int SHP> constexpr int kShapeShift = 2 + kPosBits<DIM, SHP> * (DIM + 1);
template <int DIM> constexpr int kMaxShapes = DIM == 2 ? 256 : 64;          // mode 1
constexpr int kMaxShapesGlobal = 16384;                                      // mode 2 (2D: 18 bits, 3D: 14)
constexpr int kShapeReuse = 8;                                               // mode 2: elements per shape, at least
constexpr int kShapesShared = 64;                                            // mode 1 preferred up to this many

template <int DIM>
__device__ __forceinline__ void p1_geometry(const double *__restrict__ coords, const int (&nd)[DIM + 1],
                                            double (&G)[DIM][DIM + 1], double &detJ) {
    if constexpr (DIM == 2) {
        const double x0 = coords[2 * nd[0]], y0 = coords[2 * nd[0] + 1];
        const double J00 = coords[2 * nd[1]] - x0, J01 = coords[2 * nd[1] + 1] - y0;
        const double J10 = coords[2 * nd[2]] - x0, J11 = coords[2 * nd[2] + 1] - y0;
        detJ = J00 * J11 - J01 * J10;
        const double id = 1.0 / detJ;
        // J^-1 = [[J11, -J01], [-J10, J00]] / det ; G[:,1] = J^-1[:,0], G[:,2] = J^-1[:,1]
        G[0][1] = J11 * id;  G[1][1] = -J10 * id;
        G[0][2] = -J01 * id; G[1][2] = J00 * id;
        G[0][0] = -(G[0][1] + G[0][2]);
        G[1][0] = -(G[1][1] + G[1][2]);
    } else {
        double J[3][3];
        const double *p0 = coords + 3 * nd[0];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const double *pr = coords + 3 * nd[r + 1];
#pragma unroll
            for (int c = 0; c < 3; ++c) J[r][c] = pr[c] - p0[c];
        }
        const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
        const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
        const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
        detJ = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
        const double id = 1.0 / detJ;
        // inverse = adj / det, adj[r][c] = cofactor[c][r]
        double inv[3][3];
        inv[0][0] = c00 * id;
        inv[1][0] = c01 * id;
        inv[2][0] = c02 * id;
        inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
        inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
        inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
        inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
        inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
        inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            G[d][1] = inv[d][0];
            G[d][2] = inv[d][1];
            G[d][3] = inv[d][2];
            G[d][0] = -((inv[d][0] + inv[d][1]) + inv[d][2]);
        }
    }
}

// G and detJ from the Jacobian's columns J[r][c] = X[r+1][c] - X[0][c]: the
// arithmetic of p1_geometry after its differences.
template <int DIM>
__device__ __forceinline__ void p1_geometry_j(const double (&J)[DIM][DIM], double (&G)[DIM][DIM + 1], double &detJ) {
    if constexpr (DIM == 2) {
        const double J00 = J[0][0], J01 = J[0][1], J10 = J[1][0], J11 = J[1][1];
        detJ = J00 * J11 - J01 * J10;
        const double id = 1.0 / detJ;
        G[0][1] = J11 * id;  G[1][1] = -J10 * id;
        G[0][2] = -J01 * id; G[1][2] = J00 * id;
        G[0][0] = -(G[0][1] + G[0][2]);
        G[1][0] = -(G[1][1] + G[1][2]);
    } else {
        const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
        const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
        const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
        detJ = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
        const double id = 1.0 / detJ;
        double inv[3][3];
        inv[0][0] = c00 * id;
        inv[1][0] = c01 * id;
        inv[2][0] = c02 * id;
        inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
        inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
        inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
        inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
        inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
        inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            G[d][1] = inv[d][0];
            G[d][2] = inv[d][1];
            G[d][3] = inv[d][2];
            G[d][0] = -((inv[d][0] + inv[d][1]) + inv[d][2]);
        }
    }
}

template <int DIM>
__device__ __forceinline__ void p1_jacobian(const double (&X)[DIM + 1][DIM], double (&J)[DIM][DIM]) {
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int c = 0; c < DIM; ++c) J[r][c] = X[r + 1][c] - X[0][c];
}

// Same as p1_geometry, from vertex coordinates already in registers.
template <int DIM>
__device__ __forceinline__ void p1_geometry_xyz(const double (&X)[DIM + 1][DIM], double (&G)[DIM][DIM + 1],
                                                double &detJ) {
    double J[DIM][DIM];
    p1_jacobian<DIM>(X, J);
    p1_geometry_j<DIM>(J, G, detJ);
}

// Structural zeros of a DIA Richards matrix.  Off the main diagonal the row
// kernel adds, per element, Kbar detJ (G^T G)[li][j]; the lumped mass and the
// Dirichlet rows touch only the main diagonal or write zeros.  Bit k of *mask is
// set when some element puts a nonzero factor (G^T G)[li][j] -- evaluated with
// exactly the operations of richards_rows_kernel -- on diagonal k, and for the
// main diagonal; a clear bit is a diagonal that is exactly zero in every
// assembly, whatever K, C and dt are (e.g. the edges opposite the right angles of
// a split-square grid whose coordinates are exact binary fractions).  An
// element pair whose offset is on no diagonal sets every bit (no skipping).
template <int DIM>
__global__ void dia_live_kernel(int n_elems, const int32_t *__restrict__ conn, const double *__restrict__ coords,
                                int nd, const int32_t *__restrict__ diag_off, unsigned long long *mask) {
    constexpr int NV = DIM + 1;
    __shared__ unsigned long long s_mask;
    if (threadIdx.x == 0) s_mask = 0ull;
    __syncthreads();
    unsigned long long m = 0ull;
    if (blockIdx.x == 0 && threadIdx.x < nd && diag_off[threadIdx.x] == 0) m |= 1ull << threadIdx.x;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_elems; e += gridDim.x * blockDim.x) {
        int nodes[NV];
        double X[NV][DIM];
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            nodes[j] = conn[(int64_t)NV * e + j];
#pragma unroll
            for (int d = 0; d < DIM; ++d) X[j][d] = coords[(int64_t)DIM * nodes[j] + d];
        }
        double G[DIM][NV], detJ;
        p1_geometry_xyz<DIM>(X, G, detJ);
#pragma unroll
        for (int li = 0; li < NV; ++li) {
            double gli[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                double g = G[d][0];
#pragma unroll
                for (int j = 1; j < NV; ++j) g = li == j ? G[d][j] : g;
                gli[d] = g;
            }
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                if (j == li) continue;
                double gg = 0.0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) gg = fma(gli[d], G[d][j], gg);
                if (gg == 0.0) continue;
                const int off = nodes[j] - nodes[li];
                int k = 0;
                while (k < nd && diag_off[k] != off) ++k;
                m |= k < nd ? 1ull << k : ~0ull;
            }
        }
    }
    if (m) atomicOr(&s_mask, m);
    __syncthreads();
    if (threadIdx.x == 0 && s_mask) atomicOr(mask, s_mask);
}

// Live-diagonal mask of a DIA Richards pattern (all ones for SELL patterns or on
// any failure, which only disables the skipping).  `word`: one device word of
// scratch; synchronous (plan creation only).
unsigned long long richards_dia_live_mask(const wspm_mesh *mesh, const wspm_pattern *pat,
                                          unsigned long long *word) {
    const unsigned long long all = ~0ull;
    if (!mesh || !pat || pat->n_diags <= 0 || pat->n_diags > 63 || !pat->diag_offsets || !word) return all;
    if (mesh->dim != 2 && mesh->dim != 3) return all;
    if (cudaMemset(word, 0, sizeof(unsigned long long)) != cudaSuccess) return all;
    const int blocks = (int)((mesh->n_elems + 255) / 256 < 148 * 8 ? (mesh->n_elems + 255) / 256 : 148 * 8);
    if (mesh->dim == 2)
        dia_live_kernel<2><<<blocks > 0 ? blocks : 1, 256>>>(mesh->n_elems, mesh->conn, mesh->coords, pat->n_diags,
                                                             pat->diag_offsets, word);
    else
        dia_live_kernel<3><<<blocks > 0 ? blocks : 1, 256>>>(mesh->n_elems, mesh->conn, mesh->coords, pat->n_diags,
                                                             pat->diag_offsets, word);
    unsigned long long m = 0ull;
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpy(&m, word, sizeof(m), cudaMemcpyDeviceToHost) != cudaSuccess)
        return all;
    return m;
}

// Incidence-ordered per-element values: slot o of the incidence layout gets
// elem[inc_elem[o]]; padding slots get kIncPad, a NaN bit pattern that the
// row kernel tests for (so it needs no element id per slot).
constexpr long long kIncPad = (long long)0xFFF0DEAD00000000ULL;

__global__ void incidence_gather_kernel(int n_slices, const int64_t *__restrict__ inc_ptr,
                                        const int32_t *__restrict__ inc_width, const int32_t *__restrict__ inc_elem,
                                        const double *__restrict__ elem, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = i >> 5, lane = i & 31;
    if (s >= n_slices) return;
    const int64_t ib = inc_ptr[s] + lane;
    const int w = inc_width[s];
    for (int k = 0; k < w; ++k) {
        const int64_t o = ib + (int64_t)kSlice * k;
        const int e = inc_elem[o];
        out[o] = e >= 0 ? elem[e] : __longlong_as_double(kIncPad);
    }
}

// Row kernel.  Every vertex of an element incident to node i is a column of
// row i, and the incidence word records, per element vertex, its position in
// the row.  Thread i walks the incident elements in ascending id, computes
// row "local vertex of i" of each element matrix in registers and accumulates
// into the row's slots in shared memory; vertex order inside each element and
// the element order are those of the element-walking form, so every value and
// every accumulation order are unchanged.
//
// Column data (coordinates, K) come either from a shared-memory stage filled
// once per row with all loads in flight (STAGE; two dependent memory round
// trips per row), or, for DIA patterns, straight from global memory per
// element at column i + off[position] (L1-resident: the row's columns are the
// neighbouring rows' columns too).  2D takes the stage; 3D (15 columns x 4
// values would hold occupancy to two blocks per SM) takes the direct reads.
// Either way the incidence words (and Ks) of 4 incidences are loaded together
// before the first of them is used: with one incidence at a time the 3D rows
// (24 tetrahedra per vertex) were a chain of dependent round trips (96^3 Kuhn
// grid, global shape table: 217 -> 178 us; binary 64^3 grid: 75 -> 45 us).
//
// KSM selects the per-element conductivity factor: 0 none, 1 gathered by
// element id, 2 read in incidence order (Ks_inc, built once per time step by
// incidence_gather_kernel: one coalesced load per slot, no dependent gather,
// and its pad marker replaces the element-id read).
//
// The element-local row index li selects a column of G by selects: an indexed
// register array would live in local memory.
//
// SHP (element shapes; 0: none): the incidence words carry the element's shape
// id and the geometric factors come from the shape table -- copied into shared
// memory once per block (1) or read from global memory (2); the column stage
// then holds K only.  Every value and every accumulation order are those of the
// geometry-computing form.
template <int DIM, int MW, int KSM, bool STAGE, int TB, int MINB, bool RES, int SHP>
__global__ void __launch_bounds__(TB, MINB) richards_rows_kernel(RichardsAsmArgs a) {
    constexpr bool CLS = SHP != 0;
    constexpr int PB = kPosBits<DIM, SHP>, PM = (1 << PB) - 1;   // row-position field of the incidence word
    constexpr int NV = DIM + 1;
    constexpr int CH = 4;               // incidences whose loads are issued together
    constexpr int CV = CLS ? 1 : NV;    // staged values per column (K; or coordinates and K)
    extern __shared__ double acc_sm[];  // [MW][TB] accumulators, [MW][CV][TB] column data (STAGE), shapes (CLS)
    __shared__ int s_off[MW];
    const int i = blockIdx.x * TB + threadIdx.x;
    const int s = i >> 5, lane = i & 31;
    const bool dia = a.n_diags > 0;
    if (dia)
        for (int k = threadIdx.x; k < a.n_diags; k += TB) s_off[k] = a.diag_off[k];
    double *const s_shape = acc_sm + MW * TB * (STAGE ? 1 + CV : 1);
    if constexpr (SHP == 1)
        for (int k = threadIdx.x; k < a.n_shapes * kShapeStride<DIM>; k += TB) s_shape[k] = a.shape_tab[k];
    __syncthreads();
    double res_v[2] = {0.0, 0.0};   // RES: this row's (r.r, b.b)
    do {   // one pass; break = this thread has no row (every thread reaches the RES reduction)
    if (s >= ((a.n_rows + kSlice - 1) >> 5)) break;
    const int width = dia ? a.n_diags : a.slice_width[s];
    // entry k of this row lives at vb + kstride * k
    const int64_t vb = dia ? (int64_t)i : a.slice_ptr[s] + lane;
    const int64_t kstride = dia ? a.ld : (int64_t)kSlice;
    if (i >= a.n_rows) {
        // padding rows of the last slice: keep their slots defined (zero)
        for (int k = 0; k < width; ++k) {
            a.vals[vb + kstride * k] = 0.0;
            if (a.vals32) a.vals32[vb + kstride * k] = 0.0f;
        }
        break;
    }
    double *acc = acc_sm + threadIdx.x;
    double *colv = acc_sm + MW * TB + threadIdx.x;   // column k, component c at colv[(k * CV + c) * TB]
    for (int k = 0; k < width; ++k) acc[k * TB] = 0.0;
    const int dpos = a.diag_pos[i];

    const double inv_dt = a.dt_dev ? 1.0 / *a.dt_dev : a.inv_dt;
    const double bcv = a.bc_val ? a.bc_val[i] : __longlong_as_double(0x7ff8000000000000ULL);
    double rhs_i, diag;
    if (!isnan(bcv)) {
        acc[dpos * TB] = 1.0;
        rhs_i = bcv;
        diag = 1.0;
    } else {
        const double Ci = a.C[i];
        const double tm = a.theta_m[i], tn = a.theta_n[i], hi = a.h_m[i];
        const double storage = tm - tn - Ci * hi;
        const int deg = a.inc_width[s];
        const int64_t ib = a.inc_ptr[s] + lane;
        if constexpr (STAGE) {
            // column data of the row: coordinates and K, CG columns per batch of loads in flight
            constexpr int CG = DIM == 2 ? 8 : 4;
            const int last = a.n_rows - 1;
#pragma unroll
            for (int k0 = 0; k0 < MW; k0 += CG) {
                if (k0 >= width) break;
                double xv[CG][DIM], kv[CG];
#pragma unroll
                for (int g = 0; g < CG; ++g) {
                    const int k = k0 + g;
                    if (k < width) {
                        int c = dia ? i + s_off[k] : __ldg(a.cols + vb + kstride * k);
                        c = c < 0 ? 0 : (c > last ? last : c);
                        if constexpr (!CLS) {
#pragma unroll
                            for (int d = 0; d < DIM; ++d) xv[g][d] = __ldg(a.coords + (int64_t)DIM * c + d);
                        }
                        kv[g] = __ldg(a.K + c);
                    }
                }
#pragma unroll
                for (int g = 0; g < CG; ++g) {
                    const int k = k0 + g;
                    if (k < width) {
                        if constexpr (!CLS) {
#pragma unroll
                            for (int d = 0; d < DIM; ++d) colv[(k * CV + d) * TB] = xv[g][d];
                        }
                        colv[(k * CV + CV - 1) * TB] = kv[g];
                    }
                }
            }
        }
        double bsum = 0.0;
#pragma unroll 1
        for (int k0 = 0; k0 < deg; k0 += CH) {
            uint32_t pk[CH];
            bool ok[CH];
            double kse[CH];
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                pk[c] = 0u;
                ok[c] = false;
                kse[c] = 1.0;
                if (k0 + c < deg) {
                    const int64_t o = ib + (int64_t)kSlice * (k0 + c);
                    pk[c] = __ldg(a.inc_slots + o);
                    if constexpr (KSM == 2) {
                        kse[c] = __ldg(a.Ks_inc + o);
                        ok[c] = __double_as_longlong(kse[c]) != kIncPad;
                    } else {
                        const int ev = __ldg(a.inc_elem + o);   // -1: padding of the slice
                        ok[c] = ev >= 0;
                        if (KSM == 1 && ev >= 0) kse[c] = __ldg(a.Ks_elem + ev);
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                if (!ok[c]) continue;
                const uint32_t packed = pk[c];
                const int li = packed & 3;
                double X[NV][DIM], Kv[NV];
#pragma unroll
                for (int j = 0; j < NV; ++j) {
                    const int kp = (packed >> (2 + PB * j)) & PM;
                    if constexpr (STAGE) {
                        if constexpr (!CLS) {
#pragma unroll
                            for (int d = 0; d < DIM; ++d) X[j][d] = colv[(kp * CV + d) * TB];
                        }
                        Kv[j] = colv[(kp * CV + CV - 1) * TB];
                    } else {
                        const int col = i + s_off[kp];
                        if constexpr (!CLS) {
#pragma unroll
                            for (int d = 0; d < DIM; ++d) X[j][d] = __ldg(a.coords + (int64_t)DIM * col + d);
                        }
                        Kv[j] = __ldg(a.K + col);
                    }
                }
                double Kbar = 0.0;
#pragma unroll
                for (int j = 0; j < NV; ++j) Kbar = fma(a.s[j], Kv[j], Kbar);
                if constexpr (KSM != 0) Kbar *= kse[c];
                if constexpr (CLS) {
                    const int64_t so = (int64_t)(packed >> kShapeShift<DIM, SHP>) * kShapeStride<DIM>;
                    double detJ, ggl[NV], glast;
                    if constexpr (SHP == 1) {
                        detJ = s_shape[so];
#pragma unroll
                        for (int j = 0; j < NV; ++j) ggl[j] = s_shape[so + 1 + li * NV + j];
                        glast = s_shape[so + 1 + NV * NV + li];
                    } else {
                        detJ = __ldg(a.shape_tab + so);
#pragma unroll
                        for (int j = 0; j < NV; ++j) ggl[j] = __ldg(a.shape_tab + so + 1 + li * NV + j);
                        glast = __ldg(a.shape_tab + so + 1 + NV * NV + li);
                    }
                    const double kd = Kbar * detJ;
                    const double Ml = a.mcoef[li] * detJ;
#pragma unroll
                    for (int j = 0; j < NV; ++j) {
                        double v = kd * ggl[j];
                        if (j == li) v += inv_dt * (Ml * Ci);
                        const int kpos = (packed >> (2 + PB * j)) & PM;
                        acc[kpos * TB] += v;
                    }
                    bsum += -kd * glast - inv_dt * (Ml * storage);
                } else {
                    double G[DIM][NV], detJ;
                    p1_geometry_xyz<DIM>(X, G, detJ);
                    const double kd = Kbar * detJ;
                    const double Ml = a.mcoef[li] * detJ;
                    double gli[DIM];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        double g = G[d][0];
#pragma unroll
                        for (int j = 1; j < NV; ++j) g = li == j ? G[d][j] : g;
                        gli[d] = g;
                    }
#pragma unroll
                    for (int j = 0; j < NV; ++j) {
                        double gg = 0.0;
#pragma unroll
                        for (int d = 0; d < DIM; ++d) gg = fma(gli[d], G[d][j], gg);
                        double v = kd * gg;
                        if (j == li) v += inv_dt * (Ml * Ci);
                        const int kpos = (packed >> (2 + PB * j)) & PM;
                        acc[kpos * TB] += v;
                    }
                    bsum += -kd * gli[DIM - 1] - inv_dt * (Ml * storage);
                }
            }
        }
        rhs_i = bsum;
        diag = acc[dpos * TB];
    }
    a.rhs[i] = rhs_i;
    const double dinv_i = 1.0 / (diag != 0.0 ? diag : 1.0);
    if (a.dinv) a.dinv[i] = dinv_i;
    for (int k = 0; k < width; ++k) {
        const double v = acc[k * TB];
        a.vals[vb + kstride * k] = v;
        if (a.vals32) a.vals32[vb + kstride * k] = (float)v;
    }
    if constexpr (RES) {
        // start of the refinement loop: r = b - A x0 with the row just built
        // (entries and columns in storage order, as the stand-alone kernel sums them)
        const int last = a.n_rows - 1;
        const double *x0 = a.res.x0;
        double dot = 0.0;
        for (int k = 0; k < width; ++k) {
            int c = dia ? i + s_off[k] : __ldg(a.cols + vb + kstride * k);
            c = c < 0 ? 0 : (c > last ? last : c);
            dot = fma(acc[k * TB], x0[c], dot);
        }
        const double ri = rhs_i - dot;
        a.res.r[i] = ri;
        a.res.x[i] = x0[i];
        if (a.res.dinv32) a.res.dinv32[i] = (float)dinv_i;
        res_v[0] = ri * ri;
        res_v[1] = rhs_i * rhs_i;
    }
    } while (false);
    if constexpr (RES) {
        // the block's partial sums; refine_start_kernel adds them up (no fence or ticket
        // here: every block of this latency-bound launch would hold its slot for them)
        block_sum<double, 2>(res_v);
        if (threadIdx.x == 0) {
            a.res.partials[blockIdx.x] = res_v[0];
            a.res.partials[gridDim.x + blockIdx.x] = res_v[1];
        }
    }
}

// One block after the assembly: (r.r, b.b) from the assembly blocks' partials in a
// fixed order, then the refinement loop's first decision.
__global__ void __launch_bounds__(1024) refine_start_kernel(RefineStart rs, int nb) {
    double v[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const double *pj = rs.partials + (int64_t)j * nb;
        double a0 = 0.0, a1 = 0.0;
        int b = threadIdx.x;
        for (; b + (int)blockDim.x < nb; b += 2 * (int)blockDim.x) {
            a0 += pj[b];
            a1 += pj[b + blockDim.x];
        }
        if (b < nb) a0 += pj[b];
        v[j] = a0 + a1;
    }
    block_sum<double, 2>(v);
    if (threadIdx.x == 0) ir_decide(v, rs.irs, nullptr, 1, rs.tol, rs.inner_floor, rs.maxit, rs.cond, rs.use_cond);
}

// Host-side quadrature constants from the reference rule.
void quadrature_constants(int dim, const double *Q, const double *W, int nq, double s[4], double m[4]) {
    const int nv = dim + 1;
    for (int j = 0; j < 4; ++j) s[j] = m[j] = 0.0;
    double mass[4][4] = {};
    for (int q = 0; q < nq; ++q) {
        double N[4];
        const double *p = Q + q * dim;
        if (dim == 2) { N[0] = 1 - p[0] - p[1]; N[1] = p[0]; N[2] = p[1]; }
        else { N[0] = 1.0 - p[0] - p[1] - p[2]; N[1] = p[0]; N[2] = p[1]; N[3] = p[2]; }
        for (int i = 0; i < nv; ++i) {
            s[i] += W[q] * N[i];
            for (int j = 0; j < nv; ++j) mass[i][j] += W[q] * (N[i] * N[j]);
        }
    }
    for (int i = 0; i < nv; ++i) {
        double r = 0.0;
        for (int j = 0; j < nv; ++j) r += mass[i][j];
        m[i] = r;
    }
}

template <int DIM, int MW, bool STAGE, int TB, int MINB, int SHP>
static void launch_rows(const RichardsAsmArgs &a, int ksm, int n_slices, bool res, cudaStream_t st) {
    constexpr bool CLS = SHP != 0;
    const int blocks = (n_slices * kSlice + TB - 1) / TB;
    const int cv = CLS ? 1 : DIM + 1;
    const size_t smem = (size_t)MW * TB * sizeof(double) * (STAGE ? 1 + cv : 1) +
                        (SHP == 1 ? (size_t)a.n_shapes * kShapeStride<DIM> * sizeof(double) : 0);
    auto run = [&](auto kfn) {
        if (smem > 48 * 1024) cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kfn<<<blocks, TB, smem, st>>>(a);
    };
    if (res) {
        if (ksm == 2) run(richards_rows_kernel<DIM, MW, 2, STAGE, TB, MINB, true, SHP>);
        else if (ksm == 1) run(richards_rows_kernel<DIM, MW, 1, STAGE, TB, MINB, true, SHP>);
        else run(richards_rows_kernel<DIM, MW, 0, STAGE, TB, MINB, true, SHP>);
    } else {
        if (ksm == 2) run(richards_rows_kernel<DIM, MW, 2, STAGE, TB, MINB, false, SHP>);
        else if (ksm == 1) run(richards_rows_kernel<DIM, MW, 1, STAGE, TB, MINB, false, SHP>);
        else run(richards_rows_kernel<DIM, MW, 0, STAGE, TB, MINB, false, SHP>);
    }
}

// Blocks of the assembly launch (the partial-sum slots a fused refinement start needs).
int richards_assembly_blocks(const wspm_mesh *mesh, const wspm_pattern *pat) {
    const int rows = pat->n_slices * kSlice;
    const int mw = pat->max_width;
    int tb;
    if (mesh->dim == 2) tb = mw <= 8 ? 256 : mw <= 16 ? 128 : mw <= 32 ? 64 : 32;
    else tb = (pat->n_diags > 0 && mw <= 16) ? 128 : mw <= 16 ? 128 : mw <= 32 ? 64 : 32;
    return (rows + tb - 1) / tb;
}

// ---- element shapes (plan time) -------------------------------------------------
// Distinct Jacobians by their bits, in an open-addressing table of kShapeSlots
// slots (state 0 free, 1 being written, 2 ready; keys are the Jacobian's bits).
// Every wait and probe sequence is bounded; a table that overflows, or a wait that
// gives up, sets the overflow word and the shape path is not used.
constexpr int kShapeSlots = 32768;     // > kMaxShapesGlobal, and slot ids fit the 16-bit element slots

__device__ __forceinline__ unsigned int shape_ld_acquire(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long shape_mix(unsigned long long h) {
    h ^= h >> 33; h *= 0xff51afd7ed558ccdULL; h ^= h >> 33; h *= 0xc4ceb9fe1a85ec53ULL; h ^= h >> 33;
    return h;
}

template <int DIM>
__global__ void shape_insert_kernel(wspm_mesh mesh, unsigned int *state, unsigned long long *keys,
                                    uint16_t *elem_slot, int *meta) {
    constexpr int NV = DIM + 1, NK = DIM * DIM;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < mesh.n_elems; e += gridDim.x * blockDim.x) {
        double X[NV][DIM];
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            const int v = mesh.conn[(int64_t)NV * e + j];
#pragma unroll
            for (int d = 0; d < DIM; ++d) X[j][d] = mesh.coords[(int64_t)DIM * v + d];
        }
        double J[DIM][DIM];
        p1_jacobian<DIM>(X, J);
        unsigned long long kb[NK], h = 0x9e3779b97f4a7c15ULL;
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int c = 0; c < DIM; ++c) {
                kb[r * DIM + c] = (unsigned long long)__double_as_longlong(J[r][c]);
                h = shape_mix(h ^ kb[r * DIM + c]);
            }
        int found = -1;
        for (int probe = 0; probe < kShapeSlots && found < 0; ++probe) {
            const int sl = (int)((h + (unsigned long long)probe) & (kShapeSlots - 1));
            unsigned int stv = shape_ld_acquire(state + sl);
            if (stv == 0u && atomicCAS(state + sl, 0u, 1u) == 0u) {
#pragma unroll
                for (int q = 0; q < NK; ++q) keys[(int64_t)sl * NK + q] = kb[q];
                __threadfence();
                atomicExch(state + sl, 2u);
                found = sl;
                break;
            }
            long long spins = 0;
            while ((stv = shape_ld_acquire(state + sl)) != 2u) {
                if (++spins > 4000000LL) { atomicExch(meta + 1, 1); return; }
                __nanosleep(32);
            }
            bool eq = true;
#pragma unroll
            for (int q = 0; q < NK; ++q) eq = eq && __ldcg(keys + (int64_t)sl * NK + q) == kb[q];
            if (eq) found = sl;
        }
        if (found < 0) { atomicExch(meta + 1, 1); return; }
        elem_slot[e] = (uint16_t)found;
    }
}

// One block: shape ids in slot order, and each shape's entry of the table.
template <int DIM>
__global__ void shape_table_kernel(const unsigned int *state, const unsigned long long *keys, int *slot_shape,
                                   int *meta, double *table, int max_shapes) {
    constexpr int NV = DIM + 1, NK = DIM * DIM;
    __shared__ int s_count;
    __shared__ int s_first[1024];
    // ids in ascending slot order: every thread counts the filled slots of its contiguous range, an exclusive
    // prefix over the threads (in thread order) gives each range its first id
    const int T = blockDim.x;
    const int per = (kShapeSlots + T - 1) / T;
    const int lo = min(kShapeSlots, (int)threadIdx.x * per), hi = min(kShapeSlots, lo + per);
    int mine = 0;
    for (int sl = lo; sl < hi; ++sl) mine += state[sl] == 2u ? 1 : 0;
    s_first[threadIdx.x] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        int c = 0;
        for (int t = 0; t < T; ++t) {
            const int m = s_first[t];
            s_first[t] = c;
            c += m;
        }
        meta[0] = c;
        if (c > max_shapes) meta[1] = 1;
        s_count = c;
    }
    __syncthreads();
    int next = s_first[threadIdx.x];
    for (int sl = lo; sl < hi; ++sl) slot_shape[sl] = state[sl] == 2u ? next++ : -1;
    __syncthreads();   // every slot's id written before the loop below reads other threads' slots
    if (s_count > max_shapes) return;
    for (int sl = threadIdx.x; sl < kShapeSlots; sl += blockDim.x) {
        const int id = slot_shape[sl];
        if (id < 0) continue;
        double J[DIM][DIM];
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int c = 0; c < DIM; ++c) J[r][c] = __longlong_as_double((long long)keys[(int64_t)sl * NK + r * DIM + c]);
        double G[DIM][NV], detJ;
        p1_geometry_j<DIM>(J, G, detJ);
        double *t = table + (int64_t)id * kShapeStride<DIM>;
        t[0] = detJ;
#pragma unroll
        for (int li = 0; li < NV; ++li) {
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                double gg = 0.0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) gg = fma(G[d][li], G[d][j], gg);
                t[1 + li * NV + j] = gg;
            }
            t[1 + NV * NV + li] = G[DIM - 1][li];
        }
    }
}

// Incidence words with the element's shape id above the position fields (mode
// 1: the 6-bit positions kept; mode 2: repacked into 4 bits each).
template <int DIM, int SHP>
__global__ void shape_words_kernel(int n_slices, const int64_t *__restrict__ inc_ptr,
                                   const int32_t *__restrict__ inc_width, const int32_t *__restrict__ inc_elem,
                                   const uint32_t *__restrict__ inc_slots, const uint16_t *__restrict__ elem_slot,
                                   const int *__restrict__ slot_shape, uint32_t *words) {
    constexpr int NV = DIM + 1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = i >> 5, lane = i & 31;
    if (s >= n_slices) return;
    const int64_t ib = inc_ptr[s] + lane;
    const int w = inc_width[s];
    for (int k = 0; k < w; ++k) {
        const int64_t o = ib + (int64_t)kSlice * k;
        const int e = inc_elem[o];
        const uint32_t src = inc_slots[o];
        uint32_t word = src;
        if constexpr (SHP == 2) {
            word = src & 3u;
#pragma unroll
            for (int j = 0; j < NV; ++j) word |= ((src >> (2 + 6 * j)) & 15u) << (2 + 4 * j);
        }
        if (e >= 0) word |= (uint32_t)slot_shape[elem_slot[e]] << kShapeShift<DIM, SHP>;
        words[o] = word;
    }
}

// Layout of the caller's shape buffer (bytes, 256-aligned parts): words
// [n_slices*32*max_inc] u32, element slots [n_elems] u16, slot states
// [kShapeSlots] u32, keys [kShapeSlots * dim^2] u64, slot shapes [kShapeSlots]
// i32, meta [64] i32, table [kMaxShapes * stride] f64.
struct ShapeBuffer {
    uint32_t *words; uint16_t *elem_slot; unsigned int *state; unsigned long long *keys; int *slot_shape;
    int *meta; double *table; int64_t bytes;
};
static int64_t align256(int64_t b) { return (b + 255) & ~int64_t(255); }
static ShapeBuffer carve_shapes(void *base, const wspm_mesh *mesh, const wspm_pattern *pat) {
    ShapeBuffer sb;
    char *p = (char *)base;
    int64_t off = 0;
    const int dim = mesh->dim;
    auto take = [&](int64_t bytes) { char *q = p ? p + off : nullptr; off += align256(bytes); return q; };
    sb.words = (uint32_t *)take((int64_t)pat->n_slices * kSlice * (pat->max_inc > 0 ? pat->max_inc : 1) * 4);
    sb.elem_slot = (uint16_t *)take((int64_t)mesh->n_elems * 2);
    sb.state = (unsigned int *)take((int64_t)kShapeSlots * 4);
    sb.keys = (unsigned long long *)take((int64_t)kShapeSlots * dim * dim * 8);
    sb.slot_shape = (int *)take((int64_t)kShapeSlots * 4);
    sb.meta = (int *)take(64 * 4);
    sb.table = (double *)take((int64_t)kMaxShapesGlobal * (dim == 2 ? kShapeStride<2> : kShapeStride<3>) * 8);
    sb.bytes = off;
    return sb;
}

int64_t richards_shape_bytes(const wspm_mesh *mesh, const wspm_pattern *pat) {
    if (!mesh || !pat || (mesh->dim != 2 && mesh->dim != 3)) return -1;
    return carve_shapes(nullptr, mesh, pat).bytes;
}

// Builds the shape words and table in `buf` (synchronous, plan creation).  Returns
// the number of shapes, or 0 when the mesh has too many (the caller then uses the
// geometry-computing kernel) or anything failed; *mode: 1 (table in shared memory)
// or 2 (global table, 4-bit row positions: 3D patterns of at most 16 entries per row).
int richards_build_shapes(const wspm_mesh *mesh, const wspm_pattern *pat, void *buf, const uint32_t **words,
                          const double **table, int *mode) {
    *mode = 0;
    if (!mesh || !pat || !buf || mesh->n_elems <= 0 || pat->n_slices <= 0 || !pat->inc_slots || !pat->inc_elem)
        return 0;
    if (mesh->dim != 2 && mesh->dim != 3) return 0;
    if (pat->max_width > 63) return 0;
    const ShapeBuffer sb = carve_shapes(buf, mesh, pat);
    if (cudaMemset(sb.state, 0, (size_t)kShapeSlots * 4) != cudaSuccess) return 0;
    if (cudaMemset(sb.meta, 0, 64 * 4) != cudaSuccess) return 0;
    const int blocks = (int)((mesh->n_elems + 255) / 256 < 148 * 8 ? (mesh->n_elems + 255) / 256 : 148 * 8);
    const int nsw = (pat->n_slices * kSlice + 255) / 256;
    if (mesh->dim == 2) {
        shape_insert_kernel<2><<<blocks, 256>>>(*mesh, sb.state, sb.keys, sb.elem_slot, sb.meta);
        shape_table_kernel<2><<<1, 256>>>(sb.state, sb.keys, sb.slot_shape, sb.meta, sb.table,
                                          pat->max_width <= 16 ? kMaxShapesGlobal : kMaxShapes<2>);
    } else {
        shape_insert_kernel<3><<<blocks, 256>>>(*mesh, sb.state, sb.keys, sb.elem_slot, sb.meta);
        shape_table_kernel<3><<<1, 256>>>(sb.state, sb.keys, sb.slot_shape, sb.meta, sb.table,
                                          pat->max_width <= 16 ? kMaxShapesGlobal : kMaxShapes<3>);
    }
    int meta[2] = {0, 1};
    if (cudaGetLastError() != cudaSuccess || cudaMemcpy(meta, sb.meta, sizeof(meta), cudaMemcpyDeviceToHost) != cudaSuccess)
        return 0;
    if (meta[1] != 0 || meta[0] <= 0) return 0;
    // The global table replaces a recomputation of cheap geometry with reads from L2: it is taken only when each
    // shape serves at least kShapeReuse elements on average (a structured grid), never for a mesh whose elements
    // are all distinct.  Every block copies the shared-memory table whole, so beyond kShapesShared shapes the
    // global table is the faster of the two (2D assembly at 1000^2, 162 shapes: 63.7 against 69.8 us; at 24
    // shapes the shared table wins, 59.8 against 63.7 us).
    const bool global_ok = pat->max_width <= 16 && meta[0] <= kMaxShapesGlobal &&
                           (int64_t)meta[0] * kShapeReuse <= (int64_t)mesh->n_elems;
    int md;
    if (global_ok && meta[0] > kShapesShared) md = 2;
    else if (meta[0] <= (mesh->dim == 2 ? kMaxShapes<2> : kMaxShapes<3>)) md = 1;
    else if (global_ok) md = 2;
    else return 0;
    if (mesh->dim == 2 && md == 1)
        shape_words_kernel<2, 1><<<nsw, 256>>>(pat->n_slices, pat->inc_ptr, pat->inc_width, pat->inc_elem,
                                               pat->inc_slots, sb.elem_slot, sb.slot_shape, sb.words);
    else if (mesh->dim == 2)
        shape_words_kernel<2, 2><<<nsw, 256>>>(pat->n_slices, pat->inc_ptr, pat->inc_width, pat->inc_elem,
                                               pat->inc_slots, sb.elem_slot, sb.slot_shape, sb.words);
    else if (md == 1)
        shape_words_kernel<3, 1><<<nsw, 256>>>(pat->n_slices, pat->inc_ptr, pat->inc_width, pat->inc_elem,
                                               pat->inc_slots, sb.elem_slot, sb.slot_shape, sb.words);
    else
        shape_words_kernel<3, 2><<<nsw, 256>>>(pat->n_slices, pat->inc_ptr, pat->inc_width, pat->inc_elem,
                                               pat->inc_slots, sb.elem_slot, sb.slot_shape, sb.words);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return 0;
    *words = sb.words;
    *table = sb.table;
    *mode = md;
    return meta[0];
}

static int launch_richards_assembly_impl(const wspm_mesh *mesh, const wspm_pattern *pat,
                                         const double *theta_m, const double *theta_n, const double *h_m,
                                         const double *K, const double *C, const double *Ks_elem,
                                         const double *Ks_inc, const double s[4], const double mc[4], double dt,
                                         const double *dt_dev, const double *bc_val, double *vals, float *vals32,
                                         double *rhs, double *dinv, const RefineStart *res, const uint32_t *shape_words,
                                         const double *shape_tab, int n_shapes, int shape_mode, cudaStream_t st) {
    RichardsAsmArgs a;
    const bool fused = res != nullptr;
    if (fused) a.res = *res;
    a.n_rows = pat->n_rows;
    a.slice_ptr = pat->slice_ptr; a.slice_width = pat->slice_width; a.diag_pos = pat->diag_pos;
    a.inc_ptr = pat->inc_ptr; a.inc_width = pat->inc_width; a.inc_elem = pat->inc_elem; a.inc_slots = pat->inc_slots;
    a.conn = mesh->conn; a.coords = mesh->coords;
    a.theta_m = theta_m; a.theta_n = theta_n; a.h_m = h_m; a.K = K; a.C = C; a.Ks_elem = Ks_elem; a.bc_val = bc_val;
    a.Ks_inc = Ks_inc;
    for (int j = 0; j < 4; ++j) { a.s[j] = s[j]; a.mcoef[j] = mc[j]; }
    a.inv_dt = 1.0 / dt;
    a.dt_dev = dt_dev;
    a.n_diags = pat->n_diags;
    a.ld = (int64_t)pat->n_slices * kSlice;
    a.vals = vals; a.vals32 = vals32; a.rhs = rhs; a.dinv = dinv;
    a.diag_off = pat->diag_offsets;
    a.cols = pat->cols;
    a.shape_tab = nullptr;
    a.n_shapes = 0;
    if (pat->max_width > 63) return WSPM_UNSUPPORTED;      // the incidence word holds 6-bit row positions
    const int ksm = Ks_inc ? 2 : (Ks_elem ? 1 : 0);
    const int ns = pat->n_slices;
    const int mw = pat->max_width;
    // the shape path where the plan found few element shapes (its words carry the shape ids)
    const int shp = (shape_words && shape_tab && n_shapes > 0 && mw <= 16) ? shape_mode : 0;
    const bool cls = shp != 0;
    if (cls) {
        a.inc_slots = shape_words;
        a.shape_tab = shape_tab;
        a.n_shapes = n_shapes;
    }
    // launch shapes measured on the 1024^2 triangle and 96^3 Kuhn-tetrahedron grids (B200)
    if (mesh->dim == 2) {
        if (mw <= 8) {
            if (shp == 1) launch_rows<2, 8, true, 256, 5, 1>(a, ksm, ns, fused, st);
            else if (shp == 2) launch_rows<2, 8, true, 256, 4, 2>(a, ksm, ns, fused, st);
            else launch_rows<2, 8, true, 256, 3, 0>(a, ksm, ns, fused, st);
        } else if (mw <= 16) {
            if (shp == 1) launch_rows<2, 16, true, 128, 2, 1>(a, ksm, ns, fused, st);
            else if (shp == 2) launch_rows<2, 16, true, 128, 2, 2>(a, ksm, ns, fused, st);
            else launch_rows<2, 16, true, 128, 1, 0>(a, ksm, ns, fused, st);
        } else if (mw <= 32) launch_rows<2, 32, true, 64, 1, 0>(a, ksm, ns, fused, st);
        else launch_rows<2, 64, true, 32, 1, 0>(a, ksm, ns, fused, st);
    } else {
        if (pat->n_diags > 0 && mw <= 16) {
            if (shp == 1) launch_rows<3, 16, false, 128, 8, 1>(a, ksm, ns, fused, st);
            else if (shp == 2) launch_rows<3, 16, false, 128, 10, 2>(a, ksm, ns, fused, st);
            else launch_rows<3, 16, false, 128, 8, 0>(a, ksm, ns, fused, st);
        } else if (mw <= 8) {
            if (shp == 1) launch_rows<3, 8, true, 128, 2, 1>(a, ksm, ns, fused, st);
            else if (shp == 2) launch_rows<3, 8, true, 128, 2, 2>(a, ksm, ns, fused, st);
            else launch_rows<3, 8, true, 128, 1, 0>(a, ksm, ns, fused, st);
        } else if (mw <= 16) {
            if (shp == 1) launch_rows<3, 16, true, 128, 2, 1>(a, ksm, ns, fused, st);
            else if (shp == 2) launch_rows<3, 16, true, 128, 2, 2>(a, ksm, ns, fused, st);
            else launch_rows<3, 16, true, 128, 1, 0>(a, ksm, ns, fused, st);
        } else if (mw <= 32) launch_rows<3, 32, true, 64, 1, 0>(a, ksm, ns, fused, st);
        else launch_rows<3, 64, true, 32, 1, 0>(a, ksm, ns, fused, st);
    }
    if (fused) refine_start_kernel<<<1, 1024, 0, st>>>(*res, richards_assembly_blocks(mesh, pat));
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

int launch_richards_assembly(const wspm_mesh *mesh, const wspm_pattern *pat, const double *theta_m,
                             const double *theta_n, const double *h_m, const double *K, const double *C,
                             const double *Ks_elem, const double s[4], const double mc[4], double dt,
                             const double *bc_val, double *vals, float *vals32, double *rhs, double *dinv,
                             cudaStream_t st) {
    return launch_richards_assembly_impl(mesh, pat, theta_m, theta_n, h_m, K, C, Ks_elem, nullptr, s, mc, dt,
                                         nullptr, bc_val, vals, vals32, rhs, dinv, nullptr, nullptr, nullptr, 0, 0, st);
}

int launch_richards_assembly_dev_dt(const wspm_mesh *mesh, const wspm_pattern *pat, const double *theta_m,
                                    const double *theta_n, const double *h_m, const double *K, const double *C,
                                    const double *Ks_elem, const double *Ks_inc, const double s[4],
                                    const double mc[4], const double *dt_dev, const double *bc_val, double *vals,
                                    float *vals32, double *rhs, double *dinv, const RefineStart *res,
                                    const uint32_t *shape_words, const double *shape_tab, int n_shapes,
                                    int shape_mode, cudaStream_t st) {
    return launch_richards_assembly_impl(mesh, pat, theta_m, theta_n, h_m, K, C, Ks_elem, Ks_inc, s, mc, 1.0,
                                         dt_dev, bc_val, vals, vals32, rhs, dinv, res, shape_words, shape_tab,
                                         n_shapes, shape_mode, st);
}

int launch_incidence_gather(const wspm_pattern *pat, const double *elem, double *out, cudaStream_t st) {
    const int ns = pat->n_slices;
    incidence_gather_kernel<<<(ns * kSlice + 255) / 256, 256, 0, st>>>(ns, pat->inc_ptr, pat->inc_width,
                                                                      pat->inc_elem, elem, out);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

int launch_soil(const SoilParams &sp, const double *h, int64_t n, double *C, double *K, double *theta,
                cudaStream_t st) {
    if (n <= 0) return WSPM_OK;
    int64_t b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    soil_kernel<<<(int)b, 256, 0, st>>>(sp, h, n, C, K, theta);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}

}  // namespace wspm
