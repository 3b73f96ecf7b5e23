// Allocation-free Jacobi-CG solve: wspm_cg_solve_noalloc (declared in include/wspm.h).
//
// Who needs it: callers that cannot call cudaMalloc.  The reference's own
// runtime is the typical case: JAX/XLA pre-allocates most of the GPU's memory
// for its pool when it starts, so a custom call or a host callback running
// inside a JAX program may find no free device memory to allocate a solver
// workspace from, and must not grab memory behind the pool's back.  Other
// callers run where allocation is forbidden or too slow: inside a stream
// capture (cudaMalloc is not allowed there), or in a time-stepping loop with a
// fixed memory budget.  Such callers pass only their inputs and outputs; the
// Krylov vectors, reduction partials and solver state live in the static
// device array below instead of a caller-supplied workspace.
//
// Limits and sharing:
//  * the scratch holds the CG workspace for at most WSPM_NOALLOC_MAX_ROWS rows
//    (about 11 MB of device memory, held by every GPU that loads the library
//    until the process exits); larger systems are rejected with WSPM_BAD_ARG
//    before anything is launched;
//  * every call on a device uses the same array and leaves its contents
//    behind: the solver state is cleared at the start of every call, and two
//    calls that overlap on the GPU (different streams, or different host
//    threads on one device) race on the scratch and corrupt each other;
//  * the first call on each device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current) and caches it; make that
//    first call before any stream capture.
// The solve is one launch of the same resident (cooperative) CG kernel that
// wspm_krylov_solve runs for WSPM_SOLVER_CG, so it takes the same iterations
// and returns the same iterate bit for bit; the iteration loop runs inside
// the kernel, so the number of launches does not grow with maxiter.  It never
// synchronises with the host and calls no allocating CUDA routine.
#include <mutex>
#include "krylov.cuh"
#include "graph.cuh"

namespace wspm {

constexpr int kNoallocMaxRows = WSPM_NOALLOC_MAX_ROWS;
constexpr int64_t kNoallocScratchDoubles =
    5 * (int64_t)((kNoallocMaxRows + 31) & ~31) + ((4 * kMaxPartials + 31) & ~31) + 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoallocScratchDoubles];

constexpr int kMaxDevices = 64;
static double *g_noalloc_ptr[kMaxDevices] = {};
static std::mutex g_noalloc_mu;

// Device address of the scratch array on the current device (set-up once per device).
static int noalloc_scratch(double **out) {
    int dev = 0;
    WSPM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return WSPM_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        double *p = nullptr;
        // host code must not use g_noalloc_scratch directly: it names a host-side shadow, not device memory
        WSPM_CUDA_TRY(cudaGetSymbolAddress((void **)&p, g_noalloc_scratch));
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return WSPM_OK;
}

// Result words of the solve.  The CG kernel sets `done` when it leaves its
// loop; a state that is not done (the kernel did not run to its end) is
// reported as an error, never as success.
__global__ void noalloc_result_kernel(const KrylovState *st, int32_t *result) {
    if (threadIdx.x == 0) {
        result[0] = st->done ? st->status : WSPM_CUDA_ERROR;
        result[1] = st->k;
        result[2] = 0;
        result[3] = 0;
    }
}

}  // namespace wspm

using namespace wspm;

extern "C" int wspm_cg_solve_noalloc(const wspm_pattern *pat, const double *vals, const double *b, double *x,
                                     const double *dinv, double tol, double atol, int32_t maxiter, int32_t *result,
                                     void *stream) {
    // size first: a system beyond the scratch is refused whatever the other arguments are
    if (!pat || pat->n_rows <= 0 || pat->n_rows > kNoallocMaxRows) return WSPM_BAD_ARG;
    if (!pattern_layout_ok(pat)) return WSPM_BAD_ARG;
    if (!vals || !b || !x || !result || maxiter < 0 || !(tol >= 0.0) || !(atol >= 0.0)) return WSPM_BAD_ARG;
    if (cg_workspace_doubles(pat->n_rows, 8) > kNoallocScratchDoubles) return WSPM_BAD_ARG;
    double *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc != WSPM_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const Sell A = make_sell(pat);
    int64_t used = 0;
    CgBuffers<double> w = carve_cg<double>(scratch, pat->n_rows, &used);
    // the previous call's state and barrier words are still in the scratch: clear them
    state_reset_kernel<<<1, 32, 0, st>>>((unsigned int *)w.st, (int)(sizeof(KrylovState) / 4));
    rc = cg_persistent_enqueue<double>(A, vals, b, nullptr, x, dinv, w, tol, atol, maxiter, false, nullptr, st);
    if (rc != WSPM_OK) return rc;      // WSPM_BAD_ARG: an array not on a 16-byte boundary
    noalloc_result_kernel<<<1, 32, 0, st>>>(w.st, result);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}
