// Measurement hook: streaming-read bandwidth of a device buffer
// (wspm_read_probe, declared in include/wspm.h).
//
// The resident CG kernels keep their vectors in shared memory and read the
// matrix (29.4 MB in FP32, 58.8 MB in FP64 at 1024^2) from L2 every
// iteration, so the roof that bounds them is the L2 read bandwidth, not HBM.
// This kernel measures that roof the way the CG kernels consume it: each
// block streams its own contiguous share of the buffer with 16-byte loads
// that bypass L1 (ld.global.cg), `reps` times, several loads in flight per
// thread.  For a buffer that fits in L2 the repeated passes are L2 hits; for a
// buffer much larger than L2 they measure HBM.  Timing is the caller's (CUDA
// events around two launches with different `reps`).
#include "common.cuh"

namespace wspm {

constexpr int kProbeBlock = 1024;
constexpr int kProbeUnroll = 4;

__global__ void __launch_bounds__(kProbeBlock, 2) read_probe_kernel(const float4 *__restrict__ buf, int64_t n16,
                                                                 int reps, float *out) {
    // block b owns words [b*chunk, min(n16, (b+1)*chunk))
    const int64_t chunk = (n16 + gridDim.x - 1) / gridDim.x;
    const int64_t lo = blockIdx.x * chunk;
    const int64_t hi = min(n16, lo + chunk);
    float acc = 0.f;
    for (int r = 0; r < reps; ++r) {
        int64_t i = lo + threadIdx.x;
        for (; i + (kProbeUnroll - 1) * (int64_t)kProbeBlock < hi; i += kProbeUnroll * (int64_t)kProbeBlock) {
            float4 v[kProbeUnroll];
#pragma unroll
            for (int u = 0; u < kProbeUnroll; ++u) v[u] = __ldcg(buf + i + u * (int64_t)kProbeBlock);
#pragma unroll
            for (int u = 0; u < kProbeUnroll; ++u) acc += (v[u].x + v[u].y) + (v[u].z + v[u].w);
        }
        for (; i < hi; i += kProbeBlock) {
            const float4 v = __ldcg(buf + i);
            acc += (v.x + v.y) + (v.z + v.w);
        }
    }
    float v1[1] = {acc};
    block_sum<float, 1>(v1);
    if (threadIdx.x == 0) atomicAdd(out, v1[0]);
}

}  // namespace wspm

using namespace wspm;

extern "C" int wspm_read_probe(const void *buf, int64_t n16, int32_t reps, int32_t blocks_per_sm, float *out,
                               void *stream) {
    if (!buf || !out || n16 <= 0 || reps < 0 || blocks_per_sm < 1 || blocks_per_sm > 2) return WSPM_BAD_ARG;
    if ((uintptr_t)buf % 16) return WSPM_BAD_ARG;
    int dev = 0, sms = 0;
    WSPM_CUDA_TRY(cudaGetDevice(&dev));
    WSPM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    read_probe_kernel<<<sms * blocks_per_sm, kProbeBlock, 0, (cudaStream_t)stream>>>((const float4 *)buf, n16, reps,
                                                                                      out);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}
