// CUDA-graph helpers: device-side WHILE loops built by stream capture.
//
// A loop is: (kernels that set the handle) -> WHILE(handle){ body }.  The
// body is captured into the conditional node's body graph on a private
// stream; bodies may themselves contain loops (nested conditional nodes).
// Every loop body ends with a kernel that clears the handle when its
// iteration counter reaches the caller's cap, so each loop is bounded.
#pragma once
#include "common.cuh"

namespace wspm {

__global__ void state_reset_kernel(unsigned int *words, int n_words);

inline cudaError_t make_cond_handle(cudaStream_t st, cudaGraphConditionalHandle *h) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, nullptr, nullptr);
    if (e != cudaSuccess) return e;
    if (cs != cudaStreamCaptureStatusActive) return cudaErrorIllegalState;
    return cudaGraphConditionalHandleCreate(h, g, 0, 0);
}

template <typename Body>
cudaError_t capture_while(cudaStream_t st, cudaGraphConditionalHandle h, Body body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd);
    if (e != cudaSuccess) return e;
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g, deps, nd, &p);
    if (e != cudaSuccess) return e;
    e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess) return e;
    cudaGraph_t bodyg = p.conditional.phGraph_out[0];
    cudaStream_t bs;
    e = cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    e = cudaStreamBeginCaptureToGraph(bs, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e == cudaSuccess) {
        body(bs);
        cudaGraph_t out = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(bs, &out);
        if (e == cudaSuccess) e = e2;
    }
    cudaStreamDestroy(bs);
    return e;
}

}  // namespace wspm
