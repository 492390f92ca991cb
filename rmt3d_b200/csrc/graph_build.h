// Building a step as one CUDA graph by stream capture, with conditional
// nodes for the data-dependent control: WHILE loops for the multigrid cycle
// counts and IF nodes for the branches of a step (skip after an error, revert
// the reference map).  A conditional node is added to the graph that the
// current stream is capturing into; its body is then captured from a second
// stream (cudaStreamBeginCaptureToGraph), one stream per nesting level.
//
// Every conditional handle is created with default value 0 and armed by a
// kernel right before its node: a body that is never armed never runs.
#pragma once
#include <cuda_runtime.h>

#include <string>

namespace rmt3d {

struct graph_builder {
    static constexpr int kDepth = 4;
    cudaStream_t st[kDepth] = {nullptr, nullptr, nullptr, nullptr};
    int depth = 0;       // bodies currently open
    cudaError_t err = cudaSuccess;

    int init() {
        for (int i = 0; i < kDepth; i++)
            if (!st[i] && cudaStreamCreateWithFlags(&st[i], cudaStreamNonBlocking) != cudaSuccess) return 1;
        return 0;
    }
    void release() {
        for (int i = 0; i < kDepth; i++)
            if (st[i]) cudaStreamDestroy(st[i]);
        for (int i = 0; i < kDepth; i++) st[i] = nullptr;
    }
    void note(cudaError_t e) {
        if (e != cudaSuccess && err == cudaSuccess) err = e;
    }

    // a new handle (default 0) in the graph `cur` is capturing into
    cudaGraphConditionalHandle handle(cudaStream_t cur) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        cudaGraphConditionalHandle h = 0;
        note(cudaStreamGetCaptureInfo(cur, &cs, nullptr, &g, nullptr, nullptr));
        if (err == cudaSuccess) note(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
        return h;
    }

    // Append a conditional node at the capture point of `cur` and start
    // capturing its body; returns the stream to launch the body's work on
    // (nullptr after an error).
    cudaStream_t open(cudaStream_t cur, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type) {
        if (err != cudaSuccess || depth >= kDepth) {
            if (depth >= kDepth) note(cudaErrorNotSupported);
            return nullptr;
        }
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        note(cudaStreamGetCaptureInfo(cur, &cs, nullptr, &g, &deps, &nd));
        if (err != cudaSuccess) return nullptr;
        cudaGraphNodeParams p = {};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = type;
        p.conditional.size = 1;
        cudaGraphNode_t node;
        note(cudaGraphAddNode(&node, g, deps, nd, &p));
        if (err != cudaSuccess) return nullptr;
        note(cudaStreamUpdateCaptureDependencies(cur, &node, 1, cudaStreamSetCaptureDependencies));
        cudaStream_t b = st[depth];
        note(cudaStreamBeginCaptureToGraph(b, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal));
        if (err != cudaSuccess) return nullptr;
        depth++;
        return b;
    }

    void close(cudaStream_t body) {
        if (!body) return;
        cudaGraph_t out = nullptr;
        note(cudaStreamEndCapture(body, &out));
        depth--;
    }
};

}  // namespace rmt3d
