// Host side of the wavefront engine shared by wrk_renderer (one request per
// render) and wrk_server (up to kMaxSlots requests in flight): the SoA path
// queues, the device tables the kernels read (requests, slot progress, scenes,
// admission order, generation segments), pinned mirrors for readback, and the
// CUDA graph of one chunk of bounce iterations.
#pragma once
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "wrk_internal.h"

namespace wrk {

struct EngineBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~EngineBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) {
        if (p && n <= bytes) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, n ? n : 16);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// Launch shape of the bounce loop (chosen by the autotuner or by the caller).
struct LaunchConfig {
    uint32_t chunk = 8;         // iterations per graph launch / host check
    uint32_t shadeBlock = 256;  // 128 or 256 threads per shade block
    uint32_t shadeBlocksPerSM = 4;  // in units of 256-thread blocks
};

struct Engine {
    int device = 0;
    uint32_t capacity = 0;
    int numSMs = 148;
    cudaStream_t stream = nullptr;
    // Inside a captured chunk the shadow trace of an iteration runs on `side`,
    // concurrently with that iteration's camera-ray generation and extension trace
    // (they touch disjoint queues), so each persistent kernel's tail is filled by
    // the other; the shade kernels wait for both.
    cudaStream_t side = nullptr;
    cudaEvent_t forkEv = nullptr, joinEv = nullptr;
    // likewise the glass, GGX and emissive shade kernels run on `side2`, concurrently
    // with the Lambert shade (each reads its own bucket; their appends are atomic)
    cudaStream_t side2 = nullptr;
    cudaEvent_t bucketsEv = nullptr, join2Ev = nullptr;
    EngineBuf queues, counters, tables;
    Queues q{};
    Frame* dReq = nullptr;
    SlotCtl* dCtl = nullptr;
    DevScene* dScenes = nullptr;
    uint32_t* dGenOrder = nullptr;
    GenSeg* dSeg = nullptr;
    // pinned host mirrors
    Counters* hCtr = nullptr;
    SlotCtl* hCtl = nullptr;
    Frame* hReq = nullptr;
    uint32_t* hGenOrder = nullptr;
    DevScene* hScenes = nullptr;
    LaunchConfig cfg;
    // one chunk of iterations captured as a CUDA graph (re-captured when the
    // scene parameter, the multi-scene mode or the launch shape changes)
    cudaGraphExec_t graph = nullptr;
    DevScene graphScene{};
    bool graphMulti = false;
    LaunchConfig graphCfg;
    std::vector<cudaEvent_t> stageEv;
    // device-driven loop: one graph launch repeats chunks (a conditional WHILE node)
    // until every request in the admission order finished
    cudaGraphExec_t loopGraph = nullptr;
    DevScene loopScene{};
    bool loopMulti = false;
    bool loopUnsupported = false;
    LaunchConfig loopCfg;

    ~Engine();
    // Allocates queues (capacity path entries) and tables; returns a cudaError_t.
    cudaError_t init(int dev, uint32_t cap);
    // Zeroes the queue counters (start of a render / of a server's life).
    cudaError_t reset_counters();
    // Enqueues cfg.chunk iterations (graph, or plain launches with per-stage events
    // when `timing` is set), then the readback of counters and slot progress.
    cudaError_t enqueue_chunk(const DevScene& s0, bool multi, bool timing);
    // Enqueues the device-driven loop (chunks until done or `iterLimit` iterations),
    // then the readback.  Returns cudaErrorNotSupported when conditional graph nodes
    // are unavailable (the caller then steps chunk by chunk from the host).
    cudaError_t enqueue_until_done(const DevScene& s0, bool multi, uint32_t iterLimit);
    // Adds the per-stage times of the last timed chunk.
    cudaError_t stage_times(float* ms, uint32_t* launches);
    int shade_grid() const { return numSMs * (int)cfg.shadeBlocksPerSM; }
};

}  // namespace wrk
