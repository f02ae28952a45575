// C ABI of libwrk (include/wrk.h): scene upload and BVH build, the renderer's
// host loop, and the kernel-level entry points.  Errors are returned as codes with
// a per-thread message (wrk_last_error); no exception crosses the boundary.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"
#include "wrk_internal.h"

namespace wrk {
int compact_stable(const uint32_t* stage, const uint32_t* idx, uint32_t n, uint32_t* out, uint32_t* count,
                   cudaStream_t st);
void launch_cdf(const float* cdf, uint32_t ncdf, const float* u, uint32_t n, uint32_t* out, cudaStream_t st);
void launch_rng(const uint32_t* s, const uint32_t* d, uint32_t n, uint32_t* h, float* u, cudaStream_t st);
void launch_bsdf(const float* in, uint32_t n, float* out, cudaStream_t st);
void launch_texture(const uint8_t* texels, uint32_t w, uint32_t h, const float* uv, uint32_t n, float* out,
                    cudaStream_t st);
void launch_camera_rays(const Frame& f, const uint32_t* px, const uint32_t* sm, uint32_t n, float* out,
                        cudaStream_t st);
void launch_tonemap(const float* rgb, uint32_t nfloat, uint8_t* out, int grid, int vec, cudaStream_t st);
}  // namespace wrk

using namespace wrk;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(x)                                                                                          \
    do {                                                                                               \
        cudaError_t e_ = (x);                                                                          \
        if (e_ != cudaSuccess) return fail(WRK_ERR_CUDA, "%s: %s (%s:%d)", #x, cudaGetErrorString(e_), \
                                           __FILE__, __LINE__);                                        \
    } while (0)

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~DevBuf() { if (p) cudaFree(p); }
    int alloc(size_t n) {
        if (n <= bytes && p) return WRK_OK;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (n == 0) return WRK_OK;
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) return fail(WRK_ERR_CUDA, "cudaMalloc(%zu): %s", n, cudaGetErrorString(e));
        bytes = n;
        return WRK_OK;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

int set_device(int dev) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(WRK_ERR_NO_DEVICE, "no CUDA device available");
    if (dev < 0 || dev >= n) return fail(WRK_ERR_INVALID, "device %d out of range (%d devices)", dev, n);
    CK(cudaSetDevice(dev));
    return WRK_OK;
}

// Camera basis exactly as libWR computes it on the host: wr::Camera's GLM helpers
// (libWR/include/wr/types.h:41-50; normalize = v * (1/sqrt(dot))) and
// tan(fovY/2) (libWR/src/internal/renderer.cpp:144-156).
void camera_frame(const wrk_camera& c, Frame& f) {
    auto nrm = [](float v[3]) {
        float r = 1.0f / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        v[0] = v[0] * r;
        v[1] = v[1] * r;
        v[2] = v[2] * r;
    };
    auto crs = [](const float a[3], const float b[3], float o[3]) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    for (int k = 0; k < 3; ++k) {
        f.pos[k] = c.position[k];
        f.fwd[k] = c.target[k] - c.position[k];
    }
    nrm(f.fwd);
    crs(f.fwd, c.up, f.right);
    nrm(f.right);
    crs(f.right, f.fwd, f.up);
    nrm(f.up);
    f.tanHalf = std::tan(c.fovY * 0.5f);
    f.aspect = c.aspect;
    f.focal = c.focalDistance;
    f.lens = c.lensRadius;
}

}  // namespace

namespace wrk {
// Records a failure for wrk_last_error() from entry points defined in other files.
int report_error(int code, const char* msg) { return fail(code, "%s", msg); }
}  // namespace wrk

struct wrk_scene {
    int device = 0;
    std::vector<float> vtx, nrm, uv;
    std::vector<uint32_t> idx, triMat;
    std::vector<wrk_material> mats;
    std::vector<std::vector<uint8_t>> tex;
    std::vector<uint32_t> texW, texH;
    float env[3] = {0, 0, 0};
    std::vector<float> envMap;
    uint32_t envW = 0, envH = 0;
    bool finalized = false;
    DevBuf dEnvMap;
    DevBuf dVtx, dNrm, dUv, dIdx, dTriMat, dMats, dTexels, dTexInfo, dEmissive, dCdf, dLights, dErr;
    uint4* nodes = nullptr;
    float4* tris = nullptr;
    std::vector<uint32_t> emissive;
    std::vector<float> cdf;
    wrk_bvh_info info{};
    DevScene view{};
    ~wrk_scene() {
        cudaFree(nodes);
        cudaFree(tris);
    }
};

namespace wrk {
// Accessors other translation units use (the scene's layout stays private here).
const DevScene* scene_view(const wrk_scene* s) { return s && s->finalized ? &s->view : nullptr; }
int scene_device(const wrk_scene* s) { return s ? s->device : -1; }
}  // namespace wrk

struct wrk_renderer {
    Engine eng;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evLoop0 = nullptr, evLoop1 = nullptr;
    DevBuf frameBufs, outBufs;
    ~wrk_renderer() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (evLoop0) cudaEventDestroy(evLoop0);
        if (evLoop1) cudaEventDestroy(evLoop1);
    }
};

// ---------------------------------------------------------------------------
// Engine
namespace wrk {

Engine::~Engine() {
    if (stream) cudaStreamSynchronize(stream);
    if (graph) cudaGraphExecDestroy(graph);
    if (loopGraph) cudaGraphExecDestroy(loopGraph);
    for (cudaEvent_t e : stageEv) cudaEventDestroy(e);
    if (hCtr) cudaFreeHost(hCtr);
    if (hCtl) cudaFreeHost(hCtl);
    if (hReq) cudaFreeHost(hReq);
    if (hGenOrder) cudaFreeHost(hGenOrder);
    if (hScenes) cudaFreeHost(hScenes);
    if (side) cudaStreamSynchronize(side);
    if (side2) cudaStreamSynchronize(side2);
    for (cudaEvent_t e : {forkEv, joinEv, bucketsEv, join2Ev})
        if (e) cudaEventDestroy(e);
    if (side) cudaStreamDestroy(side);
    if (side2) cudaStreamDestroy(side2);
    if (stream) cudaStreamDestroy(stream);
}

cudaError_t Engine::init(int dev, uint32_t cap) {
    device = dev;
    cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, dev);
    capacity = std::max(cap ? cap : (1u << 22), 1024u);
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)) != cudaSuccess) return e;
#ifndef WRK_NO_SHADOW_OVERLAP
    if ((e = cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&side2, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&forkEv, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&joinEv, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&bucketsEv, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&join2Ev, cudaEventDisableTiming)) != cudaSuccess)
        return e;
#endif
    if ((e = cudaMallocHost(&hCtr, sizeof(Counters))) != cudaSuccess ||
        (e = cudaMallocHost(&hCtl, sizeof(SlotCtl) * kMaxSlots)) != cudaSuccess ||
        (e = cudaMallocHost(&hReq, sizeof(Frame) * kMaxSlots)) != cudaSuccess ||
        (e = cudaMallocHost(&hGenOrder, sizeof(uint32_t) * (kMaxSlots + 4))) != cudaSuccess ||
        (e = cudaMallocHost(&hScenes, sizeof(DevScene) * kMaxScenes)) != cudaSuccess)
        return e;
    memset(hCtl, 0, sizeof(SlotCtl) * kMaxSlots);
    memset(hGenOrder, 0, sizeof(uint32_t) * (kMaxSlots + 4));
    // SoA path queues: extension x2 (5 fields), shadow x2 (4 fields), the four
    // material buckets the extension trace fills (6 fields)
    size_t C = capacity;
    const size_t fields = 2 * 5 + 2 * 4 + kBucketLambertResume * 6;
    if ((e = queues.alloc(C * fields * sizeof(float4))) != cudaSuccess) return e;
    float4* next = queues.as<float4>();
    auto take = [&]() {
        float4* p = next;
        next += C;
        return p;
    };
    for (int k = 0; k < 2; ++k) {
        PathQ& x = q.ext[k];
        x = PathQ{};
        x.ray_o = take();
        x.ray_d = take();
        x.thr = take();
        x.rad = take();
        x.st = reinterpret_cast<uint4*>(take());
        PathQ& h = q.shd[k];
        h = PathQ{};
        h.rad = take();
        h.sh_o = take();
        h.sh_d = take();
        h.sh_c = take();
    }
    q.bucket[kBucketLambertResume] = PathQ{};
    for (int b = 0; b < (int)kBucketLambertResume; ++b) {
        PathQ& x = q.bucket[b];
        x = PathQ{};
        x.ray_o = take();
        x.ray_d = take();
        x.hit = take();
        x.thr = take();
        x.rad = take();
        x.st = reinterpret_cast<uint4*>(take());
    }
    if ((e = counters.alloc(sizeof(Counters))) != cudaSuccess) return e;
    // tables: requests | slot progress | scenes | admission order | generation segments
    auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t oReq = 0, oCtl = oReq + up(sizeof(Frame) * kMaxSlots), oSc = oCtl + up(sizeof(SlotCtl) * kMaxSlots),
                 oGo = oSc + up(sizeof(DevScene) * kMaxScenes), oSeg = oGo + up(sizeof(uint32_t) * (kMaxSlots + 4)),
                 total = oSeg + up(sizeof(GenSeg) * kMaxSlots);
    if ((e = tables.alloc(total)) != cudaSuccess) return e;
    if ((e = cudaMemset(tables.p, 0, total)) != cudaSuccess) return e;
    uint8_t* t = tables.as<uint8_t>();
    dReq = reinterpret_cast<Frame*>(t + oReq);
    dCtl = reinterpret_cast<SlotCtl*>(t + oCtl);
    dScenes = reinterpret_cast<DevScene*>(t + oSc);
    dGenOrder = reinterpret_cast<uint32_t*>(t + oGo);
    dSeg = reinterpret_cast<GenSeg*>(t + oSeg);
    q.ctr = counters.as<Counters>();
    q.capacity = capacity;
    q.req = dReq;
    q.ctl = dCtl;
    q.scenes = dScenes;
    q.genOrder = dGenOrder;
    q.seg = dSeg;
    return reset_counters();
}

cudaError_t Engine::reset_counters() {
    cudaError_t e = cudaMemsetAsync(q.ctr, 0, sizeof(Counters), stream);
    if (e != cudaSuccess) return e;
    hGenOrder[kMaxSlots + 3] = 1;  // staging word for Counters::cur (the control kernel swaps first)
    return cudaMemcpyAsync(&q.ctr->cur, &hGenOrder[kMaxSlots + 3], sizeof(uint32_t), cudaMemcpyHostToDevice, stream);
}

static void launch_iteration(const Engine& E, const DevScene& s0, bool multi, cudaStream_t st, cudaEvent_t* ev) {
    if (!ev && E.side) {
        // captured chunk: the shadow trace (it reads this iteration's shadow queue and
        // updates the continuations the last iteration left in the other extension
        // buffer) overlaps generation and the extension trace (this iteration's
        // extension buffer and the material buckets); the shade kernels wait for both
        launch_control(E.q, st);
        cudaEventRecord(E.forkEv, st);
        cudaStreamWaitEvent(E.side, E.forkEv, 0);
        launch_trace_shadow(s0, E.q, multi, E.numSMs, E.side);
        cudaEventRecord(E.joinEv, E.side);
        launch_generate(E.q, E.numSMs * 8, st);
        launch_trace_extension(s0, E.q, multi, E.numSMs, st);
        cudaStreamWaitEvent(st, E.joinEv, 0);
        // the small buckets' shade kernels beside the Lambert shade
        cudaEventRecord(E.bucketsEv, st);
        cudaStreamWaitEvent(E.side2, E.bucketsEv, 0);
        for (uint32_t b : {kBucketDielectric, kBucketGGX, kBucketOther})
            launch_shade_bucket(b, s0, E.q, multi, E.shade_grid(), (int)E.cfg.shadeBlock, E.side2);
        cudaEventRecord(E.join2Ev, E.side2);
        launch_shade_bucket(kBucketLambert, s0, E.q, multi, E.shade_grid(), (int)E.cfg.shadeBlock, st);
        cudaStreamWaitEvent(st, E.join2Ev, 0);
        return;
    }
    if (ev) cudaEventRecord(ev[0], st);
    launch_control(E.q, st);
    if (ev) cudaEventRecord(ev[1], st);
    launch_generate(E.q, E.numSMs * 8, st);
    if (ev) cudaEventRecord(ev[2], st);
    launch_trace_extension(s0, E.q, multi, E.numSMs, st);
    if (ev) cudaEventRecord(ev[3], st);
    launch_trace_shadow(s0, E.q, multi, E.numSMs, st);
    if (ev) cudaEventRecord(ev[4], st);
    // four shade kernels; the fifth stage slot (Lambert resume) stays empty: the
    // shadow kernel continues those paths
    for (uint32_t b = 0; b < kNumBuckets; ++b) {
        if (b != kBucketLambertResume) launch_shade_bucket(b, s0, E.q, multi, E.shade_grid(), (int)E.cfg.shadeBlock, st);
        if (ev) cudaEventRecord(ev[5 + b], st);
    }
}

cudaError_t Engine::enqueue_chunk(const DevScene& s0, bool multi, bool timing) {
    cudaError_t e;
    if (timing) {
        while (stageEv.size() < cfg.chunk * 10) {
            cudaEvent_t ev;
            if ((e = cudaEventCreate(&ev)) != cudaSuccess) return e;
            stageEv.push_back(ev);
        }
        for (uint32_t k = 0; k < cfg.chunk; ++k) launch_iteration(*this, s0, multi, stream, &stageEv[k * 10]);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    } else {
        const bool same = graph && multi == graphMulti && memcmp(&s0, &graphScene, sizeof(DevScene)) == 0 &&
                          graphCfg.chunk == cfg.chunk && graphCfg.shadeBlock == cfg.shadeBlock &&
                          graphCfg.shadeBlocksPerSM == cfg.shadeBlocksPerSM;
        if (!same) {
            if (graph) cudaGraphExecDestroy(graph);
            graph = nullptr;
            if ((e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
            for (uint32_t k = 0; k < cfg.chunk; ++k) launch_iteration(*this, s0, multi, stream, nullptr);
            cudaGraph_t g = nullptr;
            e = cudaStreamEndCapture(stream, &g);
            if (e != cudaSuccess) return e;
            e = cudaGraphInstantiate(&graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return e;
            graphMulti = multi;
            memcpy(&graphScene, &s0, sizeof(DevScene));
            graphCfg = cfg;
        }
        if ((e = cudaGraphLaunch(graph, stream)) != cudaSuccess) return e;
    }
    if ((e = cudaMemcpyAsync(hCtr, q.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, stream)) != cudaSuccess) return e;
    return cudaMemcpyAsync(hCtl, dCtl, sizeof(SlotCtl) * kMaxSlots, cudaMemcpyDeviceToHost, stream);
}

cudaError_t Engine::enqueue_until_done(const DevScene& s0, bool multi, uint32_t iterLimit) {
    if (loopUnsupported) return cudaErrorNotSupported;
    cudaError_t e;
    const bool same = loopGraph && multi == loopMulti && memcmp(&s0, &loopScene, sizeof(DevScene)) == 0 &&
                      loopCfg.chunk == cfg.chunk && loopCfg.shadeBlock == cfg.shadeBlock &&
                      loopCfg.shadeBlocksPerSM == cfg.shadeBlocksPerSM;
    if (!same) {
        if (loopGraph) cudaGraphExecDestroy(loopGraph);
        loopGraph = nullptr;
        cudaGraph_t g = nullptr;
        if ((e = cudaGraphCreate(&g, 0)) != cudaSuccess) return e;
        cudaGraphConditionalHandle h;
        cudaGraphNodeParams np{};
        cudaGraphNode_t node;
        e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
        if (e == cudaSuccess) {
            np.type = cudaGraphNodeTypeConditional;
            np.conditional.handle = h;
            np.conditional.type = cudaGraphCondTypeWhile;
            np.conditional.size = 1;
            e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            cudaGraphDestroy(g);
            loopUnsupported = true;
            return cudaErrorNotSupported;
        }
        cudaGraph_t body = np.conditional.phGraph_out[0];
        if ((e = cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
            cudaSuccess) {
            cudaGraphDestroy(g);
            return e;
        }
        for (uint32_t k = 0; k < cfg.chunk; ++k) launch_iteration(*this, s0, multi, stream, nullptr);
        launch_loop_cond(h, q, stream);
        cudaGraph_t captured = nullptr;
        e = cudaStreamEndCapture(stream, &captured);
        if (e == cudaSuccess) e = cudaGraphInstantiate(&loopGraph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            loopGraph = nullptr;
            return e;
        }
        loopMulti = multi;
        memcpy(&loopScene, &s0, sizeof(DevScene));
        loopCfg = cfg;
    }
    hGenOrder[kMaxSlots + 2] = iterLimit;  // staging word for Counters::iterLimit
    if ((e = cudaMemcpyAsync(&q.ctr->iterLimit, &hGenOrder[kMaxSlots + 2], sizeof(uint32_t), cudaMemcpyHostToDevice,
                             stream)) != cudaSuccess)
        return e;
    if ((e = cudaGraphLaunch(loopGraph, stream)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(hCtr, q.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, stream)) != cudaSuccess) return e;
    return cudaMemcpyAsync(hCtl, dCtl, sizeof(SlotCtl) * kMaxSlots, cudaMemcpyDeviceToHost, stream);
}

cudaError_t Engine::stage_times(float* ms, uint32_t* launches) {
    for (uint32_t k = 0; k < cfg.chunk; ++k)
        for (int j = 0; j < WRK_NUM_STAGES; ++j) {
            float t = 0;
            cudaError_t e = cudaEventElapsedTime(&t, stageEv[k * 10 + j], stageEv[k * 10 + j + 1]);
            if (e != cudaSuccess) return e;
            ms[j] += t;
            launches[j] += j == WRK_STAGE_SHADE_LAMBERT_RESUME ? 0u : 1u;
        }
    return cudaSuccess;
}

}  // namespace wrk

namespace {

// Light list + power CDF exactly as Scene::finalize builds it
// (libWR/src/internal/scene.cpp:423-491): serial FP32 over triangles in order.
void build_light_cdf(wrk_scene* s) {
    s->emissive.clear();
    s->cdf.clear();
    float total = 0.0f;
    uint32_t nt = (uint32_t)s->triMat.size();
    for (uint32_t t = 0; t < nt; ++t) {
        uint32_t m = s->triMat[t];
        if (m >= s->mats.size() || s->mats[m].type != WRK_EMISSIVE) continue;
        s->emissive.push_back(t);
        const float* a = &s->vtx[3 * (size_t)s->idx[3 * t]];
        const float* b = &s->vtx[3 * (size_t)s->idx[3 * t + 1]];
        const float* c = &s->vtx[3 * (size_t)s->idx[3 * t + 2]];
        float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        float cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        float area = 0.5f * std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        const wrk_material& mm = s->mats[m];
        float power = (mm.emission[0] + mm.emission[1] + mm.emission[2]) * area;
        total += power;
        s->cdf.push_back(total);
    }
    for (float& c : s->cdf) c /= total;
}

template <class T>
int upload(DevBuf& b, const std::vector<T>& v) {
    if (v.empty()) return WRK_OK;
    int rc = b.alloc(sizeof(T) * v.size());
    if (rc) return rc;
    CK(cudaMemcpy(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return WRK_OK;
}

int check_scene(wrk_scene* s) {
    if (!s) return fail(WRK_ERR_INVALID, "null scene");
    if (!s->finalized) return fail(WRK_ERR_STATE, "scene not finalized");
    return set_device(s->device);
}

}  // namespace

extern "C" {

const char* wrk_last_error(void) { return g_err.c_str(); }
int wrk_version(void) { return 1; }

int wrk_device_count(int* count) {
    if (!count) return fail(WRK_ERR_INVALID, "null count");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    *count = e == cudaSuccess ? n : 0;
    return WRK_OK;
}
int wrk_malloc(int device, uint64_t bytes, void** ptr) {
    if (!ptr) return fail(WRK_ERR_INVALID, "null ptr");
    int rc = set_device(device);
    if (rc) return rc;
    CK(cudaMalloc(ptr, bytes ? bytes : 1));
    return WRK_OK;
}
int wrk_free(void* ptr) {
    CK(cudaFree(ptr));
    return WRK_OK;
}
int wrk_memcpy_htod(void* dst, const void* src, uint64_t bytes) {
    CK(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    return WRK_OK;
}
int wrk_memcpy_dtoh(void* dst, const void* src, uint64_t bytes) {
    CK(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return WRK_OK;
}
int wrk_synchronize(int device) {
    int rc = set_device(device);
    if (rc) return rc;
    CK(cudaDeviceSynchronize());
    return WRK_OK;
}

// ---------------------------------------------------------------------------
int wrk_scene_create(int device, wrk_scene** out) {
    if (!out) return fail(WRK_ERR_INVALID, "null out");
    int rc = set_device(device);
    if (rc) return rc;
    wrk_scene* s = new wrk_scene();
    s->device = device;
    *out = s;
    return WRK_OK;
}
int wrk_scene_destroy(wrk_scene* s) {
    if (s) {
        cudaSetDevice(s->device);
        delete s;
    }
    return WRK_OK;
}
int wrk_scene_set_geometry(wrk_scene* s, const float* vertices, uint32_t nv, const float* normals, const float* uvs,
                           const uint32_t* indices, uint32_t nt, const uint32_t* triMaterial) {
    if (!s || !vertices || !indices || !triMaterial) return fail(WRK_ERR_INVALID, "null geometry argument");
    if (s->finalized) return fail(WRK_ERR_STATE, "scene already finalized");
    if (nv == 0 || nt == 0) return fail(WRK_ERR_INVALID, "Scene has no geometry");
    for (size_t i = 0; i < 3 * (size_t)nt; ++i)
        if (indices[i] >= nv) return fail(WRK_ERR_INVALID, "index %u out of range (vertex count %u)", indices[i], nv);
    s->vtx.assign(vertices, vertices + 3 * (size_t)nv);
    s->nrm.clear();
    s->uv.clear();
    if (normals) s->nrm.assign(normals, normals + 3 * (size_t)nv);
    if (uvs) s->uv.assign(uvs, uvs + 2 * (size_t)nv);
    s->idx.assign(indices, indices + 3 * (size_t)nt);
    s->triMat.assign(triMaterial, triMaterial + nt);
    return WRK_OK;
}
int wrk_scene_set_materials(wrk_scene* s, const wrk_material* m, uint32_t n) {
    if (!s || (!m && n)) return fail(WRK_ERR_INVALID, "null materials");
    if (s->finalized) return fail(WRK_ERR_STATE, "scene already finalized");
    s->mats.assign(m, m + n);
    return WRK_OK;
}
int wrk_scene_add_texture(wrk_scene* s, const uint8_t* rgba, uint32_t w, uint32_t h, uint32_t* outId) {
    if (!s || !rgba || !outId || w == 0 || h == 0) return fail(WRK_ERR_INVALID, "bad texture arguments");
    if (s->finalized) return fail(WRK_ERR_STATE, "scene already finalized");
    s->tex.emplace_back(rgba, rgba + 4 * (size_t)w * h);
    s->texW.push_back(w);
    s->texH.push_back(h);
    *outId = (uint32_t)s->tex.size();
    return WRK_OK;
}
int wrk_scene_set_environment(wrk_scene* s, const float rgb[3]) {
    if (!s || !rgb) return fail(WRK_ERR_INVALID, "null environment");
    for (int k = 0; k < 3; ++k) s->env[k] = rgb[k];
    s->view.env[0] = rgb[0];
    s->view.env[1] = rgb[1];
    s->view.env[2] = rgb[2];
    return WRK_OK;
}

int wrk_scene_set_environment_map(wrk_scene* s, const float* rgba, uint32_t w, uint32_t h) {
    if (!s || !rgba || w == 0 || h == 0) return fail(WRK_ERR_INVALID, "bad environment map arguments");
    if (s->finalized) return fail(WRK_ERR_STATE, "scene already finalized");
    s->envMap.assign(rgba, rgba + 4 * (size_t)w * h);
    s->envW = w;
    s->envH = h;
    return WRK_OK;
}

int wrk_scene_finalize(wrk_scene* s) {
    if (!s) return fail(WRK_ERR_INVALID, "null scene");
    if (s->finalized) return WRK_OK;  // as Scene::finalize (scene.cpp:351)
    if (s->vtx.empty() || s->idx.empty()) return fail(WRK_ERR_INVALID, "Scene has no geometry");
    int rc = set_device(s->device);
    if (rc) return rc;
    uint32_t nt = (uint32_t)s->triMat.size();
    build_light_cdf(s);
    // the light records NEE reads after choosing an entry of the CDF: the emissive
    // triangle's three vertices and its material's emission, in one 64-byte record
    std::vector<float4> lights;
    for (uint32_t t : s->emissive) {
        const float* a = &s->vtx[3 * (size_t)s->idx[3 * (size_t)t]];
        const float* b = &s->vtx[3 * (size_t)s->idx[3 * (size_t)t + 1]];
        const float* c = &s->vtx[3 * (size_t)s->idx[3 * (size_t)t + 2]];
        const wrk_material& m = s->mats[s->triMat[t]];
        uint32_t tb = t;
        float tf;
        std::memcpy(&tf, &tb, sizeof(tf));
        lights.push_back(make_float4(a[0], a[1], a[2], tf));
        lights.push_back(make_float4(b[0], b[1], b[2], 0.0f));
        lights.push_back(make_float4(c[0], c[1], c[2], 0.0f));
        lights.push_back(make_float4(m.emission[0], m.emission[1], m.emission[2], 0.0f));
    }
    if ((rc = upload(s->dLights, lights))) return rc;
    if ((rc = upload(s->dVtx, s->vtx)) || (rc = upload(s->dNrm, s->nrm)) || (rc = upload(s->dUv, s->uv)) ||
        (rc = upload(s->dIdx, s->idx)) || (rc = upload(s->dTriMat, s->triMat)) || (rc = upload(s->dMats, s->mats)) ||
        (rc = upload(s->dEmissive, s->emissive)) || (rc = upload(s->dCdf, s->cdf)))
        return rc;
    // texel pool + per-texture info
    std::vector<TexInfo> ti;
    size_t total = 0;
    for (size_t i = 0; i < s->tex.size(); ++i) {
        ti.push_back(TexInfo{total, s->texW[i], s->texH[i]});
        total += (s->tex[i].size() + 15) & ~size_t(15);
    }
    if (!s->tex.empty()) {
        if ((rc = s->dTexels.alloc(total))) return rc;
        for (size_t i = 0; i < s->tex.size(); ++i)
            CK(cudaMemcpy(s->dTexels.as<uint8_t>() + ti[i].offset, s->tex[i].data(), s->tex[i].size(),
                          cudaMemcpyHostToDevice));
        if ((rc = upload(s->dTexInfo, ti))) return rc;
    }
    if ((rc = s->dErr.alloc(sizeof(uint32_t)))) return rc;
    BvhBuildResult br{};
    char err[256] = {0};
    rc = build_bvh8(s->dVtx.as<float>(), s->dIdx.as<uint32_t>(), s->dTriMat.as<uint32_t>(), nt, 0, &br, err,
                    sizeof(err));
    if (rc) return fail(rc, "%s", err);
    s->nodes = br.nodes;
    s->tris = br.tris;
    // the shade bucket of each record's material, so the trace kernel sorts a hit
    // with one load from the record it just tested
    launch_leaf_buckets(br.tris, nt, s->dMats.as<wrk_material>(), (uint32_t)s->mats.size(), 0);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(0));
    s->info.numTriangles = nt;
    s->info.numNodes = br.numNodes;
    s->info.numBinaryNodes = br.numBinary;
    s->info.depth = br.depth;
    s->info.numEmissive = (uint32_t)s->emissive.size();
    s->info.buildMs = br.ms;
    s->info.sahCost = br.sah;
    DevScene& v = s->view;
    v.vtx = s->dVtx.as<float>();
    v.nrm = s->nrm.empty() ? nullptr : s->dNrm.as<float>();
    v.uv = s->uv.empty() ? nullptr : s->dUv.as<float>();
    v.idx = s->dIdx.as<uint32_t>();
    v.triMat = s->dTriMat.as<uint32_t>();
    v.mats = s->dMats.as<wrk_material>();
    v.numMats = (uint32_t)s->mats.size();
    v.texels = s->dTexels.as<uint8_t>();
    v.tex = s->dTexInfo.as<TexInfo>();
    v.numTex = (uint32_t)s->tex.size();
    v.emissive = s->dEmissive.as<uint32_t>();
    v.cdf = s->dCdf.as<float>();
    v.lights = s->dLights.as<float4>();
    v.numEmissive = (uint32_t)s->emissive.size();
    v.numTris = nt;
    for (int k = 0; k < 3; ++k) v.env[k] = s->env[k];
    v.nodes = s->nodes;
    v.tris = s->tris;
    v.numNodes = br.numNodes;
    if (!s->envMap.empty()) {
        if ((rc = upload(s->dEnvMap, s->envMap))) return rc;
        v.envMap = s->dEnvMap.as<float4>();
        v.envW = s->envW;
        v.envH = s->envH;
    }
    s->finalized = true;
    return WRK_OK;
}

int wrk_scene_bvh_info(wrk_scene* s, wrk_bvh_info* info) {
    int rc = check_scene(s);
    if (rc) return rc;
    if (!info) return fail(WRK_ERR_INVALID, "null info");
    *info = s->info;
    return WRK_OK;
}

int wrk_scene_light_cdf(wrk_scene* s, uint32_t* tris, float* cdf, uint32_t capacity, uint32_t* count) {
    int rc = check_scene(s);
    if (rc) return rc;
    uint32_t n = (uint32_t)s->emissive.size();
    if (count) *count = n;
    if (!tris && !cdf) return WRK_OK;  // size query
    if (n > capacity) return fail(WRK_ERR_INVALID, "capacity %u < %u emissive triangles", capacity, n);
    if (n) {
        // read back what the device holds
        if (tris) CK(cudaMemcpy(tris, s->dEmissive.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
        if (cdf) CK(cudaMemcpy(cdf, s->dCdf.p, sizeof(float) * n, cudaMemcpyDeviceToHost));
    }
    return WRK_OK;
}

int wrk_scene_bvh_export(wrk_scene* s, uint32_t* nodes, float* tris) {
    int rc = check_scene(s);
    if (rc) return rc;
    if (nodes) CK(cudaMemcpy(nodes, s->nodes, sizeof(uint4) * 5 * (size_t)s->info.numNodes, cudaMemcpyDeviceToHost));
    if (tris) CK(cudaMemcpy(tris, s->tris, sizeof(float4) * 3 * (size_t)s->info.numTriangles, cudaMemcpyDeviceToHost));
    return WRK_OK;
}

int wrk_scene_buffers_get(wrk_scene* s, wrk_scene_buffers* o) {
    int rc = check_scene(s);
    if (rc) return rc;
    if (!o) return fail(WRK_ERR_INVALID, "null out");
    const DevScene& v = s->view;
    o->vertices = (uint64_t)(uintptr_t)v.vtx;
    o->normals = (uint64_t)(uintptr_t)v.nrm;
    o->uvs = (uint64_t)(uintptr_t)v.uv;
    o->indices = (uint64_t)(uintptr_t)v.idx;
    o->triMaterial = (uint64_t)(uintptr_t)v.triMat;
    o->materials = (uint64_t)(uintptr_t)v.mats;
    o->emissive = (uint64_t)(uintptr_t)v.emissive;
    o->cdf = (uint64_t)(uintptr_t)v.cdf;
    o->texels = (uint64_t)(uintptr_t)v.texels;
    o->bvhNodes = (uint64_t)(uintptr_t)v.nodes;
    o->bvhTriangles = (uint64_t)(uintptr_t)v.tris;
    o->numMaterials = v.numMats;
    o->numEmissive = v.numEmissive;
    o->numTextures = v.numTex;
    o->numTriangles = v.numTris;
    return WRK_OK;
}

// ---------------------------------------------------------------------------
int wrk_renderer_create(int device, uint32_t capacity, wrk_renderer** out) {
    if (!out) return fail(WRK_ERR_INVALID, "null out");
    int rc = set_device(device);
    if (rc) return rc;
    wrk_renderer* r = new wrk_renderer();
    cudaError_t e = r->eng.init(device, capacity);
    if (e == cudaSuccess && (cudaEventCreate(&r->ev0) != cudaSuccess || cudaEventCreate(&r->ev1) != cudaSuccess ||
                             cudaEventCreate(&r->evLoop0) != cudaSuccess || cudaEventCreate(&r->evLoop1) != cudaSuccess))
        e = cudaErrorUnknown;
    if (e != cudaSuccess) {
        delete r;
        return fail(WRK_ERR_CUDA, "renderer creation failed: %s", cudaGetErrorString(e));
    }
    *out = r;
    return WRK_OK;
}

int wrk_renderer_destroy(wrk_renderer* r) {
    if (r) {
        cudaSetDevice(r->eng.device);
        delete r;
    }
    return WRK_OK;
}

int wrk_renderer_set_launch(wrk_renderer* r, uint32_t chunk, uint32_t shadeBlock) {
    if (!r) return fail(WRK_ERR_INVALID, "null renderer");
    if (chunk < 1 || chunk > 64 || (shadeBlock != 128 && shadeBlock != 256))
        return fail(WRK_ERR_INVALID, "chunk must be 1..64 and shadeBlock 128 or 256");
    r->eng.cfg.chunk = chunk;
    r->eng.cfg.shadeBlock = shadeBlock;
    return WRK_OK;
}

}  // extern "C"

namespace wrk {
// The request record the kernels read for one render (camera basis as libWR
// computes it, settings, sums).
void fill_frame(Frame& f, const wrk_camera& cam, const wrk_render_params& p) {
    f = Frame{};
    camera_frame(cam, f);
    f.width = p.width;
    f.height = p.height;
    f.spp = p.spp;
    f.useNEE = p.useNEE ? 1u : 0u;
    f.maxBounces = p.maxBounces;
    f.seed = p.seed;
    f.sampleOffset = p.sampleOffset;
    f.maxIter = p.maxIterations ? p.maxIterations : 8u;
    f.rrStart = p.russianRouletteDepth;
    f.fireflyClamp = p.fireflyClamp;
    f.tilesX = (p.width % 8 == 0 && p.height % 4 == 0) ? p.width / 8 : 0;
    f.perSample = p.width * p.height;
    // adjacent work items take K samples of one pixel: a warp's camera paths cover
    // 32/K pixels x K samples (a tighter bundle of primary rays than 32 pixels)
    f.interleave = !f.tilesX ? 1u : (p.spp % 4 == 0 ? 4u : (p.spp % 2 == 0 ? 2u : 1u));
    f.flags = p.flags;
}
}  // namespace wrk

extern "C" {

static int render_impl(wrk_renderer* r, wrk_scene* s, const wrk_camera* cam, const wrk_render_params* p, float* d_rgb,
                       float* d_alb, float* d_nrm, wrk_render_stats* stats) {
    Engine& E = r->eng;
    Frame f;
    fill_frame(f, *cam, *p);
    size_t np = (size_t)p->width * p->height;
    int rc = r->frameBufs.alloc(np * 3 * sizeof(float4));
    if (rc) return rc;
    f.accum = r->frameBufs.as<float4>();
    // first-hit guides are summed only when the caller asks for them (two atomics
    // per camera path, ~4 % of a showcase render)
    f.albedo = d_alb ? f.accum + np : nullptr;
    f.normal = d_nrm ? f.accum + 2 * np : nullptr;
    f.err = &E.q.ctr->error;
    f.scene = 0;
    cudaStream_t st = E.stream;
    CK(cudaEventRecord(r->ev0, st));
    CK(cudaMemsetAsync(f.accum, 0, np * 3 * sizeof(float4), st));
    E.hReq[0] = f;
    E.hScenes[0] = s->view;
    SlotCtl sc{};
    sc.workTotal = (unsigned long long)np * p->spp;
    sc.state = kSlotActive;
    E.hCtl[0] = sc;
    E.hGenOrder[0] = 1;
    E.hGenOrder[1] = 0;
    CK(cudaMemcpyAsync(E.dReq, E.hReq, sizeof(Frame), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(E.dScenes, E.hScenes, sizeof(DevScene), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(E.dCtl, E.hCtl, sizeof(SlotCtl), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(E.dGenOrder, E.hGenOrder, 2 * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    CK(E.reset_counters());
    // bound on iterations: every path needs <= maxIter; waves of `capacity` paths
    unsigned long long waves = sc.workTotal / E.capacity + 2;
    unsigned long long maxIters = waves * (unsigned long long)(f.maxIter + 2) * 4ull + 64ull;
    uint32_t iters = 0;
    const bool timing = (p->flags & WRK_FLAG_STAGE_TIMING) != 0;
    float stageMs[WRK_NUM_STAGES] = {0};
    uint32_t stageN[WRK_NUM_STAGES] = {0};
    CK(cudaEventRecord(r->evLoop0, st));
    bool looped = false;
    if (!timing) {
        // device-driven: one graph launch runs chunks until the request finished
        cudaError_t e = E.enqueue_until_done(s->view, false, (uint32_t)std::min<unsigned long long>(maxIters, 0xffffffffu));
        if (e == cudaSuccess) {
            CK(cudaStreamSynchronize(st));
            iters = E.hCtr->iteration;
            if (E.hCtr->error) return fail(WRK_ERR_DEVICE, "device error flags 0x%x during render", E.hCtr->error);
            if (!slot_finished(E.hCtl[0]))
                return fail(WRK_ERR_DEVICE, "render did not converge after %u iterations", iters);
            looped = true;
        } else if (e != cudaErrorNotSupported) {
            return fail(WRK_ERR_CUDA, "device-driven render loop: %s", cudaGetErrorString(e));
        }
    }
    while (!looped) {
        CK(E.enqueue_chunk(s->view, false, timing));
        iters += E.cfg.chunk;
        CK(cudaStreamSynchronize(st));
        if (timing) CK(E.stage_times(stageMs, stageN));
        if (E.hCtr->error) return fail(WRK_ERR_DEVICE, "device error flags 0x%x during render", E.hCtr->error);
        if (E.hCtl[0].state == kSlotDone) break;
        if (iters > maxIters) return fail(WRK_ERR_DEVICE, "render did not converge after %u iterations", iters);
    }
    CK(cudaEventRecord(r->evLoop1, st));
    launch_resolve(f, p->flags & WRK_FLAG_RAW_GUIDES, d_rgb, d_alb, d_nrm, st);
    CK(cudaGetLastError());
    CK(cudaEventRecord(r->ev1, st));
    CK(cudaEventSynchronize(r->ev1));
    if (stats) {
        const Counters& h = *E.hCtr;
        stats->paths = h.paths;
        stats->extensionRays = h.extRays;
        stats->shadowRays = h.shdRays + h.shadowAnswered.v;  // + the last iteration's answered queries
        stats->shadowTraced = h.shdTraced;
        for (int b = 0; b < kNumBuckets; ++b) stats->bucketPaths[b] = h.bucketTotal[b] + h.bucket[b].v;
        stats->bucketPaths[kBucketLambert] += h.lambertTex.v;
        stats->iterations = iters;
        stats->deviceErrors = h.error;
        cudaEventElapsedTime(&stats->gpuMs, r->evLoop0, r->evLoop1);
        cudaEventElapsedTime(&stats->totalMs, r->ev0, r->ev1);
        for (int j = 0; j < WRK_NUM_STAGES; ++j) {
            stats->stageMs[j] = stageMs[j];
            stats->stageLaunches[j] = stageN[j];
        }
    }
    return WRK_OK;
}

static int check_render_args(wrk_renderer* r, wrk_scene* s, const wrk_camera* cam, const wrk_render_params* p) {
    if (!r || !cam || !p) return fail(WRK_ERR_INVALID, "null renderer/camera/params");
    int rc = check_scene(s);
    if (rc) return rc;
    if (s->device != r->eng.device) return fail(WRK_ERR_INVALID, "scene and renderer on different devices");
    if (p->width == 0 || p->height == 0 || p->spp == 0) return fail(WRK_ERR_INVALID, "empty render (w/h/spp = 0)");
    if ((uint64_t)p->width * p->height > (1ull << 31)) return fail(WRK_ERR_INVALID, "image too large");
    return WRK_OK;
}

int wrk_render_device(wrk_renderer* r, wrk_scene* s, const wrk_camera* cam, const wrk_render_params* p, float* d_rgb,
                      float* d_alb, float* d_nrm, wrk_render_stats* stats) {
    int rc = check_render_args(r, s, cam, p);
    if (rc) return rc;
    if (!d_rgb) return fail(WRK_ERR_INVALID, "null output");
    return render_impl(r, s, cam, p, d_rgb, d_alb, d_nrm, stats);
}

int wrk_render(wrk_renderer* r, wrk_scene* s, const wrk_camera* cam, const wrk_render_params* p, float* rgb,
               float* albedo, float* normal, wrk_render_stats* stats) {
    int rc = check_render_args(r, s, cam, p);
    if (rc) return rc;
    if (!rgb) return fail(WRK_ERR_INVALID, "null output");
    size_t np = (size_t)p->width * p->height;
    if ((rc = r->outBufs.alloc(np * 9 * sizeof(float)))) return rc;
    float* o = r->outBufs.as<float>();
    if ((rc = render_impl(r, s, cam, p, o, albedo ? o + 3 * np : nullptr, normal ? o + 6 * np : nullptr, stats)))
        return rc;
    CK(cudaMemcpy(rgb, o, np * 3 * sizeof(float), cudaMemcpyDeviceToHost));
    if (albedo) CK(cudaMemcpy(albedo, o + 3 * np, np * 3 * sizeof(float), cudaMemcpyDeviceToHost));
    if (normal) CK(cudaMemcpy(normal, o + 6 * np, np * 3 * sizeof(float), cudaMemcpyDeviceToHost));
    return WRK_OK;
}

// ---------------------------------------------------------------------------
int wrk_trace_closest(wrk_scene* s, const float* rays, uint32_t n, float* t, uint32_t* prim) {
    int rc = check_scene(s);
    if (rc) return rc;
    if (n && (!rays || !t || !prim)) return fail(WRK_ERR_INVALID, "null buffer");
    CK(cudaMemset(s->dErr.p, 0, sizeof(uint32_t)));
    launch_closest_query(s->view, rays, n, t, prim, s->dErr.as<uint32_t>(), 0);
    CK(cudaGetLastError());
    uint32_t e = 0;
    CK(cudaMemcpy(&e, s->dErr.p, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (e) return fail(WRK_ERR_DEVICE, "trace error flags 0x%x", e);
    return WRK_OK;
}
int wrk_trace_occluded(wrk_scene* s, const float* rays, uint32_t n, uint32_t* occ) {
    int rc = check_scene(s);
    if (rc) return rc;
    if (n && (!rays || !occ)) return fail(WRK_ERR_INVALID, "null buffer");
    CK(cudaMemset(s->dErr.p, 0, sizeof(uint32_t)));
    launch_occluded_query(s->view, rays, n, occ, s->dErr.as<uint32_t>(), 0);
    CK(cudaGetLastError());
    uint32_t e = 0;
    CK(cudaMemcpy(&e, s->dErr.p, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (e) return fail(WRK_ERR_DEVICE, "trace error flags 0x%x", e);
    return WRK_OK;
}
int wrk_compact(const uint32_t* stage, const uint32_t* idxIn, uint32_t n, uint32_t* idxOut, uint32_t* count) {
    if (!count || (n && (!stage || !idxIn || !idxOut))) return fail(WRK_ERR_INVALID, "null buffer");
    int rc = compact_stable(stage, idxIn, n, idxOut, count, 0);
    if (rc) return fail(rc, "compaction launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    CK(cudaDeviceSynchronize());
    return WRK_OK;
}
int wrk_cdf_sample(const float* cdf, uint32_t ncdf, const float* u, uint32_t n, uint32_t* out) {
    if (ncdf == 0) return fail(WRK_ERR_INVALID, "empty CDF");
    launch_cdf(cdf, ncdf, u, n, out, 0);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    return WRK_OK;
}
int wrk_rng_batch(const uint32_t* seed, const uint32_t* dim, uint32_t n, uint32_t* hash, float* u) {
    launch_rng(seed, dim, n, hash, u, 0);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    return WRK_OK;
}
int wrk_bsdf_batch(const float* in, uint32_t n, float* out) {
    launch_bsdf(in, n, out, 0);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    return WRK_OK;
}
int wrk_texture_batch(wrk_scene* s, uint32_t id, const float* uv, uint32_t n, float* out) {
    int rc = check_scene(s);
    if (rc) return rc;
    if (id == 0 || id > s->tex.size()) return fail(WRK_ERR_INVALID, "texture id %u out of range", id);
    size_t off = 0;
    for (uint32_t i = 0; i + 1 < id; ++i) off += (s->tex[i].size() + 15) & ~size_t(15);
    launch_texture(s->dTexels.as<uint8_t>() + off, s->texW[id - 1], s->texH[id - 1], uv, n, out, 0);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    return WRK_OK;
}
int wrk_camera_rays(const wrk_camera* cam, uint32_t w, uint32_t h, const uint32_t* px, const uint32_t* sm, uint32_t n,
                    uint32_t seed, float* out) {
    if (!cam || w == 0 || h == 0) return fail(WRK_ERR_INVALID, "bad camera arguments");
    Frame f{};
    camera_frame(*cam, f);
    f.width = w;
    f.height = h;
    f.seed = seed;
    launch_camera_rays(f, px, sm, n, out, 0);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    return WRK_OK;
}
int wrk_tonemap_aces(const float* rgb, uint32_t npix, uint8_t* out) {
    if (npix && (!rgb || !out)) return fail(WRK_ERR_INVALID, "null buffer");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int vec = ((uintptr_t)rgb % 16 == 0 && (uintptr_t)out % 4 == 0) ? 1 : 0;
    launch_tonemap(rgb, 3u * npix, out, sms * 8, vec, 0);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    return WRK_OK;
}

}  // extern "C"
