// Serving loop and autotuner.
//
// A wrk_server keeps scenes resident (their BVHs, textures and light CDFs stay
// where wrk_scene_finalize put them) and renders requests of different sizes,
// spp, cameras and scenes concurrently: every admitted request owns a slot of
// the engine's request table and a region of one accumulation pool, and its
// paths share the wavefront queues with every other request's (continuous
// batching: the control kernel hands the room that ending paths leave to the
// active requests in admission order, so a request admitted while others are in
// flight starts in the next iteration).  One chunk of bounce iterations is a
// captured CUDA graph replayed by wrk_server_step; between chunks the host
// admits queued requests (by free slot and HBM budget, first come first served),
// and retires finished ones (resolve to rgb / albedo / normal, optionally the
// learned denoiser).  libWR renders one image per synchronous call
// (libWR/src/internal/renderer.cpp:132-316); this has no counterpart there.
//
// Per-request results do not depend on the mix: the RNG is keyed by (request
// seed, pixel, sample), so a request's paths are the same alone and batched;
// only the order of the f32 atomic sums into its pixels changes.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <deque>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "wrk_internal.h"

namespace wrk {
const DevScene* scene_view(const wrk_scene* s);
int scene_device(const wrk_scene* s);
void fill_frame(Frame& f, const wrk_camera& cam, const wrk_render_params& p);
}  // namespace wrk

using namespace wrk;

namespace {

int sfail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return report_error(code, buf);
}
#define SCK(x)                                                                                                  \
    do {                                                                                                        \
        cudaError_t e_ = (x);                                                                                   \
        if (e_ != cudaSuccess) return sfail(WRK_ERR_CUDA, "%s: %s (%s:%d)", #x, cudaGetErrorString(e_), __FILE__, \
                                            __LINE__);                                                          \
    } while (0)

// Bytes of pool per pixel: radiance / albedo / normal sums (3 x float4), the resolved
// rgb / albedo / normal (3 x float3) and the denoised rgb (float3).
constexpr size_t kPoolBytesPerPixel = 48 + 36 + 12;

enum : int { kQueued = 0, kRunning = 1, kReady = 2 };

struct SReq {
    uint64_t ticket = 0;
    wrk_scene* scene = nullptr;
    uint32_t sceneIdx = 0;
    wrk_camera cam{};
    wrk_render_params p{};
    int slot = -1;
    size_t off = 0, bytes = 0;
    int state = kQueued;
    double tSubmit = 0, tAdmit = 0, tReady = 0;
    uint32_t admitIter = 0, doneIter = 0;
    bool denoise = false;
    size_t npx() const { return (size_t)p.width * p.height; }
};

double now_ms(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct wrk_server {
    Engine eng;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    EngineBuf pool;
    size_t poolBytes = 0;
    std::map<size_t, size_t> freeList;  // offset -> bytes
    uint32_t maxSlots = kMaxSlots;
    std::vector<wrk_scene*> scenes;
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, SReq> reqs;
    std::vector<int> order;            // slots in admission order
    uint64_t slotTicket[kMaxSlots];    // 0 = free
    uint64_t nextTicket = 1;
    wrk_denoiser* denoiser = nullptr;
    uint64_t iterations = 0;
    float lastChunkMs = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~wrk_server() {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }

    // first fit in the accumulation pool
    bool take(size_t bytes, size_t* off) {
        for (auto it = freeList.begin(); it != freeList.end(); ++it) {
            if (it->second >= bytes) {
                *off = it->first;
                size_t rest = it->second - bytes;
                size_t o = it->first + bytes;
                freeList.erase(it);
                if (rest) freeList[o] = rest;
                return true;
            }
        }
        return false;
    }
    void give(size_t off, size_t bytes) {
        auto it = freeList.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != freeList.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            freeList.erase(nx);
        }
        if (it != freeList.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                freeList.erase(it);
            }
        }
    }
    float* out_rgb(const SReq& r) const { return (float*)(pool.as<uint8_t>() + r.off + r.npx() * 48); }
    float* out_denoised(const SReq& r) const { return (float*)(pool.as<uint8_t>() + r.off + r.npx() * 84); }
};

namespace {

size_t region_bytes(const wrk_render_params& p) {
    return ((size_t)p.width * p.height * kPoolBytesPerPixel + 255) & ~size_t(255);
}

int upload_order(wrk_server* sv) {
    Engine& E = sv->eng;
    E.hGenOrder[0] = (uint32_t)sv->order.size();
    for (size_t k = 0; k < sv->order.size(); ++k) E.hGenOrder[1 + k] = (uint32_t)sv->order[k];
    SCK(cudaMemcpyAsync(E.dGenOrder, E.hGenOrder, sizeof(uint32_t) * (1 + sv->order.size()), cudaMemcpyHostToDevice,
                        E.stream));
    return WRK_OK;
}

int scene_index(wrk_server* sv, wrk_scene* s, uint32_t* idx) {
    for (size_t k = 0; k < sv->scenes.size(); ++k)
        if (sv->scenes[k] == s) {
            *idx = (uint32_t)k;
            return WRK_OK;
        }
    if (sv->scenes.size() >= kMaxScenes) return sfail(WRK_ERR_INVALID, "more than %u scenes in one server", kMaxScenes);
    const uint32_t k = (uint32_t)sv->scenes.size();
    Engine& E = sv->eng;
    E.hScenes[k] = *scene_view(s);
    SCK(cudaMemcpyAsync(E.dScenes + k, E.hScenes + k, sizeof(DevScene), cudaMemcpyHostToDevice, E.stream));
    sv->scenes.push_back(s);
    *idx = k;
    return WRK_OK;
}

// Admits queued requests in arrival order while a slot and pool room are free.
int admit(wrk_server* sv, bool* changed) {
    Engine& E = sv->eng;
    while (!sv->queue.empty()) {
        SReq& r = sv->reqs[sv->queue.front()];
        int slot = -1;
        for (uint32_t k = 0; k < sv->maxSlots; ++k)
            if (sv->slotTicket[k] == 0) {
                slot = (int)k;
                break;
            }
        size_t off = 0;
        if (slot < 0 || !sv->take(r.bytes, &off)) break;
        int rc = scene_index(sv, r.scene, &r.sceneIdx);
        if (rc) {
            sv->give(off, r.bytes);
            return rc;
        }
        r.off = off;
        r.slot = slot;
        Frame f;
        fill_frame(f, r.cam, r.p);
        const size_t np = r.npx();
        float4* acc = (float4*)(sv->pool.as<uint8_t>() + off);
        f.accum = acc;
        f.albedo = acc + np;
        f.normal = acc + 2 * np;
        f.err = &E.q.ctr->error;
        f.scene = r.sceneIdx;
        SCK(cudaMemsetAsync(acc, 0, np * 48, E.stream));
        E.hReq[slot] = f;
        SCK(cudaMemcpyAsync(E.dReq + slot, E.hReq + slot, sizeof(Frame), cudaMemcpyHostToDevice, E.stream));
        SlotCtl sc{};
        sc.workTotal = (unsigned long long)np * r.p.spp;
        sc.state = kSlotActive;
        E.hCtl[slot] = sc;
        SCK(cudaMemcpyAsync(E.dCtl + slot, E.hCtl + slot, sizeof(SlotCtl), cudaMemcpyHostToDevice, E.stream));
        sv->slotTicket[slot] = r.ticket;
        r.state = kRunning;
        r.tAdmit = now_ms(sv->t0);
        r.admitIter = (uint32_t)sv->iterations;
        sv->order.push_back(slot);
        sv->queue.pop_front();
        *changed = true;
    }
    return WRK_OK;
}

int retire(wrk_server* sv, bool* changed) {
    Engine& E = sv->eng;
    std::vector<SReq*> done;
    for (size_t k = 0; k < sv->order.size();) {
        const int slot = sv->order[k];
        if (E.hCtl[slot].state == kSlotDone) {
            auto it = sv->reqs.find(sv->slotTicket[slot]);
            if (it != sv->reqs.end()) {
                SReq* r = &it->second;
                r->doneIter = E.hCtl[slot].doneIter;
                Frame f = E.hReq[slot];
                const size_t np = r->npx();
                float* o = sv->out_rgb(*r);
                launch_resolve(f, r->p.flags & WRK_FLAG_RAW_GUIDES, o, o + 3 * np, o + 6 * np, E.stream);
                SCK(cudaGetLastError());
                done.push_back(r);
            }
            sv->slotTicket[slot] = 0;
            sv->order.erase(sv->order.begin() + (long)k);
            *changed = true;
        } else {
            ++k;
        }
    }
    if (done.empty()) return WRK_OK;
    SCK(cudaStreamSynchronize(E.stream));
    for (SReq* r : done) {
        if (r->denoise && sv->denoiser) {
            const size_t np = r->npx();
            float* o = sv->out_rgb(*r);
            int rc = wrk_denoiser_infer(sv->denoiser, o, o + 3 * np, o + 6 * np, 1, r->p.height, r->p.width,
                                        sv->out_denoised(*r));
            if (rc) return rc;
        }
        r->state = kReady;
        r->tReady = now_ms(sv->t0);
    }
    return WRK_OK;
}

}  // namespace

extern "C" {

int wrk_server_create(int device, const wrk_server_config* cfg, wrk_server** out) {
    if (!out) return sfail(WRK_ERR_INVALID, "null out");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return sfail(WRK_ERR_NO_DEVICE, "no CUDA device available");
    if (device < 0 || device >= n) return sfail(WRK_ERR_INVALID, "device %d out of range", device);
    SCK(cudaSetDevice(device));
    wrk_server_config c{};
    if (cfg) c = *cfg;
    if (c.maxRequests == 0 || c.maxRequests > kMaxSlots) c.maxRequests = kMaxSlots;
    if (c.poolBytes == 0) c.poolBytes = 4ull << 30;
    if (c.chunk == 0) c.chunk = 8;
    if (c.shadeBlock == 0) c.shadeBlock = 256;
    if (c.chunk > 64 || (c.shadeBlock != 128 && c.shadeBlock != 256))
        return sfail(WRK_ERR_INVALID, "chunk must be 1..64 and shadeBlock 128 or 256");
    wrk_server* sv = new wrk_server();
    cudaError_t e = sv->eng.init(device, c.capacity);
    if (e == cudaSuccess) e = sv->pool.alloc(c.poolBytes);
    if (e == cudaSuccess && (cudaEventCreate(&sv->e0) != cudaSuccess || cudaEventCreate(&sv->e1) != cudaSuccess))
        e = cudaErrorUnknown;
    if (e != cudaSuccess) {
        delete sv;
        return sfail(WRK_ERR_CUDA, "server creation failed: %s", cudaGetErrorString(e));
    }
    sv->eng.cfg.chunk = c.chunk;
    sv->eng.cfg.shadeBlock = c.shadeBlock;
    sv->poolBytes = c.poolBytes;
    sv->freeList[0] = c.poolBytes;
    sv->maxSlots = c.maxRequests;
    for (uint32_t k = 0; k < kMaxSlots; ++k) sv->slotTicket[k] = 0;
    *out = sv;
    return WRK_OK;
}

int wrk_server_destroy(wrk_server* sv) {
    if (sv) {
        cudaSetDevice(sv->eng.device);
        delete sv;
    }
    return WRK_OK;
}

int wrk_server_set_denoiser(wrk_server* sv, wrk_denoiser* dn) {
    if (!sv) return sfail(WRK_ERR_INVALID, "null server");
    sv->denoiser = dn;
    return WRK_OK;
}

int wrk_server_submit(wrk_server* sv, wrk_scene* s, const wrk_camera* cam, const wrk_render_params* p,
                      uint64_t* ticket) {
    if (!sv || !cam || !p || !ticket) return sfail(WRK_ERR_INVALID, "null argument");
    if (!scene_view(s)) return sfail(WRK_ERR_STATE, "scene not finalized");
    if (scene_device(s) != sv->eng.device) return sfail(WRK_ERR_INVALID, "scene and server on different devices");
    if (p->width == 0 || p->height == 0 || p->spp == 0) return sfail(WRK_ERR_INVALID, "empty render (w/h/spp = 0)");
    if ((uint64_t)p->width * p->height > (1ull << 28)) return sfail(WRK_ERR_INVALID, "image too large");
    if ((p->flags & WRK_FLAG_DENOISE) && !sv->denoiser)
        return sfail(WRK_ERR_STATE, "denoising requested but no denoiser attached");
    SReq r;
    r.ticket = sv->nextTicket++;
    r.scene = s;
    r.cam = *cam;
    r.p = *p;
    r.bytes = region_bytes(*p);
    r.denoise = (p->flags & WRK_FLAG_DENOISE) != 0;
    if (r.bytes > sv->poolBytes)
        return sfail(WRK_ERR_INVALID, "request needs %zu bytes, the pool holds %zu", r.bytes, sv->poolBytes);
    r.tSubmit = now_ms(sv->t0);
    sv->reqs[r.ticket] = r;
    sv->queue.push_back(r.ticket);
    *ticket = r.ticket;
    return WRK_OK;
}

// Admits what fits, runs one chunk of bounce iterations for every request in
// flight, and retires the requests that finished.
int wrk_server_step(wrk_server* sv, wrk_server_status* status) {
    if (!sv) return sfail(WRK_ERR_INVALID, "null server");
    SCK(cudaSetDevice(sv->eng.device));
    Engine& E = sv->eng;
    bool changed = false;
    int rc = admit(sv, &changed);
    if (rc) return rc;
    if (changed && (rc = upload_order(sv))) return rc;
    if (!sv->order.empty()) {
        const bool multi = sv->scenes.size() > 1;
        SCK(cudaEventRecord(sv->e0, E.stream));
        SCK(E.enqueue_chunk(*scene_view(sv->scenes[0]), multi, false));
        SCK(cudaEventRecord(sv->e1, E.stream));
        SCK(cudaStreamSynchronize(E.stream));
        cudaEventElapsedTime(&sv->lastChunkMs, sv->e0, sv->e1);
        sv->iterations += E.cfg.chunk;
        if (E.hCtr->error) return sfail(WRK_ERR_DEVICE, "device error flags 0x%x while serving", E.hCtr->error);
        changed = false;
        if ((rc = retire(sv, &changed))) return rc;
        if (changed && (rc = upload_order(sv))) return rc;
    }
    if (status) {
        status->queued = (uint32_t)sv->queue.size();
        status->running = (uint32_t)sv->order.size();
        uint32_t ready = 0;
        for (auto& kv : sv->reqs) ready += kv.second.state == kReady;
        status->ready = ready;
        status->iterations = sv->iterations;
        status->lastChunkMs = sv->lastChunkMs;
        status->poolFreeBytes = 0;
        for (auto& kv : sv->freeList) status->poolFreeBytes += kv.second;
    }
    return WRK_OK;
}

int wrk_server_poll(wrk_server* sv, uint64_t ticket, int* ready) {
    if (!sv || !ready) return sfail(WRK_ERR_INVALID, "null argument");
    auto it = sv->reqs.find(ticket);
    if (it == sv->reqs.end()) return sfail(WRK_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
    *ready = it->second.state == kReady;
    return WRK_OK;
}

int wrk_server_wait(wrk_server* sv, uint64_t ticket) {
    if (!sv) return sfail(WRK_ERR_INVALID, "null server");
    for (uint64_t guard = 0; guard < (1ull << 24); ++guard) {
        int ready = 0;
        int rc = wrk_server_poll(sv, ticket, &ready);
        if (rc) return rc;
        if (ready) return WRK_OK;
        wrk_server_status st{};
        if ((rc = wrk_server_step(sv, &st))) return rc;
        // nothing in flight and the request still queued: the pool or the slots
        // are held by ready results nobody has taken
        if (st.running == 0 && sv->reqs[ticket].state == kQueued)
            return sfail(WRK_ERR_STATE, "request %llu cannot be admitted: take the ready results first",
                         (unsigned long long)ticket);
    }
    return sfail(WRK_ERR_DEVICE, "request %llu did not finish", (unsigned long long)ticket);
}

static int result_impl(wrk_server* sv, uint64_t ticket, float* rgb, float* albedo, float* normal,
                       wrk_request_info* info, cudaMemcpyKind kind) {
    if (!sv) return sfail(WRK_ERR_INVALID, "null server");
    auto it = sv->reqs.find(ticket);
    if (it == sv->reqs.end()) return sfail(WRK_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
    SReq& r = it->second;
    if (r.state != kReady) return sfail(WRK_ERR_STATE, "request %llu not ready", (unsigned long long)ticket);
    const size_t np = r.npx();
    const float* o = sv->out_rgb(r);
    const float* src = (r.denoise && sv->denoiser) ? sv->out_denoised(r) : o;
    if (rgb) SCK(cudaMemcpy(rgb, src, np * 12, kind));
    if (albedo) SCK(cudaMemcpy(albedo, o + 3 * np, np * 12, kind));
    if (normal) SCK(cudaMemcpy(normal, o + 6 * np, np * 12, kind));
    if (info) {
        info->width = r.p.width;
        info->height = r.p.height;
        info->spp = r.p.spp;
        info->denoised = r.denoise && sv->denoiser ? 1u : 0u;
        info->submitMs = r.tSubmit;
        info->admitMs = r.tAdmit;
        info->readyMs = r.tReady;
        info->iterations = r.doneIter >= r.admitIter ? r.doneIter - r.admitIter : 0u;
    }
    sv->give(r.off, r.bytes);
    sv->reqs.erase(it);
    return WRK_OK;
}

int wrk_server_result(wrk_server* sv, uint64_t ticket, float* rgb, float* albedo, float* normal,
                      wrk_request_info* info) {
    return result_impl(sv, ticket, rgb, albedo, normal, info, cudaMemcpyDeviceToHost);
}
int wrk_server_result_device(wrk_server* sv, uint64_t ticket, float* d_rgb, float* d_albedo, float* d_normal,
                             wrk_request_info* info) {
    return result_impl(sv, ticket, d_rgb, d_albedo, d_normal, info, cudaMemcpyDeviceToDevice);
}

// ---------------------------------------------------------------------------
// Autotuner: times one render of the caller's workload per candidate launch
// shape (queue capacity x chunk depth x shading block size) and keeps the
// fastest.  Each capacity gets a fresh renderer; each shape renders twice and
// the second (graph captured, queues touched) is timed.
int wrk_autotune(int device, wrk_scene* s, const wrk_camera* cam, const wrk_render_params* p, wrk_tune_result* out) {
    if (!s || !cam || !p || !out) return sfail(WRK_ERR_INVALID, "null argument");
    *out = wrk_tune_result{};
    // queue capacities up to 64M paths (672 B each: 45 GB; a 512x512 frame at 256 spp
    // then runs all its paths at once, in the 8 iterations a path may take); a capacity
    // whose queues do not fit in the free device memory ends the search
    const uint32_t caps[5] = {1u << 20, 1u << 22, 1u << 24, 1u << 25, 1u << 26};
    const uint32_t chunks[3] = {4, 8, 16};
    const uint32_t blocks[2] = {128, 256};
    const size_t np = (size_t)p->width * p->height;
    float* d = nullptr;
    SCK(cudaSetDevice(device));
    SCK(cudaMalloc(&d, np * 9 * sizeof(float)));
    int rc = WRK_OK;
    out->bestMs = 3.4e38f;
    for (uint32_t ci = 0; ci < 5 && !rc; ++ci) {
        wrk_renderer* r = nullptr;
        size_t freeB = 0, totalB = 0;
        if (ci > 0 && cudaMemGetInfo(&freeB, &totalB) == cudaSuccess &&
            (size_t)caps[ci] * 672 + (size_t)512 * 1024 * 1024 > freeB)
            break;
        if ((rc = wrk_renderer_create(device, caps[ci], &r))) break;
        for (uint32_t k = 0; k < 3 && !rc; ++k)
            for (uint32_t b = 0; b < 2 && !rc; ++b) {
                if ((rc = wrk_renderer_set_launch(r, chunks[k], blocks[b]))) break;
                wrk_render_stats st{};
                if ((rc = wrk_render_device(r, s, cam, p, d, d + 3 * np, d + 6 * np, &st))) break;
                if ((rc = wrk_render_device(r, s, cam, p, d, d + 3 * np, d + 6 * np, &st))) break;
                if (out->numTrials < 32) {
                    wrk_tune_trial& t = out->trials[out->numTrials++];
                    t.capacity = caps[ci];
                    t.chunk = chunks[k];
                    t.shadeBlock = blocks[b];
                    t.ms = st.gpuMs;
                }
                if (st.gpuMs < out->bestMs) {
                    out->bestMs = st.gpuMs;
                    out->capacity = caps[ci];
                    out->chunk = chunks[k];
                    out->shadeBlock = blocks[b];
                }
            }
        wrk_renderer_destroy(r);
    }
    cudaFree(d);
    return rc;
}

}  // extern "C"
