// Internal device-side layouts of libwrk (not part of the C ABI).
//
// HBM layout
//   Scene (resident):  vertices / normals / uvs / indices / per-triangle material
//                      (the flat soup libWR uploads, scene.cpp:360-390), 64 B materials,
//                      RGBA8 texels, emissive list + power CDF, the 8-wide BVH
//                      (80 B nodes = 5 x uint4) and leaf-ordered triangle records
//                      (48 B = 3 x float4: v0|prim, e1|material, e2).
//   Path queues: a path's state travels with it from queue to queue.  Every queue
//   stores its entries SoA -- one array per field, one float4 / uint4 per entry --
//   so a kernel reading entries i..i+31 of a field, or writing the consecutive
//   positions a warp-aggregated append hands out, issues one coalesced 512-byte
//   access per field.  Fields:
//      ray_o (origin, tmin)   ray_d (direction, tmax)   hit (t, prim, material, -)
//      thr (throughput, prevPdf)   rad (radiance, pixel)   st (seed, rngDim, depth|iter<<16, flags)
//      sh_o / sh_d (shadow ray)    sh_c (NEE contribution)
//   Queues: extension (ray_o ray_d thr rad st) and shadow (sh_o = origin | request
//   slot, sh_d = direction | tmax, sh_c = contribution | continuation, and rad for
//   a path that ends after its shadow ray), each double-buffered across
//   iterations, and four material buckets (ray_o ray_d hit thr rad st).  A Lambert
//   path that sends a shadow ray has already drawn its bounce and roulette: if it
//   goes on, its next extension entry is written at once (at the front of the
//   extension buffer it will be traced from), and the shadow kernel only adds the
//   contribution to that entry's radiance when the light is visible; otherwise
//   the shadow kernel accumulates or drops it, as sh_c.w says.  No slot indirection and no free list: a path occupies exactly one
//   entry between iterations, so the room for new camera paths is the capacity
//   minus the extension and shadow entries the last iteration produced.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/wrk.h"

namespace wrk {

enum : uint32_t { kLambert = 0, kEmissive = 1, kGlass = 2, kGGX = 3, kGGXT = 4 };
// Material buckets the trace kernel sorts hits into.  Index kBucketLambertResume
// only counts the Lambert paths the shadow stage continues (it has no queue and
// no shade kernel).
enum : uint32_t {
    kBucketLambert = 0,
    kBucketDielectric = 1,
    kBucketGGX = 2,
    kBucketOther = 3,
    kBucketLambertResume = 4,
    kNumBuckets = 5
};
// The bucket of a material type; invalid material ids go to kBucketOther.
__host__ __device__ inline uint32_t bucket_of_type(uint32_t type) {
    switch (type) {
        case kLambert: return kBucketLambert;
        case kGlass:
        case kGGXT: return kBucketDielectric;
        case kGGX: return kBucketGGX;
        default: return kBucketOther;
    }
}
// A leaf record's bucket word also flags Lambert materials with an albedo or normal
// texture: their hits go to the far end of the Lambert queue (filled downward from the
// last entry), so the shade kernel's warps see plain and textured hits apart and only
// the textured ones take the texture fetches.
constexpr uint32_t kRecTextured = 8u;
__host__ __device__ inline uint32_t bucket_of_material(const wrk_material& m) {
    const uint32_t b = bucket_of_type(m.type);
    return b == kBucketLambert && (m.albedoTextureId != 0 || m.normalTextureId != 0) ? b | kRecTextured : b;
}
// st.w: flags in bits 0-7, the path's request slot in bits 8-15
enum : uint32_t { kFlagFirstHit = 1u, kFlagPrevDelta = 2u };
// What a Lambert path does after its shadow ray (sh_c.w): continue with the
// prepared extension ray, accumulate its radiance, or end unaccumulated (the
// iteration bound).
enum : uint32_t { kContExt = 0u, kContAccumulate = 1u, kContDrop = 2u };
// Start of every shadow ray's [tmin, tmax] (the light sample's distance minus it
// is tmax), so the queue does not store it.
constexpr float kShadowTmin = 1e-5f;

constexpr uint32_t kSlotShift = 8;
__host__ __device__ inline uint32_t slot_of(uint32_t stw) { return (stw >> kSlotShift) & 0xffu; }

// Requests in flight in one wavefront (each with its own camera, settings,
// accumulation buffers and scene) and scenes one engine can address.
constexpr uint32_t kMaxSlots = 64;
constexpr uint32_t kMaxScenes = 128;
enum : uint32_t { kSlotFree = 0, kSlotActive = 1, kSlotDone = 2 };

constexpr uint32_t kInvalidSlot = 0xffffffffu;
constexpr uint32_t kNoHit = 0xffffffffu;

// Device error bits (Counters::error).
enum : uint32_t { kErrStackOverflow = 1u, kErrBadIndex = 2u, kErrQueueOverflow = 4u };

struct TexInfo {
    uint64_t offset;  // byte offset into the texel pool
    uint32_t w, h;
};

struct DevScene {
    const float* vtx;
    const float* nrm;  // null when no mesh supplied normals
    const float* uv;   // null when no mesh supplied uvs
    const uint32_t* idx;
    const uint32_t* triMat;
    const wrk_material* mats;
    uint32_t numMats;
    const uint8_t* texels;
    const TexInfo* tex;
    uint32_t numTex;
    const uint32_t* emissive;
    const float* cdf;
    // per emissive entry (the order of emissive / cdf), 4 float4: v0 | triangle id,
    // v1 | 0, v2 | 0, emission | 0 -- one 64-byte record per NEE light sample
    const float4* lights;
    uint32_t numEmissive;
    uint32_t numTris;
    float env[3];
    const uint4* nodes;
    // BVH triangle records in leaf order, 3 float4 each: v0 | prim, v1 - v0 |
    // material, v2 - v0 | bucket (the material's shade bucket, set at finalize)
    const float4* tris;
    uint32_t numNodes;
    const float4* envMap;  // lat-long RGBA f32 map (null = none); used with WRK_FLAG_ENV_MAP
    uint32_t envW, envH;
};

// One queue's entries, SoA.  Fields a queue does not carry are null.  ray_d.w is the
// ray's tmax in the extension queues and the hit distance (hit.x) in the buckets.
struct PathQ {
    float4* ray_o;
    float4* ray_d;
    float4* hit;
    float4* thr;
    float4* rad;
    uint4* st;
    float4* sh_o;
    float4* sh_d;
    float4* sh_c;
};

// A queue counter alone on a 128-byte line, so appends to different queues hit
// different L2 lines instead of serializing on one.
struct alignas(128) HotCounter {
    uint32_t v;
    uint32_t pad[31];
};

// Queue counters and loop bookkeeping; lives in device memory, owned by the renderer.
// The hot counters take warp-aggregated atomics; everything after them is written
// only by the single-thread control kernel (which also keeps the statistics, so
// no kernel spends atomics on them).
struct Counters {
    HotCounter ext[2];
    HotCounter shd[2];
    HotCounter bucket[kNumBuckets];
    HotCounter lambertTex;      // textured Lambert hits, stored from the Lambert queue's last entry down
    HotCounter cont;            // Lambert continuations placed in ext[cur] this iteration
    HotCounter contDirect;      // ... of them without a shadow entry (query answered in the shade)
    HotCounter shadowAnswered;  // shadow queries the Lambert shade answered this iteration
    HotCounter fetchExtension;  // rays taken by the persistent traversal kernels this iteration
    HotCounter fetchShadow;
    uint32_t cur;          // which ext/shd buffer the current iteration consumes
    uint32_t genCount;     // paths generated this iteration
    uint32_t genExtBase;   // extension-queue index where the generated paths go
    uint32_t numSeg;       // generation segments this iteration
    uint32_t iteration;
    uint32_t error;
    uint32_t activeSlots;  // slots still active after this iteration's completion check
    uint32_t iterLimit;    // the device-driven loop stops after this many iterations
    unsigned long long extRays;
    unsigned long long shdRays;    // shadow queries: traced + answered in the Lambert shade
    unsigned long long shdTraced;  // shadow queries traced by the any-hit kernel
    unsigned long long paths;
    unsigned long long bucketTotal[kNumBuckets];
};

// One request of a batch as the kernels see it: camera basis, render settings,
// its scene and its per-pixel sums.  Lives in device memory (Queues::req).
struct Frame {
    float pos[3], fwd[3], right[3], up[3];
    float tanHalf, aspect, focal, lens;
    uint32_t width, height;
    uint32_t tilesX, perSample;  // 8x4 pixel tiles across the image (0 = row order); work items per sample
    uint32_t interleave;         // K samples of a pixel on adjacent work items (1, 2 or 4; 1 in row order)
    uint32_t spp, useNEE, maxBounces, seed, maxIter, sampleOffset;
    float rrStart, fireflyClamp;
    uint32_t scene;  // index into Queues::scenes
    uint32_t flags;  // WRK_FLAG_* of the request
    float4* accum;   // radiance sum per pixel
    float4* albedo;  // first-hit albedo sum per pixel
    float4* normal;  // first-hit normal sum per pixel
    uint32_t* err;   // device error flags (Counters::error)
};

// Progress of a request slot.  The host arms it (workTotal, state = active); the
// control kernel hands out its work items, kernels count the paths that ended,
// and the control kernel marks it done (with a device timestamp) once every work
// item was generated and every path of it ended.
struct SlotCtl {
    unsigned long long workTotal;  // pixels x spp
    unsigned long long workNext;   // work items handed out
    unsigned long long finished;   // paths ended (accumulated or dropped)
    unsigned long long doneNs;     // %globaltimer when marked done
    uint32_t state;
    uint32_t doneIter;
    uint32_t pad[2];
};

// Work items of one request generated in this iteration: extension-queue entries
// [genExtBase + extOffset, + count) take work items [workBase, + count).
struct GenSeg {
    unsigned long long workBase;
    uint32_t slot, count, extOffset, pad;
};

struct Queues {
    PathQ ext[2];
    PathQ shd[2];
    PathQ bucket[kNumBuckets];
    Counters* ctr;
    uint32_t capacity;
    uint32_t pad;
    const Frame* req;          // [kMaxSlots] request records
    SlotCtl* ctl;              // [kMaxSlots]
    const DevScene* scenes;    // [kMaxScenes]
    const uint32_t* genOrder;  // genOrder[0] = n, then n slots in admission (FIFO) order
    GenSeg* seg;               // [kMaxSlots] this iteration's generation segments
};

// ---- host-callable launchers (defined in the .cu files) ----
// `multi`: requests of the batch may use different scenes (each path looks its
// scene up through its request); otherwise every request uses scene `s`.
void launch_control(const Queues& q, cudaStream_t st);
void launch_generate(const Queues& q, int grid, cudaStream_t st);
// persistent kernels: the grid is numSMs x the kernel's resident blocks per SM
void launch_trace_extension(const DevScene& s, const Queues& q, bool multi, int numSMs, cudaStream_t st);
void launch_trace_shadow(const DevScene& s, const Queues& q, bool multi, int numSMs, cudaStream_t st);
void launch_shade_bucket(uint32_t bucket, const DevScene& s, const Queues& q, bool multi, int grid, int block,
                         cudaStream_t st);
void launch_resolve(const Frame& f, uint32_t rawGuides, float* rgb, float* albedo, float* normal, cudaStream_t st);
// End of one chunk of the device-driven loop: keeps the enclosing conditional
// WHILE graph node running while a request in the admission order has work left.
void launch_loop_cond(cudaGraphConditionalHandle h, const Queues& q, cudaStream_t st);
__host__ __device__ inline bool slot_finished(const SlotCtl& sc) {
    return sc.workNext >= sc.workTotal && sc.finished >= sc.workTotal;
}

// BVH build (bvh_build.cu)
struct BvhBuildResult {
    uint4* nodes;
    float4* tris;
    uint32_t numNodes, numBinary, depth;
    float ms;
    float sah;
};
int build_bvh8(const float* d_vtx, const uint32_t* d_idx, const uint32_t* d_triMat, uint32_t numTris,
               cudaStream_t st, BvhBuildResult* out, char* err, size_t errlen);

// Sets the per-thread message returned by wrk_last_error(); returns `code`.
int report_error(int code, const char* msg);

// Writes the shade bucket of each BVH triangle record's material into its e2.w
// (kernels_misc.cu).
void launch_leaf_buckets(float4* tris, uint32_t numTris, const wrk_material* mats, uint32_t numMats,
                         cudaStream_t st);

// standalone ray queries (trace.cu)
void launch_closest_query(const DevScene& s, const float* rays, uint32_t n, float* t, uint32_t* prim,
                          uint32_t* err, cudaStream_t st);
void launch_occluded_query(const DevScene& s, const float* rays, uint32_t n, uint32_t* occ, uint32_t* err,
                           cudaStream_t st);

}  // namespace wrk
