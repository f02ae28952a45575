// Ray traversal of the 8-wide compressed BVH: closest hit (extension rays) and
// any hit (shadow rays).  Replaces optixTrace with __closesthit__trace /
// __miss__trace (libWR/kernels/trace.cu:17-153,321-323 in trianglestrip/OfflineRenderer);
// there are no RT cores on B200, so traversal is SIMT integer/FP32 work.
//
// Per node: five 16-byte loads (__ldg, read-only path), eight quantized slab tests
// decoded with one byte permute and one directed-rounding FMA per plane.
// Internal-child hits go into an 8-bit mask permuted by the ray octant so the
// lowest set bit is the child nearest the ray's entry corner; leaf-child hits set
// bits of a triangle mask.  Pending node groups
// (child base + remaining hit bits + internal mask) go on a short stack held in
// shared memory, spilling to a bounded local array; overflow raises an error bit
// and ends the ray instead of corrupting memory.
//
// The triangle test is Moller-Trumbore written with _rn / fmaf intrinsics so the
// FP32 result is the same sequence of correctly rounded operations as the CPU
// oracle's.
#include "wrk_internal.h"
#include "wrk_shading.cuh"
#include "wrk_tri.cuh"

namespace wrk {

constexpr int kTraceBlock = 128;
#ifndef WRK_STACK_SMEM
#define WRK_STACK_SMEM 12
#endif
constexpr int kStackSmem = WRK_STACK_SMEM;
constexpr int kStackLocal = 48 - kStackSmem;
constexpr uint32_t kMaxVisits = 1u << 16;

// Byte k of w as the float 2^15 + b, exactly, without an int->float conversion:
// one byte permute builds the bits 0x4700bb00 (exponent 2^15, b in mantissa bits
// 8-15).  The 2^15 bias is folded into the per-node plane offset (see
// intersect_node), so a plane costs one permute and one FMA.
__device__ __forceinline__ float qbias(uint32_t w, uint32_t k) {
    return __uint_as_float(__byte_perm(w, 0x47000000u, 0x7504u | (k << 4)));
}

// Intersects the 8 children of a node; returns internal hits (permuted by octant)
// and the triangle mask relative to triBase.
__device__ __forceinline__ void intersect_node(const uint4* __restrict__ nodes, uint32_t idx, const Ray& r,
                                               float ix, float iy, float iz, uint32_t oct_inv, float tfar_max,
                                               uint32_t& childBase, uint32_t& triBase, uint32_t& hits,
                                               uint32_t& imask, uint32_t& tmask) {
    const uint4* n = nodes + 5 * (size_t)idx;
    uint4 n0 = __ldg(n), n1 = __ldg(n + 1), n2 = __ldg(n + 2), n3 = __ldg(n + 3), n4 = __ldg(n + 4);
    float px = __uint_as_float(n0.x), py = __uint_as_float(n0.y), pz = __uint_as_float(n0.z);
    float sx = __uint_as_float((n0.w & 0xffu) << 23) * ix;
    float sy = __uint_as_float(((n0.w >> 8) & 0xffu) << 23) * iy;
    float sz = __uint_as_float(((n0.w >> 16) & 0xffu) << 23) * iz;
    float ax = (px - r.ox) * ix, ay = (py - r.oy) * iy, az = (pz - r.oz) * iz;
    // plane t = q*s + a = (2^15 + q)*s + (a - 2^15*s).  The biased offsets are
    // rounded down for near planes and up for far planes, and the plane FMAs round
    // the same way, so the slab only grows (by at most ~1/256 of a quantization
    // step): a child box the ray crosses is never rejected.
    const float axl = __fmaf_rd(-32768.0f, sx, ax), axh = __fmaf_ru(-32768.0f, sx, ax);
    const float ayl = __fmaf_rd(-32768.0f, sy, ay), ayh = __fmaf_ru(-32768.0f, sy, ay);
    const float azl = __fmaf_rd(-32768.0f, sz, az), azh = __fmaf_ru(-32768.0f, sz, az);
    imask = n0.w >> 24;
    childBase = n1.x;
    triBase = n1.y;
    hits = 0;
    tmask = 0;
    // near/far plane words per axis: dir >= 0 -> near = lo, far = hi
    uint32_t xn0 = ix >= 0.0f ? n2.x : n3.z, xn1 = ix >= 0.0f ? n2.y : n3.w;
    uint32_t xf0 = ix >= 0.0f ? n3.z : n2.x, xf1 = ix >= 0.0f ? n3.w : n2.y;
    uint32_t yn0 = iy >= 0.0f ? n2.z : n4.x, yn1 = iy >= 0.0f ? n2.w : n4.y;
    uint32_t yf0 = iy >= 0.0f ? n4.x : n2.z, yf1 = iy >= 0.0f ? n4.y : n2.w;
    uint32_t zn0 = iz >= 0.0f ? n3.x : n4.z, zn1 = iz >= 0.0f ? n3.y : n4.w;
    uint32_t zf0 = iz >= 0.0f ? n4.z : n3.x, zf1 = iz >= 0.0f ? n4.w : n3.y;
    const float tfar_lim = tfar_max * 1.00000024f;
    uint32_t hm = 0;  // children whose slab the ray crosses, by slot
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const uint32_t k = s & 3;
        uint32_t xn = s < 4 ? xn0 : xn1, xf = s < 4 ? xf0 : xf1;
        uint32_t yn = s < 4 ? yn0 : yn1, yf = s < 4 ? yf0 : yf1;
        uint32_t zn = s < 4 ? zn0 : zn1, zf = s < 4 ? zf0 : zf1;
        float t0x = __fmaf_rd(qbias(xn, k), sx, axl);
        float t1x = __fmaf_ru(qbias(xf, k), sx, axh);
        float t0y = __fmaf_rd(qbias(yn, k), sy, ayl);
        float t1y = __fmaf_ru(qbias(yf, k), sy, ayh);
        float t0z = __fmaf_rd(qbias(zn, k), sz, azl);
        float t1z = __fmaf_ru(qbias(zf, k), sz, azh);
        // Three-input integer max / min on the float bit patterns.  Non-negative
        // floats order like their bit patterns; negative ones order reversed, which
        // only moves tn down and tf up (a larger slab, never a smaller one), and a
        // negative tf still fails against tn >= tmin >= 0.  No plane distance is
        // NaN: the inverse directions are finite (trav_init).
        float tn = __int_as_float(__vimax3_s32(__float_as_int(t0x), __float_as_int(t0y),
                                               max(__float_as_int(t0z), __float_as_int(r.tmin))));
        float tf = __int_as_float(__vimin3_s32(__float_as_int(t1x), __float_as_int(t1y),
                                               min(__float_as_int(t1z), __float_as_int(tfar_lim))));
        hm |= (tn <= tf * 1.00000024f) ? (1u << s) : 0u;
    }
    // internal hits, moved from slot s to bit s ^ oct_inv by three conditional swaps
    uint32_t ih = hm & imask;
    if (oct_inv & 1u) ih = ((ih & 0x55u) << 1) | ((ih >> 1) & 0x55u);
    if (oct_inv & 2u) ih = ((ih & 0x33u) << 2) | ((ih >> 2) & 0x33u);
    if (oct_inv & 4u) ih = ((ih & 0x0Fu) << 4) | ((ih >> 4) & 0x0Fu);
    hits = ih;
    // leaf hits: each adds its run of cnt triangles starting at bit off
    uint32_t lh = hm & ~imask;
    while (lh) {
        const uint32_t j = __ffs(lh) - 1;
        lh &= lh - 1;
        const uint32_t meta = ((j < 4 ? n1.z : n1.w) >> (8 * (j & 3u))) & 0xffu;
        const uint32_t cnt = (meta >> 5) + 1u, off = meta & 31u;
        tmask |= ((1u << cnt) - 1u) << off;
    }
}

// The four scene fields traversal needs (a DevScene has them too).
struct TraceGeom {
    const uint4* nodes;
    const float4* tris;
    uint32_t numNodes, numTris;
};

// Per-lane traversal state, kept in registers across the persistent loop's rounds.
struct Trav {
    Ray r;
    float ix, iy, iz;
    uint32_t octInv;
    uint32_t gBase;
    uint32_t gBits;  // node group: child hit bits (bits 0-7, octant order) | internal-child mask << 8
    uint32_t tBase, tMask;
    int sp;
    uint32_t visits;
    float tBest;
    // Leaf position (index into the BVH triangle records) of the best hit, kNoHit
    // while there is none; the hit's primitive and material are read from that
    // record when the ray is done, so they take no registers during traversal.
    uint32_t lBest;
};

__device__ __forceinline__ uint32_t record_prim(const float4* tris, uint32_t l) {
    return l == kNoHit ? kNoHit : __float_as_uint(__ldg(tris + 3 * (size_t)l).w);
}
__device__ __forceinline__ uint32_t record_material(const float4* tris, uint32_t l) {
    return l == kNoHit ? 0u : __float_as_uint(__ldg(tris + 3 * (size_t)l + 1).w);
}

__device__ __forceinline__ void trav_init(Trav& t, const Ray& r) {
    t.r = r;
    // Direction components below 2^-80 in magnitude are replaced by +-2^-80 for
    // the slab tests only (the triangle test uses the true direction), so inverse
    // directions and plane distances stay finite and never NaN.
    const float ooeps = 8.27180613e-25f;
    t.ix = 1.0f / (fabsf(r.dx) < ooeps ? copysignf(ooeps, r.dx) : r.dx);
    t.iy = 1.0f / (fabsf(r.dy) < ooeps ? copysignf(ooeps, r.dy) : r.dy);
    t.iz = 1.0f / (fabsf(r.dz) < ooeps ? copysignf(ooeps, r.dz) : r.dz);
    uint32_t oct = (r.dx < 0.0f ? 1u : 0u) | (r.dy < 0.0f ? 2u : 0u) | (r.dz < 0.0f ? 4u : 0u);
    t.octInv = oct ^ 7u;  // slot of the child nearest the entry corner -> bit 0
    // the root is a one-child node group
    t.gBase = 0;
    t.gBits = (1u << t.octInv) | (1u << 8);
    t.tBase = 0;
    t.tMask = 0;
    t.sp = 0;
    t.visits = 0;
    t.tBest = r.tmax;
    t.lBest = kNoHit;
}

// One traversal step: descend into the next child of the current node group
// (pushing the group's remainder), test the triangles that node exposes, and pop
// when the group is used up.  Returns true when the ray is finished.  Closest hit
// keeps ties in t with the lower primitive index; any hit stops at the first hit.
template <bool kAnyHit, class Geom>
__device__ __forceinline__ bool trav_step(const Geom& s, Trav& t, uint2* sstack, uint2* lstack,
                                          uint32_t* errFlag) {
    const int tid = threadIdx.x;
    if (++t.visits > kMaxVisits) {  // a malformed tree must not spin forever
        atomicOr(errFlag, kErrBadIndex);
        return true;
    }
    if (t.gBits & 0xffu) {
        uint32_t pos = __ffs(t.gBits) - 1;  // the lowest set bit is a hit bit
        t.gBits &= t.gBits - 1;
        uint32_t slot = pos ^ t.octInv;
        uint32_t child = t.gBase + __popc(t.gBits & (((1u << slot) - 1u) << 8));
        if (t.gBits & 0xffu) {
            uint2 e = make_uint2(t.gBase, t.gBits);
            if (t.sp < kStackSmem) sstack[t.sp * kTraceBlock + tid] = e;
            else if (t.sp < kStackSmem + kStackLocal) lstack[t.sp - kStackSmem] = e;
            else {
                atomicOr(errFlag, kErrStackOverflow);
                return true;
            }
            ++t.sp;
        }
        if (child >= s.numNodes) {
            atomicOr(errFlag, kErrBadIndex);
            return true;
        }
        uint32_t hits, imask;
        intersect_node(s.nodes, child, t.r, t.ix, t.iy, t.iz, t.octInv, t.tBest, t.gBase, t.tBase, hits, imask,
                       t.tMask);
        t.gBits = hits | (imask << 8);
        if (t.tMask && t.tBase + (31u - __clz(t.tMask)) >= s.numTris) {
            atomicOr(errFlag, kErrBadIndex);
            return true;
        }
    }
    while (t.tMask) {
        uint32_t j = __ffs(t.tMask) - 1;
        t.tMask &= t.tMask - 1;
        const float4* tp = s.tris + 3 * (size_t)(t.tBase + j);
        float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
        float th;
        // closest hit: tBest <= tmax, so the update test below implies th <= tmax;
        // any hit: tBest is tmax until the first hit, which ends the ray
        if (mt_rn(t.r, a, b, c, th) && th >= t.r.tmin && (!kAnyHit || th <= t.tBest)) {
            if (kAnyHit) {
                t.tBest = th;
                t.lBest = t.tBase + j;
                return true;
            }
            if (th < t.tBest || (th == t.tBest && __float_as_uint(a.w) < record_prim(s.tris, t.lBest))) {
                t.tBest = th;
                t.lBest = t.tBase + j;
            }
        }
    }
    if (!(t.gBits & 0xffu)) {
        if (t.sp == 0) return true;
        --t.sp;
        uint2 e = t.sp < kStackSmem ? sstack[t.sp * kTraceBlock + tid] : lstack[t.sp - kStackSmem];
        t.gBase = e.x;
        t.gBits = e.y;
    }
    return false;
}

template <bool kAnyHit>
__device__ __forceinline__ bool traverse(const DevScene& s, const Ray& r, float& tBest, uint32_t& pBest,
                                         uint32_t& mBest, uint2* sstack, uint32_t* errFlag) {
    uint2 lstack[kStackLocal];
    Trav t;
    trav_init(t, r);
    while (!trav_step<kAnyHit>(s, t, sstack, lstack, errFlag)) {
    }
    tBest = t.tBest;
    pBest = record_prim(s.tris, t.lBest);
    mBest = record_material(s.tris, t.lBest);
    return t.lBest != kNoHit;
}

__device__ __forceinline__ Ray load_ray8(const float* p) {
    float4 a = *reinterpret_cast<const float4*>(p);
    float4 b = *reinterpret_cast<const float4*>(p + 4);
    return Ray{a.x, a.y, a.z, b.x, b.y, b.z, a.w, b.w};
}

__global__ void __launch_bounds__(kTraceBlock) k_closest_query(DevScene s, const float* __restrict__ rays, uint32_t n,
                                                               float* tOut, uint32_t* pOut, uint32_t* err) {
    __shared__ uint2 sstack[kStackSmem * kTraceBlock];
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Ray r = load_ray8(rays + 8 * (size_t)i);
    float t;
    uint32_t p, m;
    bool hit = traverse<false>(s, r, t, p, m, sstack, err);
    tOut[i] = hit ? t : __int_as_float(0x7f800000);
    pOut[i] = hit ? p : kNoHit;
}

__global__ void __launch_bounds__(kTraceBlock) k_occluded_query(DevScene s, const float* __restrict__ rays,
                                                                uint32_t n, uint32_t* out, uint32_t* err) {
    __shared__ uint2 sstack[kStackSmem * kTraceBlock];
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Ray r = load_ray8(rays + 8 * (size_t)i);
    float t;
    uint32_t p, m;
    out[i] = traverse<true>(s, r, t, p, m, sstack, err) ? 1u : 0u;
}

void launch_closest_query(const DevScene& s, const float* rays, uint32_t n, float* t, uint32_t* prim, uint32_t* err,
                          cudaStream_t st) {
    if (!n) return;
    k_closest_query<<<(n + kTraceBlock - 1) / kTraceBlock, kTraceBlock, 0, st>>>(s, rays, n, t, prim, err);
}
void launch_occluded_query(const DevScene& s, const float* rays, uint32_t n, uint32_t* occ, uint32_t* err,
                           cudaStream_t st) {
    if (!n) return;
    k_occluded_query<<<(n + kTraceBlock - 1) / kTraceBlock, kTraceBlock, 0, st>>>(s, rays, n, occ, err);
}

// ---------------------------------------------------------------------------
// Wavefront trace kernels.  A path's state travels with it: a lane reads its ray
// from the input queue entry it fetched and, when the ray is done, copies the
// whole entry into the next queue at the position a warp-aggregated append (one
// ballot per destination, one atomicAdd by the lowest lane) handed out, so the
// lanes of a warp write consecutive entries.  Queue entries are read and written
// once per pass, so they go through the cache with the streaming (evict-first)
// policy (__ldcs / __stcs) and leave L1 to the BVH nodes and triangle records.
__device__ __forceinline__ uint32_t warp_append_pos(uint32_t* counter, bool pred, uint32_t cap, uint32_t* err) {
    uint32_t b = __ballot_sync(0xffffffffu, pred);
    if (!b) return kInvalidSlot;
    uint32_t lane = threadIdx.x & 31u;
    uint32_t leader = __ffs(b) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(b));
    base = __shfl_sync(0xffffffffu, base, leader);
    uint32_t pos = base + __popc(b & ((1u << lane) - 1u));
    if (pred && pos >= cap) {
        atomicOr(err, kErrQueueOverflow);
        return kInvalidSlot;
    }
    return pred ? pos : kInvalidSlot;
}

__device__ __forceinline__ PathQ pick_bucket(const Queues& q, uint32_t b) {
    switch (b) {
        case kBucketLambert: return q.bucket[kBucketLambert];
        case kBucketDielectric: return q.bucket[kBucketDielectric];
        case kBucketGGX: return q.bucket[kBucketGGX];
        default: return q.bucket[kBucketOther];
    }
}

// Persistent traversal: each warp keeps its lanes busy by fetching new rays from
// the queue (one warp-aggregated atomic on a per-launch fetch counter) whenever
// fewer than kRefillAt lanes still have a ray in flight, instead of waiting for
// the slowest ray of a fixed batch (Aila & Laine 2009, "Understanding the
// efficiency of ray traversal on GPUs").
#ifndef WRK_REFILL_AT
#define WRK_REFILL_AT 16
#endif
// Resident blocks per SM of each persistent trace kernel (its register budget is
// 65536 / (128 x blocks)); the grid is that many blocks per SM.
#ifndef WRK_TRACE_EXT_BLOCKS
#define WRK_TRACE_EXT_BLOCKS 9
#endif
#ifndef WRK_TRACE_SHADOW_BLOCKS
#define WRK_TRACE_SHADOW_BLOCKS 8
#endif
constexpr int kRefillAt = WRK_REFILL_AT;
template <bool kAnyHit, bool kMulti>
struct TraceBlocks {
    static constexpr int value = kMulti ? 8 : (kAnyHit ? WRK_TRACE_SHADOW_BLOCKS : WRK_TRACE_EXT_BLOCKS);
};

// Adds a miss's environment term and accumulates the path into its request's sums
// (__miss__trace + the raygen miss branch, trace.cu:143-148).
__device__ __forceinline__ void miss_accumulate(const DevScene& sc, const Frame& f, float4 th, float4 rd, float3 dir) {
    float3 e = make_float3(sc.env[0], sc.env[1], sc.env[2]);
    if ((f.flags & WRK_FLAG_ENV_MAP) && sc.envMap) e = env_lookup(sc.envMap, sc.envW, sc.envH, dir);
    float3 L = make_float3(rd.x + th.x * e.x, rd.y + th.y * e.y, rd.z + th.z * e.z);
    L = clamp_fireflies(L, f.fireflyClamp);
    atomicAdd(f.accum + __float_as_uint(rd.w), make_float4(L.x, L.y, L.z, 0.0f));
}

__device__ __forceinline__ void count_ended_t(SlotCtl* ctl, bool ended, uint32_t slot) {
    const uint32_t m = __ballot_sync(0xffffffffu, ended);
    if (!m) return;
    const uint32_t peers = __match_any_sync(0xffffffffu, ended ? slot : 0xffffffffu) & m;
    if (ended && (uint32_t)(__ffs(peers) - 1) == (threadIdx.x & 31u))
        atomicAdd(&ctl[slot].finished, (unsigned long long)__popc(peers));
}

// kMulti: the batch's requests may use different scenes; a lane loads the
// geometry of its ray's scene when it fetches the ray.  Otherwise scene s0.
template <bool kAnyHit, bool kMulti>
__global__ void __launch_bounds__(kTraceBlock, (TraceBlocks<kAnyHit, kMulti>::value))
    k_trace_persistent(DevScene s0, Queues q) {
    __shared__ uint2 sstack[kStackSmem * kTraceBlock];
    uint2 lstack[kStackLocal];
    Counters* c = q.ctr;
    const uint32_t cur = c->cur;
    const uint32_t n = min(kAnyHit ? c->shd[cur].v : c->ext[cur].v, q.capacity);
    const PathQ in = kAnyHit ? q.shd[cur] : q.ext[cur];
    uint32_t* fetch = kAnyHit ? &c->fetchShadow.v : &c->fetchExtension.v;
    const uint32_t lane = threadIdx.x & 31u;
    // the shadow stage continues every Lambert path it traces (statistics slot)
    if (kAnyHit && blockIdx.x == 0 && threadIdx.x == 0) c->bucket[kBucketLambertResume].v = n;
    Trav t;
    TraceGeom geo{s0.nodes, s0.tris, s0.numNodes, s0.numTris};
    uint32_t sceneIdx = 0;
    uint32_t idx = 0;
    bool active = false, exhausted = false;
    while (true) {
        uint32_t idle = __ballot_sync(0xffffffffu, !active && !exhausted);
        if (idle) {
            uint32_t leader = __ffs(idle) - 1, base = 0;
            if (lane == leader) base = atomicAdd(fetch, (uint32_t)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (!active && !exhausted) {
                idx = base + __popc(idle & ((1u << lane) - 1u));
                if (idx < n) {
                    float4 o = kAnyHit ? __ldcs(in.sh_o + idx) : __ldcs(in.ray_o + idx);
                    float4 d = kAnyHit ? __ldcs(in.sh_d + idx) : __ldcs(in.ray_d + idx);
                    // a shadow entry keeps its request slot where tmin would be
                    const uint32_t slot = kAnyHit ? __float_as_uint(o.w) : slot_of(__ldcs(&in.st[idx].w));
                    if (kAnyHit) o.w = kShadowTmin;
                    if constexpr (kMulti) {
                        sceneIdx = q.req[slot].scene;
                        const DevScene& sc = q.scenes[sceneIdx];
                        geo = TraceGeom{sc.nodes, sc.tris, sc.numNodes, sc.numTris};
                    }
                    trav_init(t, Ray{o.x, o.y, o.z, d.x, d.y, d.z, o.w, d.w});
                    active = true;
                } else {
                    exhausted = true;
                }
            }
        }
        if (__all_sync(0xffffffffu, exhausted && !active)) break;
        // once the queue is drained nothing can refill a lane: run to completion
        const int refillAt = __any_sync(0xffffffffu, exhausted) ? 1 : kRefillAt;
        bool fin = false;
        do {
            if (active && !fin) fin = trav_step<kAnyHit>(geo, t, sstack, lstack, &c->error);
        } while (__popc(__ballot_sync(0xffffffffu, active && !fin)) >= refillAt);
        const bool done = active && fin;
        if (kAnyHit) {
            // Shadow stage of __raygen__trace (trace.cu:27-51): add the NEE
            // contribution if nothing lies in [tmin, tmax], then carry out what the
            // Lambert shade decided for the path after its shadow ray: continue
            // with the prepared extension ray, accumulate, or drop.
            uint32_t cont = kContDrop, slot = 0;
            if (done) {
                const float4 cc = __ldcs(in.sh_c + idx);
                const uint32_t w = __float_as_uint(cc.w);
                const bool lit = t.lBest == kNoHit;
                cont = w & 3u;
                slot = __float_as_uint(in.sh_o[idx].w);
                if (cont == kContExt) {
                    // the continuing path's entry waits in the next extension queue
                    const uint32_t pos = w >> 2;
                    if (lit && pos < q.capacity) {
                        const PathQ o = cur ? q.ext[0] : q.ext[1];
                        const float4 rd = o.rad[pos];
                        o.rad[pos] = make_float4(rd.x + cc.x, rd.y + cc.y, rd.z + cc.z, rd.w);
                    }
                } else if (cont == kContAccumulate) {
                    float4 rd = in.rad[idx];
                    if (lit) rd = make_float4(rd.x + cc.x, rd.y + cc.y, rd.z + cc.z, rd.w);
                    const Frame& f = q.req[slot];
                    const float3 L = clamp_fireflies(make_float3(rd.x, rd.y, rd.z), f.fireflyClamp);
                    atomicAdd(f.accum + __float_as_uint(rd.w), make_float4(L.x, L.y, L.z, 0.0f));
                }
            }
            count_ended_t(q.ctl, done && cont != kContExt, slot);
        } else {
            uint32_t bucket = kNumBuckets;
            float4 th = make_float4(0, 0, 0, 0), rd = make_float4(0, 0, 0, 0);
            uint4 st = make_uint4(0, 0, 0, 0);
            bool missed = false;
            uint32_t pBest = kNoHit, mBest = 0;
            if (done) {
                th = __ldcs(in.thr + idx);
                rd = __ldcs(in.rad + idx);
                st = __ldcs(in.st + idx);
                // prim, material and material bucket from the hit's record (just
                // tested, so cached)
                pBest = record_prim(geo.tris, t.lBest);
                mBest = record_material(geo.tris, t.lBest);
                const Frame& f = q.req[slot_of(st.w)];
                if (pBest != kNoHit) bucket = __float_as_uint(__ldg(geo.tris + 3 * (size_t)t.lBest + 2).w);
                else if constexpr (kMulti) miss_accumulate(q.scenes[sceneIdx], f, th, rd, make_float3(t.r.dx, t.r.dy, t.r.dz));
                else miss_accumulate(s0, f, th, rd, make_float3(t.r.dx, t.r.dy, t.r.dz));
                missed = pBest == kNoHit;
            }
            count_ended_t(q.ctl, missed, slot_of(st.w));
            // textured Lambert hits fill the Lambert queue from its last entry down
            const bool texL = bucket == (kBucketLambert | kRecTextured);
            if (bucket != kNumBuckets) bucket = texL ? (uint32_t)kBucketLambert : min(bucket, (uint32_t)kBucketOther);
            uint32_t pos = kInvalidSlot;
#pragma unroll
            for (uint32_t b = 0; b < kBucketLambertResume; ++b) {
                uint32_t pb = warp_append_pos(&c->bucket[b].v, bucket == b && !texL, q.capacity, &c->error);
                if (bucket == b && !texL) pos = pb;
            }
            {
                const uint32_t pt = warp_append_pos(&c->lambertTex.v, texL, q.capacity, &c->error);
                if (texL && pt != kInvalidSlot) pos = q.capacity - 1u - pt;
            }
            if (pos != kInvalidSlot) {
                const PathQ o = pick_bucket(q, bucket);
                __stcs(o.ray_o + pos, make_float4(t.r.ox, t.r.oy, t.r.oz, t.r.tmin));
                __stcs(o.ray_d + pos, make_float4(t.r.dx, t.r.dy, t.r.dz, t.tBest));
                o.hit[pos] = make_float4(t.tBest, __uint_as_float(pBest), __uint_as_float(mBest),
                                         __uint_as_float(t.lBest));
                __stcs(o.thr + pos, th);
                __stcs(o.rad + pos, rd);
                __stcs(o.st + pos, st);
            }
        }
        if (done) active = false;
    }
}

void launch_trace_extension(const DevScene& s, const Queues& q, bool multi, int numSMs, cudaStream_t st) {
    if (multi) k_trace_persistent<false, true><<<numSMs * TraceBlocks<false, true>::value, kTraceBlock, 0, st>>>(s, q);
    else k_trace_persistent<false, false><<<numSMs * TraceBlocks<false, false>::value, kTraceBlock, 0, st>>>(s, q);
}
void launch_trace_shadow(const DevScene& s, const Queues& q, bool multi, int numSMs, cudaStream_t st) {
    if (multi) k_trace_persistent<true, true><<<numSMs * TraceBlocks<true, true>::value, kTraceBlock, 0, st>>>(s, q);
    else k_trace_persistent<true, false><<<numSMs * TraceBlocks<true, false>::value, kTraceBlock, 0, st>>>(s, q);
}

}  // namespace wrk
