// Wavefront path-tracing kernels: per-iteration control, camera-path generation,
// material-bucketed shading, and the final resolve.  Together with the trace
// kernels (trace.cu) they replace libWR's host loop and its raygen / closest-hit /
// shade / compact programs (paths inside trianglestrip/OfflineRenderer):
//   libWR/src/internal/renderer.cpp:190-313, libWR/kernels/trace.cu:17-319,
//   libWR/kernels/shade.cu:24-85, libWR/kernels/materials/*.cuh,
//   libWR/kernels/compact.cu:6-17.
//
// A path's state travels with it through SoA queues (see wrk_internal.h).  Each
// iteration:
//   control   (1 thread)  swaps the extension/shadow queue buffers, clears the
//                         material buckets, and sizes the batch of new camera paths
//                         by the room the live paths leave
//   generate              camera rays for the next (sample, pixel) work items,
//                         appended to the extension queue
//   trace_extension       closest hit -> material bucket, or miss -> accumulate
//   trace_shadow          any hit for pending NEE rays; adds the contribution if
//                         unoccluded, then continues / accumulates / drops the path
//   shade<bucket> x4      closest-hit attributes, guides, emission, BSDF, RR;
//                         appends to the next extension / shadow queue
// A path carries its own iteration count; after `maxIter` iterations (8 = the
// reference host loop's cap) a live path is dropped unaccumulated, as libWR does.
// RNG is keyed by (pixel, sample), so the image does not depend on queue order.
#include "wrk_internal.h"
#include "wrk_shading.cuh"
#include "wrk_tri.cuh"

namespace wrk {

constexpr int kShadeBlock = 256;

__device__ __forceinline__ uint32_t append_pos(uint32_t* counter, bool pred, uint32_t cap, uint32_t* err) {
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

// Paths that ended in this warp, counted per request slot with one atomic per
// distinct slot (warp-aggregated with __match_any_sync).  All lanes call it.
__device__ __forceinline__ void count_ended(SlotCtl* ctl, bool ended, uint32_t slot) {
    const uint32_t m = __ballot_sync(0xffffffffu, ended);
    if (!m) return;
    const uint32_t peers = __match_any_sync(0xffffffffu, ended ? slot : 0xffffffffu) & m;
    if (ended && (uint32_t)(__ffs(peers) - 1) == (threadIdx.x & 31u))
        atomicAdd(&ctl[slot].finished, (unsigned long long)__popc(peers));
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// One thread: folds the last iteration's statistics, swaps the queue buffers,
// marks finished requests done, and hands the room the live paths leave to the
// active requests' remaining work items in admission (FIFO) order.
__global__ void k_control(Queues q) {
    Counters* c = q.ctr;
    for (int b = 0; b < kNumBuckets; ++b) c->bucketTotal[b] += c->bucket[b].v;
    c->bucketTotal[kBucketLambert] += c->lambertTex.v;
    c->lambertTex.v = 0;
    uint32_t cur = c->cur ^ 1u;
    uint32_t out = cur ^ 1u;
    c->cur = cur;
    // the Lambert continuations the last iteration placed at the front of ext[out];
    // those whose shadow query the shade answered have no shadow entry and count
    // as live paths here
    c->ext[out].v = c->cont.v;
    c->cont.v = 0;
    const uint32_t direct = c->contDirect.v;
    c->contDirect.v = 0;
    c->shdRays += c->shadowAnswered.v;
    c->shadowAnswered.v = 0;
    c->shd[out].v = 0;
    for (int b = 0; b < kNumBuckets; ++b) c->bucket[b].v = 0;
    c->fetchExtension.v = 0;
    c->fetchShadow.v = 0;
    // every live path holds one extension or shadow entry: the rest is room for new ones
    uint32_t live = c->ext[cur].v + c->shd[cur].v + direct;
    if (c->ext[cur].v > q.capacity || c->shd[cur].v > q.capacity || live > q.capacity) {
        c->error |= kErrQueueOverflow;
        live = q.capacity;
    }
    unsigned long long room = q.capacity - live;
    const uint32_t n = min(q.genOrder[0], kMaxSlots);
    uint32_t g = 0, ns = 0, active = 0;
    const unsigned long long now = global_ns();
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t slot = q.genOrder[1 + k];
        if (slot >= kMaxSlots) continue;
        SlotCtl& sc = q.ctl[slot];
        if (sc.state != kSlotActive) continue;
        if (slot_finished(sc)) {
            sc.state = kSlotDone;
            sc.doneNs = now;
            sc.doneIter = c->iteration;
            continue;
        }
        ++active;
        const unsigned long long take = min(sc.workTotal - sc.workNext, room);
        if (take == 0) continue;
        q.seg[ns] = GenSeg{sc.workNext, slot, (uint32_t)take, g, 0u};
        ++ns;
        sc.workNext += take;
        room -= take;
        g += (uint32_t)take;
    }
    c->activeSlots = active;
    c->numSeg = ns;
    c->genCount = g;
    c->genExtBase = c->ext[cur].v;
    c->ext[cur].v += g;
    c->paths += g;
    c->extRays += c->ext[cur].v;
    c->shdRays += c->shd[cur].v;
    c->shdTraced += c->shd[cur].v;
    c->iteration += 1;
}

void launch_control(const Queues& q, cudaStream_t st) { k_control<<<1, 1, 0, st>>>(q); }

// One thread: the conditional graph node repeats its chunk while any request in the
// admission order is still active and unfinished, no device error was raised and
// the iteration bound is not reached.
__global__ void k_loop_cond(cudaGraphConditionalHandle h, Queues q) {
    const Counters* c = q.ctr;
    const uint32_t n = min(q.genOrder[0], kMaxSlots);
    bool busy = false;
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t slot = q.genOrder[1 + k];
        if (slot < kMaxSlots && q.ctl[slot].state == kSlotActive && !slot_finished(q.ctl[slot])) busy = true;
    }
    const bool go = busy && c->error == 0 && c->iteration < c->iterLimit;
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

void launch_loop_cond(cudaGraphConditionalHandle h, const Queues& q, cudaStream_t st) {
    k_loop_cond<<<1, 1, 0, st>>>(h, q);
}

// Camera ray for (pixel, sample) of the request a work item belongs to: trace.cu:54-125.
__global__ void __launch_bounds__(kShadeBlock) k_generate(Queues q) {
    __shared__ GenSeg seg[kMaxSlots];
    Counters* c = q.ctr;
    const uint32_t g = c->genCount;
    const uint32_t eb = c->genExtBase;
    const uint32_t ns = min(c->numSeg, kMaxSlots);
    for (uint32_t k = threadIdx.x; k < ns; k += blockDim.x) seg[k] = q.seg[k];
    __syncthreads();
    const PathQ o = c->cur ? q.ext[1] : q.ext[0];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < g; i += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = ns;  // the last segment starting at or before i
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (seg[mid].extOffset <= i) lo = mid;
            else hi = mid;
        }
        const GenSeg sg = seg[lo];
        const Frame& f = q.req[sg.slot];
        const uint32_t e = eb + i;
        const unsigned long long w = sg.workBase + (i - sg.extOffset);
        const uint32_t perSample = f.perSample, width = f.width, tilesX = f.tilesX;
        // blocks of K samples: within a block, each group of 32 work items covers
        // 32/K consecutive pixel positions, with the K samples of a pixel adjacent
        const uint32_t K = f.interleave;
        const unsigned long long blk = (unsigned long long)perSample * K;
        const uint32_t idx = (uint32_t)(w % blk), ln = idx & 31u;
        uint32_t sample = f.sampleOffset + (uint32_t)(w / blk) * K + ln % K;
        uint32_t j = (idx >> 5) * (32u / K) + ln / K;
        uint32_t x, y;
        if (tilesX) {
            uint32_t tile = j >> 5, lane = j & 31u;
            x = (tile % tilesX) * 8u + (lane & 7u);
            y = (tile / tilesX) * 4u + (lane >> 3);
        } else {
            x = j % width;
            y = j / width;
        }
        uint32_t pixel = y * width + x;
        uint32_t seed = path_seed(pixel, sample, f.seed);
        uint32_t js = seed;
        float r1 = lcg_randf(js);
        float r2 = lcg_randf(js);
        float nx = (2.0f * ((float)x + r1) / (float)width - 1.0f) * f.aspect;
        float ny = 1.0f - 2.0f * ((float)y + r2) / (float)f.height;
        float3 fwd = f3(f.fwd[0], f.fwd[1], f.fwd[2]), rt = f3(f.right[0], f.right[1], f.right[2]),
               up = f3(f.up[0], f.up[1], f.up[2]), pos = f3(f.pos[0], f.pos[1], f.pos[2]);
        const float tanHalf = f.tanHalf;
        float3 dir = normalize(add(add(fwd, mul(mul(rt, nx), tanHalf)), mul(mul(up, ny), tanHalf)));
        float3 ro = pos, rd = dir;
        const float lens = f.lens, focal = f.focal;
        if (lens > 0.0f && focal > 0.0f) {
            float r3 = lcg_randf(js), r4 = lcg_randf(js);
            float th = 2.0f * 3.14159265f * r3;
            float rad = sqrtf(r4) * lens;
            float sn, ct;
            sincosf(th, &sn, &ct);
            float3 off = f3(rt.x * rad * ct + up.x * rad * sn, rt.y * rad * ct + up.y * rad * sn,
                            rt.z * rad * ct + up.z * rad * sn);
            float3 fp = f3(pos.x + dir.x * focal, pos.y + dir.y * focal, pos.z + dir.z * focal);
            ro = f3(pos.x + off.x, pos.y + off.y, pos.z + off.z);
            rd = normalize(f3(fp.x - ro.x, fp.y - ro.y, fp.z - ro.z));
        }
        __stcs(o.ray_o + e, make_float4(ro.x, ro.y, ro.z, 0.0001f));
        __stcs(o.ray_d + e, make_float4(rd.x, rd.y, rd.z, 1e20f));
        __stcs(o.thr + e, make_float4(1.0f, 1.0f, 1.0f, 1.0f));
        __stcs(o.rad + e, make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(pixel)));
        __stcs(o.st + e, make_uint4(seed, 0u, 0u, kFlagFirstHit | kFlagPrevDelta | (sg.slot << kSlotShift)));
    }
}

void launch_generate(const Queues& q, int grid, cudaStream_t st) { k_generate<<<grid, kShadeBlock, 0, st>>>(q); }

// ---------------------------------------------------------------------------
// Closest-hit attributes (trace.cu:167-264): projected barycentrics, geometric and
// interpolated shading normals (both flipped to face the ray), uv.
struct HitAttr {
    float3 pos, n, ng, e1, e2;
    float u, v;
    uint32_t mat, prim;
};

__device__ __forceinline__ float3 vtx3(const float* v, uint32_t i) {
    return f3(__ldg(v + 3 * i), __ldg(v + 3 * i + 1), __ldg(v + 3 * i + 2));
}

// The hit triangle's v0, v1 - v0 and v2 - v0 come from its BVH leaf record (at the
// leaf position the trace kernel stored with the hit: three independent 16-byte
// loads instead of index -> vertex chains); the builder writes them with correctly
// rounded subtractions, the same values sub(v1, v0), sub(v2, v0) give.  Indices are
// loaded only for interpolated normals and uvs.
__device__ __forceinline__ HitAttr hit_program(const DevScene& s, float3 o, float3 d, float t, uint32_t prim,
                                               uint32_t mat, uint32_t leafPos) {
    HitAttr h;
    float3 hp = f3(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
    const float4* tp = s.tris + 3 * (size_t)leafPos;
    const float4 ta = __ldg(tp), tb = __ldg(tp + 1), tc = __ldg(tp + 2);
    uint32_t i0 = 0, i1 = 0, i2 = 0;
    if (s.nrm || s.uv) {
        i0 = __ldg(s.idx + 3 * prim);
        i1 = __ldg(s.idx + 3 * prim + 1);
        i2 = __ldg(s.idx + 3 * prim + 2);
    }
    float3 a = f3(ta.x, ta.y, ta.z);
    float3 e1 = f3(tb.x, tb.y, tb.z), e2 = f3(tc.x, tc.y, tc.z);
    float3 gn = normalize(cross(e1, e2));
    float3 vp = sub(hp, a);
    float d00 = dot(e1, e1), d01 = dot(e1, e2), d11 = dot(e2, e2), d20 = dot(vp, e1), d21 = dot(vp, e2);
    float den = d00 * d11 - d01 * d01;
    float bv = (d11 * d20 - d01 * d21) / fmaxf(den, 1e-8f);
    float bw = (d00 * d21 - d01 * d20) / fmaxf(den, 1e-8f);
    float bu = 1.0f - bv - bw;
    float3 sn = gn;
    if (s.nrm) {
        float3 n0 = vtx3(s.nrm, i0), n1 = vtx3(s.nrm, i1), n2 = vtx3(s.nrm, i2);
        if (length(n0) > 1e-6f && length(n1) > 1e-6f && length(n2) > 1e-6f) {
            sn = normalize(add(add(mul(bu, n0), mul(bv, n1)), mul(bw, n2)));
            if (dot(sn, gn) < 0.0f) sn = neg(sn);
        }
    }
    h.ng = dot(gn, d) > 0.0f ? neg(gn) : gn;
    h.n = dot(sn, d) > 0.0f ? neg(sn) : sn;
    h.pos = hp;
    h.e1 = e1;
    h.e2 = e2;
    h.mat = mat;
    h.prim = prim;
    if (s.uv) {
        h.u = bu * __ldg(s.uv + 2 * i0) + bv * __ldg(s.uv + 2 * i1) + bw * __ldg(s.uv + 2 * i2);
        h.v = bu * __ldg(s.uv + 2 * i0 + 1) + bv * __ldg(s.uv + 2 * i1 + 1) + bw * __ldg(s.uv + 2 * i2 + 1);
    } else {
        h.u = h.v = 0.0f;
    }
    return h;
}

// getMaterialAlbedo (materials.cuh:25-29): 1-based texture id, else the constant.
__device__ __forceinline__ float3 albedo_of(const DevScene& s, const wrk_material& m, float u, float v) {
    if (m.albedoTextureId != 0 && m.albedoTextureId <= s.numTex) {
        TexInfo ti = s.tex[m.albedoTextureId - 1];
        if (ti.w == 0) return f3(1, 1, 1);
        float4 c = tex_fetch(s.texels + ti.offset, ti.w, ti.h, u, v);
        return f3(c.x, c.y, c.z);
    }
    return f3(m.albedo[0], m.albedo[1], m.albedo[2]);
}

// getEffectiveNormal (normal_map.cuh:40-60).
__device__ __forceinline__ float3 normal_mapped(const DevScene& s, const wrk_material& m, const HitAttr& h) {
    if (m.normalTextureId > 0 && m.normalTextureId <= s.numTex) {
        TexInfo ti = s.tex[m.normalTextureId - 1];
        float4 c = ti.w ? tex_fetch(s.texels + ti.offset, ti.w, ti.h, h.u, h.v) : make_float4(0.5f, 0.5f, 1.0f, 1.0f);
        float3 tg, bt;
        frame(h.n, tg, bt);
        float3 q = f3(c.x * 2.0f - 1.0f, c.y * 2.0f - 1.0f, c.z * 2.0f - 1.0f);
        return normalize(f3(tg.x * q.x + bt.x * q.y + h.n.x * q.z, tg.y * q.x + bt.y * q.y + h.n.y * q.z,
                            tg.z * q.x + bt.z * q.y + h.n.z * q.z));
    }
    return h.n;
}

// kOutCont: a Lambert path whose shadow query was answered in the shade (its light
// blocks the ray) and that continues: only its next extension entry is written.
enum : int { kOutNone = 0, kOutExt = 1, kOutShadow = 2, kOutDone = 3, kOutCont = 4 };

struct PathRegs {
    float3 o, d, thr, rad;
    float prevPdf;
    uint32_t pixel, seed, dim, depth, iter, flags;
};

__device__ __forceinline__ void accumulate(const Frame& f, const PathRegs& r) {
    float3 L = clamp_fireflies(r.rad, f.fireflyClamp);
    atomicAdd(f.accum + r.pixel, make_float4(L.x, L.y, L.z, 0.0f));
}

// setupNextBounce (material_common.cuh:55-71); returns the outcome.
__device__ __forceinline__ int next_bounce(const Frame& f, PathRegs& r, const HitAttr& h, float3 nd) {
    r.d = nd;
    r.o = offset_origin(h.pos, h.n, nd);
    r.depth += 1;
    if (r.depth >= f.maxBounces) {
        accumulate(f, r);
        return kOutDone;
    }
    return kOutExt;
}

__device__ __forceinline__ bool rr(const Frame& f, PathRegs& r, bool delta) {
    float3 nt;
    float xi = rnd_dim(r.seed, r.dim++);
    if (!russian_roulette(r.thr, r.depth, f.rrStart, xi, nt, delta)) {
        accumulate(f, r);
        return false;
    }
    r.thr = nt;
    return true;
}

// NEE light sample (lambertian.cuh:17-63, ggx_material.cuh:51-95): picks a light
// through the power CDF, samples a point on it; returns false if not facing.
struct LightSample {
    float3 toLight, le;
    float dist, d2, lpdf, cosTheta;
    uint32_t light;  // the sampled entry of the emissive list
};
// The light record (emissive list order): v0 | triangle id, v1, v2, emission.
__device__ __forceinline__ bool sample_light(const DevScene& s, PathRegs& r, const HitAttr& h, LightSample& ls) {
    float lu = rnd_dim(r.seed, r.dim++);
    uint32_t li = cdf_lower_bound(lu, s.cdf, s.numEmissive);
    const float4* lr = s.lights + 4 * (size_t)li;
    const float4 l0 = __ldg(lr), l1 = __ldg(lr + 1), l2 = __ldg(lr + 2), l3 = __ldg(lr + 3);
    float3 a = f3(l0.x, l0.y, l0.z), b = f3(l1.x, l1.y, l1.z), c = f3(l2.x, l2.y, l2.z);
    // two uniforms in one call: the earlier dimension is the first argument
    float u1 = rnd_dim(r.seed, r.dim++);
    float u2 = rnd_dim(r.seed, r.dim++);
    float3 ln;
    float la;
    float3 lp = sample_triangle(u1, u2, a, b, c, ln, la);
    float3 tl = f3(lp.x - h.pos.x, lp.y - h.pos.y, lp.z - h.pos.z);
    float d2 = dot(tl, tl);
    float dist = sqrtf(d2);
    tl = f3(tl.x / dist, tl.y / dist, tl.z / dist);
    float ct = dot(h.n, tl);
    float cl = -dot(ln, tl);
    if (!(ct > 0.0f && cl > 0.0f)) return false;
    float pa = 1.0f / ((float)s.numEmissive * la);
    ls.lpdf = pa * d2 / fmaxf(cl, 1e-8f);
    ls.toLight = tl;
    ls.dist = dist;
    ls.d2 = d2;
    ls.cosTheta = ct;
    ls.le = f3(l3.x, l3.y, l3.z);
    ls.light = li;
    return true;
}

// A Lambert hit that sends a shadow ray: the shadow ray, its contribution, and what
// the path does after the visibility test (kCont*; the path's next ray is in the
// path registers when it continues).
struct ShadowOut {
    float3 o, d, c;
    float dist;
    uint32_t cont;
    uint32_t light;     // the emissive-list entry of the light the ray aims at
    bool answered;      // the shadow query was answered here (the light blocks the ray)
};

// Shades entry i of a bucket; the path's next state is left in r (and so for a
// shadow ray).  Returns kOutExt / kOutShadow for a continuing path, kOutDone when
// it ended (accumulated or dropped).
template <uint32_t kBucket>
__device__ __forceinline__ int shade_one(const DevScene& s, const PathQ& in, uint32_t i, const Frame& f, PathRegs& r,
                                         ShadowOut& so, float4 o4, float4 d4, float4 h4, float4 t4, float4 r4,
                                         uint4 st) {
    r.o = f3(o4.x, o4.y, o4.z);
    r.d = f3(d4.x, d4.y, d4.z);
    r.thr = f3(t4.x, t4.y, t4.z);
    r.prevPdf = t4.w;
    r.rad = f3(r4.x, r4.y, r4.z);
    r.pixel = __float_as_uint(r4.w);
    r.seed = st.x;
    r.dim = st.y;
    r.depth = st.z & 0xffffu;
    r.iter = st.z >> 16;
    r.flags = st.w;
    uint32_t mat = __float_as_uint(h4.z);
    uint32_t prim = __float_as_uint(h4.y);
    uint32_t leafPos = __float_as_uint(h4.w);
    if (prim >= s.numTris || leafPos >= s.numTris) {
        atomicOr(f.err, kErrBadIndex);
        return kOutDone;
    }
    HitAttr h = hit_program(s, r.o, r.d, h4.x, prim, mat, leafPos);
    const bool matOk = mat < s.numMats;
    // getMaterialAlbedo is a pure function of (material, uv): fetched once for the
    // first-hit guide and the Lambert / dielectric shading (their buckets only ever
    // hold valid material ids)
    constexpr bool kShadeAlbedo = kBucket == kBucketLambert || kBucket == kBucketDielectric;
    float3 al = f3(0.0f, 0.0f, 0.0f);
    if (kShadeAlbedo || (matOk && f.albedo && (r.flags & kFlagFirstHit))) al = albedo_of(s, s.mats[mat], h.u, h.v);
    // first-hit guides (trace.cu:267-286)
    if (r.flags & kFlagFirstHit) {
        if (matOk) {
            if (f.albedo) atomicAdd(f.albedo + r.pixel, make_float4(al.x, al.y, al.z, 0.0f));
            if (f.normal) atomicAdd(f.normal + r.pixel, make_float4(h.ng.x, h.ng.y, h.ng.z, 0.0f));
        }
        r.flags &= ~kFlagFirstHit;
    }
    int out = kOutNone;
    if (kBucket == kBucketOther) {
        if (!matOk) return kOutDone;  // shade.cu:35-38: terminated without accumulation
        const wrk_material& m = s.mats[mat];
        if (m.type == kEmissive) {  // emission with MIS (trace.cu:288-316)
            float w = 1.0f;
            if (f.useNEE && r.depth > 0 && !(r.flags & kFlagPrevDelta) && s.numEmissive > 0) {
                float area = 0.5f * length(cross(h.e1, h.e2));
                float d2 = h4.x * h4.x;
                float cl = fabsf(dot(h.ng, r.d));
                float pa = 1.0f / ((float)s.numEmissive * area);
                float lpdf = pa * d2 / fmaxf(cl, 1e-8f);
                w = power_heuristic(r.prevPdf, lpdf);
            }
            float3 em = f3(m.emission[0], m.emission[1], m.emission[2]);
            r.rad = add(r.rad, mul(mul(r.thr, em), w));
        }
        accumulate(f, r);  // shadeEmissive / default branch: terminateRay
        return kOutDone;
    }
    const wrk_material& m = s.mats[mat];
    if (m.normalTextureId > 0) h.n = normal_mapped(s, m, h);
    if (kBucket == kBucketLambert) {
        bool shadow = false;
        if (f.useNEE && s.numEmissive > 0) {
            LightSample ls;
            if (sample_light(s, r, h, ls)) {
                float bpdf = cosine_pdf(ls.cosTheta);
                float w = power_heuristic(ls.lpdf, bpdf);
                float3 fb = f3(al.x / kPi * ls.cosTheta, al.y / kPi * ls.cosTheta, al.z / kPi * ls.cosTheta);
                float3 con = f3(r.thr.x * fb.x * ls.le.x * w / ls.lpdf, r.thr.y * fb.y * ls.le.y * w / ls.lpdf,
                                r.thr.z * fb.z * ls.le.z * w / ls.lpdf);
                if (finite3(con) && con.x >= 0.0f && con.y >= 0.0f && con.z >= 0.0f) {
                    so.o = offset_origin(h.pos, h.n, ls.toLight);
                    so.d = ls.toLight;
                    so.dist = ls.dist;
                    so.c = con;
                    so.light = ls.light;
                    shadow = true;
                }
            }
        }
        // cosine bounce (lambertian.cuh:65-147): its draws follow the light
        // sample's three whether or not a shadow ray is sent
        float3 tg, bt;
        frame(h.n, tg, bt);
        float u1 = rnd_dim(r.seed, r.dim++);
        float u2 = rnd_dim(r.seed, r.dim++);
        float pdf;
        float3 loc = cosine_hemisphere(u1, u2, pdf);
        float3 wd = to_world(loc, h.n, tg, bt);
        r.thr = mul(r.thr, al);
        r.prevPdf = pdf;
        r.flags &= ~kFlagPrevDelta;
        if (!shadow) {
            if (!rr(f, r, false)) return kOutDone;
            out = next_bounce(f, r, h, wd);
        } else {
            // The shadow ray is traced in the next iteration and the path goes on
            // after it (the reference resumes shading there).  Nothing below
            // depends on its outcome, so roulette, depth and the iteration bound
            // are applied now and the shadow kernel carries them out, adding the
            // contribution first if the light is visible.
            if (r.iter + 1u >= f.maxIter) return kOutDone;  // dropped with its shadow ray
            r.iter += 1u;
            float3 nt;
            const float xi = rnd_dim(r.seed, r.dim++);
            if (!russian_roulette(r.thr, r.depth, f.rrStart, xi, nt, false)) {
                so.cont = kContAccumulate;
            } else {
                r.thr = nt;
                r.d = wd;
                r.o = offset_origin(h.pos, h.n, wd);
                r.depth += 1;
                if (r.depth >= f.maxBounces) so.cont = kContAccumulate;
                else if (r.iter + 1u >= f.maxIter) so.cont = kContDrop;
                else {
                    r.iter += 1u;
                    so.cont = kContExt;
                }
            }
            // The shadow ray offset 1e-4 along the normal but ending 1e-5 short of
            // the light often hits the light triangle itself: then the query's
            // answer (occluded) is known here, the shadow kernel has nothing to do,
            // and the path only continues, accumulates or ends.
            const Ray sr{so.o.x, so.o.y, so.o.z, so.d.x, so.d.y, so.d.z, kShadowTmin, so.dist - kShadowTmin};
            if (so.light < s.numEmissive && light_blocks(s.lights + 4 * (size_t)so.light, sr)) {
                so.answered = true;
                if (so.cont == kContExt) return kOutCont;
                if (so.cont == kContAccumulate) accumulate(f, r);
                return kOutDone;
            }
            return kOutShadow;
        }
    } else if (kBucket == kBucketDielectric) {
        float3 wo = neg(r.d);
        float ci = dot(wo, h.n);
        float ei = 1.0f, et = m.ior;
        float3 n = h.n;
        if (ci < 0.0f) { ci = -ci; n = neg(n); ei = m.ior; et = 1.0f; }
        float F = fresnel_dielectric(ci, ei, et);
        float xi = rnd_dim(r.seed, r.dim++);
        if (xi < F) {
            r.d = sub(r.d, mul(n, 2.0f * dot(r.d, n)));
            r.thr = f3(r.thr.x * al.x, r.thr.y * al.y, r.thr.z * al.z);
        } else {
            float eta = ei / et;
            float s2 = eta * eta * (1.0f - ci * ci);
            if (s2 >= 1.0f) {
                r.d = sub(r.d, mul(n, 2.0f * dot(r.d, n)));
                r.thr = f3(r.thr.x * al.x, r.thr.y * al.y, r.thr.z * al.z);
            } else {
                float ct = sqrtf(fmaxf(0.0f, 1.0f - s2));
                float3 rf = add(mul(eta, r.d), mul(n, eta * ci - ct));
                r.d = rf;
                r.thr = f3(r.thr.x * al.x, r.thr.y * al.y, r.thr.z * al.z);
                float k = shading_correction(rf, h.n, h.ng);
                r.thr = f3(r.thr.x * k, r.thr.y * k, r.thr.z * k);
            }
        }
        r.flags |= kFlagPrevDelta;
        if (!rr(f, r, true)) return kOutDone;
        out = next_bounce(f, r, h, r.d);
    } else {  // GGX reflection
        float3 wo = neg(r.d);
        float3 alb = f3(m.albedo[0], m.albedo[1], m.albedo[2]);
        if (f.useNEE && s.numEmissive > 0) {
            LightSample ls;
            if (sample_light(s, r, h, ls)) {
                float3 fb = ggx_eval(wo, ls.toLight, h.n, alb, m.roughness, m.metallic, m.ior);
                float bpdf = ggx_pdf(wo, ls.toLight, h.n, m.roughness);
                float w = power_heuristic(ls.lpdf, bpdf);
                float3 con = f3(r.thr.x * fb.x * ls.le.x * ls.cosTheta * w / ls.lpdf,
                                r.thr.y * fb.y * ls.le.y * ls.cosTheta * w / ls.lpdf,
                                r.thr.z * fb.z * ls.le.z * ls.cosTheta * w / ls.lpdf);
                if (finite3(con) && con.x >= 0.0f && con.y >= 0.0f && con.z >= 0.0f)
                    r.rad = f3(r.rad.x + con.x, r.rad.y + con.y, r.rad.z + con.z);
            }
        }
        float3 tg, bt;
        frame(h.n, tg, bt);
        float3 wi = f3(0, 0, 0);
        float pdf = 0.0f;
        float u0 = rnd_dim(r.seed, r.dim++);
        float u1 = rnd_dim(r.seed, r.dim++);
        ggx_sample(wo, h.n, tg, bt, m.roughness, u0, u1, wi, pdf);
        float ct = dot(h.n, wi);
        if (pdf < 1e-5f || ct <= 0.0f) {
            accumulate(f, r);
            return kOutDone;
        }
        float3 fb = ggx_eval(wo, wi, h.n, alb, m.roughness, m.metallic, m.ior);
        if (!finite3(fb)) {
            accumulate(f, r);
            return kOutDone;
        }
        r.thr = f3(r.thr.x * fb.x * ct / pdf, r.thr.y * fb.y * ct / pdf, r.thr.z * fb.z * ct / pdf);
        r.prevPdf = pdf;
        r.flags &= ~kFlagPrevDelta;
        if (!rr(f, r, false)) return kOutDone;
        out = next_bounce(f, r, h, wi);
    }
    // continuing path: the reference's host loop stops after maxIter iterations
    // (renderer.cpp:213) and drops whatever is still alive
    if (out == kOutExt || out == kOutShadow) {
        if (r.iter + 1u >= f.maxIter) return kOutDone;  // dropped, nothing accumulated
        r.iter += 1u;
    }
    return out;
}

#ifndef WRK_SHADE_MIN_BLOCKS
#define WRK_SHADE_MIN_BLOCKS 4
#endif
// Shades one bucket.  A path's request (camera, settings, sums) comes from the
// slot in its state word; with kMulti its scene too, otherwise every path is in
// scene s0.  Paths that end are counted for their request.
template <uint32_t kBucket, bool kMulti, int kBlock>
__global__ void __launch_bounds__(kBlock, WRK_SHADE_MIN_BLOCKS * 256 / kBlock) k_shade(DevScene s0, Queues q) {
    Counters* c = q.ctr;
    const uint32_t cur = c->cur, nxt = cur ^ 1u;
    // the Lambert queue holds plain hits at [0, n) and textured ones at the far end,
    // [capacity - nt, capacity): threads take the plain ones first
    const uint32_t n = min(c->bucket[kBucket].v, q.capacity);
    const uint32_t nt = kBucket == kBucketLambert ? min(c->lambertTex.v, q.capacity - n) : 0u;
    const uint32_t total = n + nt;
    const PathQ in = q.bucket[kBucket];
    const PathQ ext = nxt ? q.ext[1] : q.ext[0];
    const PathQ shd = nxt ? q.shd[1] : q.shd[0];
    for (uint32_t base = blockIdx.x * blockDim.x; base < total; base += gridDim.x * blockDim.x) {
        const uint32_t t = base + threadIdx.x;
        const uint32_t i = t < n ? t : q.capacity - 1u - (t - n);
        PathRegs r;
        ShadowOut so;
        so.cont = kContDrop;
        so.answered = false;
        int out = kOutNone;
        uint32_t slot = 0;
        if (t < total) {
            // queue fields are read once: streaming loads keep L1 for materials,
            // textures, triangle and light records
            float4 o4 = __ldcs(in.ray_o + i), d4 = __ldcs(in.ray_d + i), h4 = __ldcs(in.hit + i), t4 = __ldcs(in.thr + i),
                   r4 = __ldcs(in.rad + i);
            uint4 st = __ldcs(in.st + i);
            slot = slot_of(st.w);
            const Frame& f = q.req[slot];
            if constexpr (kMulti) {
                out = shade_one<kBucket>(q.scenes[f.scene], in, i, f, r, so, o4, d4, h4, t4, r4, st);
            } else {
                out = shade_one<kBucket>(s0, in, i, f, r, so, o4, d4, h4, t4, r4, st);
            }
        }
        count_ended(q.ctl, out == kOutDone, slot);
        uint32_t pe = append_pos(&c->ext[nxt].v, out == kOutExt, q.capacity, &c->error);
        uint32_t ps = append_pos(&c->shd[nxt].v, out == kOutShadow, q.capacity, &c->error);
        // A Lambert path that continues after its shadow ray is placed now in the
        // extension buffer it will be traced from two iterations on (this
        // iteration's input, no longer read); the control kernel of the next
        // iteration starts that queue after these entries.
        // (decided from the outcome alone, so the three appends' atomics are issued
        // together; a queue overflow fails the whole render, whatever is written)
        const bool cx = (out == kOutShadow && so.cont == kContExt) || out == kOutCont;
        const uint32_t pc = append_pos(&c->cont.v, cx, q.capacity, &c->error);
        // shadow queries answered here: counted as traced, and the continuations
        // they leave (no shadow entry) held as live paths until traced
        {
            const uint32_t ans = __ballot_sync(0xffffffffu, so.answered);
            const uint32_t direct = __ballot_sync(0xffffffffu, out == kOutCont && pc != kInvalidSlot);
            if ((threadIdx.x & 31u) == 0) {
                if (ans) atomicAdd(&c->shadowAnswered.v, (uint32_t)__popc(ans));
                if (direct) atomicAdd(&c->contDirect.v, (uint32_t)__popc(direct));
            }
        }
        // entries are written once and read in a later pass: streaming stores
        if (pe != kInvalidSlot || pc != kInvalidSlot) {
            const PathQ o = pe != kInvalidSlot ? ext : (cur ? q.ext[1] : q.ext[0]);
            const uint32_t p = pe != kInvalidSlot ? pe : pc;
            __stcs(o.ray_o + p, make_float4(r.o.x, r.o.y, r.o.z, 0.0f));
            __stcs(o.ray_d + p, make_float4(r.d.x, r.d.y, r.d.z, 1e20f));
            __stcs(o.thr + p, make_float4(r.thr.x, r.thr.y, r.thr.z, r.prevPdf));
            __stcs(o.rad + p, make_float4(r.rad.x, r.rad.y, r.rad.z, __uint_as_float(r.pixel)));
            __stcs(o.st + p, make_uint4(r.seed, r.dim, (r.depth & 0xffffu) | (r.iter << 16), r.flags));
        }
        if (ps != kInvalidSlot) {
            // sh_o.w: the request slot (every shadow ray starts at kShadowTmin);
            // sh_c.w: the continuation code | the continuing path's position << 2
            uint32_t w = so.cont;
            if (cx) w = pc == kInvalidSlot ? (uint32_t)kContDrop : kContExt | (pc << 2);
            if (so.cont == kContAccumulate) __stcs(shd.rad + ps, make_float4(r.rad.x, r.rad.y, r.rad.z, __uint_as_float(r.pixel)));
            __stcs(shd.sh_o + ps, make_float4(so.o.x, so.o.y, so.o.z, __uint_as_float(slot)));
            __stcs(shd.sh_d + ps, make_float4(so.d.x, so.d.y, so.d.z, so.dist - kShadowTmin));
            __stcs(shd.sh_c + ps, make_float4(so.c.x, so.c.y, so.c.z, __uint_as_float(w)));
        }
    }
}

template <bool kMulti, int kBlock>
static void launch_shade_t(uint32_t b, const DevScene& s, const Queues& q, int grid, cudaStream_t st) {
    switch (b) {
        case kBucketLambert: k_shade<kBucketLambert, kMulti, kBlock><<<grid, kBlock, 0, st>>>(s, q); break;
        case kBucketDielectric: k_shade<kBucketDielectric, kMulti, kBlock><<<grid, kBlock, 0, st>>>(s, q); break;
        case kBucketGGX: k_shade<kBucketGGX, kMulti, kBlock><<<grid, kBlock, 0, st>>>(s, q); break;
        case kBucketLambertResume: break;  // continued by the shadow kernel
        default: k_shade<kBucketOther, kMulti, kBlock><<<grid, kBlock, 0, st>>>(s, q); break;
    }
}

void launch_shade_bucket(uint32_t b, const DevScene& s, const Queues& q, bool multi, int grid, int block,
                         cudaStream_t st) {
    if (block == 128) {
        if (multi) launch_shade_t<true, 128>(b, s, q, grid * 2, st);
        else launch_shade_t<false, 128>(b, s, q, grid * 2, st);
    } else {
        if (multi) launch_shade_t<true, 256>(b, s, q, grid, st);
        else launch_shade_t<false, 256>(b, s, q, grid, st);
    }
}

// rgb = sum * (1/spp) as renderer.cpp:308-313; guides averaged unless raw.
__global__ void k_resolve(Frame f, uint32_t raw, float* rgb, float* albedo, float* normal) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t n = f.width * f.height;
    if (i >= n) return;
    float inv = 1.0f / (float)f.spp;
    float4 a = f.accum[i];
    rgb[3 * i] = a.x * inv;
    rgb[3 * i + 1] = a.y * inv;
    rgb[3 * i + 2] = a.z * inv;
    float g = raw ? 1.0f : inv;
    if (albedo) {
        float4 b = f.albedo[i];
        albedo[3 * i] = b.x * g;
        albedo[3 * i + 1] = b.y * g;
        albedo[3 * i + 2] = b.z * g;
    }
    if (normal) {
        float4 b = f.normal[i];
        normal[3 * i] = b.x * g;
        normal[3 * i + 1] = b.y * g;
        normal[3 * i + 2] = b.z * g;
    }
}

void launch_resolve(const Frame& f, uint32_t raw, float* rgb, float* albedo, float* normal, cudaStream_t st) {
    uint32_t n = f.width * f.height;
    k_resolve<<<(n + 255) / 256, 256, 0, st>>>(f, raw, rgb, albedo, normal);
}

}  // namespace wrk
