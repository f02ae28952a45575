// Stand-alone device kernels behind the kernel-level C entry points: stable
// ballot/prefix-sum compaction, light-CDF selection, RNG, the BSDF math batch,
// texture fetch, camera rays, and the ACES tonemap.  These are the same device
// functions the renderer uses, exposed one at a time for parity checks.  Also the
// finalize-time pass that completes the BVH's triangle records for shading.
#include <algorithm>
#include <mutex>

#include "wrk_internal.h"
#include "wrk_shading.cuh"

namespace wrk {

// ---- compaction (libWR/kernels/compact.cu:6-17 in trianglestrip/OfflineRenderer,
// order-preserving here).  Pass 1 counts survivors per 1024-element tile with warp
// ballots; pass 2 scans the tile counts in one block; pass 3 re-ballots and writes
// each survivor at tileBase + warpBase + rank-in-warp.
constexpr int kCompactTile = 1024;

__global__ void k_compact_count(const uint32_t* __restrict__ stage, const uint32_t* __restrict__ idx, uint32_t n,
                                uint32_t* tileCount) {
    __shared__ uint32_t warpCnt[kCompactTile / 32];
    uint32_t i = blockIdx.x * kCompactTile + threadIdx.x;
    bool keep = i < n && stage[idx[i]] != 3u;
    uint32_t b = __ballot_sync(0xffffffffu, keep);
    if ((threadIdx.x & 31) == 0) warpCnt[threadIdx.x >> 5] = __popc(b);
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t v = warpCnt[threadIdx.x];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) tileCount[blockIdx.x] = v;
    }
}

__global__ void k_compact_scan(uint32_t* tileCount, uint32_t tiles, uint32_t* total) {
    // single block of 1024 threads, sequential over chunks of 1024 tiles
    __shared__ uint32_t warpSum[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < tiles; base += blockDim.x) {
        uint32_t i = base + threadIdx.x;
        uint32_t v = i < tiles ? tileCount[i] : 0u;
        uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        uint32_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (lane == 31) warpSum[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t s = warpSum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= (uint32_t)o) s += y;
            }
            warpSum[lane] = s;
        }
        __syncthreads();
        uint32_t incl = x + (w ? warpSum[w - 1] : 0u);
        if (i < tiles) tileCount[i] = carry + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_compact_write(const uint32_t* __restrict__ stage, const uint32_t* __restrict__ idx, uint32_t n,
                                const uint32_t* __restrict__ tileBase, uint32_t* out) {
    __shared__ uint32_t warpOff[kCompactTile / 32];
    uint32_t i = blockIdx.x * kCompactTile + threadIdx.x;
    uint32_t v = i < n ? idx[i] : 0u;
    bool keep = i < n && stage[v] != 3u;
    uint32_t b = __ballot_sync(0xffffffffu, keep);
    uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warpOff[w] = __popc(b);
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t x = warpOff[threadIdx.x];
        uint32_t incl = x;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (threadIdx.x >= (uint32_t)o) incl += y;
        }
        warpOff[threadIdx.x] = incl - x;
    }
    __syncthreads();
    if (keep) out[tileBase[blockIdx.x] + warpOff[w] + __popc(b & ((1u << lane) - 1u))] = v;
}

int compact_stable(const uint32_t* stage, const uint32_t* idx, uint32_t n, uint32_t* out, uint32_t* count,
                   cudaStream_t st) {
    // in 64 bits: n + 1023 wraps for n > 2^32 - 1024 (at most 4,194,304 tiles fit a grid)
    const uint32_t tiles = (uint32_t)(((uint64_t)n + kCompactTile - 1) / kCompactTile);
    if (tiles == 0) return cudaMemsetAsync(count, 0, sizeof(uint32_t), st) == cudaSuccess ? WRK_OK : WRK_ERR_CUDA;
    uint32_t* tileCount = nullptr;
    if (cudaMallocAsync(&tileCount, sizeof(uint32_t) * tiles, st) != cudaSuccess) return WRK_ERR_CUDA;
    k_compact_count<<<tiles, kCompactTile, 0, st>>>(stage, idx, n, tileCount);
    k_compact_scan<<<1, 1024, 0, st>>>(tileCount, tiles, count);
    k_compact_write<<<tiles, kCompactTile, 0, st>>>(stage, idx, n, tileCount, out);
    cudaFreeAsync(tileCount, st);
    return cudaGetLastError() == cudaSuccess ? WRK_OK : WRK_ERR_CUDA;
}

// ---- light CDF / RNG ----
__global__ void k_cdf(const float* cdf, uint32_t ncdf, const float* u, uint32_t n, uint32_t* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = cdf_lower_bound(u[i], cdf, ncdf);
}
__global__ void k_rng(const uint32_t* seed, const uint32_t* dim, uint32_t n, uint32_t* h, float* u) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        h[i] = pcg_hash_dim(seed[i], dim[i]);
        u[i] = rnd_dim(seed[i], dim[i]);
    }
}

// ---- BSDF batch: record layout documented in include/wrk.h (20 in, 34 out) ----
__global__ void k_bsdf(const float* __restrict__ in, uint32_t n, float* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* q = in + 20 * (size_t)i;
    float* o = out + 34 * (size_t)i;
    float3 wo = f3(q[0], q[1], q[2]), wi = f3(q[3], q[4], q[5]), nn = f3(q[6], q[7], q[8]), al = f3(q[9], q[10], q[11]);
    float rough = q[12], metal = q[13], ior = q[14], u0 = q[15], u1 = q[16], u2 = q[17];
    uint32_t depth = (uint32_t)q[18];
    float rrs = q[19];
    float3 e = ggx_eval(wo, wi, nn, al, rough, metal, ior);
    o[0] = e.x; o[1] = e.y; o[2] = e.z;
    float gp = ggx_pdf(wo, wi, nn, rough);
    o[3] = gp;
    float3 tg, bt;
    frame(nn, tg, bt);
    float3 sw = f3(0, 0, 0);
    float sp = 0.0f;
    ggx_sample(wo, nn, tg, bt, rough, u0, u1, sw, sp);
    bool ok = sp > 0.0f || sp != sp;
    if (!ok) sw = f3(0, 0, 0);
    o[4] = sw.x; o[5] = sw.y; o[6] = sw.z; o[7] = sp; o[8] = ok ? 1.0f : 0.0f;
    o[9] = fresnel_dielectric(fabsf(dot(wo, nn)), 1.0f, ior);
    float cp;
    float3 ch = cosine_hemisphere(u0, u1, cp);
    o[10] = ch.x; o[11] = ch.y; o[12] = ch.z; o[13] = cp;
    float cpdf = cosine_pdf(dot(nn, wi));
    o[14] = power_heuristic(gp, cpdf);
    o[15] = cpdf;
    float3 nt = f3(0, 0, 0);
    bool sv = russian_roulette(al, depth, rrs, u2, nt, metal > 0.5f);
    o[16] = sv ? 1.0f : 0.0f;
    o[17] = nt.x; o[18] = nt.y; o[19] = nt.z;
    o[20] = tg.x; o[21] = tg.y; o[22] = tg.z; o[23] = bt.x; o[24] = bt.y; o[25] = bt.z;
    float3 ln;
    float la;
    float3 pp = sample_triangle(u0, u1, wo, wi, nn, ln, la);
    o[26] = pp.x; o[27] = pp.y; o[28] = pp.z; o[29] = la; o[30] = ln.x; o[31] = ln.y; o[32] = ln.z;
    o[33] = shading_correction(wi, nn, normalize(wo));
}

__global__ void k_texture(const uint8_t* texels, uint32_t w, uint32_t h, const float* uv, uint32_t n, float* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 c = tex_fetch(texels, w, h, uv[2 * i], uv[2 * i + 1]);
    out[4 * i] = c.x; out[4 * i + 1] = c.y; out[4 * i + 2] = c.z; out[4 * i + 3] = c.w;
}

__global__ void k_camera_rays(Frame f, const uint32_t* pixels, const uint32_t* samples, uint32_t n, float* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t pixel = pixels[i], sample = samples[i];
    uint32_t x = pixel % f.width, y = pixel / f.width;
    uint32_t js = path_seed(pixel, sample, f.seed);
    float r1 = lcg_randf(js);
    float r2 = lcg_randf(js);
    float nx = (2.0f * ((float)x + r1) / (float)f.width - 1.0f) * f.aspect;
    float ny = 1.0f - 2.0f * ((float)y + r2) / (float)f.height;
    float3 fwd = f3(f.fwd[0], f.fwd[1], f.fwd[2]), rt = f3(f.right[0], f.right[1], f.right[2]),
           up = f3(f.up[0], f.up[1], f.up[2]), pos = f3(f.pos[0], f.pos[1], f.pos[2]);
    float3 dir = normalize(add(add(fwd, mul(mul(rt, nx), f.tanHalf)), mul(mul(up, ny), f.tanHalf)));
    float3 o = pos, d = dir;
    if (f.lens > 0.0f && f.focal > 0.0f) {
        float r3 = lcg_randf(js), r4 = lcg_randf(js);
        float th = 2.0f * 3.14159265f * r3;
        float rad = sqrtf(r4) * f.lens;
        float ct = cosf(th), sn = sinf(th);
        float3 off = f3(rt.x * rad * ct + up.x * rad * sn, rt.y * rad * ct + up.y * rad * sn,
                        rt.z * rad * ct + up.z * rad * sn);
        float3 fp = f3(pos.x + dir.x * f.focal, pos.y + dir.y * f.focal, pos.z + dir.z * f.focal);
        o = f3(pos.x + off.x, pos.y + off.y, pos.z + off.z);
        d = normalize(f3(fp.x - o.x, fp.y - o.y, fp.z - o.z));
    }
    float* q = out + 8 * (size_t)i;
    q[0] = o.x; q[1] = o.y; q[2] = o.z; q[3] = 0.0001f;
    q[4] = d.x; q[5] = d.y; q[6] = d.z; q[7] = 1e20f;
}

// 16 bytes in (4 floats), 4 bytes out per thread-step: vectorized grid-stride tonemap.
__global__ void k_tonemap(const float* __restrict__ rgb, uint32_t nfloat, uint8_t* __restrict__ out, int vec) {
    uint32_t stride = gridDim.x * blockDim.x;
    uint32_t n4 = vec ? nfloat / 4 : 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
        float4 v = reinterpret_cast<const float4*>(rgb)[i];
        uchar4 b = make_uchar4(aces_byte(v.x), aces_byte(v.y), aces_byte(v.z), aces_byte(v.w));
        reinterpret_cast<uchar4*>(out)[i] = b;
    }
    for (uint32_t i = n4 * 4 + blockIdx.x * blockDim.x + threadIdx.x; i < nfloat; i += stride) out[i] = aces_byte(rgb[i]);
}

__global__ void k_leaf_buckets(float4* tris, uint32_t nt, const wrk_material* __restrict__ mats, uint32_t numMats) {
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < nt; l += gridDim.x * blockDim.x) {
        const uint32_t mat = __float_as_uint(tris[3 * (size_t)l + 1].w);
        const uint32_t b = mat < numMats ? bucket_of_material(mats[mat]) : (uint32_t)kBucketOther;
        tris[3 * (size_t)l + 2].w = __uint_as_float(b);
    }
}

void launch_leaf_buckets(float4* tris, uint32_t numTris, const wrk_material* mats, uint32_t numMats,
                         cudaStream_t st) {
    if (!numTris) return;
    const uint32_t grid = (uint32_t)std::min<uint64_t>(((uint64_t)numTris + 255) / 256, 148u * 16u);
    k_leaf_buckets<<<grid, 256, 0, st>>>(tris, numTris, mats, numMats);
}

void launch_cdf(const float* cdf, uint32_t ncdf, const float* u, uint32_t n, uint32_t* out, cudaStream_t st) {
    if (n) k_cdf<<<(n + 255) / 256, 256, 0, st>>>(cdf, ncdf, u, n, out);
}
void launch_rng(const uint32_t* s, const uint32_t* d, uint32_t n, uint32_t* h, float* u, cudaStream_t st) {
    if (n) k_rng<<<(n + 255) / 256, 256, 0, st>>>(s, d, n, h, u);
}
void launch_bsdf(const float* in, uint32_t n, float* out, cudaStream_t st) {
    if (n) k_bsdf<<<(n + 127) / 128, 128, 0, st>>>(in, n, out);
}
void launch_texture(const uint8_t* texels, uint32_t w, uint32_t h, const float* uv, uint32_t n, float* out,
                    cudaStream_t st) {
    if (n) k_texture<<<(n + 255) / 256, 256, 0, st>>>(texels, w, h, uv, n, out);
}
void launch_camera_rays(const Frame& f, const uint32_t* px, const uint32_t* sm, uint32_t n, float* out,
                        cudaStream_t st) {
    if (n) k_camera_rays<<<(n + 255) / 256, 256, 0, st>>>(f, px, sm, n, out);
}
void launch_tonemap(const float* rgb, uint32_t nfloat, uint8_t* out, int grid, int vec, cudaStream_t st) {
    if (nfloat) k_tonemap<<<grid, 256, 0, st>>>(rgb, nfloat, out, vec);
}

}  // namespace wrk

// ---------------------------------------------------------------------------
// Compaction for callers that cannot allocate device memory.
//
// wrk_compact obtains its per-tile count buffer with cudaMallocAsync.  Some
// callers cannot let a library allocate: a serving process that reserved its
// whole device-memory budget up front and must not grow, a framework whose own
// allocator has to own every device byte, and hosts that forbid allocation after
// start-up so that memory use stays fixed.  For them wrk_compact_noalloc keeps
// that scratch in a fixed array that is part of the library image itself (loaded
// with the module into each device's primary context, and held there until the
// process exits or that context is reset), so the call allocates nothing.
//
// The first call on each device resolves the array's device address (with
// cudaGetSymbolAddress, that device current); make that first call before any
// stream capture begins.  The address is kept for the life of the process, so
// this entry point supports neither a cudaDeviceReset of that device after its
// first call (the module is reloaded elsewhere and the kept address dangles) nor
// a caller that makes a non-primary driver context current on the device.
//
// Limit: at most kNoAllocMaxTiles tiles of 1024 entries (67,108,864 input
// indices), i.e. 256 KiB of scratch per GPU.  Every call shares this one array
// and it keeps the previous call's values; each call writes every tile count it
// reads before reading it, so nothing has to be cleared first.  Calls that overlap
// on the GPU (other host threads, other streams) race on the array and must be
// serialized by the caller.
namespace wrk {
namespace {

constexpr uint32_t kNoAllocMaxTiles = 65536;
static __device__ __align__(256) uint32_t g_compactScratch[kNoAllocMaxTiles];

constexpr int kMaxDevices = 64;
std::mutex g_scratchMutex;
uint32_t* g_scratchAddr[kMaxDevices] = {nullptr};

// The array's name in host code is only a host-side handle of the device symbol,
// not a device address: resolve the device address once per device, with that
// device current, and pass the pointer to the kernels.
int scratch_for_current_device(uint32_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return report_error(WRK_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return report_error(WRK_ERR_INVALID, "device index out of range");
    std::lock_guard<std::mutex> lock(g_scratchMutex);
    if (!g_scratchAddr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_compactScratch);
        if (e != cudaSuccess) return report_error(WRK_ERR_CUDA, cudaGetErrorString(e));
        g_scratchAddr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_scratchAddr[dev];
    return WRK_OK;
}

}  // namespace
}  // namespace wrk

extern "C" int wrk_compact_noalloc(const uint32_t* d_stage, const uint32_t* d_idxIn, uint32_t n, uint32_t* d_idxOut,
                                   uint32_t* d_count) {
    using namespace wrk;
    if (!d_count || (n && (!d_stage || !d_idxIn || !d_idxOut)))
        return report_error(WRK_ERR_INVALID, "wrk_compact_noalloc: null buffer");
    // in 64 bits, so that n close to 2^32 cannot wrap to zero tiles and pass the limit
    const uint64_t tiles64 = ((uint64_t)n + kCompactTile - 1) / kCompactTile;
    if (tiles64 > kNoAllocMaxTiles)
        return report_error(WRK_ERR_INVALID,
                            "wrk_compact_noalloc: n exceeds the fixed scratch limit of 67108864 indices "
                            "(65536 tiles of 1024); use wrk_compact");
    const uint32_t tiles = (uint32_t)tiles64;
    uint32_t* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    if (tiles == 0) {
        cudaError_t e = cudaMemset(d_count, 0, sizeof(uint32_t));
        return e == cudaSuccess ? WRK_OK : report_error(WRK_ERR_CUDA, cudaGetErrorString(e));
    }
    k_compact_count<<<tiles, kCompactTile>>>(d_stage, d_idxIn, n, scratch);
    k_compact_scan<<<1, 1024>>>(scratch, tiles, d_count);
    k_compact_write<<<tiles, kCompactTile>>>(d_stage, d_idxIn, n, scratch, d_idxOut);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return e == cudaSuccess ? WRK_OK : report_error(WRK_ERR_CUDA, cudaGetErrorString(e));
}
