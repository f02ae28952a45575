// Learned denoiser: a 4-level U-Net (3x3 convolutions, 32/64/128/256 channels,
// average-pool down, nearest up, concatenated skips) on the 9-channel input libWR
// hands its denoiser -- radiance, first-hit albedo and normal
// (libWR/src/internal/denoiser.cpp:98-116, guides from libWR/kernels/trace.cu:267-287).
// It replaces the closed OptiX AI denoiser (denoiser.cpp:171, optixDenoiserInvoke).
//
// Every convolution runs on the tcgen05 kernels of conv_tc.cu (forward, data
// gradient through flipped / transposed weights, weight gradient); the rest are
// bandwidth-bound elementwise kernels here.  Training: L1 loss in log space on a
// residual prediction (output = log1p(radiance) + network), Adam on f32 master
// weights that are re-laid-out to bf16 after every step.
//
// Activations NHWC bf16.  Buffers per level l (resolution H/2^l):
//   x0[16] a0[32] cat0[96] a6[32] dec0[32] out[16 f32]       level 0
//   p1[32] a1[64] cat1[192] a5[64] dec1[64]                   level 1
//   p2[64] a2[128] cat2[384] a4[128] dec2[128]                level 2
//   p3[128] a3[256] b3[256]                                   level 3
// cat_l = [up(deeper) | skip s_l]; the encoder's second convolution writes s_l
// straight into its slice of cat_l, the upsample writes the other slice.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "conv_tc.h"
#include "wrk_internal.h"

namespace wrk {
namespace dn {

using conv::Epilogue;

constexpr int kLayers = 15;
struct LayerDef {
    uint32_t cin, cout, level;
    bool relu;
};
// e0a e0b e1a e1b e2a e2b e3a e3b d2a d2b d1a d1b d0a d0b head
constexpr LayerDef kDefs[kLayers] = {{16, 32, 0, true},  {32, 32, 0, true},   {32, 64, 1, true},   {64, 64, 1, true},
                                     {64, 128, 2, true}, {128, 128, 2, true}, {128, 256, 3, true}, {256, 256, 3, true},
                                     {384, 128, 2, true}, {128, 128, 2, true}, {192, 64, 1, true},  {64, 64, 1, true},
                                     {96, 32, 0, true},  {32, 32, 0, true},   {32, 3, 0, false}};

__host__ __device__ inline uint32_t pad16(uint32_t c) { return (c + 15) / 16 * 16; }

// ---------------------------------------------------------------------------
// elementwise kernels
__device__ __forceinline__ float lg(float x) { return log1pf(fmaxf(x, 0.0f)); }

// (rgb, albedo, normal) f32 [B][h][w][3] -> x0 bf16 [B][H][W][16] (H >= h, W >= w, edge-clamped)
__global__ void k_pack(const float* rgb, const float* alb, const float* nrm, uint32_t B, uint32_t h, uint32_t w,
                       uint32_t H, uint32_t W, __nv_bfloat16* x0) {
    size_t n = (size_t)B * H * W;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t b = (uint32_t)(i / ((size_t)H * W));
        uint32_t r = (uint32_t)(i % ((size_t)H * W));
        uint32_t y = min(r / W, h - 1), x = min(r % W, w - 1);
        size_t s = ((size_t)b * h + y) * w + x;
        float v[16];
        for (int c = 0; c < 3; ++c) {
            v[c] = lg(rgb[3 * s + c]);
            v[3 + c] = alb ? alb[3 * s + c] : 0.0f;
            v[6 + c] = nrm ? nrm[3 * s + c] : 0.0f;
        }
        for (int c = 9; c < 16; ++c) v[c] = 0.0f;
        uint32_t p[8];
        for (int j = 0; j < 8; ++j) {
            __nv_bfloat162 t = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
            p[j] = *(uint32_t*)&t;
        }
        uint4* o = (uint4*)(x0 + i * 16);
        o[0] = make_uint4(p[0], p[1], p[2], p[3]);
        o[1] = make_uint4(p[4], p[5], p[6], p[7]);
    }
}

__device__ __forceinline__ void bf8_to_f(uint4 u, float (&f)[8]) {
    const __nv_bfloat162* h = (const __nv_bfloat162*)&u;
    for (int j = 0; j < 4; ++j) {
        float2 t = __bfloat1622float2(h[j]);
        f[2 * j] = t.x;
        f[2 * j + 1] = t.y;
    }
}
__device__ __forceinline__ uint4 f_to_bf8(const float (&f)[8]) {
    uint4 u;
    uint32_t* p = (uint32_t*)&u;
    for (int j = 0; j < 4; ++j) {
        __nv_bfloat162 t = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
        p[j] = *(uint32_t*)&t;
    }
    return u;
}

// 2x2 average pool: src [B][H][W][stride] channels [off, off+C) -> dst [B][H/2][W/2][C]
__global__ void k_pool2(const __nv_bfloat16* src, uint32_t stride, uint32_t off, uint32_t C, uint32_t B, uint32_t H,
                        uint32_t W, __nv_bfloat16* dst) {
    const uint32_t g = C / 8, h = H / 2, w = W / 2;
    size_t n = (size_t)B * h * w * g;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t cg = (uint32_t)(i % g);
        size_t p = i / g;
        uint32_t x = (uint32_t)(p % w), y = (uint32_t)((p / w) % h), b = (uint32_t)(p / ((size_t)w * h));
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                size_t sp = ((size_t)b * H + 2 * y + dy) * W + 2 * x + dx;
                float f[8];
                bf8_to_f(*(const uint4*)(src + sp * stride + off + cg * 8), f);
                for (int j = 0; j < 8; ++j) acc[j] += f[j];
            }
        for (int j = 0; j < 8; ++j) acc[j] *= 0.25f;
        *(uint4*)(dst + p * C + cg * 8) = f_to_bf8(acc);
    }
}

// nearest 2x upsample: src [B][h][w][C] -> dst [B][2h][2w][stride] channels [0, C)
__global__ void k_up2(const __nv_bfloat16* src, uint32_t C, uint32_t B, uint32_t h, uint32_t w, __nv_bfloat16* dst,
                      uint32_t stride) {
    const uint32_t g = C / 8, H = 2 * h, W = 2 * w;
    size_t n = (size_t)B * H * W * g;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t cg = (uint32_t)(i % g);
        size_t p = i / g;
        uint32_t x = (uint32_t)(p % W), y = (uint32_t)((p / W) % H), b = (uint32_t)(p / ((size_t)W * H));
        size_t sp = ((size_t)b * h + y / 2) * w + x / 2;
        *(uint4*)(dst + p * stride + cg * 8) = *(const uint4*)(src + sp * C + cg * 8);
    }
}

// gradient of the upsample: g[B][h][w][C] = sum of the 4 children of dcat[.., 0:C), x (mask > 0)
__global__ void k_up2_bwd(const float* dcat, uint32_t stride, uint32_t C, uint32_t B, uint32_t h, uint32_t w,
                          const __nv_bfloat16* mask, __nv_bfloat16* g) {
    const uint32_t G = C / 8, H = 2 * h, W = 2 * w;
    size_t n = (size_t)B * h * w * G;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t cg = (uint32_t)(i % G);
        size_t p = i / G;
        uint32_t x = (uint32_t)(p % w), y = (uint32_t)((p / w) % h), b = (uint32_t)(p / ((size_t)w * h));
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                const float* s = dcat + (((size_t)b * H + 2 * y + dy) * W + 2 * x + dx) * stride + cg * 8;
                float4 u = *(const float4*)s, v = *(const float4*)(s + 4);
                acc[0] += u.x; acc[1] += u.y; acc[2] += u.z; acc[3] += u.w;
                acc[4] += v.x; acc[5] += v.y; acc[6] += v.z; acc[7] += v.w;
            }
        float m[8];
        bf8_to_f(*(const uint4*)(mask + p * C + cg * 8), m);
        for (int j = 0; j < 8; ++j)
            if (!(m[j] > 0.0f)) acc[j] = 0.0f;
        *(uint4*)(g + p * C + cg * 8) = f_to_bf8(acc);
    }
}

// skip gradient: g[B][H][W][C] = (dcat[.., off:off+C) + dp[parent] / 4) x (s > 0), s = cat[.., off:off+C)
__global__ void k_skip_bwd(const float* dcat, uint32_t stride, uint32_t off, uint32_t C, uint32_t B, uint32_t H,
                           uint32_t W, const float* dp, const __nv_bfloat16* cat, __nv_bfloat16* g) {
    const uint32_t G = C / 8;
    size_t n = (size_t)B * H * W * G;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t cg = (uint32_t)(i % G);
        size_t p = i / G;
        uint32_t x = (uint32_t)(p % W), y = (uint32_t)((p / W) % H), b = (uint32_t)(p / ((size_t)W * H));
        const float* s = dcat + p * stride + off + cg * 8;
        const float* q = dp + (((size_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + cg * 8;
        float m[8];
        bf8_to_f(*(const uint4*)(cat + p * stride + off + cg * 8), m);
        float v[8];
        for (int j = 0; j < 8; ++j) v[j] = m[j] > 0.0f ? s[j] + 0.25f * q[j] : 0.0f;
        *(uint4*)(g + p * C + cg * 8) = f_to_bf8(v);
    }
}

// bias gradient: db[c] += sum_p g[p][c]
__global__ void k_bias_grad(const __nv_bfloat16* g, size_t P, uint32_t C, uint32_t cValid, float* db) {
    extern __shared__ float red[];
    const uint32_t c = threadIdx.x % C, lanes = blockDim.x / C;
    const uint32_t r = threadIdx.x / C;
    float acc = 0.0f;
    if (r < lanes)
        for (size_t p = blockIdx.x * (size_t)lanes + r; p < P; p += (size_t)gridDim.x * lanes)
            acc += __bfloat162float(g[p * C + c]);
    red[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < cValid) {
        float s = 0.0f;
        for (uint32_t k = 0; k < lanes; ++k) s += red[k * C + threadIdx.x];
        atomicAdd(db + threadIdx.x, s);
    }
}

// L1 loss in log space on the residual prediction; writes the head's gradient (bf16,
// 16 channels, 3 used) and accumulates the loss sum.
__global__ void k_loss(const float* out, const float* rgb, const float* target, size_t P, float scale,
                       __nv_bfloat16* gHead, float* lossSum) {
    float acc = 0.0f;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < P; p += (size_t)gridDim.x * blockDim.x) {
        __nv_bfloat16 gv[16];
        for (int c = 0; c < 16; ++c) gv[c] = __float2bfloat16_rn(0.0f);
        for (int c = 0; c < 3; ++c) {
            float pred = lg(rgb[3 * p + c]) + out[16 * p + c];
            float d = pred - lg(target[3 * p + c]);
            acc += fabsf(d);
            gv[c] = __float2bfloat16_rn(d > 0.0f ? scale : (d < 0.0f ? -scale : 0.0f));
        }
        uint4* o = (uint4*)(gHead + 16 * p);
        o[0] = *(uint4*)&gv[0];
        o[1] = *(uint4*)&gv[8];
    }
    for (int s = 16; s > 0; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
    if ((threadIdx.x & 31) == 0) atomicAdd(lossSum, acc);
}

// denoised radiance = expm1(log1p(rgb) + head), cropped to [B][h][w][3]
__global__ void k_unpack(const float* out, const float* rgb, uint32_t B, uint32_t h, uint32_t w, uint32_t H,
                         uint32_t W, float* dst) {
    size_t n = (size_t)B * h * w;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t b = (uint32_t)(i / ((size_t)h * w)), r = (uint32_t)(i % ((size_t)h * w));
        uint32_t y = r / w, x = r % w;
        size_t q = ((size_t)b * H + y) * W + x;
        for (int c = 0; c < 3; ++c) dst[3 * i + c] = fmaxf(expm1f(lg(rgb[3 * i + c]) + out[16 * q + c]), 0.0f);
    }
}

// Adam (Kingma & Ba 2015) on the flat f32 parameter array.
__global__ void k_adam(float* w, const float* g, float* m, float* v, size_t n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.0f - b1) * gi;
        float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// f32 master W[co][tap][ci] -> forward bf16 Wf[co][tap][ci] (rows >= cout stay zero) and
// data-gradient bf16 Wd[ci][tap][coPad] = W[co][8 - tap][ci].
__global__ void k_relayout(const float* W, uint32_t cout, uint32_t cin, uint32_t coPad, __nv_bfloat16* Wf,
                           __nv_bfloat16* Wd) {
    size_t n = (size_t)cout * 9 * cin;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t ci = (uint32_t)(i % cin);
        uint32_t tap = (uint32_t)((i / cin) % 9);
        uint32_t co = (uint32_t)(i / ((size_t)9 * cin));
        __nv_bfloat16 b = __float2bfloat16_rn(W[i]);
        Wf[i] = b;
        if (Wd) Wd[((size_t)ci * 9 + (8 - tap)) * coPad + co] = b;
    }
}

inline int grid_for(size_t n, int block = 256) {
    size_t g = (n + block - 1) / block;
    return (int)std::min<size_t>(std::max<size_t>(g, 1), 148 * 16);
}

}  // namespace dn
}  // namespace wrk

using namespace wrk;
using namespace wrk::dn;

namespace {
thread_local std::string g_dnerr;
int dfail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    report_error(code, buf);
    return code;
}
#define DCK(x)                                                                                                \
    do {                                                                                                      \
        cudaError_t e_ = (x);                                                                                 \
        if (e_ != cudaSuccess) return dfail(WRK_ERR_CUDA, "%s: %s (%s:%d)", #x, cudaGetErrorString(e_), __FILE__, \
                                            __LINE__);                                                        \
    } while (0)

struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~DBuf() { if (p) cudaFree(p); }
    int alloc(size_t n) {
        if (p && n <= bytes) return 0;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (cudaMalloc(&p, std::max<size_t>(n, 16)) != cudaSuccess) return 1;
        bytes = n;
        return 0;
    }
    template <class T> T* as() const { return (T*)p; }
};
}  // namespace

struct wrk_denoiser {
    int device = 0;
    int numSMs = 148;
    cudaStream_t stream = nullptr;
    uint32_t step = 0;
    // parameters: flat f32 (per layer W [cout][9][cin] then b [cout])
    size_t woff[kLayers], boff[kLayers], nparams = 0;
    DBuf params, grads, adamM, adamV, wf[kLayers], wd[kLayers], err, lossSum;
    // activations / gradients for the current shape
    uint32_t B = 0, H = 0, W = 0;
    DBuf x0, a[kLayers], cat[3], pool[3], out, g[kLayers], dcat[3], dp[3];
    DBuf inPad, scratchIn[3];
    bool shapeReady = false;
    // plans and tensor maps for the current shape
    conv::FwdPlan fplan[kLayers];
    conv::FwdPlan dplan[kLayers][2];
    conv::WgradPlan wplan[kLayers];
    CUtensorMap fin[kLayers], fw[kLayers], din[kLayers], dwmap[kLayers][2], wg[kLayers], wx[kLayers];
    uint32_t dsplit[kLayers];
    // device time of the last inference / training step (events on `stream`)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float lastMs = 0.0f;
    ~wrk_denoiser() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

uint32_t lvl_h(const wrk_denoiser* d, uint32_t l) { return d->H >> l; }
uint32_t lvl_w(const wrk_denoiser* d, uint32_t l) { return d->W >> l; }

// Input tensor (buffer, channels) of layer i, and where its output goes.
struct IO {
    void* in;
    uint32_t inC;
    void* out;
    uint32_t outStride, outOffset;
};
IO layer_io(wrk_denoiser* d, int i) {
    auto A = [&](int k) { return d->a[k].p; };
    switch (i) {
        case 0: return {d->x0.p, 16, A(0), 32, 0};
        case 1: return {A(0), 32, d->cat[0].p, 96, 64};
        case 2: return {d->pool[0].p, 32, A(2), 64, 0};
        case 3: return {A(2), 64, d->cat[1].p, 192, 128};
        case 4: return {d->pool[1].p, 64, A(4), 128, 0};
        case 5: return {A(4), 128, d->cat[2].p, 384, 256};
        case 6: return {d->pool[2].p, 128, A(6), 256, 0};
        case 7: return {A(6), 256, A(7), 256, 0};
        case 8: return {d->cat[2].p, 384, A(8), 128, 0};
        case 9: return {A(8), 128, A(9), 128, 0};
        case 10: return {d->cat[1].p, 192, A(10), 64, 0};
        case 11: return {A(10), 64, A(11), 64, 0};
        case 12: return {d->cat[0].p, 96, A(12), 32, 0};
        case 13: return {A(12), 32, A(13), 32, 0};
        default: return {A(13), 32, d->out.p, 16, 0};
    }
}

int alloc_params(wrk_denoiser* d, uint32_t seed) {
    size_t n = 0;
    for (int i = 0; i < kLayers; ++i) {
        d->woff[i] = n;
        n += (size_t)kDefs[i].cout * 9 * kDefs[i].cin;
        d->boff[i] = n;
        n += kDefs[i].cout;
    }
    d->nparams = n;
    if (d->params.alloc(n * 4) || d->grads.alloc(n * 4) || d->adamM.alloc(n * 4) || d->adamV.alloc(n * 4) ||
        d->err.alloc(4) || d->lossSum.alloc(4))
        return dfail(WRK_ERR_CUDA, "denoiser parameter allocation failed");
    // He-uniform initialisation (seeded); the head starts near zero so the
    // untrained network passes its input through.
    std::vector<float> h(n, 0.0f);
    std::mt19937 rng(seed);
    for (int i = 0; i < kLayers; ++i) {
        float fan = 9.0f * kDefs[i].cin;
        float a = std::sqrt(6.0f / fan) * (i == kLayers - 1 ? 0.05f : 1.0f);
        std::uniform_real_distribution<float> U(-a, a);
        for (size_t k = 0; k < (size_t)kDefs[i].cout * 9 * kDefs[i].cin; ++k) h[d->woff[i] + k] = U(rng);
    }
    DCK(cudaMemcpy(d->params.p, h.data(), n * 4, cudaMemcpyHostToDevice));
    DCK(cudaMemset(d->adamM.p, 0, n * 4));
    DCK(cudaMemset(d->adamV.p, 0, n * 4));
    for (int i = 0; i < kLayers; ++i) {
        const LayerDef& L = kDefs[i];
        uint32_t coPad = pad16(L.cout);
        size_t fb = (size_t)coPad * 9 * L.cin * 2, db = (size_t)L.cin * 9 * coPad * 2;
        if (d->wf[i].alloc(fb) || (i > 0 && d->wd[i].alloc(db))) return dfail(WRK_ERR_CUDA, "weight allocation failed");
        DCK(cudaMemset(d->wf[i].p, 0, fb));
        if (i > 0) DCK(cudaMemset(d->wd[i].p, 0, db));
    }
    return WRK_OK;
}

int relayout_all(wrk_denoiser* d) {
    for (int i = 0; i < kLayers; ++i) {
        const LayerDef& L = kDefs[i];
        size_t n = (size_t)L.cout * 9 * L.cin;
        k_relayout<<<grid_for(n), 256, 0, d->stream>>>(d->params.as<float>() + d->woff[i], L.cout, L.cin, pad16(L.cout),
                                                       d->wf[i].as<__nv_bfloat16>(),
                                                       i > 0 ? d->wd[i].as<__nv_bfloat16>() : nullptr);
    }
    DCK(cudaGetLastError());
    return WRK_OK;
}

// Buffers, launch plans and tensor maps for batch B at H x W (multiples of 128 x 64).
int set_shape(wrk_denoiser* d, uint32_t B, uint32_t H, uint32_t W) {
    if (d->shapeReady && d->B == B && d->H == H && d->W == W) return WRK_OK;
    if (B == 0 || H % 64 || W % 128) return dfail(WRK_ERR_INVALID, "denoiser shape %ux%u not a multiple of 128x64", W, H);
    d->shapeReady = false;
    d->B = B;
    d->H = H;
    d->W = W;
    auto px = [&](uint32_t l) { return (size_t)B * lvl_h(d, l) * lvl_w(d, l); };
    bool bad = d->x0.alloc(px(0) * 16 * 2) || d->out.alloc(px(0) * 16 * 4);
    const uint32_t catC[3] = {96, 192, 384}, poolC[3] = {32, 64, 128};
    for (int l = 0; l < 3; ++l) {
        bad = bad || d->cat[l].alloc(px(l) * catC[l] * 2) || d->dcat[l].alloc(px(l) * catC[l] * 4) ||
              d->pool[l].alloc(px(l + 1) * poolC[l] * 2) || d->dp[l].alloc(px(l + 1) * poolC[l] * 4);
    }
    for (int i = 0; i < kLayers; ++i) {
        const LayerDef& L = kDefs[i];
        bad = bad || d->a[i].alloc(px(L.level) * pad16(L.cout) * 2) || d->g[i].alloc(px(L.level) * pad16(L.cout) * 2);
    }
    if (bad) return dfail(WRK_ERR_CUDA, "denoiser activation allocation failed (%ux%u x %u)", W, H, B);
    for (int i = 0; i < kLayers; ++i) {
        const LayerDef& L = kDefs[i];
        const uint32_t h = lvl_h(d, L.level), w = lvl_w(d, L.level), coPad = pad16(L.cout);
        IO io = layer_io(d, i);
        if (conv::plan_fwd(B, h, w, L.cin, coPad, d->numSMs, &d->fplan[i]))
            return dfail(WRK_ERR_INVALID, "no forward plan for layer %d", i);
        int ch = d->fplan[i].chunk;
        if (conv::make_input_map(d->fplan[i], io.in, &d->fin[i]) ||
            (!d->fplan[i].halo && conv::make_weight_map(&d->fw[i], d->wf[i].p, 9 * L.cin, coPad, ch, coPad)))
            return dfail(WRK_ERR_CUDA, "tensor map encoding failed (layer %d)", i);
        // weight gradient: G = g[i] (coPad channels), X = layer input
        if (conv::plan_wgrad(B, h, w, L.cin, coPad, d->numSMs, &d->wplan[i]))
            return dfail(WRK_ERR_INVALID, "no weight-gradient plan for layer %d", i);
        d->wplan[i].shape.coutStore = L.cout;
        if (conv::make_act_map(&d->wg[i], d->g[i].p, coPad, w, h, B, d->wplan[i].ca) ||
            conv::make_act_map(&d->wx[i], io.in, L.cin, w, h, B, d->wplan[i].cb))
            return dfail(WRK_ERR_CUDA, "tensor map encoding failed (layer %d wgrad)", i);
        // data gradient: input g[i] (coPad), weights Wd [cin][9][coPad], output cin channels
        if (i > 0) {
            d->dsplit[i] = L.cin > 256 ? 2 : 1;
            uint32_t n = L.cin / d->dsplit[i];
            for (uint32_t s = 0; s < d->dsplit[i]; ++s) {
                if (conv::plan_fwd(B, h, w, coPad, n, d->numSMs, &d->dplan[i][s]))
                    return dfail(WRK_ERR_INVALID, "no data-gradient plan for layer %d", i);
                d->dplan[i][s].shape.wRow0 = s * n;
                int dc = d->dplan[i][s].chunk;
                if (!d->dplan[i][s].halo && conv::make_weight_map(&d->dwmap[i][s], d->wd[i].p, 9 * coPad, L.cin, dc, n))
                    return dfail(WRK_ERR_CUDA, "tensor map encoding failed (layer %d dgrad)", i);
            }
            if (conv::make_input_map(d->dplan[i][0], d->g[i].p, &d->din[i]))
                return dfail(WRK_ERR_CUDA, "tensor map encoding failed (layer %d dgrad input)", i);
        }
    }
    d->shapeReady = true;
    return WRK_OK;
}

int conv_forward(wrk_denoiser* d, int i) {
    const LayerDef& L = kDefs[i];
    IO io = layer_io(d, i);
    Epilogue ep{};
    ep.bias = d->params.as<float>() + d->boff[i];
    ep.nBias = L.cout;
    ep.out = io.out;
    ep.outStride = io.outStride;
    ep.outOffset = io.outOffset;
    ep.coutValid = i == kLayers - 1 ? 16u : L.cout;  // head: padded channels are written as zero
    ep.relu = L.relu;
    ep.outF32 = i == kLayers - 1;
    DCK(conv::launch_fwd(d->fplan[i], d->fin[i], d->fw[i], d->wf[i].p, ep, d->err.as<uint32_t>(), d->stream));
    return WRK_OK;
}

int forward(wrk_denoiser* d) {
    const uint32_t B = d->B;
    int rc;
    for (int i = 0; i < kLayers; ++i) {
        if ((rc = conv_forward(d, i))) return rc;
        // pool after each encoder level's second convolution
        if (i == 1 || i == 3 || i == 5) {
            int l = (i - 1) / 2;
            const uint32_t catC[3] = {96, 192, 384}, off[3] = {64, 128, 256}, C[3] = {32, 64, 128};
            size_t n = (size_t)B * lvl_h(d, l + 1) * lvl_w(d, l + 1) * C[l] / 8;
            k_pool2<<<grid_for(n), 256, 0, d->stream>>>(d->cat[l].as<__nv_bfloat16>(), catC[l], off[l], C[l], B,
                                                        lvl_h(d, l), lvl_w(d, l), d->pool[l].as<__nv_bfloat16>());
        }
        // upsample into the decoder's concat buffer before its first convolution
        if (i == 7 || i == 9 || i == 11) {
            int l = i == 7 ? 2 : i == 9 ? 1 : 0;
            const uint32_t C[3] = {64, 128, 256}, catC[3] = {96, 192, 384};
            size_t n = (size_t)B * lvl_h(d, l) * lvl_w(d, l) * C[l] / 8;
            k_up2<<<grid_for(n), 256, 0, d->stream>>>(d->a[i].as<__nv_bfloat16>(), C[l], B, lvl_h(d, l + 1),
                                                      lvl_w(d, l + 1), d->cat[l].as<__nv_bfloat16>(), catC[l]);
        }
    }
    DCK(cudaGetLastError());
    return WRK_OK;
}

// Activation that masks the data gradient flowing into layer i's input (the ReLU
// output the input came from), or null when the input is not a ReLU output of one
// tensor (concat buffers and pooled tensors are handled by k_up2_bwd / k_skip_bwd).
const void* input_mask(wrk_denoiser* d, int i) {
    switch (i) {
        case 1: return d->a[0].p;
        case 3: return d->a[2].p;
        case 5: return d->a[4].p;
        case 7: return d->a[6].p;
        case 9: return d->a[8].p;
        case 11: return d->a[10].p;
        case 13: return d->a[12].p;
        case 14: return d->a[13].p;
        default: return nullptr;
    }
}

int backward(wrk_denoiser* d) {
    const uint32_t B = d->B;
    DCK(cudaMemsetAsync(d->grads.p, 0, d->nparams * 4, d->stream));
    for (int i = kLayers - 1; i >= 0; --i) {
        const LayerDef& L = kDefs[i];
        const uint32_t h = lvl_h(d, L.level), w = lvl_w(d, L.level), coPad = pad16(L.cout);
        // weight and bias gradients
        DCK(conv::launch_wgrad(d->wplan[i], d->wg[i], d->wx[i], d->grads.as<float>() + d->woff[i],
                               d->err.as<uint32_t>(), d->stream));
        {
            // g has coPad channels; only the layer's real output channels have a bias
            uint32_t lanes = std::max(1u, 256u / coPad);
            size_t P = (size_t)B * h * w;
            k_bias_grad<<<(unsigned)std::min<size_t>(1184, (P + lanes - 1) / lanes), lanes * coPad,
                          lanes * coPad * 4, d->stream>>>(d->g[i].as<__nv_bfloat16>(), P, coPad, L.cout,
                                                          d->grads.as<float>() + d->boff[i]);
        }
        if (i == 0) break;
        // data gradient into the layer's input
        const void* mask = input_mask(d, i);
        const uint32_t targetLayer = (uint32_t)i - 1;  // the G it produces (when masked)
        for (uint32_t s = 0; s < d->dsplit[i]; ++s) {
            Epilogue ep{};
            uint32_t n = L.cin / d->dsplit[i];
            ep.coutValid = n;
            ep.relu = 0;
            if (mask) {
                ep.out = d->g[targetLayer].p;
                ep.outStride = L.cin;
                ep.outOffset = s * n;
                ep.outF32 = 0;
                ep.mask = (const __nv_bfloat16*)mask;
                ep.maskStride = L.cin;
                ep.maskOffset = s * n;
            } else {
                // concat or pooled input: f32 gradient, split by the combine kernels
                void* dst = nullptr;
                switch (i) {
                    case 12: dst = d->dcat[0].p; break;
                    case 10: dst = d->dcat[1].p; break;
                    case 8: dst = d->dcat[2].p; break;
                    case 6: dst = d->dp[2].p; break;
                    case 4: dst = d->dp[1].p; break;
                    case 2: dst = d->dp[0].p; break;
                }
                ep.out = dst;
                ep.outStride = L.cin;
                ep.outOffset = s * n;
                ep.outF32 = 1;
            }
            DCK(conv::launch_fwd(d->dplan[i][s], d->din[i], d->dwmap[i][s], d->wd[i].p, ep, d->err.as<uint32_t>(),
                                 d->stream));
        }
        // combine kernels that produce the G of the layer below
        const uint32_t catC[3] = {96, 192, 384};
        if (i == 12 || i == 10 || i == 8) {  // gradient of up(deeper) -> G of the deeper layer's output
            int l = i == 12 ? 0 : i == 10 ? 1 : 2;
            int below = i - 1;  // 11, 9, 7
            const uint32_t C[3] = {64, 128, 256};
            size_t n = (size_t)B * lvl_h(d, l + 1) * lvl_w(d, l + 1) * C[l] / 8;
            k_up2_bwd<<<grid_for(n), 256, 0, d->stream>>>(d->dcat[l].as<float>(), catC[l], C[l], B, lvl_h(d, l + 1),
                                                          lvl_w(d, l + 1), d->a[below].as<__nv_bfloat16>(),
                                                          d->g[below].as<__nv_bfloat16>());
        }
        if (i == 6 || i == 4 || i == 2) {  // pooled input -> G of the skip tensor s_l (layer i-1)
            int l = i == 6 ? 2 : i == 4 ? 1 : 0;
            const uint32_t off[3] = {64, 128, 256}, C[3] = {32, 64, 128};
            size_t n = (size_t)B * lvl_h(d, l) * lvl_w(d, l) * C[l] / 8;
            k_skip_bwd<<<grid_for(n), 256, 0, d->stream>>>(d->dcat[l].as<float>(), catC[l], off[l], C[l], B, lvl_h(d, l),
                                                           lvl_w(d, l), d->dp[l].as<float>(),
                                                           d->cat[l].as<__nv_bfloat16>(), d->g[i - 1].as<__nv_bfloat16>());
        }
    }
    DCK(cudaGetLastError());
    return WRK_OK;
}

}  // namespace

namespace {

int check_err(wrk_denoiser* d, const char* what) {
    uint32_t e = 0;
    DCK(cudaMemcpyAsync(&e, d->err.p, 4, cudaMemcpyDeviceToHost, d->stream));
    DCK(cudaStreamSynchronize(d->stream));
    if (e) return dfail(WRK_ERR_DEVICE, "%s: a convolution kernel timed out waiting on its pipeline (flags 0x%x)", what, e);
    return WRK_OK;
}

int run_loss(wrk_denoiser* d, const float* rgb, const float* target, float* loss) {
    size_t P = (size_t)d->B * d->H * d->W;
    DCK(cudaMemsetAsync(d->lossSum.p, 0, 4, d->stream));
    k_loss<<<grid_for(P), 256, 0, d->stream>>>(d->out.as<float>(), rgb, target, P, 1.0f / (float)(3 * P),
                                               d->g[kLayers - 1].as<__nv_bfloat16>(), d->lossSum.as<float>());
    DCK(cudaGetLastError());
    if (loss) {
        float s = 0;
        DCK(cudaMemcpyAsync(&s, d->lossSum.p, 4, cudaMemcpyDeviceToHost, d->stream));
        DCK(cudaStreamSynchronize(d->stream));
        *loss = s / (float)(3 * P);
    }
    return WRK_OK;
}

int fwd_bwd(wrk_denoiser* d, const float* rgb, const float* alb, const float* nrm, const float* target, uint32_t B,
            uint32_t H, uint32_t W, float* loss) {
    if (!d || !rgb || !target) return dfail(WRK_ERR_INVALID, "null denoiser argument");
    DCK(cudaSetDevice(d->device));
    int rc = set_shape(d, B, H, W);
    if (rc) return rc;
    DCK(cudaMemsetAsync(d->err.p, 0, 4, d->stream));
    size_t P = (size_t)B * H * W;
    k_pack<<<grid_for(P), 256, 0, d->stream>>>(rgb, alb, nrm, B, H, W, H, W, d->x0.as<__nv_bfloat16>());
    if ((rc = forward(d)) || (rc = run_loss(d, rgb, target, nullptr)) || (rc = backward(d))) return rc;
    if (loss) {
        float s = 0;
        DCK(cudaMemcpyAsync(&s, d->lossSum.p, 4, cudaMemcpyDeviceToHost, d->stream));
        DCK(cudaStreamSynchronize(d->stream));
        *loss = s / (float)(3 * P);
    }
    return check_err(d, "denoiser forward/backward");
}

// One Adam step (Kingma & Ba 2015) with the current gradients, then the bf16 re-layout.
int adam_step(wrk_denoiser* d, float lr) {
    d->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.0f - std::pow(b1, (float)d->step), c2 = 1.0f - std::pow(b2, (float)d->step);
    k_adam<<<grid_for(d->nparams), 256, 0, d->stream>>>(d->params.as<float>(), d->grads.as<float>(),
                                                        d->adamM.as<float>(), d->adamV.as<float>(), d->nparams, lr, b1,
                                                        b2, 1e-8f, c1, c2);
    DCK(cudaGetLastError());
    return relayout_all(d);
}

}  // namespace

extern "C" {

int wrk_conv3x3_forward(const void* x, uint32_t B, uint32_t H, uint32_t W, uint32_t Cin, const void* w,
                        const float* bias, uint32_t Cout, uint32_t flags, void* out) {
    if (!x || !w || !out) return dfail(WRK_ERR_INVALID, "null conv argument");
    if (Cin % 16 || Cout == 0 || Cout > 256 || H % 8 || W % 16 || B == 0)
        return dfail(WRK_ERR_INVALID, "conv shape unsupported (Cin %% 16, Cout <= 256, H %% 8, W %% 16)");
    int dev = 0, sms = 148;
    DCK(cudaGetDevice(&dev));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t N = pad16(Cout);
    DBuf wpad, err;
    const void* wp = w;
    if (N != Cout) {  // pad the weight rows to a multiple of 16 with zeros
        if (wpad.alloc((size_t)N * 9 * Cin * 2)) return dfail(WRK_ERR_CUDA, "weight padding allocation failed");
        DCK(cudaMemset(wpad.p, 0, (size_t)N * 9 * Cin * 2));
        DCK(cudaMemcpy(wpad.p, w, (size_t)Cout * 9 * Cin * 2, cudaMemcpyDeviceToDevice));
        wp = wpad.p;
    }
    if (err.alloc(4)) return dfail(WRK_ERR_CUDA, "allocation failed");
    DCK(cudaMemset(err.p, 0, 4));
    conv::FwdPlan plan;
    if (conv::plan_fwd(B, H, W, Cin, N, (uint32_t)sms, &plan)) return dfail(WRK_ERR_INVALID, "no conv plan");
    CUtensorMap mx, mw;
    memset(&mw, 0, sizeof(mw));
    if (conv::make_input_map(plan, x, &mx) ||
        (!plan.halo && conv::make_weight_map(&mw, wp, 9 * Cin, N, plan.chunk, N)))
        return dfail(WRK_ERR_CUDA, "tensor map encoding failed (pointers must be 16-byte aligned)");
    Epilogue ep{};
    ep.bias = bias;
    ep.nBias = bias ? Cout : 0;
    ep.out = out;
    ep.outStride = Cout;
    ep.coutValid = Cout;
    ep.relu = flags & 1u;
    ep.outF32 = (flags >> 1) & 1u;
    DCK(conv::launch_fwd(plan, mx, mw, wp, ep, err.as<uint32_t>(), 0));
    uint32_t e = 0;
    DCK(cudaMemcpy(&e, err.p, 4, cudaMemcpyDeviceToHost));
    if (e) return dfail(WRK_ERR_DEVICE, "conv kernel timed out (flags 0x%x)", e);
    return WRK_OK;
}

int wrk_conv3x3_wgrad(const void* g, const void* x, uint32_t B, uint32_t H, uint32_t W, uint32_t Cin, uint32_t Cout,
                      float* dw) {
    if (!g || !x || !dw) return dfail(WRK_ERR_INVALID, "null conv argument");
    int dev = 0, sms = 148;
    DCK(cudaGetDevice(&dev));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    conv::WgradPlan plan;
    if (conv::plan_wgrad(B, H, W, Cin, Cout, (uint32_t)sms, &plan))
        return dfail(WRK_ERR_INVALID, "weight-gradient shape unsupported (Cin, Cout multiples of 16, H %% 8, W %% 16)");
    DBuf err;
    if (err.alloc(4)) return dfail(WRK_ERR_CUDA, "allocation failed");
    DCK(cudaMemset(err.p, 0, 4));
    CUtensorMap mg, mx;
    if (conv::make_act_map(&mg, g, Cout, W, H, B, plan.ca) || conv::make_act_map(&mx, x, Cin, W, H, B, plan.cb))
        return dfail(WRK_ERR_CUDA, "tensor map encoding failed (pointers must be 16-byte aligned)");
    DCK(conv::launch_wgrad(plan, mg, mx, dw, err.as<uint32_t>(), 0));
    uint32_t e = 0;
    DCK(cudaMemcpy(&e, err.p, 4, cudaMemcpyDeviceToHost));
    if (e) return dfail(WRK_ERR_DEVICE, "weight-gradient kernel timed out (flags 0x%x)", e);
    return WRK_OK;
}

int wrk_denoiser_create(int device, uint32_t seed, wrk_denoiser** out) {
    if (!out) return dfail(WRK_ERR_INVALID, "null out");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return dfail(WRK_ERR_NO_DEVICE, "no CUDA device available");
    if (device < 0 || device >= n) return dfail(WRK_ERR_INVALID, "device %d out of range", device);
    DCK(cudaSetDevice(device));
    wrk_denoiser* d = new wrk_denoiser();
    d->device = device;
    cudaDeviceGetAttribute(&d->numSMs, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&d->ev0) != cudaSuccess || cudaEventCreate(&d->ev1) != cudaSuccess) {
        delete d;
        return dfail(WRK_ERR_CUDA, "stream creation failed");
    }
    int rc = alloc_params(d, seed);
    if (!rc) rc = relayout_all(d);
    if (!rc && cudaStreamSynchronize(d->stream) != cudaSuccess) rc = dfail(WRK_ERR_CUDA, "denoiser init failed");
    if (rc) {
        delete d;
        return rc;
    }
    *out = d;
    return WRK_OK;
}

int wrk_denoiser_destroy(wrk_denoiser* d) {
    if (d) {
        cudaSetDevice(d->device);
        cudaStreamSynchronize(d->stream);
        delete d;
    }
    return WRK_OK;
}

int wrk_denoiser_num_params(wrk_denoiser* d, uint64_t* n) {
    if (!d || !n) return dfail(WRK_ERR_INVALID, "null argument");
    *n = d->nparams;
    return WRK_OK;
}

int wrk_denoiser_get_params(wrk_denoiser* d, float* h, uint64_t n) {
    if (!d || !h || n != d->nparams) return dfail(WRK_ERR_INVALID, "parameter buffer must hold %zu floats", d ? d->nparams : 0);
    DCK(cudaSetDevice(d->device));
    DCK(cudaStreamSynchronize(d->stream));
    DCK(cudaMemcpy(h, d->params.p, n * 4, cudaMemcpyDeviceToHost));
    return WRK_OK;
}

int wrk_denoiser_set_params(wrk_denoiser* d, const float* h, uint64_t n) {
    if (!d || !h || n != d->nparams) return dfail(WRK_ERR_INVALID, "parameter buffer must hold %zu floats", d ? d->nparams : 0);
    DCK(cudaSetDevice(d->device));
    DCK(cudaStreamSynchronize(d->stream));
    DCK(cudaMemcpy(d->params.p, h, n * 4, cudaMemcpyHostToDevice));
    DCK(cudaMemset(d->adamM.p, 0, n * 4));
    DCK(cudaMemset(d->adamV.p, 0, n * 4));
    d->step = 0;
    int rc = relayout_all(d);
    if (rc) return rc;
    DCK(cudaStreamSynchronize(d->stream));
    return WRK_OK;
}

int wrk_denoiser_gradients(wrk_denoiser* d, const float* rgb, const float* alb, const float* nrm, const float* target,
                           uint32_t B, uint32_t H, uint32_t W, float* h_grads, float* loss) {
    int rc = fwd_bwd(d, rgb, alb, nrm, target, B, H, W, loss);
    if (rc) return rc;
    if (h_grads) DCK(cudaMemcpy(h_grads, d->grads.p, d->nparams * 4, cudaMemcpyDeviceToHost));
    return WRK_OK;
}

int wrk_denoiser_train_step(wrk_denoiser* d, const float* rgb, const float* alb, const float* nrm, const float* target,
                            uint32_t B, uint32_t H, uint32_t W, float lr, float* loss) {
    if (!d) return dfail(WRK_ERR_INVALID, "null denoiser");
    DCK(cudaSetDevice(d->device));
    DCK(cudaEventRecord(d->ev0, d->stream));
    int rc = fwd_bwd(d, rgb, alb, nrm, target, B, H, W, loss);
    if (rc) return rc;
    if ((rc = adam_step(d, lr))) return rc;
    DCK(cudaEventRecord(d->ev1, d->stream));
    DCK(cudaStreamSynchronize(d->stream));
    cudaEventElapsedTime(&d->lastMs, d->ev0, d->ev1);
    return WRK_OK;
}

// Data-parallel training: the gradients of the last forward / backward pass are
// copied out (device to device), averaged across ranks by the caller's collective,
// written back, and applied.
int wrk_denoiser_grads_copy(wrk_denoiser* d, float* d_out) {
    if (!d || !d_out) return dfail(WRK_ERR_INVALID, "null argument");
    DCK(cudaSetDevice(d->device));
    DCK(cudaMemcpyAsync(d_out, d->grads.p, d->nparams * 4, cudaMemcpyDeviceToDevice, d->stream));
    DCK(cudaStreamSynchronize(d->stream));
    return WRK_OK;
}

int wrk_denoiser_grads_set(wrk_denoiser* d, const float* d_in) {
    if (!d || !d_in) return dfail(WRK_ERR_INVALID, "null argument");
    DCK(cudaSetDevice(d->device));
    DCK(cudaMemcpyAsync(d->grads.p, d_in, d->nparams * 4, cudaMemcpyDeviceToDevice, d->stream));
    DCK(cudaStreamSynchronize(d->stream));
    return WRK_OK;
}

int wrk_denoiser_apply(wrk_denoiser* d, float lr) {
    if (!d) return dfail(WRK_ERR_INVALID, "null denoiser");
    DCK(cudaSetDevice(d->device));
    int rc = adam_step(d, lr);
    if (rc) return rc;
    DCK(cudaStreamSynchronize(d->stream));
    return WRK_OK;
}

// Weights file: "WRKUNET1", u64 count, u64 metadata bytes, count bf16 bit patterns
// (the precision inference uses), then the metadata (JSON text).
int wrk_denoiser_load(wrk_denoiser* d, const char* path) {
    if (!d || !path) return dfail(WRK_ERR_INVALID, "null argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return dfail(WRK_ERR_INVALID, "cannot open denoiser weights %s", path);
    char magic[8];
    uint64_t count = 0, metaLen = 0;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "WRKUNET1", 8) == 0 &&
              std::fread(&count, 8, 1, f) == 1 && std::fread(&metaLen, 8, 1, f) == 1 && count == d->nparams;
    std::vector<uint16_t> bits(ok ? count : 0);
    ok = ok && std::fread(bits.data(), 2, count, f) == count;
    std::fclose(f);
    if (!ok) return dfail(WRK_ERR_INVALID, "%s is not a weights file for this network (%zu parameters)", path, d->nparams);
    std::vector<float> h(count);
    for (size_t i = 0; i < count; ++i) {
        uint32_t u = (uint32_t)bits[i] << 16;
        std::memcpy(&h[i], &u, 4);
    }
    return wrk_denoiser_set_params(d, h.data(), count);
}

int wrk_denoiser_last_ms(wrk_denoiser* d, float* ms) {
    if (!d || !ms) return dfail(WRK_ERR_INVALID, "null argument");
    *ms = d->lastMs;
    return WRK_OK;
}

int wrk_denoiser_infer(wrk_denoiser* d, const float* rgb, const float* alb, const float* nrm, uint32_t B, uint32_t H,
                       uint32_t W, float* out) {
    if (!d || !rgb || !out || B == 0 || H == 0 || W == 0) return dfail(WRK_ERR_INVALID, "bad denoiser arguments");
    DCK(cudaSetDevice(d->device));
    const uint32_t Hp = (H + 63) / 64 * 64, Wp = (W + 127) / 128 * 128;
    int rc = set_shape(d, B, Hp, Wp);
    if (rc) return rc;
    DCK(cudaMemsetAsync(d->err.p, 0, 4, d->stream));
    DCK(cudaEventRecord(d->ev0, d->stream));
    size_t P = (size_t)B * Hp * Wp;
    k_pack<<<grid_for(P), 256, 0, d->stream>>>(rgb, alb, nrm, B, H, W, Hp, Wp, d->x0.as<__nv_bfloat16>());
    if ((rc = forward(d))) return rc;
    k_unpack<<<grid_for((size_t)B * H * W), 256, 0, d->stream>>>(d->out.as<float>(), rgb, B, H, W, Hp, Wp, out);
    DCK(cudaGetLastError());
    DCK(cudaEventRecord(d->ev1, d->stream));
    rc = check_err(d, "denoiser inference");
    if (!rc) cudaEventElapsedTime(&d->lastMs, d->ev0, d->ev1);
    return rc;
}

}  // extern "C"
