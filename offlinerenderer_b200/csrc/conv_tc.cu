// BF16 3x3 convolutions on the 5th-generation tensor cores (tcgen05 + TMEM + TMA),
// the compute of the learned denoiser that stands in for libWR's closed OptiX AI
// denoiser (libWR/src/internal/denoiser.cpp:17-195, optixDenoiserInvoke at :171).
//
// Layout: activations NHWC bf16, dense channels (C a multiple of 16); weights
// [Cout][3*3][Cin] bf16 (K-major: k = tap*Cin + ci, tap = dy*3 + dx).
//
// k_conv_fwd  -- implicit GEMM, M = 128 output pixels (a 16 x 8 pixel tile),
//                N = Cout (padded to 16, <= 256), K = 9 taps x Cin.  Every K step is
//                one TMA load of the input tile shifted by the tap (zero fill at the
//                image border comes from the TMA out-of-bounds fill) plus one TMA load
//                of the weight slice, both K-major in 32/64/128-byte swizzled rows.
//                Persistent CTAs walk the tiles; one thread issues tcgen05.mma into a
//                double-buffered TMEM accumulator while four warps run the previous
//                tile's epilogue (bias, ReLU, optional ReLU-derivative mask of another
//                tensor, bf16 or f32 store at a channel offset of a wider buffer).
//                Used for the forward pass and, with flipped / transposed weights, for
//                the data gradient.
// k_conv_wgrad -- weight gradient dW[co][tap][ci] = sum_p G[p][co] X[p+tap][ci]:
//                M = 128 output channels, N = input channels, K = pixels; both
//                operands are loaded channel-contiguous (MN-major) so the tap shift
//                lands on the pixel coordinates of the TMA box, never on the
//                16-byte-aligned channel coordinate.  Split over pixel ranges, f32
//                vector atomics into dW.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "conv_tc.h"
#include "tc_conv.cuh"

namespace wrk {
namespace conv {

using namespace tc;

constexpr uint32_t kTileW = 16, kTileH = 8, kTileP = 128;

__host__ __device__ inline uint32_t round_up(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

// ---------------------------------------------------------------------------
// Epilogue of one 128-pixel tile: thread (warp w, lane l) owns TMEM lane / tile
// row 32w + l and its N accumulator columns starting at `col`.
__device__ __forceinline__ void fwd_epilogue(const FwdShape& sh, const Epilogue& ep, uint32_t tmem, uint32_t col,
                                             uint32_t warp, uint32_t lane, uint32_t b, uint32_t h0, uint32_t w0,
                                             uint32_t tileW = kTileW) {
    const uint32_t row = warp * 32 + lane;
    const uint32_t h = h0 + row / tileW, w = w0 + row % tileW;
    const size_t pix = ((size_t)b * sh.H + h) * sh.W + w;
    for (uint32_t c0 = 0; c0 < sh.N; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + ((warp * 32u) << 16) + col + c0, v);
        if (c0 >= ep.coutValid) continue;
        const uint32_t nv = min(16u, ep.coutValid - c0);
#pragma unroll
        for (uint32_t j = 0; j < 16; ++j) {
            float x = v[j];
            if (ep.bias && c0 + j < ep.nBias) x += ep.bias[c0 + j];
            if (ep.relu) x = fmaxf(x, 0.0f);
            v[j] = x;
        }
        if (ep.mask) {
            const __nv_bfloat16* m = ep.mask + pix * ep.maskStride + ep.maskOffset + c0;
#pragma unroll
            for (uint32_t j = 0; j < 16; ++j)
                if (j < nv && !(__bfloat162float(m[j]) > 0.0f)) v[j] = 0.0f;
        }
        if (ep.outF32) {
            float* o = (float*)ep.out + pix * ep.outStride + ep.outOffset + c0;
            if (nv == 16 && ((uintptr_t)o & 15u) == 0) {
#pragma unroll
                for (uint32_t j = 0; j < 16; j += 4) {
                    float4 x = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
                    if (ep.accumulate) {
                        float4 y = *(float4*)(o + j);
                        x.x += y.x;
                        x.y += y.y;
                        x.z += y.z;
                        x.w += y.w;
                    }
                    *(float4*)(o + j) = x;
                }
            } else {
                for (uint32_t j = 0; j < nv; ++j) o[j] = ep.accumulate ? o[j] + v[j] : v[j];
            }
        } else {
            __nv_bfloat16* o = (__nv_bfloat16*)ep.out + pix * ep.outStride + ep.outOffset + c0;
            if (nv == 16 && ((uintptr_t)o & 15u) == 0) {
                uint32_t p[8];
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j) {
                    __nv_bfloat162 t = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
                    p[j] = *(uint32_t*)&t;
                }
                *(uint4*)o = make_uint4(p[0], p[1], p[2], p[3]);
                *(uint4*)(o + 8) = make_uint4(p[4], p[5], p[6], p[7]);
            } else {
                for (uint32_t j = 0; j < nv; ++j) o[j] = __float2bfloat16_rn(v[j]);
            }
        }
    }
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Persistent: each CTA walks tiles blockIdx.x, += gridDim.x.  Warps 0-3 run the
// epilogue, warp 4 the TMA producer, warp 5 the MMA issuer.  The stage ring runs
// across tile boundaries, and the accumulator is double-buffered in TMEM (columns
// [0, N) and [N, 2N)), so the epilogue of one tile overlaps the next tile's loads
// and MMAs.
template <int CHUNK>
__global__ void __launch_bounds__(192, 1)
    k_conv_fwd(const __grid_constant__ CUtensorMap mx, const __grid_constant__ CUtensorMap mw, FwdShape sh, Epilogue ep,
               uint32_t* err) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    constexpr uint32_t kRow = CHUNK * 2;  // bytes per pixel row / weight row in a stage
    constexpr uint32_t kABytes = kTileP * kRow;
    const uint32_t bBytes = round_up(sh.N * kRow, 1024);
    const uint32_t stageBytes = kABytes + bBytes;
    const uint32_t S = sh.stages;
    uint64_t* bars = (uint64_t*)(smem + S * stageBytes);
    // bars: full[S] empty[S] accFull[2] accEmpty[2] drain
    uint32_t* tmemSlot = (uint32_t*)(bars + 2 * S + 5);
    volatile uint32_t* abortFlag = tmemSlot + 1;
    const uint32_t base = smem_u32(smem);
    auto full = [&](uint32_t s) { return smem_u32(bars + s); };
    auto empty = [&](uint32_t s) { return smem_u32(bars + S + s); };
    auto accFull = [&](uint32_t b) { return smem_u32(bars + 2 * S + b); };
    auto accEmpty = [&](uint32_t b) { return smem_u32(bars + 2 * S + 2 + b); };
    const uint32_t drain = smem_u32(bars + 2 * S + 4);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < S; ++s) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        for (uint32_t b = 0; b < 2; ++b) {
            mbar_init(accFull(b), 1);
            mbar_init(accEmpty(b), 128);
        }
        mbar_init(drain, 1);
        *abortFlag = 0;
        fence_mbar_init();
        prefetch_map(&mx);
        prefetch_map(&mw);
    }
    if (warp == 0) {
        tmem_alloc(smem_u32(tmemSlot), sh.tmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmemSlot;

    const uint32_t perImg = sh.tilesX * sh.tilesY;
    const uint32_t numTiles = sh.B * perImg;
    const uint32_t nChunk = sh.Cin / CHUNK;
    const uint32_t kSteps = 9 * nChunk;

    if (warp == 4) {
        if (lane == 0) {  // TMA producer
            uint32_t kg = 0, issued = 0;
            for (uint32_t tile = blockIdx.x; tile < numTiles && !*abortFlag; tile += gridDim.x) {
                const uint32_t b = tile / perImg, rem = tile % perImg;
                const int h0 = (int)((rem / sh.tilesX) * kTileH), w0 = (int)((rem % sh.tilesX) * kTileW);
                for (uint32_t k = 0; k < kSteps; ++k, ++kg) {
                    const uint32_t s = kg % S, round = kg / S;
                    if (*abortFlag || !mbar_wait(empty(s), (round & 1u) ^ 1u)) {
                        *abortFlag = 1;
                        break;
                    }
                    const uint32_t tap = k / nChunk, cc = k % nChunk;
                    const int dy = (int)(tap / 3) - 1, dx = (int)(tap % 3) - 1;
                    mbar_expect_tx(full(s), kABytes + sh.N * kRow);
                    tma_load_4d(base + s * stageBytes, &mx, full(s), (int)(cc * CHUNK), w0 + dx, h0 + dy, (int)b);
                    tma_load_2d(base + s * stageBytes + kABytes, &mw, full(s), (int)(tap * sh.Cin + cc * CHUNK),
                                (int)sh.wRow0);
                    ++issued;
                }
            }
            if (*abortFlag) {  // let the copies in flight land before the block exits (bounded)
                for (uint32_t k = issued > S ? issued - S : 0; k < issued; ++k) mbar_wait(full(k % S), (k / S) & 1u);
            }
        }
    } else if (warp == 5) {
        if (lane == 0) {  // MMA issuer
            const uint32_t idesc = idesc_bf16(sh.N, false, false);
            const uint32_t layout = layout_for_row_bytes(kRow);
            uint32_t kg = 0, it = 0;
            for (uint32_t tile = blockIdx.x; tile < numTiles && !*abortFlag; tile += gridDim.x, ++it) {
                const uint32_t buf = it & 1u, use = it >> 1;
                if (!mbar_wait(accEmpty(buf), (use & 1u) ^ 1u)) {
                    *abortFlag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t acc = tmem + buf * sh.N;
                for (uint32_t k = 0; k < kSteps; ++k, ++kg) {
                    const uint32_t s = kg % S, round = kg / S;
                    if (*abortFlag || !mbar_wait(full(s), round & 1u)) {
                        *abortFlag = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a0 = base + s * stageBytes, b0 = a0 + kABytes;
#pragma unroll
                    for (uint32_t kk = 0; kk < CHUNK / 16; ++kk) {
                        const uint64_t ad = sdesc(a0 + kk * 32, 16, 8 * kRow, layout);
                        const uint64_t bd = sdesc(b0 + kk * 32, 16, 8 * kRow, layout);
                        umma_bf16(acc, ad, bd, idesc, (k | kk) ? 1u : 0u);
                    }
                    umma_commit(empty(s));
                }
                umma_commit(accFull(buf));
            }
            // every MMA this thread issued has completed before TMEM is released
            umma_commit(drain);
            mbar_wait(drain, 0);
        }
    } else {
        // epilogue warps 0-3
        uint32_t it = 0;
        for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++it) {
            const uint32_t buf = it & 1u, use = it >> 1;
            const bool ready = mbar_wait(accFull(buf), use & 1u);
            // warp-uniform decision: tcgen05.ld below is .sync.aligned
            const bool go = __all_sync(0xffffffffu, ready && !*abortFlag);
            tc_fence_after();
            if (!go) {
                *abortFlag = 1;
                break;
            }
            const uint32_t b = tile / perImg, rem = tile % perImg;
            fwd_epilogue(sh, ep, tmem, buf * sh.N, warp, lane, b, (rem / sh.tilesX) * kTileH,
                         (rem % sh.tilesX) * kTileW);
            tc_fence_before();
            mbar_arrive(accEmpty(buf));
        }
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *abortFlag) atomicOr(err, 1u);
    if (warp == 0) tmem_dealloc(tmem, sh.tmemCols);
}

// ---------------------------------------------------------------------------
// Small-N variant (N <= 128, 9*Cin*N bf16 weights <= 72 KB): the whole weight tensor
// stays in shared memory for the CTA's life, and each 8 x 16 pixel tile needs one
// TMA load per 8-channel group of its 10 x 18 pixel halo.  Operands use the
// non-swizzled K-major layout (8 x 16-byte core matrices): the halo is stored
// [channel group][pixel][8 channels], so the view of the 128 output pixels shifted
// by tap (dy, dx) starts (dy*10 + dx) * 16 bytes in, with core matrices (8
// consecutive pixels of one row) 160 bytes apart along M and 2944 bytes (one
// 2880-byte channel group, padded to 128 bytes) apart along K: all nine taps are descriptors into the same halo, and the input crosses
// L2 -> shared memory once instead of nine times.
constexpr uint32_t kHaloW = 10, kHaloH = 18, kHaloPix = kHaloW * kHaloH, kHTileW = 8, kHTileH = 16;
// one channel group of a halo: 180 pixels x 16 bytes = 2880, padded so every TMA
// destination stays 128-byte aligned
constexpr uint32_t kHaloGroupBytes = 2944;

// CIN > 0: the input channel count is a compile-time constant, so the MMA issuer's
// 9 x CIN/16 descriptors are fixed offsets from one base descriptor per tile
// (0 = read sh.Cin at run time).
template <int CIN>
__global__ void __launch_bounds__(192, 1)
    k_conv_fwd_halo(const __grid_constant__ CUtensorMap mh, const __nv_bfloat16* __restrict__ wgt, FwdShape sh,
                    Epilogue ep, uint32_t* err) {
    if (CIN > 0) sh.Cin = CIN;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const uint32_t G = sh.Cin / 8;                      // channel groups
    const uint32_t haloBytes = G * kHaloPix * 16;       // bytes one stage's TMA loads deliver
    const uint32_t stageBytes = round_up(G * kHaloGroupBytes, 1024);
    const uint32_t wBytes = round_up(9 * sh.Cin * sh.N * 2, 1024);
    const uint32_t S = sh.stages;
    uint8_t* wsm = smem + S * stageBytes;
    uint64_t* bars = (uint64_t*)(wsm + wBytes);
    uint32_t* tmemSlot = (uint32_t*)(bars + 2 * S + 5);
    volatile uint32_t* abortFlag = tmemSlot + 1;
    const uint32_t base = smem_u32(smem), wbase = smem_u32(wsm);
    auto full = [&](uint32_t s) { return smem_u32(bars + s); };
    auto empty = [&](uint32_t s) { return smem_u32(bars + S + s); };
    auto accFull = [&](uint32_t b) { return smem_u32(bars + 2 * S + b); };
    auto accEmpty = [&](uint32_t b) { return smem_u32(bars + 2 * S + 2 + b); };
    const uint32_t drain = smem_u32(bars + 2 * S + 4);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;

    // weights -> shared memory, [k group][n][8 channels] (k = tap * Cin + ci)
    {
        const uint32_t K = 9 * sh.Cin, units = K / 8 * sh.N;
        for (uint32_t u = threadIdx.x; u < units; u += blockDim.x) {
            const uint32_t kg = u / sh.N, n = u % sh.N;
            const uint4 v = *reinterpret_cast<const uint4*>(wgt + (size_t)(n + sh.wRow0) * K + kg * 8);
            *reinterpret_cast<uint4*>(wsm + ((size_t)kg * sh.N + n) * 16) = v;
        }
        fence_proxy_async();
    }
    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < S; ++s) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        for (uint32_t b = 0; b < 2; ++b) {
            mbar_init(accFull(b), 1);
            mbar_init(accEmpty(b), 128);
        }
        mbar_init(drain, 1);
        *abortFlag = 0;
        fence_mbar_init();
        prefetch_map(&mh);
    }
    if (warp == 0) {
        tmem_alloc(smem_u32(tmemSlot), sh.tmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmemSlot;

    const uint32_t perImg = sh.tilesX * sh.tilesY;  // 8 x 16 tiles
    const uint32_t numTiles = sh.B * perImg;

    if (warp == 4) {
        if (lane == 0) {  // TMA producer: one halo per tile
            uint32_t it = 0, issued = 0;
            for (uint32_t tile = blockIdx.x; tile < numTiles && !*abortFlag; tile += gridDim.x, ++it) {
                const uint32_t s = it % S, round = it / S;
                if (!mbar_wait(empty(s), (round & 1u) ^ 1u)) {
                    *abortFlag = 1;
                    break;
                }
                const uint32_t b = tile / perImg, rem = tile % perImg;
                const int h0 = (int)((rem / sh.tilesX) * kHTileH), w0 = (int)((rem % sh.tilesX) * kHTileW);
                mbar_expect_tx(full(s), haloBytes);
                for (uint32_t g = 0; g < G; ++g)
                    tma_load_4d(base + s * stageBytes + g * kHaloGroupBytes, &mh, full(s), (int)(g * 8), w0 - 1,
                                h0 - 1, (int)b);
                ++issued;
            }
            if (*abortFlag) {
                for (uint32_t k = issued > S ? issued - S : 0; k < issued; ++k) mbar_wait(full(k % S), (k / S) & 1u);
            }
        }
    } else if (warp == 5) {
        if (lane == 0) {  // MMA issuer
            const uint32_t idesc = idesc_bf16(sh.N, false, false);
            const uint32_t lboA = kHaloGroupBytes, sboA = kHaloW * 16;  // K step of 8 channels, M step of 8 pixels
            const uint32_t lboB = sh.N * 16, sboB = 8 * 16;
            uint32_t it = 0;
            for (uint32_t tile = blockIdx.x; tile < numTiles && !*abortFlag; tile += gridDim.x, ++it) {
                const uint32_t buf = it & 1u, use = it >> 1;
                const uint32_t s = it % S, round = it / S;
                if (!mbar_wait(accEmpty(buf), (use & 1u) ^ 1u) || !mbar_wait(full(s), round & 1u)) {
                    *abortFlag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t acc = tmem + buf * sh.N;
                // descriptors advance by (byte offset >> 4) in their low 14-bit address field
                const uint64_t a0 = sdesc(base + s * stageBytes, lboA, sboA, 0);
                const uint64_t b0 = sdesc(wbase, lboB, sboB, 0);
                const uint32_t nUnits = sh.N;  // lboB >> 4
                constexpr uint32_t kKC = CIN > 0 ? CIN / 16 : 8;
#pragma unroll
                for (uint32_t tap = 0; tap < 9; ++tap) {
                    const uint32_t shift = ((tap / 3) * kHaloW + (tap % 3));  // 16-byte units
#pragma unroll
                    for (uint32_t kk = 0; kk < kKC; ++kk) {
                        if (CIN == 0 && kk >= sh.Cin / 16) break;
                        const uint64_t ad = a0 + (2 * kk * (kHaloGroupBytes >> 4) + shift);
                        const uint64_t bd = b0 + ((tap * sh.Cin + 16 * kk) / 8) * nUnits;
                        umma_bf16(acc, ad, bd, idesc, (tap | kk) ? 1u : 0u);
                    }
                }
                umma_commit(empty(s));
                umma_commit(accFull(buf));
            }
            umma_commit(drain);
            mbar_wait(drain, 0);
        }
    } else {
        uint32_t it = 0;
        for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++it) {
            const uint32_t buf = it & 1u, use = it >> 1;
            const bool ready = mbar_wait(accFull(buf), use & 1u);
            const bool go = __all_sync(0xffffffffu, ready && !*abortFlag);
            tc_fence_after();
            if (!go) {
                *abortFlag = 1;
                break;
            }
            const uint32_t b = tile / perImg, rem = tile % perImg;
            fwd_epilogue(sh, ep, tmem, buf * sh.N, warp, lane, b, (rem / sh.tilesX) * kHTileH,
                         (rem % sh.tilesX) * kHTileW, kHTileW);
            tc_fence_before();
            mbar_arrive(accEmpty(buf));
        }
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *abortFlag) atomicOr(err, 1u);
    if (warp == 0) tmem_dealloc(tmem, sh.tmemCols);
}

// ---------------------------------------------------------------------------
template <int CA, int CB>
__global__ void __launch_bounds__(128, 1)
    k_conv_wgrad(const __grid_constant__ CUtensorMap mg, const __grid_constant__ CUtensorMap mx, WgradShape sh,
                 float* dW, uint32_t* err) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    constexpr uint32_t kRowA = CA * 2, kRowB = CB * 2;
    constexpr uint32_t kAtomA = kTileP * kRowA, kAtomB = kTileP * kRowB;  // one channel group x 128 pixels
    constexpr uint32_t kAtomsA = 128 / CA;
    constexpr uint32_t kABytes = kAtomsA * kAtomA;  // 32 KB
    const uint32_t nAtomsB = sh.NB / CB;
    const uint32_t bBytes = nAtomsB * kAtomB;
    const uint32_t stageBytes = kABytes + bBytes;
    const uint32_t S = sh.stages;
    uint64_t* bars = (uint64_t*)(smem + S * stageBytes);
    uint32_t* tmemSlot = (uint32_t*)(bars + 2 * S + 1);
    volatile uint32_t* abortFlag = tmemSlot + 1;
    const uint32_t base = smem_u32(smem);
    auto full = [&](uint32_t s) { return smem_u32(bars + s); };
    auto empty = [&](uint32_t s) { return smem_u32(bars + S + s); };
    const uint32_t accum = smem_u32(bars + 2 * S);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;

    const uint32_t tap = blockIdx.z % 9, coBlock = blockIdx.z / 9;
    const uint32_t co0 = coBlock * 128, ci0 = blockIdx.y * sh.NB;
    const uint32_t loadedA = min(kAtomsA, (sh.Cout - co0 + CA - 1) / CA);
    const uint32_t t0 = blockIdx.x * sh.tilesPerCta;
    const uint32_t t1 = min(sh.tilesTotal, t0 + sh.tilesPerCta);
    const int dy = (int)(tap / 3) - 1, dx = (int)(tap % 3) - 1;

    // output-channel groups past Cout are never loaded: zero them once
    if (loadedA < kAtomsA) {
        for (uint32_t s = 0; s < S; ++s) {
            uint4* z = (uint4*)(smem + s * stageBytes + loadedA * kAtomA);
            const uint32_t n16 = (kAtomsA - loadedA) * kAtomA / 16;
            for (uint32_t i = threadIdx.x; i < n16; i += blockDim.x) z[i] = make_uint4(0, 0, 0, 0);
        }
        fence_proxy_async();
    }
    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < S; ++s) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        mbar_init(accum, 1);
        *abortFlag = 0;
        fence_mbar_init();
        prefetch_map(&mg);
        prefetch_map(&mx);
    }
    if (warp == 1) {
        tmem_alloc(smem_u32(tmemSlot), sh.tmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmemSlot;
    const uint32_t perImg = sh.tilesX * sh.tilesY;
    const uint32_t kSteps = t1 > t0 ? t1 - t0 : 0;

    if (warp == 0 && lane == 0) {
        uint32_t issued = 0;
        for (uint32_t k = 0; k < kSteps; ++k) {
            const uint32_t s = k % S, round = k / S;
            if (*abortFlag || !mbar_wait(empty(s), (round & 1u) ^ 1u)) {
                *abortFlag = 1;
                break;
            }
            const uint32_t t = t0 + k;
            const uint32_t b = t / perImg, rem = t % perImg;
            const int h0 = (int)((rem / sh.tilesX) * kTileH), w0 = (int)((rem % sh.tilesX) * kTileW);
            mbar_expect_tx(full(s), loadedA * kAtomA + bBytes);
            const uint32_t sa = base + s * stageBytes;
            for (uint32_t a = 0; a < loadedA; ++a)
                tma_load_4d(sa + a * kAtomA, &mg, full(s), (int)(co0 + a * CA), w0, h0, (int)b);
            for (uint32_t a = 0; a < nAtomsB; ++a)
                tma_load_4d(sa + kABytes + a * kAtomB, &mx, full(s), (int)(ci0 + a * CB), w0 + dx, h0 + dy, (int)b);
            ++issued;
        }
        if (*abortFlag) {
            for (uint32_t k = issued > S ? issued - S : 0; k < issued; ++k) mbar_wait(full(k % S), (k / S) & 1u);
        }
    } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = idesc_bf16(sh.NB, true, true);
        const uint32_t layA = layout_for_row_bytes(kRowA), layB = layout_for_row_bytes(kRowB);
        for (uint32_t k = 0; k < kSteps; ++k) {
            const uint32_t s = k % S, round = k / S;
            if (*abortFlag || !mbar_wait(full(s), round & 1u)) {
                *abortFlag = 1;
                break;
            }
            tc_fence_after();
            const uint32_t a0 = base + s * stageBytes, b0 = a0 + kABytes;
#pragma unroll
            for (uint32_t kk = 0; kk < kTileP / 16; ++kk) {
                // 16 pixels = two 8-row groups; LBO = next channel group, SBO = next 8 pixels
                const uint64_t ad = sdesc(a0 + kk * 16 * kRowA, kAtomA, 8 * kRowA, layA);
                const uint64_t bd = sdesc(b0 + kk * 16 * kRowB, kAtomB, 8 * kRowB, layB);
                umma_bf16(tmem, ad, bd, idesc, (k | kk) ? 1u : 0u);
            }
            umma_commit(empty(s));
        }
        umma_commit(accum);
    }
    __syncwarp();

    const bool ready = mbar_wait(accum, 0);
    __syncwarp();
    tc_fence_after();
    if (!ready || *abortFlag) {
        if (threadIdx.x == 0) atomicOr(err, 1u);
    } else if (kSteps > 0) {
        const uint32_t co = co0 + warp * 32 + lane;
        for (uint32_t c0 = 0; c0 < sh.NB; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((warp * 32u) << 16) + c0, v);
            if (co < sh.coutStore) {
                float* o = dW + ((size_t)co * 9 + tap) * sh.Cin + ci0 + c0;
#pragma unroll
                for (uint32_t j = 0; j < 16; j += 4) atomicAdd((float4*)(o + j), make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]));
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) tmem_dealloc(tmem, sh.tmemCols);
}

// ---------------------------------------------------------------------------
// host side
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

static CUtensorMapSwizzle swizzle_for(uint32_t rowBytes) {
    return rowBytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                           : rowBytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
}

int make_act_map(CUtensorMap* m, const void* base, uint32_t C, uint32_t W, uint32_t H, uint32_t B, uint32_t boxC) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return 1;
    if (((uintptr_t)base & 15u) || (C * 2) % 16 || boxC * 2 > 128 || (boxC * 2) % 32) return 2;
    cuuint64_t dims[4] = {C, W, H, B};
    cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    cuuint32_t box[4] = {boxC, kTileW, kTileH, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(boxC * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : 3;
}

int make_weight_map(CUtensorMap* m, const void* base, uint32_t K, uint32_t rows, uint32_t boxK, uint32_t boxRows) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return 1;
    if (((uintptr_t)base & 15u) || (K * 2) % 16 || boxRows > 256) return 2;
    cuuint64_t dims[2] = {K, rows};
    cuuint64_t strides[1] = {(cuuint64_t)K * 2};
    cuuint32_t box[2] = {boxK, boxRows};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(boxK * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : 3;
}

static uint32_t pow2_cols(uint32_t n) {
    uint32_t c = 32;
    while (c < n) c <<= 1;
    return c;
}

// Dynamic shared memory that keeps (blocks per SM) x (TMEM columns) within the 512
// columns of an SM: the allocation of a block that does not fit would wait.
static uint32_t smem_for(uint32_t need, uint32_t tmemCols) {
    const uint32_t smPool = 228 * 1024, perBlockReserve = 1024;
    uint32_t maxBlocks = std::max(1u, 512u / tmemCols);
    uint32_t s = need;
    while (smPool / (s + perBlockReserve) > maxBlocks) s += 1024;
    return s;
}

int chunk_for(uint32_t c) { return c % 64 == 0 ? 64 : c % 32 == 0 ? 32 : 16; }

int plan_fwd(uint32_t B, uint32_t H, uint32_t W, uint32_t Cin, uint32_t N, uint32_t numSMs, FwdPlan* p) {
    if (Cin == 0 || Cin % 16 || N == 0 || N % 16 || N > 256 || W % kTileW || H % kTileH || B == 0) return 1;
    FwdShape& sh = p->shape;
    sh.B = B;
    sh.H = H;
    sh.W = W;
    sh.Cin = Cin;
    sh.N = N;
    sh.tilesX = W / kTileW;
    sh.tilesY = H / kTileH;
    sh.tmemCols = pow2_cols(2 * N);  // double-buffered accumulator
    sh.wRow0 = 0;
    p->chunk = chunk_for(Cin);
    const uint32_t row = p->chunk * 2;
    const uint32_t stage = kTileP * row + round_up(N * row, 1024);
    uint32_t S = std::max(2u, std::min(8u, (100u * 1024u) / stage));
    if (S * stage > 200u * 1024u) S = std::max(2u, (200u * 1024u) / stage);
    sh.stages = S;
    p->smem = smem_for(S * stage + (2 * S + 5) * 8 + 16 + 1024, sh.tmemCols);
    p->halo = false;
    const uint32_t wBytes = round_up(9 * Cin * N * 2, 1024);
    if (N <= 128 && wBytes <= 72u * 1024u && H % kHTileH == 0 && W % kHTileW == 0) {
        // small N: weights resident, one halo per 8 x 16 tile
        p->halo = true;
        sh.tilesX = W / kHTileW;
        sh.tilesY = H / kHTileH;
        const uint32_t hs = round_up(Cin / 8 * kHaloGroupBytes, 1024);
        uint32_t Sh = std::max(2u, std::min(4u, (200u * 1024u - wBytes) / hs));
        sh.stages = Sh;
        p->smem = smem_for(Sh * hs + wBytes + (2 * Sh + 5) * 8 + 16 + 1024, sh.tmemCols);
    }
    const uint32_t tiles = B * sh.tilesX * sh.tilesY;
    const uint32_t perSM = std::max(1u, std::min(228u * 1024u / (p->smem + 1024u), 512u / sh.tmemCols));
    p->grid = std::min(tiles, perSM * numSMs);
    return 0;
}

static int make_halo_map(CUtensorMap* m, const void* base, uint32_t C, uint32_t W, uint32_t H, uint32_t B) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return 1;
    if (((uintptr_t)base & 15u) || (C * 2) % 16) return 2;
    cuuint64_t dims[4] = {C, W, H, B};
    cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    cuuint32_t box[4] = {8, kHaloW, kHaloH, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : 3;
}

int make_input_map(const FwdPlan& p, const void* x, CUtensorMap* mx) {
    const FwdShape& sh = p.shape;
    if (p.halo) return make_halo_map(mx, x, sh.Cin, sh.W, sh.H, sh.B);
    return make_act_map(mx, x, sh.Cin, sh.W, sh.H, sh.B, p.chunk);
}

int plan_wgrad(uint32_t B, uint32_t H, uint32_t W, uint32_t Cin, uint32_t Cout, uint32_t numSMs, WgradPlan* p) {
    if (Cin == 0 || Cin % 16 || Cout == 0 || Cout % 16 || W % kTileW || H % kTileH || B == 0) return 1;
    WgradShape& sh = p->shape;
    sh.B = B;
    sh.H = H;
    sh.W = W;
    sh.Cin = Cin;
    sh.Cout = Cout;
    sh.coutStore = Cout;
    sh.tilesX = W / kTileW;
    sh.tilesY = H / kTileH;
    sh.tilesTotal = B * sh.tilesX * sh.tilesY;
    sh.NB = Cin <= 256 ? Cin : (Cin % 2 == 0 && (Cin / 2) % 16 == 0 ? Cin / 2 : 0);
    if (sh.NB == 0 || sh.NB > 256) return 1;
    sh.ciBlocks = Cin / sh.NB;
    sh.coBlocks = (Cout + 127) / 128;
    p->ca = std::min<uint32_t>(64, (uint32_t)chunk_for(Cout));
    p->cb = chunk_for(sh.NB);
    if (128 % p->ca) return 1;
    sh.tmemCols = pow2_cols(sh.NB);
    const uint32_t stage = 128 * kTileP * 2 + sh.NB * kTileP * 2;
    uint32_t S = std::max(2u, std::min(6u, (200u * 1024u) / stage));
    sh.stages = S;
    p->smem = smem_for(S * stage + (2 * S + 1) * 8 + 16 + 1024, sh.tmemCols);
    const uint32_t cells = 9 * sh.ciBlocks * sh.coBlocks;
    uint32_t splits = std::max(1u, (2 * numSMs + cells - 1) / cells);
    splits = std::min(splits, sh.tilesTotal);
    sh.tilesPerCta = (sh.tilesTotal + splits - 1) / splits;
    splits = (sh.tilesTotal + sh.tilesPerCta - 1) / sh.tilesPerCta;
    p->grid = dim3(splits, sh.ciBlocks, 9 * sh.coBlocks);
    return 0;
}

template <class K>
static cudaError_t set_smem(K kern, uint32_t bytes) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t launch_fwd(const FwdPlan& p, const CUtensorMap& mx, const CUtensorMap& mw, const void* w,
                       const Epilogue& ep, uint32_t* err, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    if (p.halo) {
        const __nv_bfloat16* wb = (const __nv_bfloat16*)w;
#define WRK_HALO_CASE(C)                                                                       \
    case C:                                                                                    \
        e = set_smem(k_conv_fwd_halo<C>, p.smem);                                             \
        if (e == cudaSuccess) k_conv_fwd_halo<C><<<p.grid, 192, p.smem, st>>>(mx, wb, p.shape, ep, err); \
        break;
        switch (p.shape.Cin) {
            WRK_HALO_CASE(16)
            WRK_HALO_CASE(32)
            WRK_HALO_CASE(64)
            WRK_HALO_CASE(96)
            default:
                e = set_smem(k_conv_fwd_halo<0>, p.smem);
                if (e == cudaSuccess) k_conv_fwd_halo<0><<<p.grid, 192, p.smem, st>>>(mx, wb, p.shape, ep, err);
                break;
        }
#undef WRK_HALO_CASE
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    switch (p.chunk) {
        case 64:
            e = set_smem(k_conv_fwd<64>, p.smem);
            if (e == cudaSuccess) k_conv_fwd<64><<<p.grid, 192, p.smem, st>>>(mx, mw, p.shape, ep, err);
            break;
        case 32:
            e = set_smem(k_conv_fwd<32>, p.smem);
            if (e == cudaSuccess) k_conv_fwd<32><<<p.grid, 192, p.smem, st>>>(mx, mw, p.shape, ep, err);
            break;
        default:
            e = set_smem(k_conv_fwd<16>, p.smem);
            if (e == cudaSuccess) k_conv_fwd<16><<<p.grid, 192, p.smem, st>>>(mx, mw, p.shape, ep, err);
            break;
    }
    return e != cudaSuccess ? e : cudaGetLastError();
}

#define WRK_WGRAD_CASE(A, B)                                                                        \
    if (p.ca == A && p.cb == B) {                                                                   \
        e = set_smem(k_conv_wgrad<A, B>, p.smem);                                                   \
        if (e == cudaSuccess) k_conv_wgrad<A, B><<<p.grid, 128, p.smem, st>>>(mg, mx, p.shape, dW, err); \
        return e != cudaSuccess ? e : cudaGetLastError();                                           \
    }

cudaError_t launch_wgrad(const WgradPlan& p, const CUtensorMap& mg, const CUtensorMap& mx, float* dW, uint32_t* err,
                         cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    WRK_WGRAD_CASE(64, 64)
    WRK_WGRAD_CASE(64, 32)
    WRK_WGRAD_CASE(64, 16)
    WRK_WGRAD_CASE(32, 64)
    WRK_WGRAD_CASE(32, 32)
    WRK_WGRAD_CASE(32, 16)
    WRK_WGRAD_CASE(16, 64)
    WRK_WGRAD_CASE(16, 32)
    WRK_WGRAD_CASE(16, 16)
    return cudaErrorInvalidValue;
}

}  // namespace conv
}  // namespace wrk
