// Host interface of the tcgen05 convolution kernels (conv_tc.cu).
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace wrk {
namespace conv {

struct FwdShape {
    uint32_t B, H, W, Cin, N;  // N = output channels padded to a multiple of 16 (<= 256)
    uint32_t tilesX, tilesY;   // 16 x 8 pixel tiles
    uint32_t stages, tmemCols;
    uint32_t wRow0;            // first weight row (output channel) this launch computes
};

// What the forward kernel does with the accumulator of output channel co < coutValid:
// (+ bias[co]) -> (ReLU) -> (x 0 where mask <= 0) -> store to out[pixel*outStride + outOffset + co]
// as bf16 or f32 (f32 may accumulate into what is there).
struct Epilogue {
    const float* bias;  // bias[co] added for co < nBias
    uint32_t nBias;
    void* out;
    uint32_t outStride, outOffset, coutValid;
    uint32_t relu, outF32, accumulate;
    const __nv_bfloat16* mask;
    uint32_t maskStride, maskOffset;
};

struct WgradShape {
    uint32_t B, H, W, Cin, Cout;  // Cout = channels of G (a multiple of 16)
    uint32_t coutStore;           // rows of dW that exist (<= Cout)
    uint32_t tilesX, tilesY, tilesTotal, tilesPerCta;
    uint32_t NB;  // input channels per block (= N of the MMA)
    uint32_t ciBlocks, coBlocks;
    uint32_t stages, tmemCols;
};

struct FwdPlan {
    FwdShape shape;
    int chunk;
    uint32_t smem, grid;
    bool halo;  // small-N kernel: resident weights, one halo load per 8 x 16 tile
};
struct WgradPlan {
    WgradShape shape;
    uint32_t ca, cb, smem;
    dim3 grid;
};

int chunk_for(uint32_t channels);
// Tensor maps: activations NHWC bf16 (box = boxC channels x 16 x 8 pixels); weights
// as a 2-D [rows][K] bf16 matrix (box = boxK x boxRows).  Return 0 on success.
int make_act_map(CUtensorMap* m, const void* base, uint32_t C, uint32_t W, uint32_t H, uint32_t B, uint32_t boxC);
int make_weight_map(CUtensorMap* m, const void* base, uint32_t K, uint32_t rows, uint32_t boxK, uint32_t boxRows);
int plan_fwd(uint32_t B, uint32_t H, uint32_t W, uint32_t Cin, uint32_t N, uint32_t numSMs, FwdPlan* p);
int plan_wgrad(uint32_t B, uint32_t H, uint32_t W, uint32_t Cin, uint32_t Cout, uint32_t numSMs, WgradPlan* p);
// Input tensor map for a forward plan (tiled or halo boxes); 0 on success.  The halo
// kernel reads the weights straight from memory: its `mw` is not used, so only the
// tiled kernel needs make_weight_map.
int make_input_map(const FwdPlan& p, const void* x, CUtensorMap* mx);
cudaError_t launch_fwd(const FwdPlan& p, const CUtensorMap& mx, const CUtensorMap& mw, const void* w,
                       const Epilogue& ep, uint32_t* err, cudaStream_t st);
cudaError_t launch_wgrad(const WgradPlan& p, const CUtensorMap& mg, const CUtensorMap& mx, float* dW, uint32_t* err,
                         cudaStream_t st);

}  // namespace conv
}  // namespace wrk
