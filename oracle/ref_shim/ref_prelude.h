// Host prelude for compiling libWR's device headers (kernels/*.cuh) with g++ so
// that the reference's own shading/sampling code can serve as the oracle's pin
// and as the CPU baseline.  Supplies host versions of the few device intrinsics
// those headers call.  Test infrastructure only.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <algorithm>
#include <atomic>
#include <cuda_runtime.h>

// The kernels define M_PI as a float literal unless the platform already did;
// the reference's MSVC build does not, so drop glibc's double M_PI here.
#undef M_PI

using std::min;
using std::isnan;
using std::isinf;

// Correctly rounded 1/sqrt: the same convention the oracle port and the CUDA
// renderer use (the device rsqrtf is an approximation with no host equivalent).
inline float rsqrtf(float x) { return (float)(1.0 / std::sqrt((double)x)); }

inline float atomicAdd(float* a, float v) { return std::atomic_ref<float>(*a).fetch_add(v); }
inline unsigned int atomicAdd(unsigned int* a, unsigned int v) {
    return std::atomic_ref<unsigned int>(*a).fetch_add(v);
}

// Texture objects are host pointers to an orc_texture; filtering is the oracle's
// bilinear fetch (wrap addressing, normalized float, 8-bit weight fractions).
template <class T> T tex2D(cudaTextureObject_t obj, float u, float v);
template <> float4 tex2D<float4>(cudaTextureObject_t obj, float u, float v);
