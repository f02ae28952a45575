// Image output of libWR's test layer (libWR/test/helpers/image.h:1-11,
// image.cpp:14-49): exposure 2.2, ACES filmic fit, gamma 1/2.2, 8-bit RGB PNG.
// Same namespace and signature, so libWR test mains compile unchanged; the tone
// map runs on the GPU (wrk_tonemap_aces) and failures throw std::runtime_error.
#pragma once
#include <cstdint>

#include "wr/types.h"

namespace test_helpers {

void savePNG(const char* filename, const wr::Vec3* image, uint32_t width, uint32_t height);
// Additive: the linear radiance as an OpenEXR (32-bit float B G R) or Radiance
// RGBE file, no tone map.
void saveEXR(const char* filename, const wr::Vec3* image, uint32_t width, uint32_t height);
void saveHDR(const char* filename, const wr::Vec3* image, uint32_t width, uint32_t height);

}  // namespace test_helpers
