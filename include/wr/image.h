// Image output of libWR's test layer (libWR/test/helpers/image.h:1-11,
// image.cpp:14-49): exposure 2.2, ACES filmic fit, gamma 1/2.2, 8-bit RGB PNG.
// Same namespace and signature, so libWR test code calling savePNG compiles
// unchanged; the tone map runs on the GPU (wrk_tonemap_aces) and failures throw
// std::runtime_error.  Defined inline over the C ABI (plain float pointers), so
// libwrk.so does not depend on which Vec3 the caller compiled with.
//
// Not included by wr/wr.h (libWR's umbrella header does not include its test
// helpers either): a program that links libWR's own helpers/image.cpp keeps its
// savePNG, one that wants this one includes wr/image.h.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>

#include "wr/types.h"
#include "wrk.h"

namespace test_helpers {

inline void savePNG(const char* filename, const wr::Vec3* image, uint32_t width, uint32_t height) {
    if (wrk_image_save_png(filename, reinterpret_cast<const float*>(image), width, height) != WRK_OK)
        throw std::runtime_error(std::string("savePNG(") + (filename ? filename : "") + "): " + wrk_last_error());
}
// Additive: the linear radiance as an OpenEXR (32-bit float B G R) or Radiance
// RGBE file, no tone map.
inline void saveEXR(const char* filename, const wr::Vec3* image, uint32_t width, uint32_t height) {
    if (wrk_exr_write(filename, reinterpret_cast<const float*>(image), width, height) != WRK_OK)
        throw std::runtime_error(std::string("saveEXR(") + (filename ? filename : "") + "): " + wrk_last_error());
}
inline void saveHDR(const char* filename, const wr::Vec3* image, uint32_t width, uint32_t height) {
    if (wrk_hdr_write(filename, reinterpret_cast<const float*>(image), width, height) != WRK_OK)
        throw std::runtime_error(std::string("saveHDR(") + (filename ? filename : "") + "): " + wrk_last_error());
}

}  // namespace test_helpers
