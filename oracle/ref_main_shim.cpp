// Test infrastructure (oracle side; the product never links it).
//
// Linked into libWR's own test programs (libWR/test/cornell_box_var_test.cpp,
// material_showcase_test.cpp, rough_glass_test.cpp of trianglestrip/OfflineRenderer),
// which oracle/Makefile compiles UNMODIFIED from the reference checkout against this
// repository's include/wr headers (with the reference's vendored GLM, so wr::Vec3 is
// glm::vec3 exactly as in libWR) and links with libwrk.so.  Two hooks let a test
// check what such a program rendered:
//
//  * test_helpers::savePNG -- writes the float image the program passes in to
//    "<png path>.f32" (u32 width, u32 height, then width*height*3 floats) and then
//    calls libWR's own savePNG (libWR/test/helpers/image.cpp:23-49, compiled with
//    its function renamed wr_reference_savePNG), so the PNG is the reference
//    writer's.
//  * the linker's --wrap of wr::Renderer::renderNative (the library call every
//    inline wr::Renderer::render ends in) -- before rendering, writes the scene the
//    library holds (read back through the C ABI), the camera and the render
//    parameters to "wr_capture.bin" in the working directory.  The test renders
//    exactly that scene with the oracle.
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#include <wr/wr.h>

#include "wrk.h"

namespace test_helpers {
void wr_reference_savePNG(const char* filename, const wr::Vec3* image, uint32_t width, uint32_t height);

void savePNG(const char* filename, const wr::Vec3* image, uint32_t width, uint32_t height) {
    std::string path = std::string(filename) + ".f32";
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + path);
    uint32_t hdr[2] = {width, height};
    std::fwrite(hdr, sizeof(hdr), 1, f);
    std::fwrite(image, sizeof(float) * 3, (size_t)width * height, f);
    std::fclose(f);
    wr_reference_savePNG(filename, image, width, height);
}
}  // namespace test_helpers

namespace {

template <class T>
std::vector<T> from_device(uint64_t ptr, size_t n) {
    std::vector<T> h(n);
    if (n && ptr && wrk_memcpy_dtoh(h.data(), reinterpret_cast<const void*>(ptr), n * sizeof(T)) != WRK_OK)
        throw std::runtime_error(std::string("capture: read-back failed: ") + wrk_last_error());
    return h;
}

template <class T>
void put(FILE* f, const std::vector<T>& v) {
    uint64_t n = v.size();
    std::fwrite(&n, sizeof(n), 1, f);
    if (n) std::fwrite(v.data(), sizeof(T), v.size(), f);
}

void capture(wr::Scene* scene, const wrk_camera& cam, const wrk_render_params& rp, bool denoise) {
    scene->finalize();
    wrk_scene_buffers b{};
    if (wrk_scene_buffers_get(scene->native(), &b) != WRK_OK)
        throw std::runtime_error(std::string("capture: ") + wrk_last_error());
    std::vector<uint32_t> idx = from_device<uint32_t>(b.indices, 3 * (size_t)b.numTriangles);
    uint32_t nv = 0;
    for (uint32_t i : idx) nv = i + 1 > nv ? i + 1 : nv;
    FILE* f = std::fopen("wr_capture.bin", "wb");
    if (!f) throw std::runtime_error("capture: cannot write wr_capture.bin");
    std::fwrite("WRCAPT01", 8, 1, f);
    std::fwrite(&cam, sizeof(cam), 1, f);
    std::fwrite(&rp, sizeof(rp), 1, f);
    uint32_t dn = denoise ? 1u : 0u;
    std::fwrite(&dn, sizeof(dn), 1, f);
    float env[3];
    scene->environmentRadianceRGB(env);
    std::fwrite(env, sizeof(env), 1, f);
    put(f, from_device<float>(b.vertices, 3 * (size_t)nv));
    put(f, from_device<float>(b.normals, b.normals ? 3 * (size_t)nv : 0));
    put(f, from_device<float>(b.uvs, b.uvs ? 2 * (size_t)nv : 0));
    put(f, idx);
    put(f, from_device<uint32_t>(b.triMaterial, b.numTriangles));
    put(f, from_device<wrk_material>(b.materials, b.numMaterials));
    std::fclose(f);
}

}  // namespace

// wr::Renderer::renderNative(Scene*, const wrk_camera&, const wrk_render_params&,
// float*, float*, float*, bool, const char*): a non-virtual member, so `this` comes
// first; the name is the Itanium mangling oracle/Makefile passes to --wrap.
extern "C" {
void __real__ZN2wr8Renderer12renderNativeEPNS_5SceneERK10wrk_cameraRK17wrk_render_paramsPfS9_S9_bPKc(
    wr::Renderer* self, wr::Scene* scene, const wrk_camera& cam, const wrk_render_params& rp, float* rgb,
    float* albedo, float* normal, bool denoise, const char* weights);

void __wrap__ZN2wr8Renderer12renderNativeEPNS_5SceneERK10wrk_cameraRK17wrk_render_paramsPfS9_S9_bPKc(
    wr::Renderer* self, wr::Scene* scene, const wrk_camera& cam, const wrk_render_params& rp, float* rgb,
    float* albedo, float* normal, bool denoise, const char* weights) {
    if (scene) capture(scene, cam, rp, denoise);
    __real__ZN2wr8Renderer12renderNativeEPNS_5SceneERK10wrk_cameraRK17wrk_render_paramsPfS9_S9_bPKc(
        self, scene, cam, rp, rgb, albedo, normal, denoise, weights);
}
}
