// CPU oracle C API -- test infrastructure only (called from tests/ through ctypes
// and from bench.py's CPU-baseline leg).  Never linked by the product library.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

// 64-byte material record; same field meaning as libWR's MaterialData
// (libWR/src/internal/gpu_types.h:28-37).
typedef struct {
    float albedo[4];
    float emission[4];
    float ior;
    uint32_t type;  // 0 Lambertian, 1 Emissive, 2 Glass, 3 GGXReflection, 4 GGXTransmission
    float roughness;
    float metallic;
    uint32_t albedoTextureId;  // 1-based, 0 = constant albedo
    uint32_t normalTextureId;  // 1-based, 0 = none
    uint32_t pad[2];
} orc_material;

typedef struct {
    const uint8_t* rgba;  // width*height*4 bytes, row-major
    uint32_t width, height;
} orc_texture;

typedef struct {
    const float* vertices;  // 3 floats per vertex
    const float* normals;   // 3 floats per vertex or NULL
    const float* uvs;       // 2 floats per vertex or NULL
    const uint32_t* indices;  // 3 per triangle
    const uint32_t* triMaterial;  // 1 per triangle
    uint32_t numVertices, numTriangles;
    const orc_material* materials;
    uint32_t numMaterials;
    const orc_texture* textures;
    uint32_t numTextures;
    float envRadiance[3];
} orc_scene_desc;

typedef struct {
    float position[3], target[3], up[3];
    float fovY, aspect, focalDistance, lensRadius;
} orc_camera;

typedef struct {
    uint32_t width, height, spp;
    uint32_t useNEE;
    uint32_t maxBounces;
    float rrStartDepth;
    float fireflyClamp;
    uint32_t seed;           // 0 = reference seed formula
    uint32_t maxIterations;  // wavefront iterations per path; 8 = reference host loop
    uint32_t drawOrder;      // 0 = paired draws left-to-right (device build), 1 = right-to-left (g++ host build)
    uint32_t sampleBegin;    // render samples [sampleBegin, sampleBegin+spp)
    uint32_t pixelBegin, pixelEnd;  // pixel sub-range (pixelEnd 0 = all)
} orc_render_params;

typedef struct {
    uint64_t extensionRays, shadowRays, paths;
} orc_stats;

void* orc_scene_create(const orc_scene_desc* d);
void orc_scene_destroy(void* s);
uint32_t orc_scene_num_emissive(void* s);
void orc_scene_light_cdf(void* s, uint32_t* tris, float* cdf);

// Renders into accum-style buffers: rgb = sum/spp (as renderer.cpp:308-313);
// albedo/normal are raw per-pixel sums (as trace.cu:277-283). Any may be NULL.
void orc_render(void* s, const orc_camera* cam, const orc_render_params* p, float* rgb,
                float* albedo, float* normal, int threads, orc_stats* stats);

// Ray queries.  rays: 8 floats each (ox,oy,oz,tmin,dx,dy,dz,tmax).
// out_t/out_prim: closest hit (prim 0xffffffff on miss).  mode 0 = FP32
// Moller-Trumbore via the BVH, 1 = FP64 over all triangles (exact reference),
// 2 = the same FP64 test on the triangles a BVH walk with conservatively widened
// FP64 boxes reaches (equal to mode 1, fast enough for millions of triangles).
void orc_closest(void* s, const float* rays, uint32_t n, int mode, float* out_t, uint32_t* out_prim,
                 int threads);
void orc_occluded(void* s, const float* rays, uint32_t n, uint32_t* out, int threads);

// Camera rays for (pixel, sample): out 8 floats per ray as above.
void orc_camera_rays(const orc_camera* cam, uint32_t width, uint32_t height, const uint32_t* pixels,
                     const uint32_t* samples, uint32_t n, uint32_t seed, float* out);

// Per-function batches (FP32 when prec == 0, FP64 transcription when prec == 1,
// FP32 with correctly rounded sin / cos / pow -- the device library's -- when prec
// == 2; results returned as double).  See orc_api.cpp for the record layouts.
void orc_bsdf_batch(const float* in, uint32_t n, int prec, double* out);
void orc_rng_batch(const uint32_t* seeds, const uint32_t* dims, uint32_t n, uint32_t* hash, float* u);
void orc_cdf_batch(const float* cdf, uint32_t ncdf, const float* u, uint32_t n, uint32_t* out);
void orc_tonemap(const float* rgb, uint32_t npix, uint8_t* out);
void orc_texture_batch(const orc_texture* t, const float* uv, uint32_t n, float* out);
// Stable filter: keeps idx[i] whose stage[idx[i]] != 3 (Terminated); returns count.
uint32_t orc_compact(const uint32_t* stage, const uint32_t* idx, uint32_t n, uint32_t* out);

#ifdef __cplusplus
}
#endif
