/* wrk.h -- C ABI of the B200 wavefront path tracer (libwrk.so).
 *
 * Plain C: opaque handles, POD structs, pointers and sizes; every call returns
 * an int status (WRK_OK = 0) and wrk_last_error() gives the message of the last
 * failure on the calling thread.  No exception crosses this boundary; the C++
 * layer (include/wr/*.h) rethrows failures as std::runtime_error, the error
 * convention of libWR's CUDA_CHECK / CU_CHECK macros
 * (libWR/src/internal/cuda_utils.h:13-39).
 *
 * Each entry point names the libWR interface it replaces
 * (paths inside trianglestrip/OfflineRenderer).
 */
#ifndef WRK_H
#define WRK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    WRK_OK = 0,
    WRK_ERR_INVALID = 1,   /* bad argument or size */
    WRK_ERR_CUDA = 2,      /* CUDA runtime failure */
    WRK_ERR_STATE = 3,     /* call out of order (e.g. render before finalize) */
    WRK_ERR_NO_DEVICE = 4, /* no CUDA device / extension unusable */
    WRK_ERR_DEVICE = 5     /* a kernel reported an internal error (stack overflow, bad index) */
};

enum { WRK_LAMBERTIAN = 0, WRK_EMISSIVE = 1, WRK_GLASS = 2, WRK_GGX_REFLECTION = 3, WRK_GGX_TRANSMISSION = 4 };

/* 64-byte material record; field meaning of MaterialData
 * (libWR/src/internal/gpu_types.h:28-37). */
typedef struct {
    float albedo[4];
    float emission[4];
    float ior;
    uint32_t type;
    float roughness;
    float metallic;
    uint32_t albedoTextureId; /* 1-based texture id, 0 = constant albedo */
    uint32_t normalTextureId; /* 1-based texture id, 0 = no normal map */
    uint32_t pad[2];
} wrk_material;

/* wr::Camera (libWR/include/wr/types.h:16-51); fovY in radians, vertical. */
typedef struct {
    float position[3], target[3], up[3];
    float fovY, aspect, focalDistance, lensRadius;
} wrk_camera;

/* wr::RenderParams (libWR/include/wr/renderer.h:25-36) plus additive fields. */
typedef struct {
    uint32_t width, height, spp;
    uint32_t useNEE;
    uint32_t maxBounces;
    float russianRouletteDepth;
    float fireflyClamp;
    uint32_t seed;          /* 0 = the reference's per-pixel seed formula (trace.cu:58) */
    uint32_t maxIterations; /* wavefront iterations a path may use; 0 = 8, the reference host loop's cap (renderer.cpp:213) */
    uint32_t flags;         /* WRK_FLAG_* */
    uint32_t sampleOffset;  /* render sample indices [sampleOffset, sampleOffset+spp): splits one image across calls / GPUs */
} wrk_render_params;

/* Guides (albedo / normal) are returned averaged over spp; with this flag they
 * are the raw per-pixel sums libWR keeps (trace.cu:277-283). */
#define WRK_FLAG_RAW_GUIDES 1u
/* Record CUDA events around every kernel of the loop (on the renderer's stream)
 * and report per-stage device time in wrk_render_stats.stageMs. */
#define WRK_FLAG_STAGE_TIMING 2u
/* Served requests: pass the result through the server's learned denoiser. */
#define WRK_FLAG_DENOISE 4u
/* Rays that miss take their radiance from the scene's environment map (lat-long,
 * bilinear, wrap in u, clamp in v: getEnvironmentRadiance of
 * libWR/kernels/utils/environment_sampling.cuh:10-52).  libWR's own miss program
 * adds only the uniform radiance (libWR/kernels/trace.cu:143-148), which stays the
 * default. */
#define WRK_FLAG_ENV_MAP 8u

enum {
    WRK_STAGE_CONTROL = 0,
    WRK_STAGE_GENERATE = 1,
    WRK_STAGE_TRACE_EXTENSION = 2,
    WRK_STAGE_TRACE_SHADOW = 3,
    WRK_STAGE_SHADE_LAMBERT = 4,
    WRK_STAGE_SHADE_DIELECTRIC = 5,
    WRK_STAGE_SHADE_GGX = 6,
    WRK_STAGE_SHADE_EMISSIVE = 7,
    WRK_STAGE_SHADE_LAMBERT_RESUME = 8, /* kept for layout; always 0: the shadow stage continues these paths */
    WRK_NUM_STAGES = 9
};

typedef struct {
    uint64_t paths;          /* camera paths started */
    uint64_t extensionRays;  /* closest-hit rays traced */
    uint64_t shadowRays;     /* any-hit (shadow) queries answered, by traversal or by the
                                light-triangle test of the Lambert shade */
    uint32_t iterations;     /* wavefront iterations issued */
    uint32_t deviceErrors;   /* internal device error flags raised (0 = none) */
    float gpuMs;             /* device time of the render loop (CUDA events) */
    float totalMs;           /* device time including uploads / readback */
    float stageMs[9];        /* per-stage device time (WRK_FLAG_STAGE_TIMING), indexed by WRK_STAGE_* */
    uint32_t stageLaunches[9];
    uint64_t bucketPaths[5]; /* paths shaded per bucket: Lambert, dielectric, GGX, emissive/other, and the
                                Lambert paths the shadow stage continued after their shadow ray */
    uint64_t shadowTraced;   /* the part of shadowRays the any-hit kernel traced (the rest were
                                answered by the Lambert shade's light-triangle test) */
} wrk_render_stats;

typedef struct {
    uint32_t numTriangles;
    uint32_t numNodes;     /* 8-wide BVH nodes (80 bytes each) */
    uint32_t numBinaryNodes;
    uint32_t depth;        /* 8-wide depth */
    uint32_t numEmissive;
    float buildMs;         /* GPU time of the BVH build */
    float sahCost;         /* SAH cost of the 8-wide tree (node visits + triangle tests per ray, area-weighted) */
} wrk_bvh_info;

typedef struct wrk_scene wrk_scene;
typedef struct wrk_renderer wrk_renderer;

const char* wrk_last_error(void);
int wrk_version(void);

/* ---- device memory helpers (for callers without their own allocator) ---- */
int wrk_device_count(int* count);
int wrk_malloc(int device, uint64_t bytes, void** ptr);
int wrk_free(void* ptr);
int wrk_memcpy_htod(void* dst, const void* src, uint64_t bytes);
int wrk_memcpy_dtoh(void* dst, const void* src, uint64_t bytes);
int wrk_synchronize(int device);

/* ---- scene: replaces wr::Scene (libWR/include/wr/scene.h:33-101,
 *      libWR/src/internal/scene.cpp:91-557) ---- */
int wrk_scene_create(int device, wrk_scene** out);
int wrk_scene_destroy(wrk_scene* s);
/* Flat triangle soup as Scene::addTriangleMesh accumulates it (scene.cpp:190-244):
 * vertices 3 floats each; normals (3 each) and uvs (2 each) may be NULL. */
int wrk_scene_set_geometry(wrk_scene* s, const float* vertices, uint32_t numVertices, const float* normals,
                           const float* uvs, const uint32_t* indices, uint32_t numTriangles,
                           const uint32_t* triMaterial);
int wrk_scene_set_materials(wrk_scene* s, const wrk_material* materials, uint32_t numMaterials);
/* RGBA8 texture (Scene::loadTexture, scene.cpp:246-264); returns the 1-based id. */
int wrk_scene_add_texture(wrk_scene* s, const uint8_t* rgba, uint32_t width, uint32_t height, uint32_t* outId);
int wrk_scene_set_environment(wrk_scene* s, const float rgb[3]);
/* Environment map (Scene::setEnvironmentMap, scene.cpp:289-348): width*height RGBA f32
 * texels, row 0 = the +y pole (v = 0); kept on the device after finalize. */
int wrk_scene_set_environment_map(wrk_scene* s, const float* rgba, uint32_t width, uint32_t height);
/* Scene::finalize (scene.cpp:350-557): uploads, builds the emissive list and power
 * CDF (same serial FP32 order as scene.cpp:423-491), builds the 8-wide BVH on the GPU
 * (replaces optixAccelBuild, scene.cpp:493-550). */
int wrk_scene_finalize(wrk_scene* s);
int wrk_scene_bvh_info(wrk_scene* s, wrk_bvh_info* info);
/* Light list / CDF readback (getEmissiveTrianglesBuffer, getEmissiveTriangleCDFBuffer):
 * the emissive triangle ids and their power CDF as the device holds them; *count
 * receives the number of entries.  With tris and cdf both NULL this is a size query;
 * otherwise capacity below the count is WRK_ERR_INVALID. */
int wrk_scene_light_cdf(wrk_scene* s, uint32_t* tris, float* cdf, uint32_t capacity, uint32_t* count);

/* Copies the 8-wide BVH to host memory for inspection: nodes = numNodes * 20 u32
 * (five 16-byte words each), tris = numTriangles * 12 floats (v0|prim, e1|material,
 * e2|bucket per triangle, in leaf order; bucket = the material's shade queue: 0
 * Lambert, 1 glass / rough glass, 2 GGX, 3 emissive or other, plus 8 for a Lambert
 * material with an albedo or normal texture, as a u32).  Sizes come from
 * wrk_scene_bvh_info. */
int wrk_scene_bvh_export(wrk_scene* s, uint32_t* nodes, float* tris);

/* Device addresses of a finalized scene's buffers: the getters of wr::Scene
 * (libWR/include/wr/scene.h:70-93); bvhNodes stands in for the GAS handle. */
typedef struct {
    uint64_t vertices, normals, uvs, indices, triMaterial, materials, emissive, cdf, texels, bvhNodes, bvhTriangles;
    uint32_t numMaterials, numEmissive, numTextures, numTriangles;
} wrk_scene_buffers;
int wrk_scene_buffers_get(wrk_scene* s, wrk_scene_buffers* out);

/* ---- renderer: replaces wr::Renderer::render (libWR/src/internal/renderer.cpp:132-316) ---- */
/* capacity = path slots in flight (0 = chosen from the device). */
int wrk_renderer_create(int device, uint32_t capacity, wrk_renderer** out);
int wrk_renderer_destroy(wrk_renderer* r);
/* Launch shape of the bounce loop: iterations per captured CUDA graph launch
 * (1..64, default 8) and threads per shading block (128 or 256, default 256);
 * wrk_autotune picks them. */
int wrk_renderer_set_launch(wrk_renderer* r, uint32_t chunk, uint32_t shadeBlock);
/* Synchronous render into HOST buffers of width*height*3 floats: rgb = sum/spp
 * (renderer.cpp:308-313), albedo / normal first-hit guides (may be NULL). */
int wrk_render(wrk_renderer* r, wrk_scene* s, const wrk_camera* cam, const wrk_render_params* p, float* rgb,
               float* albedo, float* normal, wrk_render_stats* stats);
/* Same render into DEVICE buffers (float3 per pixel), enqueued on the renderer's
 * stream; the call returns after the loop has finished on the device. */
int wrk_render_device(wrk_renderer* r, wrk_scene* s, const wrk_camera* cam, const wrk_render_params* p, float* d_rgb,
                      float* d_albedo, float* d_normal, wrk_render_stats* stats);

/* ---- serving loop: no counterpart in libWR, which renders one image per
 *      synchronous Renderer::render call (libWR/src/internal/renderer.cpp:132-316) ----
 * A server keeps scenes resident and renders many requests (any size, spp, camera,
 * scene) at once: admitted requests share one set of wavefront queues, new ones
 * join while others are in flight (admission by free slot and by room in an
 * accumulation pool of poolBytes, first come first served), and each step runs one
 * captured CUDA graph of `chunk` bounce iterations for all of them.  A request's
 * image is the same alone and in the mix (RNG keyed by seed, pixel and sample)
 * up to the order of f32 sums.  Scenes must outlive the server. */
typedef struct wrk_server wrk_server;
typedef struct wrk_denoiser wrk_denoiser;
typedef struct {
    uint32_t capacity;     /* path entries in flight (0 = 4M) */
    uint32_t maxRequests;  /* concurrent requests (0 or > 64 = 64) */
    uint64_t poolBytes;    /* HBM for per-request buffers, 96 bytes per pixel (0 = 4 GiB) */
    uint32_t chunk;        /* bounce iterations per step (0 = 8) */
    uint32_t shadeBlock;   /* 128 or 256 (0 = 256) */
} wrk_server_config;
typedef struct {
    uint32_t queued, running, ready;
    uint64_t iterations;   /* bounce iterations run so far */
    float lastChunkMs;     /* device time of the last step's chunk */
    uint64_t poolFreeBytes;
} wrk_server_status;
typedef struct {
    uint32_t width, height, spp, denoised;
    double submitMs, admitMs, readyMs; /* host clock, ms since the server was created */
    uint32_t iterations;               /* bounce iterations from admission to completion */
} wrk_request_info;
int wrk_server_create(int device, const wrk_server_config* cfg, wrk_server** out);
int wrk_server_destroy(wrk_server* s);
/* Requests flagged WRK_FLAG_DENOISE are passed through this denoiser. */
int wrk_server_set_denoiser(wrk_server* s, wrk_denoiser* d);
int wrk_server_submit(wrk_server* s, wrk_scene* scene, const wrk_camera* cam, const wrk_render_params* p,
                      uint64_t* ticket);
/* Admits, runs one chunk for every request in flight, retires finished ones. */
int wrk_server_step(wrk_server* s, wrk_server_status* status);
int wrk_server_poll(wrk_server* s, uint64_t ticket, int* ready);
/* Steps until the request is ready.  A ready request keeps its pool region until
 * its result is taken; when ready results fill the pool (or the slots) so that the
 * awaited request can never be admitted, this returns WRK_ERR_STATE. */
int wrk_server_wait(wrk_server* s, uint64_t ticket);
/* Copies a ready request's images (width*height*3 floats each; rgb is the denoised
 * image when the request asked for it; albedo / normal may be NULL) to host memory
 * (or device memory: _device) and releases the request. */
int wrk_server_result(wrk_server* s, uint64_t ticket, float* rgb, float* albedo, float* normal,
                      wrk_request_info* info);
int wrk_server_result_device(wrk_server* s, uint64_t ticket, float* d_rgb, float* d_albedo, float* d_normal,
                             wrk_request_info* info);

/* ---- autotuner: no counterpart in libWR.  Times one render of the given
 *      workload per launch shape (capacity 1M/4M/16M/32M/64M paths x chunk 4/8/16
 *      x shading block 128/256) and returns the fastest.  Capacities from 4M up are
 *      tried only while their queues (672 bytes per path) plus 512 MB fit in the
 *      device's free memory, so numTrials is 6 to 30. ---- */
typedef struct {
    uint32_t capacity, chunk, shadeBlock;
    float ms;
} wrk_tune_trial;
typedef struct {
    uint32_t capacity, chunk, shadeBlock;
    float bestMs;
    uint32_t numTrials;
    wrk_tune_trial trials[32];
} wrk_tune_result;
int wrk_autotune(int device, wrk_scene* scene, const wrk_camera* cam, const wrk_render_params* p,
                 wrk_tune_result* out);

/* ---- kernel-level entry points (device pointers; synchronous) ---- */
/* Closest hit (optixTrace + __closesthit__trace, trace.cu:127-141):
 * rays = 8 floats each (ox,oy,oz,tmin,dx,dy,dz,tmax); t = +inf and prim = 0xffffffff on miss. */
int wrk_trace_closest(wrk_scene* s, const float* d_rays, uint32_t n, float* d_t, uint32_t* d_prim);
/* Visibility (the Shadow stage of __raygen__trace, trace.cu:27-51): 1 = occluded. */
int wrk_trace_occluded(wrk_scene* s, const float* d_rays, uint32_t n, uint32_t* d_occluded);
/* Stable compaction (compact.cu:6-17): keeps idxIn[i] whose stage[idxIn[i]] != 3,
 * in input order; *d_count receives the survivor count. */
int wrk_compact(const uint32_t* d_stage, const uint32_t* d_idxIn, uint32_t n, uint32_t* d_idxOut, uint32_t* d_count);
/* wrk_compact without any allocation -- no counterpart in the reference (its
 * compact kernel is handed buffers the renderer allocated).  For callers that may
 * not allocate device memory (a fixed, pre-reserved memory budget; an allocator
 * that must own all device memory): the per-tile counts live in a 256 KiB array
 * built into the library, so n is limited to 67,108,864 indices (larger n returns
 * WRK_ERR_INVALID).  The first call on a device resolves that array's address and
 * should come before any stream capture; the address is kept for the life of the
 * process, so a cudaDeviceReset of that device after the first call, or a
 * non-primary driver context made current on it, is not supported.  All calls
 * share the array: calls that overlap on the GPU race and must be serialized by
 * the caller. */
int wrk_compact_noalloc(const uint32_t* d_stage, const uint32_t* d_idxIn, uint32_t n, uint32_t* d_idxOut,
                        uint32_t* d_count);
/* Light selection (sampleEmissiveTriangle, sampling.cuh:116-135). */
int wrk_cdf_sample(const float* d_cdf, uint32_t ncdf, const float* d_u, uint32_t n, uint32_t* d_out);
/* PCG hash with dimension and its uniform (sampling.cuh:24-38). */
int wrk_rng_batch(const uint32_t* d_seed, const uint32_t* d_dim, uint32_t n, uint32_t* d_hash, float* d_u);
/* BSDF / sampling math on the device for batches of records (20 floats in, 34 out):
 * GGX eval/pdf/VNDF sample, dielectric Fresnel, cosine warp, MIS power heuristic,
 * Russian roulette, frames, triangle sampling, shading correction. */
int wrk_bsdf_batch(const float* d_in, uint32_t n, float* d_out);
/* Bilinear RGBA8 texture fetch (wrap, normalized float) of texture id of a finalized scene. */
int wrk_texture_batch(wrk_scene* s, uint32_t textureId, const float* d_uv, uint32_t n, float* d_out);
/* Camera rays for (pixel, sample) pairs (the depth-0 branch of __raygen__trace). */
int wrk_camera_rays(const wrk_camera* cam, uint32_t width, uint32_t height, const uint32_t* d_pixels,
                    const uint32_t* d_samples, uint32_t n, uint32_t seed, float* d_rays);
/* Exposure 2.2, ACES filmic fit, gamma 1/2.2, 8-bit (libWR/test/helpers/image.cpp:14-49). */
int wrk_tonemap_aces(const float* d_rgb, uint32_t numPixels, uint8_t* d_out);
/* savePNG of libWR's test layer (libWR/test/helpers/image.cpp:23-49): host float RGB
 * (width*height*3) tone mapped on the GPU as above and written as an 8-bit RGB PNG. */
int wrk_image_save_png(const char* path, const float* rgb, uint32_t width, uint32_t height);
/* Writes host RGB8 bytes (width*height*3) as a PNG file (zlib deflate); 0 on success. */
int wrk_png_write(const char* path, const uint8_t* rgb8, uint32_t width, uint32_t height);
/* HDR outputs of linear host float RGB (width*height*3, rows top to bottom), no tone
 * map (the next step after accumulation; libWR writes only the 8-bit PNG of
 * libWR/test/helpers/image.cpp:23-49):
 * OpenEXR 2 scan-line file, uncompressed, channels B G R as 32-bit float. */
int wrk_exr_write(const char* path, const float* rgb, uint32_t width, uint32_t height);
/* Radiance .hdr (RGBE, run-length scan lines for 8 <= width < 32768, else flat). */
int wrk_hdr_write(const char* path, const float* rgb, uint32_t width, uint32_t height);

/* ---- learned denoiser: replaces the OptiX AI denoiser of libWR
 *      (libWR/src/internal/denoiser.cpp:17-195: optixDenoiserCreate :30-35,
 *      guide layers :98-116, optixDenoiserInvoke :171-184) ---- */
/* 3x3 convolution, stride 1, zero padding, on the tensor cores (bf16 in, f32
 * accumulate).  x: bf16 NHWC [B][H][W][Cin]; w: bf16 [Cout][3][3][Cin]; bias: f32
 * [Cout] or NULL; out: NHWC [B][H][W][Cout], bf16 or (flags & 2) f32; flags & 1 =
 * ReLU.  Cin a multiple of 16, Cout <= 256, H a multiple of 8, W of 16; device
 * pointers 16-byte aligned.  Kernel-level entry of the denoiser's convolution. */
#define WRK_CONV_RELU 1u
#define WRK_CONV_F32_OUT 2u
int wrk_conv3x3_forward(const void* d_x, uint32_t B, uint32_t H, uint32_t W, uint32_t Cin, const void* d_w,
                        const float* d_bias, uint32_t Cout, uint32_t flags, void* d_out);
/* Weight gradient of that convolution: dw[Cout][3][3][Cin] (f32) += sum over pixels
 * of g[p][co] * x[p + tap][ci]; g: bf16 NHWC [B][H][W][Cout]. */
int wrk_conv3x3_wgrad(const void* d_g, const void* d_x, uint32_t B, uint32_t H, uint32_t W, uint32_t Cin,
                      uint32_t Cout, float* d_dw);

/* A 4-level U-Net (32/64/128/256 channels) on radiance + albedo + normal, weights
 * initialised from `seed`.  Parameters are one f32 array: per layer W [Cout][3][3][Cin]
 * then bias [Cout], layers in the order e0a e0b e1a e1b e2a e2b e3a e3b d2a d2b d1a
 * d1b d0a d0b head. */
int wrk_denoiser_create(int device, uint32_t seed, wrk_denoiser** out);
int wrk_denoiser_destroy(wrk_denoiser* d);
int wrk_denoiser_num_params(wrk_denoiser* d, uint64_t* n);
int wrk_denoiser_get_params(wrk_denoiser* d, float* h_params, uint64_t n);
/* Sets the weights (host array) and resets the optimizer state. */
int wrk_denoiser_set_params(wrk_denoiser* d, const float* h_params, uint64_t n);
/* One forward + backward pass on device images [B][H][W][3] f32 (rgb, albedo, normal,
 * target; H a multiple of 64, W of 128): the L1 loss of log1p(radiance) and the
 * parameter gradients (copied to h_grads when not NULL). */
int wrk_denoiser_gradients(wrk_denoiser* d, const float* d_rgb, const float* d_albedo, const float* d_normal,
                           const float* d_target, uint32_t B, uint32_t H, uint32_t W, float* h_grads, float* loss);
/* Data-parallel training: copy the last pass's gradients out to device memory
 * (num_params floats), overwrite them (e.g. with the average across ranks), and
 * apply one Adam step with the current gradients. */
int wrk_denoiser_grads_copy(wrk_denoiser* d, float* d_out);
int wrk_denoiser_grads_set(wrk_denoiser* d, const float* d_in);
int wrk_denoiser_apply(wrk_denoiser* d, float lr);
/* The same followed by one Adam step with learning rate lr. */
int wrk_denoiser_train_step(wrk_denoiser* d, const float* d_rgb, const float* d_albedo, const float* d_normal,
                            const float* d_target, uint32_t B, uint32_t H, uint32_t W, float lr, float* loss);
/* Loads weights written by offlinerenderer_b200.denoise_train ("WRKUNET1" file:
 * count, metadata length, bf16 parameters, JSON metadata); resets the optimizer. */
int wrk_denoiser_load(wrk_denoiser* d, const char* path);
/* Device time (CUDA events on the denoiser's stream) of the last inference or
 * training step. */
int wrk_denoiser_last_ms(wrk_denoiser* d, float* ms);
/* Denoises device images [B][H][W][3] f32 of any size (padded internally) into d_out. */
int wrk_denoiser_infer(wrk_denoiser* d, const float* d_rgb, const float* d_albedo, const float* d_normal, uint32_t B,
                       uint32_t H, uint32_t W, float* d_out);

#ifdef __cplusplus
}
#endif
#endif /* WRK_H */
