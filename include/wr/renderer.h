// wr::Renderer (libWR/include/wr/renderer.h:10-65).  RenderParams keeps libWR's
// fields; the fields after fireflyClamp are additive extensions.
#pragma once
#include <cstdint>

#include <stdexcept>

#include "wr/scene.h"
#include "wr/types.h"
#include "wrk.h"

namespace wr {

struct RendererConfig {
    uint32_t maxBounces = 8;
    bool useNEE = true;
    float russianRouletteDepth = 3;
};

// libWR's OptiX AI denoiser settings.  Here `enabled` runs the learned U-Net
// denoiser, which always uses the albedo and normal guides it was trained with
// (useAlbedo / useNormal / hdrIntensity are accepted and not needed).
struct DenoiserConfig {
    bool enabled = false;
    bool useAlbedo = false;
    bool useNormal = false;
    float hdrIntensity = 1.0f;
    // --- additive extension ---
    const char* weightsPath = nullptr;  // WRKUNET1 file; null = $WRK_DENOISER_WEIGHTS, else
                                        // weights/unet_scale.wrkw next to libwrk.so
};

struct RenderParams {
    uint32_t width;
    uint32_t height;
    uint32_t spp = 1;
    DenoiserConfig denoiser;

    bool useNEE = true;
    uint32_t maxBounces = 8;
    float russianRouletteDepth = 3.0f;
    float fireflyClamp = 0.0f;

    // --- additive extensions ---
    uint32_t seed = 0;              // 0 = libWR's per-pixel seed formula
    Vec3* albedoOut = nullptr;      // first-hit albedo guide, averaged over spp
    Vec3* normalOut = nullptr;      // first-hit normal guide, averaged over spp
    bool rawGuides = false;         // guides as per-pixel sums (libWR's buffers)
    uint32_t maxIterations = 8;     // wavefront iterations per path (8 = libWR's host loop)
    bool useEnvironmentMap = false; // misses read Scene::setEnvironmentMap's map (libWR: uniform only)
};

struct RenderStats {
    uint64_t paths = 0, extensionRays = 0, shadowRays = 0;
    uint64_t shadowTraced = 0;  // the part of shadowRays traced by the any-hit kernel
    uint32_t iterations = 0;
    float gpuMs = 0.0f, totalMs = 0.0f;
};

struct RendererImpl;

class Renderer {
public:
    Renderer(const RendererConfig& config = {});
    Renderer(const RendererConfig& config, int deviceId);
    ~Renderer();

    // Renders width*height pixels into outputBuffer (sum/spp, renderer.cpp:289-313);
    // with params.denoiser.enabled the learned denoiser runs on the result.
    void render(Scene* scene, const Camera& camera, Vec3* outputBuffer, const RenderParams& params) {
        if (!scene || !outputBuffer) throw std::runtime_error("render: null scene or output buffer");
        wrk_camera c{};
        c.position[0] = camera.position.x, c.position[1] = camera.position.y, c.position[2] = camera.position.z;
        c.target[0] = camera.target.x, c.target[1] = camera.target.y, c.target[2] = camera.target.z;
        c.up[0] = camera.up.x, c.up[1] = camera.up.y, c.up[2] = camera.up.z;
        c.fovY = camera.fovY;
        c.aspect = camera.aspect;
        c.focalDistance = camera.focalDistance;
        c.lensRadius = camera.lensRadius;
        wrk_render_params rp{};
        rp.width = params.width;
        rp.height = params.height;
        rp.spp = params.spp;
        rp.useNEE = params.useNEE ? 1u : 0u;
        rp.maxBounces = params.maxBounces;
        rp.russianRouletteDepth = params.russianRouletteDepth;
        rp.fireflyClamp = params.fireflyClamp;
        rp.seed = params.seed;
        rp.maxIterations = params.maxIterations;
        rp.flags = (params.rawGuides ? WRK_FLAG_RAW_GUIDES : 0u) | (params.useEnvironmentMap ? WRK_FLAG_ENV_MAP : 0u);
        renderNative(scene, c, rp, reinterpret_cast<float*>(outputBuffer), reinterpret_cast<float*>(params.albedoOut),
                     reinterpret_cast<float*>(params.normalOut), params.denoiser.enabled, params.denoiser.weightsPath);
    }
    // libWR's legacy overload (renderer.cpp:318-335).
    void render(Scene* scene, const Camera& camera, Vec3* outputBuffer, uint32_t width, uint32_t height,
                uint32_t spp = 1, bool denoiser = false) {
        RenderParams p;
        p.width = width;
        p.height = height;
        p.spp = spp;
        p.denoiser.enabled = denoiser;
        p.denoiser.useAlbedo = true;
        p.denoiser.useNormal = true;
        render(scene, camera, outputBuffer, p);
    }

    // Additive: statistics of the last render.
    const RenderStats& lastStats() const;

    // Additive: the Vec3-free form the inline render calls (libwrk.so exports only
    // this one).  Host buffers of width*height*3 floats; albedo / normal may be null;
    // denoise runs the learned denoiser with weightsPath (null = the default weights).
    void renderNative(Scene* scene, const wrk_camera& camera, const wrk_render_params& params, float* rgb,
                      float* albedo, float* normal, bool denoise, const char* weightsPath);

private:
    RendererImpl* m_impl;
    RendererConfig m_config;
};

}  // namespace wr
