// wr::Renderer (libWR/include/wr/renderer.h:10-65).  RenderParams keeps libWR's
// fields; the fields after fireflyClamp are additive extensions.
#pragma once
#include <cstdint>

#include "wr/scene.h"
#include "wr/types.h"

struct wrk_renderer;

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
    uint32_t iterations = 0;
    float gpuMs = 0.0f, totalMs = 0.0f;
};

struct RendererImpl;

class Renderer {
public:
    Renderer(const RendererConfig& config = {});
    Renderer(const RendererConfig& config, int deviceId);
    ~Renderer();

    void render(Scene* scene, const Camera& camera, Vec3* outputBuffer, const RenderParams& params);
    void render(Scene* scene, const Camera& camera, Vec3* outputBuffer, uint32_t width, uint32_t height,
                uint32_t spp = 1, bool denoiser = false);

    // Additive: statistics of the last render.
    const RenderStats& lastStats() const;

private:
    RendererImpl* m_impl;
    RendererConfig m_config;
};

}  // namespace wr
