// Drop-in check of the C++ API: builds a Cornell box the way libWR's test mains do
// (trianglestrip/OfflineRenderer libWR/test/cornell_box_var_test.cpp:138-174:
// Context -> createScene -> add materials / meshes -> finalize -> createRenderer ->
// render), then writes the float image to the path in argv[1] as raw RGB floats.
#include <wr/wr.h>

#include <cstdio>
#include <stdexcept>
#include <vector>

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    wr::Context context;
    wr::Scene* scene = context.createScene();
    uint32_t white = scene->addLambertianMaterial(wr::Vec3(0.73f, 0.73f, 0.73f));
    uint32_t red = scene->addLambertianMaterial(wr::Vec3(0.63f, 0.065f, 0.05f));
    uint32_t light = scene->addEmissiveMaterial(wr::Vec3(17.0f, 12.0f, 4.0f));
    uint32_t glass = scene->addGlassMaterial(wr::Vec3(0.999f, 0.999f, 0.999f), 1.5f);
    uint32_t metal = scene->addGGXReflectionMaterial(wr::Vec3(0.95f, 0.64f, 0.54f), 0.3f, 1.0f);
    {
        float v[] = {0, 0, 0, 1, 0, 0, 1, 0, 1, 0, 0, 1};
        uint32_t i[] = {0, 1, 2, 0, 2, 3};
        float uv[] = {0, 0, 1, 0, 1, 1, 0, 1};
        scene->addTriangleMesh(std::span(v, 12), std::span(i, 6), std::span(uv, 8), white);
    }
    {
        float v[] = {1, 0, 0, 1, 1, 0, 1, 1, 1, 1, 0, 1};
        uint32_t i[] = {0, 1, 2, 0, 2, 3};
        scene->addTriangleMesh(std::span(v, 12), std::span(i, 6), red);
    }
    {
        float v[] = {0.35f, 0.999f, 0.35f, 0.65f, 0.999f, 0.35f, 0.65f, 0.999f, 0.65f, 0.35f, 0.999f, 0.65f};
        uint32_t i[] = {0, 1, 2, 0, 2, 3};
        scene->addTriangleMesh(std::span(v, 12), std::span(i, 6), light);
    }
    {
        float v[] = {0.2f, 0.1f, 0.4f, 0.5f, 0.1f, 0.4f, 0.35f, 0.5f, 0.5f};
        uint32_t i[] = {0, 1, 2};
        float n[] = {0, 0, -1, 0, 0, -1, 0, 0, -1};
        scene->addTriangleMesh(std::span(v, 9), std::span(i, 3), std::span(n, 9), std::span<const float>(), glass);
    }
    {
        float v[] = {0.6f, 0.1f, 0.6f, 0.9f, 0.1f, 0.6f, 0.75f, 0.6f, 0.7f};
        uint32_t i[] = {0, 1, 2};
        scene->addTriangleMesh(std::span(v, 9), std::span(i, 3), metal);
    }
    scene->setEnvironmentRadiance(wr::Vec3(0.1f, 0.1f, 0.1f));
    scene->finalize();
    wr::Renderer* renderer = context.createRenderer();
    wr::Camera camera;
    camera.position = wr::Vec3(0.5f, 0.5f, -1.4f);
    camera.target = wr::Vec3(0.5f, 0.5f, 0.0f);
    camera.up = wr::Vec3(0.0f, 1.0f, 0.0f);
    camera.fovY = wr::radians(40.0f);
    camera.aspect = 1.0f;
    const uint32_t W = 48, H = 48;
    std::vector<wr::Vec3> image(W * H), albedo(W * H), normal(W * H);
    wr::RenderParams p;
    p.width = W;
    p.height = H;
    p.spp = 8;
    p.maxBounces = 8;
    p.russianRouletteDepth = 3.0f;
    p.albedoOut = albedo.data();
    p.normalOut = normal.data();
    renderer->render(scene, camera, image.data(), p);
    bool threw = false;
    try {
        renderer->render(scene, camera, image.data(), W, H, 0, false);  // spp 0 is rejected
    } catch (const std::runtime_error&) {
        threw = true;
    }
    // libWR's legacy call with the denoiser on (renderer.cpp:318-335)
    std::vector<wr::Vec3> denoised(W * H);
    renderer->render(scene, camera, denoised.data(), W, H, 8, true);
    FILE* f = std::fopen(argv[1], "wb");
    std::fwrite(image.data(), sizeof(wr::Vec3), image.size(), f);
    std::fwrite(albedo.data(), sizeof(wr::Vec3), albedo.size(), f);
    std::fwrite(normal.data(), sizeof(wr::Vec3), normal.size(), f);
    std::fwrite(denoised.data(), sizeof(wr::Vec3), denoised.size(), f);
    std::fclose(f);
    std::printf("paths=%llu rays=%llu threw=%d\n", (unsigned long long)renderer->lastStats().paths,
                (unsigned long long)renderer->lastStats().extensionRays, threw ? 1 : 0);
    delete renderer;
    delete scene;
    return threw ? 0 : 3;
}
