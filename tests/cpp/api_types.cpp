// Compile-and-link check of the drop-in C++ API's types (no GPU needed; the
// program is built, not run).  With GLM on the include path wr::Vec3 must be
// glm::vec3 and the GLM calls libWR's test programs make on it must compile
// (libWR/test/cornell_box_var_test.cpp:153 uses glm::radians); without GLM the
// fallback Vec3 must serve the same libWR calls.
#include <wr/image.h>
#include <wr/wr.h>

#include <type_traits>
#include <vector>

#ifdef WR_EXPECT_GLM
static_assert(std::is_same_v<wr::Vec3, glm::vec3>, "wr::Vec3 must be glm::vec3 when GLM is present");
#endif

int main() {
    wr::Context context;
    wr::Scene* scene = context.createScene();
    uint32_t white = scene->addLambertianMaterial(wr::Vec3(0.73f, 0.73f, 0.73f));
    uint32_t glass = scene->addGlassMaterial(wr::Vec3(0.999f), 1.5f);
    (void)glass;
    float v[] = {0, 0, 0, 1, 0, 0, 0, 1, 0};
    uint32_t i[] = {0, 1, 2};
    scene->addTriangleMesh(std::span(v, 9), std::span(i, 3), white);
    scene->setEnvironmentRadiance(wr::Vec3(0.1f, 0.2f, 0.3f));
    wr::Vec3 env = scene->getEnvironmentRadiance();
    scene->finalize();
    wr::Camera camera;
    camera.position = wr::Vec3(0.0f, 1.5f, 4.5f);
    camera.target = wr::Vec3(0.0f, 1.0f, 0.0f);
#ifdef WR_EXPECT_GLM
    camera.fovY = glm::radians(45.0f);
    wr::Vec3 d = glm::normalize(camera.target - camera.position) * 2.0f + glm::cross(camera.up, env);
    wr::Mat4 view = camera.getViewMatrix() * camera.getProjectionMatrix();
    (void)view;
#else
    camera.fovY = wr::radians(45.0f);
    wr::Vec3 d = wr::normalize(camera.target - camera.position) * 2.0f + wr::cross(camera.up, env);
#endif
    (void)d;
    wr::Renderer* renderer = context.createRenderer();
    std::vector<wr::Vec3> image(16 * 16);
    renderer->render(scene, camera, image.data(), 16, 16, 1, false);
    test_helpers::savePNG("unused.png", image.data(), 16, 16);
    delete renderer;
    delete scene;
    return 0;
}
