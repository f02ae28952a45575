// libWR-style test-layer output through the C++ API: writes a small HDR gradient
// with test_helpers::saveEXR and test_helpers::saveHDR (host-only, no GPU needed).
#include <cstdio>
#include <vector>

#include "wr/image.h"
#include "wr/wr.h"

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    const uint32_t w = 24, h = 10;
    std::vector<wr::Vec3> img(w * h);
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) img[y * w + x] = wr::Vec3{0.25f * x, 0.5f * y + 0.125f, 100.0f / (1 + x + y)};
    try {
        test_helpers::saveEXR(argv[1], img.data(), w, h);
        test_helpers::saveHDR(argv[2], img.data(), w, h);
        test_helpers::saveEXR(nullptr, img.data(), w, h);  // must throw
    } catch (const std::exception& e) {
        std::printf("threw: %s\n", e.what());
        return 0;
    }
    return 1;
}
