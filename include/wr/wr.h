// Umbrella header of the drop-in C++ API (libWR/include/wr/wr.h): the same four
// headers.  The test-layer image writers are in wr/image.h, included separately.
#pragma once

#include "wr/types.h"
#include "wr/context.h"
#include "wr/scene.h"
#include "wr/renderer.h"

namespace wr {

constexpr int VERSION_MAJOR = 1;
constexpr int VERSION_MINOR = 0;
constexpr int VERSION_PATCH = 0;

}  // namespace wr
