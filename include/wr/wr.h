// Umbrella header of the drop-in C++ API (libWR/include/wr/wr.h).
#pragma once

#include "wr/context.h"
#include "wr/image.h"
#include "wr/renderer.h"
#include "wr/scene.h"
#include "wr/types.h"

namespace wr {

constexpr int VERSION_MAJOR = 1;
constexpr int VERSION_MINOR = 0;
constexpr int VERSION_PATCH = 0;

}  // namespace wr
