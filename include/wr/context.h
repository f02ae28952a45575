// wr::Context (libWR/include/wr/context.h:12-29).
#pragma once
#include <cstdint>

namespace wr {

class Scene;
class Renderer;

struct ContextConfig {
    int deviceId = 0;
    int logLevel = 4;  // kept for source compatibility (libWR passes it to OptiX)
    bool enableValidation = false;
};

// Selects the CUDA device; scenes and renderers it creates live on that device.
class Context {
public:
    Context(const ContextConfig& config = {});
    ~Context();

    Scene* createScene();
    Renderer* createRenderer();

    int getDeviceId() const;

private:
    int m_device = 0;
};

}  // namespace wr
