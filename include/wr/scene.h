// wr::Scene and wr::Texture2D (libWR/include/wr/scene.h:11-103): same methods and
// argument meaning; the acceleration structure is the library's own 8-wide BVH
// built on the GPU at finalize().
#pragma once
#include <cstdint>
#include <span>
#include <string>

#include "wr/types.h"
#include "wrk.h"

namespace wr {

struct SceneBuildConfig {
    bool allowUpdate = false;
    bool allowCompaction = true;
    bool preferFastTrace = true;
};

struct SceneImpl;
class Scene;

using DevicePtr = unsigned long long;
using TraversableHandle = unsigned long long;
using TextureHandle = unsigned long long;

// RGBA8 textures loaded from PNG files; ids are 1-based (0 = none).
class Texture2D {
public:
    static uint32_t create(Scene* scene, const std::string& path);
    static void destroy(Scene* scene, uint32_t textureId);
};

class Scene {
public:
    Scene();
    explicit Scene(int deviceId);
    ~Scene();

    // Material creation (returns the material id), with libWR's defaults for the
    // fields a material type does not take (scene.cpp:91-168).
    uint32_t addLambertianMaterial(const Vec3& albedo) { return addLambertianMaterial(albedo, 0u); }
    uint32_t addLambertianMaterial(const Vec3& albedo, uint32_t albedoTextureId) {
        return addMaterialRecord(material(WRK_LAMBERTIAN, albedo.x, albedo.y, albedo.z, 0.0f, 0.0f, 0.0f, 1.0f, 1.0f,
                                          0.0f, albedoTextureId));
    }
    uint32_t addEmissiveMaterial(const Vec3& emission) {
        return addMaterialRecord(
            material(WRK_EMISSIVE, 0.0f, 0.0f, 0.0f, emission.x, emission.y, emission.z, 1.0f, 0.0f, 0.0f, 0u));
    }
    uint32_t addGlassMaterial(const Vec3& albedo, float ior) {
        return addMaterialRecord(material(WRK_GLASS, albedo.x, albedo.y, albedo.z, 0.0f, 0.0f, 0.0f, ior, 0.0f, 0.0f, 0u));
    }
    uint32_t addGGXReflectionMaterial(const Vec3& albedo, float roughness, float metallic = 0.0f) {
        return addMaterialRecord(material(WRK_GGX_REFLECTION, albedo.x, albedo.y, albedo.z, 0.0f, 0.0f, 0.0f, 1.5f,
                                          roughness, metallic, 0u));
    }
    uint32_t addGGXTransmissionMaterial(const Vec3& albedo, float roughness, float ior) {
        return addMaterialRecord(material(WRK_GGX_TRANSMISSION, albedo.x, albedo.y, albedo.z, 0.0f, 0.0f, 0.0f, ior,
                                          roughness, 0.0f, 0u));
    }

    void setMaterialNormalMap(uint32_t materialId, uint32_t normalTextureId);

    // Geometry: xyz triples, index triples, optional normals (xyz) and uvs (uv).
    void addTriangleMesh(std::span<const float> vertices, std::span<const uint32_t> indices, uint32_t materialId);
    void addTriangleMesh(std::span<const float> vertices, std::span<const uint32_t> indices,
                         std::span<const float> uvs, uint32_t materialId);
    void addTriangleMesh(std::span<const float> vertices, std::span<const uint32_t> indices,
                         std::span<const float> normals, std::span<const float> uvs, uint32_t materialId);

    void setEnvironmentRadiance(const Vec3& radiance) { setEnvironmentRadianceRGB(radiance.x, radiance.y, radiance.z); }
    // Loads a Radiance .hdr map; stored with the scene.  libWR's miss program
    // shades with the uniform radiance only (trace.cu:143-148), and so does this.
    void setEnvironmentMap(const std::string& hdrPath);

    void finalize(const SceneBuildConfig& config = {});

    // Device buffers (valid after finalize)
    DevicePtr getVerticesBuffer() const;
    DevicePtr getNormalsBuffer() const;
    DevicePtr getIndicesBuffer() const;
    DevicePtr getTriangleMaterialIdsBuffer() const;
    DevicePtr getMaterialsBuffer() const;
    TraversableHandle getGASHandle() const;  // the BVH node array
    uint32_t getNumMaterials() const;
    Vec3 getEnvironmentRadiance() const {
        float c[3];
        environmentRadianceRGB(c);
        return Vec3(c[0], c[1], c[2]);
    }
    uint64_t getEnvironmentMapTexture() const;
    uint32_t getEnvironmentMapWidth() const;
    uint32_t getEnvironmentMapHeight() const;
    DevicePtr getEmissiveTrianglesBuffer() const;
    DevicePtr getEmissiveTriangleCDFBuffer() const;
    uint32_t getNumEmissiveTriangles() const;
    DevicePtr getTexturesBuffer() const;
    uint32_t getNumTextures() const;
    DevicePtr getUVsBuffer() const;

    uint32_t loadTexture(const std::string& path);
    void destroyTexture(uint32_t textureId);

    // Additive: texture from memory (RGBA8, width*height*4 bytes); returns its id.
    uint32_t addTexture(const uint8_t* rgba, uint32_t width, uint32_t height);
    // Additive: the C-ABI handle (valid after finalize).
    wrk_scene* native() const;

    // Additive: the Vec3-free forms the inline members above call.  libwrk.so
    // exports only these, so its symbols do not depend on the caller's Vec3.
    uint32_t addMaterialRecord(const wrk_material& m);
    void setEnvironmentRadianceRGB(float r, float g, float b);
    void environmentRadianceRGB(float rgb[3]) const;
    static wrk_material material(uint32_t type, float ar, float ag, float ab, float er, float eg, float eb, float ior,
                                 float roughness, float metallic, uint32_t albedoTextureId) {
        wrk_material m{};
        m.albedo[0] = ar;
        m.albedo[1] = ag;
        m.albedo[2] = ab;
        m.emission[0] = er;
        m.emission[1] = eg;
        m.emission[2] = eb;
        m.ior = ior;
        m.type = type;
        m.roughness = roughness;
        m.metallic = metallic;
        m.albedoTextureId = albedoTextureId;
        return m;
    }

private:
    SceneImpl* m_impl;
};

}  // namespace wr
