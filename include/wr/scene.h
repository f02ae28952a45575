// wr::Scene and wr::Texture2D (libWR/include/wr/scene.h:11-103): same methods and
// argument meaning; the acceleration structure is the library's own 8-wide BVH
// built on the GPU at finalize().
#pragma once
#include <cstdint>
#include <span>
#include <string>

#include "wr/types.h"

struct wrk_scene;

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

    // Material creation (returns the material id)
    uint32_t addLambertianMaterial(const Vec3& albedo);
    uint32_t addLambertianMaterial(const Vec3& albedo, uint32_t albedoTextureId);
    uint32_t addEmissiveMaterial(const Vec3& emission);
    uint32_t addGlassMaterial(const Vec3& albedo, float ior);
    uint32_t addGGXReflectionMaterial(const Vec3& albedo, float roughness, float metallic = 0.0f);
    uint32_t addGGXTransmissionMaterial(const Vec3& albedo, float roughness, float ior);

    void setMaterialNormalMap(uint32_t materialId, uint32_t normalTextureId);

    // Geometry: xyz triples, index triples, optional normals (xyz) and uvs (uv).
    void addTriangleMesh(std::span<const float> vertices, std::span<const uint32_t> indices, uint32_t materialId);
    void addTriangleMesh(std::span<const float> vertices, std::span<const uint32_t> indices,
                         std::span<const float> uvs, uint32_t materialId);
    void addTriangleMesh(std::span<const float> vertices, std::span<const uint32_t> indices,
                         std::span<const float> normals, std::span<const float> uvs, uint32_t materialId);

    void setEnvironmentRadiance(const Vec3& radiance);
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
    Vec3 getEnvironmentRadiance() const;
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

private:
    SceneImpl* m_impl;
};

}  // namespace wr
