// Drop-in C++ API (include/wr/*.h) on top of the C ABI (include/wrk.h).
//
// Mirrors libWR's public classes (trianglestrip/OfflineRenderer,
// libWR/src/internal/{context,scene,renderer}.cpp): materials are appended with
// libWR's defaults, meshes are accumulated as one flat triangle soup (indices
// rebased, absent normals / uvs zero-padded), and finalize() hands everything to
// libwrk, which builds the light CDF and the BVH on the GPU.  Failures of the C
// ABI are rethrown as std::runtime_error, libWR's error convention
// (libWR/src/internal/cuda_utils.h:13-39).
//
// Only the members without a Vec3 / Camera / RenderParams in their signature are
// defined here; the others are inline in include/wr/*.h and call these, so the
// library serves callers whose wr::Vec3 is glm::vec3 as well as the GLM-free one.
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <fstream>
#include <iterator>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/wr/wr.h"
#include "../../include/wrk.h"

namespace wr {
namespace {

void check(int rc, const char* what) {
    if (rc != WRK_OK) throw std::runtime_error(std::string("wrk error in ") + what + ": " + wrk_last_error());
}

std::vector<uint8_t> read_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("Failed to open: " + path);
    return std::vector<uint8_t>(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
}

uint32_t be32(const uint8_t* p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }

// PNG -> RGBA8: 8-bit grey / grey+alpha / RGB / RGBA / palette, non-interlaced.
void decode_png(const std::vector<uint8_t>& d, std::vector<uint8_t>& rgba, uint32_t& w, uint32_t& h) {
    static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', 0x0d, 0x0a, 0x1a, 0x0a};
    if (d.size() < 8 || std::memcmp(d.data(), sig, 8) != 0) throw std::runtime_error("not a PNG file");
    size_t pos = 8;
    uint8_t depth = 0, ctype = 0, interlace = 0;
    std::vector<uint8_t> idat, plte, trns;
    while (pos + 8 <= d.size()) {
        uint32_t len = be32(&d[pos]);
        std::string type(reinterpret_cast<const char*>(&d[pos + 4]), 4);
        if (pos + 12 + (size_t)len > d.size()) throw std::runtime_error("truncated PNG");
        const uint8_t* body = &d[pos + 8];
        if (type == "IHDR") {
            w = be32(body);
            h = be32(body + 4);
            depth = body[8];
            ctype = body[9];
            interlace = body[12];
        } else if (type == "PLTE") {
            plte.assign(body, body + len);
        } else if (type == "tRNS") {
            trns.assign(body, body + len);
        } else if (type == "IDAT") {
            idat.insert(idat.end(), body, body + len);
        } else if (type == "IEND") {
            break;
        }
        pos += 12 + len;
    }
    if (depth != 8 || interlace != 0) throw std::runtime_error("PNG: only 8-bit non-interlaced images are supported");
    int ch = ctype == 0 ? 1 : ctype == 2 ? 3 : ctype == 3 ? 1 : ctype == 4 ? 2 : ctype == 6 ? 4 : 0;
    if (!ch || w == 0 || h == 0) throw std::runtime_error("PNG: unsupported color type");
    size_t stride = (size_t)w * ch;
    std::vector<uint8_t> raw((stride + 1) * h);
    uLongf rawLen = (uLongf)raw.size();
    if (uncompress(raw.data(), &rawLen, idat.data(), (uLong)idat.size()) != Z_OK || rawLen != raw.size())
        throw std::runtime_error("PNG: zlib stream error");
    std::vector<uint8_t> img(stride * h), prev(stride, 0);
    for (uint32_t y = 0; y < h; ++y) {
        uint8_t f = raw[y * (stride + 1)];
        const uint8_t* in = &raw[y * (stride + 1) + 1];
        uint8_t* out = &img[y * stride];
        for (size_t x = 0; x < stride; ++x) {
            int a = x >= (size_t)ch ? out[x - ch] : 0, b = prev[x], c = x >= (size_t)ch ? prev[x - ch] : 0;
            int v = in[x];
            if (f == 1) v += a;
            else if (f == 2) v += b;
            else if (f == 3) v += (a + b) >> 1;
            else if (f == 4) {
                int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
                v += (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
            }
            out[x] = (uint8_t)v;
        }
        std::memcpy(prev.data(), out, stride);
    }
    rgba.resize((size_t)w * h * 4);
    for (size_t i = 0; i < (size_t)w * h; ++i) {
        uint8_t* o = &rgba[4 * i];
        const uint8_t* s = &img[i * ch];
        switch (ctype) {
            case 0: o[0] = o[1] = o[2] = s[0]; o[3] = 255; break;
            case 2: o[0] = s[0]; o[1] = s[1]; o[2] = s[2]; o[3] = 255; break;
            case 3: {
                size_t k = s[0];
                if (3 * k + 2 >= plte.size()) throw std::runtime_error("PNG: palette index out of range");
                o[0] = plte[3 * k]; o[1] = plte[3 * k + 1]; o[2] = plte[3 * k + 2];
                o[3] = k < trns.size() ? trns[k] : 255;
                break;
            }
            case 4: o[0] = o[1] = o[2] = s[0]; o[3] = s[1]; break;
            default: o[0] = s[0]; o[1] = s[1]; o[2] = s[2]; o[3] = s[3]; break;
        }
    }
}

// Radiance .hdr (RGBE, flat or new-style run-length scanlines) -> RGBA float.
void decode_hdr(const std::vector<uint8_t>& d, std::vector<float>& rgba, uint32_t& w, uint32_t& h) {
    size_t pos = 0;
    auto line = [&]() {
        std::string s;
        while (pos < d.size() && d[pos] != '\n') s += (char)d[pos++];
        ++pos;
        return s;
    };
    std::string l = line();
    if (l.rfind("#?", 0) != 0) throw std::runtime_error("not a Radiance HDR file");
    while (pos < d.size() && !(l = line()).empty()) {
    }
    l = line();
    int H = 0, W = 0;
    if (std::sscanf(l.c_str(), "-Y %d +X %d", &H, &W) != 2 || W <= 0 || H <= 0)
        throw std::runtime_error("HDR: unsupported orientation");
    w = (uint32_t)W;
    h = (uint32_t)H;
    std::vector<uint8_t> rgbe((size_t)W * H * 4);
    for (int y = 0; y < H; ++y) {
        uint8_t* row = &rgbe[(size_t)y * W * 4];
        if (pos + 4 <= d.size() && d[pos] == 2 && d[pos + 1] == 2 && W >= 8 && W < 32768) {
            pos += 4;
            for (int c = 0; c < 4; ++c)
                for (int x = 0; x < W;) {
                    if (pos >= d.size()) throw std::runtime_error("HDR: truncated");
                    int n = d[pos++];
                    if (n > 128) {
                        n -= 128;
                        uint8_t v = d[pos++];
                        for (int k = 0; k < n && x < W; ++k) row[4 * x++ + c] = v;
                    } else {
                        for (int k = 0; k < n && x < W; ++k) row[4 * x++ + c] = d[pos++];
                    }
                }
        } else {
            if (pos + (size_t)W * 4 > d.size()) throw std::runtime_error("HDR: truncated");
            std::memcpy(row, &d[pos], (size_t)W * 4);
            pos += (size_t)W * 4;
        }
    }
    rgba.resize((size_t)W * H * 4);
    for (size_t i = 0; i < (size_t)W * H; ++i) {
        const uint8_t* e = &rgbe[4 * i];
        float f = e[3] ? std::ldexp(1.0f, (int)e[3] - 136) : 0.0f;
        rgba[4 * i] = e[0] * f;
        rgba[4 * i + 1] = e[1] * f;
        rgba[4 * i + 2] = e[2] * f;
        rgba[4 * i + 3] = 1.0f;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
Context::Context(const ContextConfig& config) : m_device(config.deviceId) {
    int n = 0;
    check(wrk_device_count(&n), "Context");
    if (n == 0) throw std::runtime_error("wrk: no CUDA device available");
    if (m_device < 0 || m_device >= n) throw std::runtime_error("wrk: device id out of range");
}
Context::~Context() {}
Scene* Context::createScene() { return new Scene(m_device); }
Renderer* Context::createRenderer() { return new Renderer(RendererConfig{}, m_device); }
int Context::getDeviceId() const { return m_device; }

// ---------------------------------------------------------------------------
struct SceneImpl {
    int device = 0;
    std::vector<float> vertices, normals, uvs;
    std::vector<uint32_t> indices, triMat;
    std::vector<wrk_material> materials;
    std::vector<std::vector<uint8_t>> textures;
    std::vector<uint32_t> texW, texH;
    std::vector<float> envMap;
    uint32_t envW = 0, envH = 0;
    float env[3] = {0.0f, 0.0f, 0.0f};
    bool hasNormals = false, hasUVs = false, finalized = false;
    wrk_scene* handle = nullptr;
    wrk_scene_buffers bufs{};
    ~SceneImpl() {
        if (handle) wrk_scene_destroy(handle);
    }
    uint32_t add(const wrk_material& m) {
        materials.push_back(m);
        return (uint32_t)materials.size() - 1;
    }
};

Scene::Scene() : m_impl(new SceneImpl()) {}
Scene::Scene(int deviceId) : m_impl(new SceneImpl()) { m_impl->device = deviceId; }
Scene::~Scene() { delete m_impl; }

uint32_t Scene::addMaterialRecord(const wrk_material& m) {
    if (m_impl->finalized) throw std::runtime_error("Scene already finalized");
    return m_impl->add(m);
}
void Scene::setMaterialNormalMap(uint32_t materialId, uint32_t normalTextureId) {
    if (materialId >= m_impl->materials.size()) throw std::runtime_error("Invalid material ID");
    m_impl->materials[materialId].normalTextureId = normalTextureId;
}

void Scene::addTriangleMesh(std::span<const float> v, std::span<const uint32_t> i, uint32_t mat) {
    addTriangleMesh(v, i, std::span<const float>(), std::span<const float>(), mat);
}
void Scene::addTriangleMesh(std::span<const float> v, std::span<const uint32_t> i, std::span<const float> uv,
                            uint32_t mat) {
    addTriangleMesh(v, i, std::span<const float>(), uv, mat);
}
// scene.cpp:190-244: indices rebased by the vertex offset, normals / uvs padded with
// zeros for meshes that do not supply them, one material id per triangle.
void Scene::addTriangleMesh(std::span<const float> v, std::span<const uint32_t> idx, std::span<const float> nrm,
                            std::span<const float> uv, uint32_t mat) {
    SceneImpl& s = *m_impl;
    if (s.finalized) throw std::runtime_error("Scene already finalized");
    uint32_t off = (uint32_t)(s.vertices.size() / 3);
    size_t nv = v.size() / 3;
    s.vertices.insert(s.vertices.end(), v.begin(), v.begin() + 3 * nv);
    if (!nrm.empty() && nrm.size() >= nv * 3) {
        s.hasNormals = true;
        s.normals.insert(s.normals.end(), nrm.begin(), nrm.begin() + 3 * nv);
    } else {
        s.normals.insert(s.normals.end(), 3 * nv, 0.0f);
    }
    if (!uv.empty() && uv.size() >= nv * 2) {
        s.hasUVs = true;
        s.uvs.insert(s.uvs.end(), uv.begin(), uv.begin() + 2 * nv);
    } else {
        s.uvs.insert(s.uvs.end(), 2 * nv, 0.0f);
    }
    size_t nt = idx.size() / 3;
    for (size_t k = 0; k < 3 * nt; ++k) s.indices.push_back(off + idx[k]);
    s.triMat.insert(s.triMat.end(), nt, mat);
}

void Scene::setEnvironmentRadianceRGB(float r, float g, float b) {
    m_impl->env[0] = r;
    m_impl->env[1] = g;
    m_impl->env[2] = b;
}
void Scene::environmentRadianceRGB(float rgb[3]) const {
    for (int k = 0; k < 3; ++k) rgb[k] = m_impl->env[k];
}
void Scene::setEnvironmentMap(const std::string& path) {
    decode_hdr(read_file(path), m_impl->envMap, m_impl->envW, m_impl->envH);
}

uint32_t Scene::loadTexture(const std::string& path) {
    std::vector<uint8_t> rgba;
    uint32_t w = 0, h = 0;
    try {
        decode_png(read_file(path), rgba, w, h);
    } catch (const std::exception& e) {
        throw std::runtime_error("Failed to load texture: " + path + " (" + e.what() + ")");
    }
    return addTexture(rgba.data(), w, h);
}
uint32_t Scene::addTexture(const uint8_t* rgba, uint32_t w, uint32_t h) {
    if (m_impl->finalized) throw std::runtime_error("Scene already finalized");
    m_impl->textures.emplace_back(rgba, rgba + (size_t)w * h * 4);
    m_impl->texW.push_back(w);
    m_impl->texH.push_back(h);
    return (uint32_t)m_impl->textures.size();
}
// scene.cpp:266-275: the texture keeps its id; a destroyed texture samples as white.
void Scene::destroyTexture(uint32_t id) {
    if (id == 0 || id > m_impl->textures.size()) return;
    m_impl->textures[id - 1].clear();
}
uint32_t Texture2D::create(Scene* scene, const std::string& path) { return scene->loadTexture(path); }
void Texture2D::destroy(Scene* scene, uint32_t id) { scene->destroyTexture(id); }

void Scene::finalize(const SceneBuildConfig&) {
    SceneImpl& s = *m_impl;
    if (s.finalized) return;
    if (s.vertices.empty() || s.indices.empty()) throw std::runtime_error("Scene has no geometry");
    check(wrk_scene_create(s.device, &s.handle), "wrk_scene_create");
    check(wrk_scene_set_geometry(s.handle, s.vertices.data(), (uint32_t)(s.vertices.size() / 3),
                                 s.hasNormals ? s.normals.data() : nullptr, s.hasUVs ? s.uvs.data() : nullptr,
                                 s.indices.data(), (uint32_t)s.triMat.size(), s.triMat.data()),
          "wrk_scene_set_geometry");
    check(wrk_scene_set_materials(s.handle, s.materials.data(), (uint32_t)s.materials.size()),
          "wrk_scene_set_materials");
    for (size_t i = 0; i < s.textures.size(); ++i) {
        uint32_t id = 0;
        // a destroyed texture keeps its slot as a 1x1 white texel
        static const uint8_t white[4] = {255, 255, 255, 255};
        bool gone = s.textures[i].empty();
        check(wrk_scene_add_texture(s.handle, gone ? white : s.textures[i].data(), gone ? 1 : s.texW[i],
                                    gone ? 1 : s.texH[i], &id),
              "wrk_scene_add_texture");
    }
    check(wrk_scene_set_environment(s.handle, s.env), "wrk_scene_set_environment");
    if (!s.envMap.empty())
        check(wrk_scene_set_environment_map(s.handle, s.envMap.data(), s.envW, s.envH),
              "wrk_scene_set_environment_map");
    check(wrk_scene_finalize(s.handle), "wrk_scene_finalize");
    check(wrk_scene_buffers_get(s.handle, &s.bufs), "wrk_scene_buffers_get");
    s.finalized = true;
}

DevicePtr Scene::getVerticesBuffer() const { return m_impl->bufs.vertices; }
DevicePtr Scene::getNormalsBuffer() const { return m_impl->bufs.normals; }
DevicePtr Scene::getIndicesBuffer() const { return m_impl->bufs.indices; }
DevicePtr Scene::getTriangleMaterialIdsBuffer() const { return m_impl->bufs.triMaterial; }
DevicePtr Scene::getMaterialsBuffer() const { return m_impl->bufs.materials; }
TraversableHandle Scene::getGASHandle() const { return m_impl->bufs.bvhNodes; }
uint32_t Scene::getNumMaterials() const { return (uint32_t)m_impl->materials.size(); }
uint64_t Scene::getEnvironmentMapTexture() const { return 0; }
uint32_t Scene::getEnvironmentMapWidth() const { return m_impl->envW; }
uint32_t Scene::getEnvironmentMapHeight() const { return m_impl->envH; }
DevicePtr Scene::getEmissiveTrianglesBuffer() const { return m_impl->bufs.emissive; }
DevicePtr Scene::getEmissiveTriangleCDFBuffer() const { return m_impl->bufs.cdf; }
uint32_t Scene::getNumEmissiveTriangles() const { return m_impl->bufs.numEmissive; }
DevicePtr Scene::getTexturesBuffer() const { return m_impl->bufs.texels; }
uint32_t Scene::getNumTextures() const { return (uint32_t)m_impl->textures.size(); }
DevicePtr Scene::getUVsBuffer() const { return m_impl->bufs.uvs; }
wrk_scene* Scene::native() const { return m_impl->handle; }

// ---------------------------------------------------------------------------
struct RendererImpl {
    int device = 0;
    wrk_renderer* handle = nullptr;
    RenderStats stats;
    // the learned denoiser (created on the first denoised render) and its device buffers
    wrk_denoiser* denoiser = nullptr;
    std::string weights;
    void* dbuf = nullptr;
    size_t dbufBytes = 0;
    ~RendererImpl() {
        if (dbuf) wrk_free(dbuf);
        if (denoiser) wrk_denoiser_destroy(denoiser);
        if (handle) wrk_renderer_destroy(handle);
    }
};

// Default weights: $WRK_DENOISER_WEIGHTS, else weights/unet_scale.wrkw beside this library.
static std::string default_weights() {
    if (const char* e = std::getenv("WRK_DENOISER_WEIGHTS")) return e;
    Dl_info info{};
    if (dladdr(reinterpret_cast<void*>(&wrk_version), &info) && info.dli_fname) {
        std::string lib = info.dli_fname;
        size_t slash = lib.find_last_of('/');
        return (slash == std::string::npos ? std::string(".") : lib.substr(0, slash)) + "/weights/unet_scale.wrkw";
    }
    return "weights/unet_scale.wrkw";
}

Renderer::Renderer(const RendererConfig& config) : Renderer(config, 0) {}
Renderer::Renderer(const RendererConfig& config, int deviceId) : m_impl(new RendererImpl()), m_config(config) {
    m_impl->device = deviceId;
    try {
        check(wrk_renderer_create(deviceId, 0, &m_impl->handle), "wrk_renderer_create");
    } catch (...) {
        delete m_impl;
        throw;
    }
}
Renderer::~Renderer() { delete m_impl; }
const RenderStats& Renderer::lastStats() const { return m_impl->stats; }

void Renderer::renderNative(Scene* scene, const wrk_camera& c, const wrk_render_params& rp, float* out,
                            float* albedoOut, float* normalOut, bool denoise, const char* weightsPath) {
    if (!scene || !out) throw std::runtime_error("render: null scene or output buffer");
    scene->finalize();
    wrk_render_stats st{};
    if (!denoise) {
        check(wrk_render(m_impl->handle, scene->native(), &c, &rp, out, albedoOut, normalOut, &st), "wrk_render");
    } else {
        // libWR denoises inside render (renderer.cpp:289-313, denoiser.cpp:17-195): render
        // rgb + averaged guides into device memory, denoise, copy the result out.
        const std::string path = weightsPath ? weightsPath : default_weights();
        if (!m_impl->denoiser) check(wrk_denoiser_create(m_impl->device, 1, &m_impl->denoiser), "wrk_denoiser_create");
        if (m_impl->weights != path) {
            check(wrk_denoiser_load(m_impl->denoiser, path.c_str()), "wrk_denoiser_load");
            m_impl->weights = path;
        }
        const size_t np = (size_t)rp.width * rp.height, bytes = np * 12 * sizeof(float);
        if (m_impl->dbufBytes < bytes) {
            if (m_impl->dbuf) wrk_free(m_impl->dbuf);
            m_impl->dbuf = nullptr;
            m_impl->dbufBytes = 0;
            check(wrk_malloc(m_impl->device, bytes, &m_impl->dbuf), "wrk_malloc");
            m_impl->dbufBytes = bytes;
        }
        float* d = static_cast<float*>(m_impl->dbuf);
        wrk_render_params dp = rp;
        dp.flags &= ~WRK_FLAG_RAW_GUIDES;  // the network takes guides averaged over spp
        check(wrk_render_device(m_impl->handle, scene->native(), &c, &dp, d, d + 3 * np, d + 6 * np, &st),
              "wrk_render_device");
        check(wrk_denoiser_infer(m_impl->denoiser, d, d + 3 * np, d + 6 * np, 1, rp.height, rp.width, d + 9 * np),
              "wrk_denoiser_infer");
        check(wrk_memcpy_dtoh(out, d + 9 * np, np * 3 * sizeof(float)), "wrk_memcpy_dtoh");
        const float g = (rp.flags & WRK_FLAG_RAW_GUIDES) ? (float)rp.spp : 1.0f;
        float* guides[2] = {albedoOut, normalOut};
        for (int k = 0; k < 2; ++k) {
            if (!guides[k]) continue;
            check(wrk_memcpy_dtoh(guides[k], d + 3 * (k + 1) * np, np * 3 * sizeof(float)), "wrk_memcpy_dtoh");
            if (g != 1.0f)
                for (size_t i = 0; i < 3 * np; ++i) guides[k][i] = guides[k][i] * g;
        }
    }
    m_impl->stats.paths = st.paths;
    m_impl->stats.extensionRays = st.extensionRays;
    m_impl->stats.shadowRays = st.shadowRays;
    m_impl->stats.shadowTraced = st.shadowTraced;
    m_impl->stats.iterations = st.iterations;
    m_impl->stats.gpuMs = st.gpuMs;
    m_impl->stats.totalMs = st.totalMs;
}

}  // namespace wr

// ---------------------------------------------------------------------------
// PNG output (test_helpers::savePNG, libWR/test/helpers/image.cpp:23-49)
namespace wrk {
int report_error(int code, const char* msg);
}

namespace {

void put_be32(std::vector<uint8_t>& o, uint32_t v) {
    o.push_back((uint8_t)(v >> 24));
    o.push_back((uint8_t)(v >> 16));
    o.push_back((uint8_t)(v >> 8));
    o.push_back((uint8_t)v);
}

void put_chunk(std::vector<uint8_t>& o, const char* type, const uint8_t* data, size_t n) {
    put_be32(o, (uint32_t)n);
    const size_t start = o.size();
    o.insert(o.end(), type, type + 4);
    if (n) o.insert(o.end(), data, data + n);
    uLong crc = crc32(0L, Z_NULL, 0);
    crc = crc32(crc, o.data() + start, (uInt)(o.size() - start));
    put_be32(o, (uint32_t)crc);
}

}  // namespace

extern "C" int wrk_png_write(const char* path, const uint8_t* rgb8, uint32_t width, uint32_t height) {
    if (!path || !rgb8 || width == 0 || height == 0) return wrk::report_error(WRK_ERR_INVALID, "png: bad arguments");
    std::vector<uint8_t> raw((size_t)height * (1 + 3 * (size_t)width));
    for (uint32_t y = 0; y < height; ++y) {
        uint8_t* row = raw.data() + (size_t)y * (1 + 3 * (size_t)width);
        row[0] = 0;  // filter: none
        std::memcpy(row + 1, rgb8 + (size_t)y * 3 * width, 3 * (size_t)width);
    }
    uLongf zlen = compressBound((uLong)raw.size());
    std::vector<uint8_t> z(zlen);
    if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK)
        return wrk::report_error(WRK_ERR_INVALID, "png: deflate failed");
    std::vector<uint8_t> png = {0x89, 'P', 'N', 'G', 0x0d, 0x0a, 0x1a, 0x0a};
    uint8_t ihdr[13];
    for (int k = 0; k < 4; ++k) {
        ihdr[k] = (uint8_t)(width >> (24 - 8 * k));
        ihdr[4 + k] = (uint8_t)(height >> (24 - 8 * k));
    }
    ihdr[8] = 8;   // bit depth
    ihdr[9] = 2;   // colour type RGB
    ihdr[10] = 0;  // deflate
    ihdr[11] = 0;  // adaptive filtering
    ihdr[12] = 0;  // no interlace
    put_chunk(png, "IHDR", ihdr, 13);
    put_chunk(png, "IDAT", z.data(), zlen);
    put_chunk(png, "IEND", nullptr, 0);
    FILE* f = std::fopen(path, "wb");
    if (!f) return wrk::report_error(WRK_ERR_INVALID, (std::string("png: cannot open ") + path).c_str());
    const bool ok = std::fwrite(png.data(), 1, png.size(), f) == png.size();
    std::fclose(f);
    return ok ? WRK_OK : wrk::report_error(WRK_ERR_INVALID, "png: write failed");
}

extern "C" int wrk_image_save_png(const char* path, const float* rgb, uint32_t width, uint32_t height) {
    if (!path || !rgb || width == 0 || height == 0) return wrk::report_error(WRK_ERR_INVALID, "png: bad arguments");
    const size_t np = (size_t)width * height;
    void* d = nullptr;
    int dev = 0, n = 0;
    if (wrk_device_count(&n) || n == 0) return wrk::report_error(WRK_ERR_NO_DEVICE, "no CUDA device available");
    int rc = wrk_malloc(dev, np * 12 + np * 3 + 16, &d);
    if (rc) return rc;
    float* df = static_cast<float*>(d);
    uint8_t* db = reinterpret_cast<uint8_t*>(df + 3 * np);
    std::vector<uint8_t> bytes(np * 3);
    if (!(rc = wrk_memcpy_htod(df, rgb, np * 12)) && !(rc = wrk_tonemap_aces(df, (uint32_t)np, db)))
        rc = wrk_memcpy_dtoh(bytes.data(), db, np * 3);
    wrk_free(d);
    if (rc) return rc;
    return wrk_png_write(path, bytes.data(), width, height);
}

// ---------------------------------------------------------------------------
// HDR outputs of the linear radiance (no tone map): OpenEXR and Radiance RGBE.
namespace {

void put_le32(std::vector<uint8_t>& o, uint32_t v) {
    for (int k = 0; k < 4; ++k) o.push_back((uint8_t)(v >> (8 * k)));
}
void put_le64(std::vector<uint8_t>& o, uint64_t v) {
    for (int k = 0; k < 8; ++k) o.push_back((uint8_t)(v >> (8 * k)));
}
void put_f32(std::vector<uint8_t>& o, float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    put_le32(o, u);
}
void put_cstr(std::vector<uint8_t>& o, const char* s) { o.insert(o.end(), s, s + std::strlen(s) + 1); }
// One header attribute: name, type name, byte size, value.
void put_attr(std::vector<uint8_t>& o, const char* name, const char* type, const std::vector<uint8_t>& v) {
    put_cstr(o, name);
    put_cstr(o, type);
    put_le32(o, (uint32_t)v.size());
    o.insert(o.end(), v.begin(), v.end());
}

int write_file(const char* path, const std::vector<uint8_t>& bytes, const char* what) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return wrk::report_error(WRK_ERR_INVALID, (std::string(what) + ": cannot open " + path).c_str());
    const bool ok = std::fwrite(bytes.data(), 1, bytes.size(), f) == bytes.size();
    std::fclose(f);
    return ok ? WRK_OK : wrk::report_error(WRK_ERR_INVALID, (std::string(what) + ": write failed").c_str());
}

// Radiance RGBE of one pixel (Ward's shared-exponent encoding): the largest
// component's binary exponent e is shared, mantissas scaled by 256 / 2^e.
void rgbe(const float* c, uint8_t* out) {
    const float v = std::max(c[0], std::max(c[1], c[2]));
    if (!(v >= 1e-32f)) {  // also NaN
        out[0] = out[1] = out[2] = out[3] = 0;
        return;
    }
    int e;
    const float m = std::frexp(v, &e);  // v = m * 2^e, m in [0.5, 1)
    const float scale = m * 256.0f / v;
    for (int k = 0; k < 3; ++k) out[k] = (uint8_t)std::max(0.0f, c[k] * scale);
    out[3] = (uint8_t)(e + 128);
}

}  // namespace

extern "C" int wrk_exr_write(const char* path, const float* rgb, uint32_t width, uint32_t height) {
    if (!path || !rgb || width == 0 || height == 0 || width > (1u << 30) / 12 || height > (1u << 30))
        return wrk::report_error(WRK_ERR_INVALID, "exr: bad arguments");
    // OpenEXR 2 single-part scan-line file, no compression, one scan line per
    // block, channels B G R (alphabetical, as the format requires) as 32-bit float.
    std::vector<uint8_t> o = {0x76, 0x2f, 0x31, 0x01};
    put_le32(o, 2u);
    std::vector<uint8_t> ch;
    for (const char* name : {"B", "G", "R"}) {
        put_cstr(ch, name);
        put_le32(ch, 2u);                          // pixel type FLOAT
        ch.push_back(0);                           // pLinear
        ch.push_back(0), ch.push_back(0), ch.push_back(0);
        put_le32(ch, 1u);                          // x sampling
        put_le32(ch, 1u);                          // y sampling
    }
    ch.push_back(0);
    put_attr(o, "channels", "chlist", ch);
    put_attr(o, "compression", "compression", {0});
    std::vector<uint8_t> win;
    put_le32(win, 0), put_le32(win, 0), put_le32(win, width - 1), put_le32(win, height - 1);
    put_attr(o, "dataWindow", "box2i", win);
    put_attr(o, "displayWindow", "box2i", win);
    put_attr(o, "lineOrder", "lineOrder", {0});
    std::vector<uint8_t> one;
    put_f32(one, 1.0f);
    put_attr(o, "pixelAspectRatio", "float", one);
    std::vector<uint8_t> ctr;
    put_f32(ctr, 0.0f), put_f32(ctr, 0.0f);
    put_attr(o, "screenWindowCenter", "v2f", ctr);
    put_attr(o, "screenWindowWidth", "float", one);
    o.push_back(0);  // end of header
    const uint64_t rowBytes = 12ull * width, blockBytes = 8 + rowBytes;
    const uint64_t first = o.size() + 8ull * height;
    for (uint32_t y = 0; y < height; ++y) put_le64(o, first + y * blockBytes);
    o.reserve(first + height * blockBytes);
    for (uint32_t y = 0; y < height; ++y) {
        put_le32(o, y);
        put_le32(o, (uint32_t)rowBytes);
        const float* row = rgb + (size_t)y * 3 * width;
        for (int c = 2; c >= 0; --c)  // B, G, R planes of the scan line
            for (uint32_t x = 0; x < width; ++x) put_f32(o, row[3 * x + c]);
    }
    return write_file(path, o, "exr");
}

extern "C" int wrk_hdr_write(const char* path, const float* rgb, uint32_t width, uint32_t height) {
    if (!path || !rgb || width == 0 || height == 0) return wrk::report_error(WRK_ERR_INVALID, "hdr: bad arguments");
    std::string head = "#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y " + std::to_string(height) + " +X " +
                       std::to_string(width) + "\n";
    std::vector<uint8_t> o(head.begin(), head.end());
    std::vector<uint8_t> px(4 * (size_t)width);
    const bool rle = width >= 8 && width < 32768;
    for (uint32_t y = 0; y < height; ++y) {
        for (uint32_t x = 0; x < width; ++x) rgbe(rgb + 3 * ((size_t)y * width + x), &px[4 * (size_t)x]);
        if (!rle) {  // flat scan line (the run-length form needs 8 <= width < 32768)
            o.insert(o.end(), px.begin(), px.end());
            continue;
        }
        // run-length form: marker 2 2 width, then each component plane as literal
        // runs of at most 128 bytes (count byte, bytes)
        o.push_back(2), o.push_back(2), o.push_back((uint8_t)(width >> 8)), o.push_back((uint8_t)width);
        for (int c = 0; c < 4; ++c)
            for (uint32_t x = 0; x < width;) {
                const uint32_t n = std::min<uint32_t>(128, width - x);
                o.push_back((uint8_t)n);
                for (uint32_t k = 0; k < n; ++k) o.push_back(px[4 * (size_t)(x + k) + c]);
                x += n;
            }
    }
    return write_file(path, o, "hdr");
}


