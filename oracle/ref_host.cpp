// Reference-on-the-host driver -- test infrastructure only.
//
// Compiles the reference's own shading, sampling, GGX and material headers
// (libWR/kernels/*.cuh, compiled where they lie in the reference checkout) on the
// CPU through the small shim in oracle/ref_shim, and drives them with the
// oracle's CPU BVH.  Built into oracle/_ref/libref.so by oracle/Makefile.  Used to
//   * pin the oracle's restatement (orc_render.cpp) against the reference code,
//   * time the reference's shading on the host cores as bench.py's CPU baseline.
// The per-path loop and the raygen / closest-hit logic (libWR/kernels/trace.cu,
// libWR/kernels/shade.cu, libWR/src/internal/renderer.cpp) run OptiX device
// programs in the reference and cannot be compiled here, so they are restated
// below against the reference's own RayState / HitInfo / LaunchParams types.
#include "ref_shim/ref_prelude.h"
#define printf(...) ((void)0)
#include "vector_math.cuh"
#include "sampling.cuh"
#include "ggx.cuh"
#include "materials.cuh"
#include "utils/atomic_ops.cuh"
#include "utils/fresnel.cuh"
#include "utils/ray_offset.cuh"
#include "utils/normal_map.cuh"
#include "materials/emissive.cuh"
#include "materials/lambertian.cuh"
#include "materials/glass.cuh"
#include "materials/ggx_material.cuh"
#include "materials/ggx_transmission.cuh"
#undef printf

#include "port/orc_geom.h"

#include <wr/types.h>
#include "helpers/image.h"

#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using wr::internal::HitInfo;
using wr::internal::LaunchParams;
using wr::internal::MaterialData;
using wr::internal::RayState;

template <> float4 tex2D<float4>(cudaTextureObject_t obj, float u, float v) {
    const orc_texture* t = reinterpret_cast<const orc_texture*>(obj);
    float c[4];
    orc::tex_fetch(t->rgba, t->width, t->height, u, v, c);
    return make_float4(c[0], c[1], c[2], c[3]);
}

namespace {

struct RefScene {
    orc::Scene* s;
    std::vector<orc_texture> texDesc;
    std::vector<cudaTextureObject_t> texObj;
    std::vector<MaterialData> mats;
};

LaunchParams make_params(const RefScene& rs, const orc_render_params* p, float3* accum, float3* alb, float3* nrm) {
    const orc::Scene& s = *rs.s;
    LaunchParams lp{};
    lp.geometry.vertices = s.vtx.data();
    lp.geometry.normals = s.hasNormals ? s.nrm.data() : nullptr;
    lp.geometry.indices = s.idx.data();
    lp.geometry.triangleMaterialIds = s.triMat.data();
    lp.geometry.uvs = s.hasUVs ? s.uv.data() : nullptr;
    lp.accumBuffer = accum;
    lp.albedoBuffer = alb;
    lp.normalBuffer = nrm;
    lp.materials = rs.mats.data();
    lp.numMaterials = (uint32_t)rs.mats.size();
    lp.textures = rs.texObj.empty() ? nullptr : rs.texObj.data();
    lp.numTextures = (uint32_t)rs.texObj.size();
    lp.emissiveTriangles = s.emissive.data();
    lp.emissiveTriangleCDF = s.cdf.data();
    lp.numEmissiveTriangles = (uint32_t)s.emissive.size();
    lp.environmentRadiance = make_float4(s.env[0], s.env[1], s.env[2], 0.0f);
    lp.width = p->width;
    lp.height = p->height;
    lp.useNEE = p->useNEE;
    lp.maxBounces = p->maxBounces;
    lp.rrStartDepth = p->rrStartDepth;
    lp.fireflyClamp = p->fireflyClamp;
    return lp;
}

// trace.cu:54-125 (camera ray at depth 0), written with the reference helpers.
void gen_camera(RayState& ray, const LaunchParams& lp, const orc::CamBasis& cb, uint32_t pixel, uint32_t sample,
                uint32_t userSeed) {
    using namespace wr::internal;
    uint32_t px = pixel % lp.width, py = pixel / lp.width;
    uint32_t seed = (pixel * 1664525u + sample * 1013904223u) ^ 0x9e3779b9u;
    if (userSeed != 0u) seed ^= pcg_hash(userSeed);
    uint32_t js = seed;
    float r1 = randf(js);
    float r2 = randf(js);
    float ndcX = (2.0f * (px + r1) / lp.width - 1.0f) * cb.aspect;
    float ndcY = 1.0f - 2.0f * (py + r2) / lp.height;
    float3 pos = make_float3(cb.pos.x, cb.pos.y, cb.pos.z);
    float3 fwd = make_float3(cb.fwd.x, cb.fwd.y, cb.fwd.z);
    float3 rgt = make_float3(cb.right.x, cb.right.y, cb.right.z);
    float3 up = make_float3(cb.up.x, cb.up.y, cb.up.z);
    float3 dir = normalize(fwd + rgt * ndcX * cb.tanHalf + up * ndcY * cb.tanHalf);
    if (cb.lens > 0.0f && cb.focal > 0.0f) {
        float r3 = randf(js), r4 = randf(js);
        float th = 2.0f * 3.14159265f * r3;
        float rad = sqrtf(r4) * cb.lens;
        float3 off = make_float3(rgt.x * rad * cosf(th) + up.x * rad * sinf(th),
                                 rgt.y * rad * cosf(th) + up.y * rad * sinf(th),
                                 rgt.z * rad * cosf(th) + up.z * rad * sinf(th));
        float3 fp = make_float3(pos.x + dir.x * cb.focal, pos.y + dir.y * cb.focal, pos.z + dir.z * cb.focal);
        ray.origin = make_float3(pos.x + off.x, pos.y + off.y, pos.z + off.z);
        ray.direction = normalize(make_float3(fp.x - ray.origin.x, fp.y - ray.origin.y, fp.z - ray.origin.z));
    } else {
        ray.origin = pos;
        ray.direction = dir;
    }
    ray.throughput = make_float3(1, 1, 1);
    ray.radiance = make_float3(0, 0, 0);
    ray.pixelIndex = pixel;
    ray.depth = 0;
    ray.stage = RayStage::Trace;
    ray.seed = seed;
    ray.tMin = 0.0001f;
    ray.tMax = 1e20f;
    ray.isFirstHit = true;
    ray.prevPdf = 1.0f;
    ray.prevWasDelta = true;
    ray.rngDimension = 0;
    ray.neeDone = 0;
}

// trace.cu:155-319 (closest-hit program) with the reference helpers.
void closest_hit(RayState& ray, HitInfo& hit, const LaunchParams& lp, float t, uint32_t primIdx) {
    using namespace wr::internal;
    float3 hitPos = ray.origin + t * ray.direction;
    const float* V = lp.geometry.vertices;
    uint32_t i0 = lp.geometry.indices[primIdx * 3], i1 = lp.geometry.indices[primIdx * 3 + 1],
             i2 = lp.geometry.indices[primIdx * 3 + 2];
    float3 v0 = make_float3(V[i0 * 3], V[i0 * 3 + 1], V[i0 * 3 + 2]);
    float3 v1 = make_float3(V[i1 * 3], V[i1 * 3 + 1], V[i1 * 3 + 2]);
    float3 v2 = make_float3(V[i2 * 3], V[i2 * 3 + 1], V[i2 * 3 + 2]);
    float3 e1 = v1 - v0, e2 = v2 - v0;
    float3 gN = normalize(cross(e1, e2));
    float3 vp = hitPos - v0;
    float d00 = dot(e1, e1), d01 = dot(e1, e2), d11 = dot(e2, e2), d20 = dot(vp, e1), d21 = dot(vp, e2);
    float den = d00 * d11 - d01 * d01;
    float bv = (d11 * d20 - d01 * d21) / fmaxf(den, 1e-8f);
    float bw = (d00 * d21 - d01 * d20) / fmaxf(den, 1e-8f);
    float bu = 1.0f - bv - bw;
    float3 sN = gN;
    if (lp.geometry.normals) {
        const float* N = lp.geometry.normals;
        float3 n0 = make_float3(N[i0 * 3], N[i0 * 3 + 1], N[i0 * 3 + 2]);
        float3 n1 = make_float3(N[i1 * 3], N[i1 * 3 + 1], N[i1 * 3 + 2]);
        float3 n2 = make_float3(N[i2 * 3], N[i2 * 3 + 1], N[i2 * 3 + 2]);
        if (length(n0) > 1e-6f && length(n1) > 1e-6f && length(n2) > 1e-6f) {
            sN = normalize(bu * n0 + bv * n1 + bw * n2);
            if (dot(sN, gN) < 0.0f) sN = -sN;
        }
    }
    float3 nF = dot(gN, ray.direction) > 0.0f ? -gN : gN;
    float3 sNF = dot(sN, ray.direction) > 0.0f ? -sN : sN;
    hit.position = hitPos;
    hit.normal = sNF;
    hit.geometricNormal = nF;
    hit.materialId = lp.geometry.triangleMaterialIds[primIdx];
    hit.primIndex = primIdx;
    if (lp.geometry.uvs) {
        const float* U = lp.geometry.uvs;
        hit.uv = make_float2(bu * U[i0 * 2] + bv * U[i1 * 2] + bw * U[i2 * 2],
                             bu * U[i0 * 2 + 1] + bv * U[i1 * 2 + 1] + bw * U[i2 * 2 + 1]);
    } else {
        hit.uv = make_float2(0, 0);
    }
    if (ray.isFirstHit) {
        if (hit.materialId < lp.numMaterials) {
            float3 al = getMaterialAlbedo(lp.materials[hit.materialId], hit.uv,
                                          reinterpret_cast<const cudaTextureObject_t*>(lp.textures), lp.numTextures);
            if (lp.albedoBuffer) atomicAddFloat3(&lp.albedoBuffer[ray.pixelIndex], al);
            if (lp.normalBuffer) atomicAddFloat3(&lp.normalBuffer[ray.pixelIndex], nF);
        }
        ray.isFirstHit = false;
    }
    if (hit.materialId < lp.numMaterials) {
        const MaterialData& m = lp.materials[hit.materialId];
        if (m.type == MaterialType::Emissive) {
            float w = 1.0f;
            if (lp.useNEE && ray.depth > 0 && !ray.prevWasDelta && lp.numEmissiveTriangles > 0) {
                float area = 0.5f * length(cross(e1, e2));
                float d2 = t * t;
                float cl = fabsf(dot(nF, ray.direction));
                float pa = 1.0f / (lp.numEmissiveTriangles * area);
                float lpdf = pa * d2 / fmaxf(cl, 1e-8f);
                w = powerHeuristic(ray.prevPdf, lpdf);
            }
            float3 em = make_float3(m.emission.x, m.emission.y, m.emission.z);
            ray.radiance = ray.radiance + ray.throughput * em * w;
        }
    }
}

// Per-path view of renderer.cpp:190-284 with the shade dispatch of shade.cu:24-85.
void run_path(const orc::Scene& s, const LaunchParams& lp, const orc::CamBasis& cb, uint32_t pixel,
              uint32_t sample, uint32_t userSeed, uint32_t iters, uint64_t& ext, uint64_t& shd) {
    using namespace wr::internal;
    RayState ray{};
    HitInfo hit{};
    ray.stage = RayStage::Trace;
    for (uint32_t it = 0; it < iters; ++it) {
        if (ray.stage == RayStage::Shadow) {
            float o[3] = {ray.origin.x, ray.origin.y, ray.origin.z}, d[3] = {ray.direction.x, ray.direction.y, ray.direction.z};
            shd++;
            if (!orc::occluded32(s, o, d, ray.tMin, ray.tMax)) ray.radiance = ray.radiance + ray.shadowContribution;
            ray.direction = ray.savedDirection;
            ray.stage = RayStage::Shade;
        } else if (ray.stage == RayStage::Trace) {
            if (ray.depth == 0 && it == 0) gen_camera(ray, lp, cb, pixel, sample, userSeed);
            float o[3] = {ray.origin.x, ray.origin.y, ray.origin.z}, d[3] = {ray.direction.x, ray.direction.y, ray.direction.z};
            float t;
            uint32_t prim;
            ext++;
            if (!orc::closest32(s, o, d, ray.tMin, ray.tMax, t, prim)) {
                float3 env = make_float3(lp.environmentRadiance.x, lp.environmentRadiance.y, lp.environmentRadiance.z);
                ray.radiance = ray.radiance + ray.throughput * env;
                atomicAddFloat3(&lp.accumBuffer[ray.pixelIndex], clampFireflies(ray.radiance, lp.fireflyClamp));
                return;
            }
            closest_hit(ray, hit, lp, t, prim);
            ray.stage = RayStage::Shade;
        }
        if (ray.stage == RayStage::Shade) {
            if (hit.materialId >= lp.numMaterials) return;
            const MaterialData& m = lp.materials[hit.materialId];
            HitInfo eh = hit;
            if (m.normalTextureId > 0)
                eh.normal = getEffectiveNormal(m, hit, reinterpret_cast<const cudaTextureObject_t*>(lp.textures),
                                               lp.numTextures);
            switch (m.type) {
                case MaterialType::Emissive: shadeEmissive(ray, eh, m, &lp); break;
                case MaterialType::Lambertian: shadeLambertian(ray, eh, m, &lp); break;
                case MaterialType::Glass: shadeGlass(ray, eh, m, &lp); break;
                case MaterialType::GGXReflection: shadeGGX(ray, eh, m, &lp); break;
                case MaterialType::GGXTransmission: shadeGGXTransmission(ray, eh, m, &lp); break;
                default: terminateRay(ray, &lp); break;
            }
        }
        if (ray.stage == RayStage::Terminated) return;
    }
}

}  // namespace

extern "C" {

void* ref_scene_create(const orc_scene_desc* d) {
    RefScene* rs = new RefScene();
    rs->s = orc::scene_from_desc(d);
    rs->texDesc.assign(d->textures, d->textures + d->numTextures);
    for (size_t i = 0; i < rs->texDesc.size(); ++i)
        rs->texObj.push_back((cudaTextureObject_t) reinterpret_cast<uintptr_t>(&rs->texDesc[i]));
    rs->mats.resize(d->numMaterials);
    static_assert(sizeof(MaterialData) == sizeof(orc_material), "material record size");
    std::memcpy(rs->mats.data(), d->materials, sizeof(orc_material) * d->numMaterials);
    return rs;
}

void ref_scene_destroy(void* p) {
    RefScene* rs = (RefScene*)p;
    delete rs->s;
    delete rs;
}

void ref_render(void* p, const orc_camera* cam, const orc_render_params* rp, float* rgb, float* albedo, float* normal,
                int threads, orc_stats* stats) {
    RefScene* rs = (RefScene*)p;
    uint32_t np = rp->width * rp->height;
    uint32_t pb = rp->pixelBegin, pe = rp->pixelEnd ? rp->pixelEnd : np;
    std::vector<float3> accum(np, make_float3(0, 0, 0));
    if (albedo) std::memset(albedo, 0, sizeof(float) * 3 * (size_t)np);
    if (normal) std::memset(normal, 0, sizeof(float) * 3 * (size_t)np);
    LaunchParams lp = make_params(*rs, rp, accum.data(), (float3*)albedo, (float3*)normal);
    orc::CamBasis cb = orc::cam_basis(*cam);
    uint32_t iters = rp->maxIterations ? rp->maxIterations : 8;
    uint64_t ext = 0, shd = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : ext, shd)
#endif
    for (int64_t px = pb; px < (int64_t)pe; ++px)
        for (uint32_t k = 0; k < rp->spp; ++k)
            run_path(*rs->s, lp, cb, (uint32_t)px, rp->sampleBegin + k, rp->seed, iters, ext, shd);
    float inv = 1.0f / (float)rp->spp;
    if (rgb)
        for (uint32_t i = 0; i < np; ++i) {
            rgb[3 * i] = accum[i].x * inv;
            rgb[3 * i + 1] = accum[i].y * inv;
            rgb[3 * i + 2] = accum[i].z * inv;
        }
    if (stats) {
        stats->extensionRays = ext;
        stats->shadowRays = shd;
        stats->paths = (uint64_t)(pe - pb) * rp->spp;
    }
}

// Same record layout as orc_bsdf_batch (FP32), evaluated by the reference functions.
void ref_bsdf_batch(const float* in, uint32_t n, double* out) {
    using namespace wr::internal;
    for (uint32_t i = 0; i < n; ++i) {
        const float* q = in + 20 * (size_t)i;
        double* o = out + 34 * (size_t)i;
        float3 wo = make_float3(q[0], q[1], q[2]), wi = make_float3(q[3], q[4], q[5]), n3 = make_float3(q[6], q[7], q[8]);
        float3 al = make_float3(q[9], q[10], q[11]);
        float rough = q[12], metal = q[13], ior = q[14], u0 = q[15], u1 = q[16], u2 = q[17];
        uint32_t depth = (uint32_t)q[18];
        float rr = q[19];
        float3 e = evaluateGGXReflection(wo, wi, n3, al, rough, metal, ior);
        o[0] = e.x; o[1] = e.y; o[2] = e.z;
        float gp = ggxReflectionPdf(wo, wi, n3, rough);
        o[3] = gp;
        float3 tg, bt;
        createCoordinateFrame(n3, tg, bt);
        float3 sw = make_float3(0, 0, 0);
        float sp = 0;
        sampleGGXReflection(wo, n3, tg, bt, rough, u0, u1, sw, sp);
        bool ok = sp > 0.0f || sp != sp;
        if (!ok) sw = make_float3(0, 0, 0);
        o[4] = sw.x; o[5] = sw.y; o[6] = sw.z; o[7] = sp; o[8] = ok ? 1.0 : 0.0;
        o[9] = fresnelDielectric(fabsf(dot(wo, n3)), 1.0f, ior);
        float cp;
        float3 ch = sampleCosineHemisphere(u0, u1, cp);
        o[10] = ch.x; o[11] = ch.y; o[12] = ch.z; o[13] = cp;
        float cpdf = cosineHemispherePdf(dot(n3, wi));
        o[14] = powerHeuristic(gp, cpdf);
        o[15] = cpdf;
        float3 nt = make_float3(0, 0, 0);
        bool sv = russianRoulette(al, depth, rr, u2, nt, metal > 0.5f);
        o[16] = sv ? 1.0 : 0.0;
        o[17] = nt.x; o[18] = nt.y; o[19] = nt.z;
        o[20] = tg.x; o[21] = tg.y; o[22] = tg.z; o[23] = bt.x; o[24] = bt.y; o[25] = bt.z;
        float3 ln;
        float la;
        float3 pp = sampleTriangle(u0, u1, wo, wi, n3, ln, la);
        o[26] = pp.x; o[27] = pp.y; o[28] = pp.z; o[29] = la; o[30] = ln.x; o[31] = ln.y; o[32] = ln.z;
        o[33] = asymmetricScatteringCorrection(wi, n3, normalize(wo));
    }
}

void ref_rng_batch(const uint32_t* seeds, const uint32_t* dims, uint32_t n, uint32_t* hash, float* u) {
    for (uint32_t i = 0; i < n; ++i) {
        hash[i] = wr::internal::pcg_hash(seeds[i], dims[i]);
        u[i] = wr::internal::rnd_dim(seeds[i], dims[i]);
    }
}

void ref_cdf_batch(const float* cdf, uint32_t ncdf, const float* u, uint32_t n, uint32_t* out) {
    for (uint32_t i = 0; i < n; ++i) out[i] = wr::internal::sampleEmissiveTriangle(u[i], cdf, ncdf);
}

// Camera basis through the reference's public wr::Camera helpers (GLM).
void ref_camera_basis(const orc_camera* c, float* out12) {
    wr::Camera cam;
    cam.position = wr::Vec3(c->position[0], c->position[1], c->position[2]);
    cam.target = wr::Vec3(c->target[0], c->target[1], c->target[2]);
    cam.up = wr::Vec3(c->up[0], c->up[1], c->up[2]);
    cam.fovY = c->fovY;
    wr::Vec3 f = cam.getForward(), r = cam.getRight(), u = cam.getUp();
    float v[12] = {f.x, f.y, f.z, r.x, r.y, r.z, u.x, u.y, u.z, tanf(cam.fovY * 0.5f), 0, 0};
    std::memcpy(out12, v, sizeof(v));
}

// The reference's PNG writer (exposure, ACES, gamma, 8-bit) on a linear image.
void ref_save_png(const char* path, const float* rgb, uint32_t w, uint32_t h) {
    test_helpers::savePNG(path, reinterpret_cast<const wr::Vec3*>(rgb), w, h);
}

}  // extern "C"
