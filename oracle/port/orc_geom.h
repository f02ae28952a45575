// CPU oracle -- test infrastructure only (see orc_render.cpp).
//
// Geometry side of the oracle, shared by the restated renderer (orc_render.cpp)
// and the driver that runs the reference's own shading headers on the host
// (oracle/ref_host.cpp): scene storage, the light CDF, RGBA8 texture filtering,
// a CPU binned-SAH BVH with Moller-Trumbore intersection, and the camera basis.
#pragma once
#include "orc_api.h"
#include "orc_shading.h"

#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>

namespace orc {

using V3f = V3<float>;
using V3d = V3<double>;

enum : uint32_t { kLambert = 0, kEmissive = 1, kGlass = 2, kGGX = 3, kGGXT = 4 };
enum : uint32_t { kStageTrace = 0, kStageShade = 1, kStageShadow = 2, kStageDone = 3 };

struct Tex {
    std::vector<uint8_t> px;
    uint32_t w = 0, h = 0;
};

// Bilinear RGBA8 fetch with wrap addressing and normalized-float read, the
// texture mode the reference configures (scene.cpp:403-408).  The hardware filter
// keeps 8 fractional bits of the interpolation weights; the weights here are
// rounded to 1/256 the same way, then blended in FP32.
inline void tex_fetch(const uint8_t* px, uint32_t w, uint32_t h, float u, float v, float out[4]) {
    float uw = u - std::floor(u), vw = v - std::floor(v);
    float x = uw * (float)w - 0.5f, y = vw * (float)h - 0.5f;
    float fx = std::floor(x), fy = std::floor(y);
    float ax = std::rint((x - fx) * 256.0f) * (1.0f / 256.0f);
    float ay = std::rint((y - fy) * 256.0f) * (1.0f / 256.0f);
    int ix = (int)fx, iy = (int)fy;
    int x0 = ((ix % (int)w) + (int)w) % (int)w, y0 = ((iy % (int)h) + (int)h) % (int)h;
    int x1 = (x0 + 1) % (int)w, y1 = (y0 + 1) % (int)h;
    const uint8_t* t00 = px + ((size_t)y0 * w + x0) * 4;
    const uint8_t* t10 = px + ((size_t)y0 * w + x1) * 4;
    const uint8_t* t01 = px + ((size_t)y1 * w + x0) * 4;
    const uint8_t* t11 = px + ((size_t)y1 * w + x1) * 4;
    float bx = 1.0f - ax, by = 1.0f - ay;
    for (int c = 0; c < 4; ++c) {
        float a = (float)t00[c] / 255.0f, b = (float)t10[c] / 255.0f;
        float cc = (float)t01[c] / 255.0f, d = (float)t11[c] / 255.0f;
        out[c] = (a * bx + b * ax) * by + (cc * bx + d * ax) * ay;
    }
}

struct BNode {
    float lo[3], hi[3];
    uint32_t left;   // internal: index of left child (right = left+1); leaf: first prim slot
    uint32_t count;  // 0 = internal
};

struct Scene {
    std::vector<float> vtx, nrm, uv;
    std::vector<uint32_t> idx, triMat;
    std::vector<orc_material> mats;
    std::vector<Tex> tex;
    float env[3] = {0, 0, 0};
    bool hasNormals = false, hasUVs = false;
    std::vector<uint32_t> emissive;
    std::vector<float> cdf;
    // BVH
    std::vector<BNode> nodes;
    std::vector<uint32_t> primOrder;
    std::vector<float> triV0, triE1, triE2;  // per triangle, 3 floats each
    uint32_t nt = 0;

    V3f vert(uint32_t i) const { return {vtx[3 * i], vtx[3 * i + 1], vtx[3 * i + 2]}; }
};

// ---------------------------------------------------------------------------
// Light list and power CDF (scene.cpp:423-491): serial FP32 prefix of
// (ex+ey+ez)*area over emissive triangles in triangle order, divided by the total.
inline void build_light_cdf(Scene& s) {
    s.emissive.clear();
    s.cdf.clear();
    float total = 0.0f;
    for (uint32_t t = 0; t < s.nt; ++t) {
        uint32_t m = s.triMat[t];
        if (m >= s.mats.size() || s.mats[m].type != kEmissive) continue;
        s.emissive.push_back(t);
        V3f a = s.vert(s.idx[3 * t]), b = s.vert(s.idx[3 * t + 1]), c = s.vert(s.idx[3 * t + 2]);
        V3f e1{b.x - a.x, b.y - a.y, b.z - a.z}, e2{c.x - a.x, c.y - a.y, c.z - a.z};
        V3f cr{e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x};
        float area = 0.5f * std::sqrt(cr.x * cr.x + cr.y * cr.y + cr.z * cr.z);
        const orc_material& mm = s.mats[m];
        float power = (mm.emission[0] + mm.emission[1] + mm.emission[2]) * area;
        total += power;
        s.cdf.push_back(total);
    }
    for (float& c : s.cdf) c /= total;
}

// ---------------------------------------------------------------------------
// CPU BVH: binary, binned SAH (16 bins x 3 axes), leaves of <= 4 triangles.
struct BuildPrim {
    float lo[3], hi[3], c[3];
};

inline void build_bvh(Scene& s) {
    uint32_t n = s.nt;
    std::vector<BuildPrim> bp(n);
    s.triV0.resize(3 * (size_t)n);
    s.triE1.resize(3 * (size_t)n);
    s.triE2.resize(3 * (size_t)n);
    for (uint32_t t = 0; t < n; ++t) {
        V3f a = s.vert(s.idx[3 * t]), b = s.vert(s.idx[3 * t + 1]), c = s.vert(s.idx[3 * t + 2]);
        float* v0 = &s.triV0[3 * (size_t)t];
        float* e1 = &s.triE1[3 * (size_t)t];
        float* e2 = &s.triE2[3 * (size_t)t];
        v0[0] = a.x; v0[1] = a.y; v0[2] = a.z;
        e1[0] = b.x - a.x; e1[1] = b.y - a.y; e1[2] = b.z - a.z;
        e2[0] = c.x - a.x; e2[1] = c.y - a.y; e2[2] = c.z - a.z;
        float p[3][3] = {{a.x, a.y, a.z}, {b.x, b.y, b.z}, {c.x, c.y, c.z}};
        for (int k = 0; k < 3; ++k) {
            bp[t].lo[k] = std::min(p[0][k], std::min(p[1][k], p[2][k]));
            bp[t].hi[k] = std::max(p[0][k], std::max(p[1][k], p[2][k]));
            bp[t].c[k] = 0.5f * (bp[t].lo[k] + bp[t].hi[k]);
        }
    }
    s.primOrder.resize(n);
    for (uint32_t i = 0; i < n; ++i) s.primOrder[i] = i;
    s.nodes.clear();
    s.nodes.reserve(2 * (size_t)n + 1);
    struct Task { uint32_t node, begin, end; };
    std::vector<Task> stack;
    s.nodes.push_back(BNode{});
    stack.push_back({0, 0, n});
    auto area = [](const float lo[3], const float hi[3]) {
        float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        if (dx < 0) return 0.0f;
        return 2.0f * (dx * dy + dy * dz + dz * dx);
    };
    const int B = 16;
    while (!stack.empty()) {
        Task tk = stack.back();
        stack.pop_back();
        BNode nd{};
        float clo[3], chi[3];
        for (int k = 0; k < 3; ++k) {
            nd.lo[k] = clo[k] = std::numeric_limits<float>::infinity();
            nd.hi[k] = chi[k] = -std::numeric_limits<float>::infinity();
        }
        for (uint32_t i = tk.begin; i < tk.end; ++i) {
            const BuildPrim& q = bp[s.primOrder[i]];
            for (int k = 0; k < 3; ++k) {
                nd.lo[k] = std::min(nd.lo[k], q.lo[k]);
                nd.hi[k] = std::max(nd.hi[k], q.hi[k]);
                clo[k] = std::min(clo[k], q.c[k]);
                chi[k] = std::max(chi[k], q.c[k]);
            }
        }
        uint32_t cnt = tk.end - tk.begin;
        int bestAxis = -1, bestSplit = -1;
        float bestCost = std::numeric_limits<float>::infinity();
        if (cnt > 4) {
            for (int ax = 0; ax < 3; ++ax) {
                float ext = chi[ax] - clo[ax];
                if (!(ext > 0)) continue;
                float blo[B][3], bhi[B][3];
                uint32_t bc[B] = {0};
                for (int b = 0; b < B; ++b)
                    for (int k = 0; k < 3; ++k) { blo[b][k] = INFINITY; bhi[b][k] = -INFINITY; }
                float scale = (float)B / ext;
                for (uint32_t i = tk.begin; i < tk.end; ++i) {
                    const BuildPrim& q = bp[s.primOrder[i]];
                    int b = std::min(B - 1, (int)((q.c[ax] - clo[ax]) * scale));
                    bc[b]++;
                    for (int k = 0; k < 3; ++k) { blo[b][k] = std::min(blo[b][k], q.lo[k]); bhi[b][k] = std::max(bhi[b][k], q.hi[k]); }
                }
                float rArea[B];
                uint32_t rCnt[B];
                float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
                uint32_t c = 0;
                for (int b = B - 1; b > 0; --b) {
                    c += bc[b];
                    for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], blo[b][k]); hi[k] = std::max(hi[k], bhi[b][k]); }
                    rArea[b] = area(lo, hi);
                    rCnt[b] = c;
                }
                for (int k = 0; k < 3; ++k) { lo[k] = INFINITY; hi[k] = -INFINITY; }
                c = 0;
                for (int b = 0; b < B - 1; ++b) {
                    c += bc[b];
                    for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], blo[b][k]); hi[k] = std::max(hi[k], bhi[b][k]); }
                    if (c == 0 || rCnt[b + 1] == 0) continue;
                    float cost = area(lo, hi) * c + rArea[b + 1] * rCnt[b + 1];
                    if (cost < bestCost) { bestCost = cost; bestAxis = ax; bestSplit = b; }
                }
            }
        }
        uint32_t mid = tk.begin;
        if (bestAxis >= 0) {
            float ext = chi[bestAxis] - clo[bestAxis];
            float scale = (float)B / ext;
            auto it = std::partition(s.primOrder.begin() + tk.begin, s.primOrder.begin() + tk.end, [&](uint32_t p) {
                int b = std::min(B - 1, (int)((bp[p].c[bestAxis] - clo[bestAxis]) * scale));
                return b <= bestSplit;
            });
            mid = (uint32_t)(it - s.primOrder.begin());
        } else if (cnt > 4) {
            mid = tk.begin + cnt / 2;  // all centroids coincide: split by count
        }
        if (cnt <= 4 || mid == tk.begin || mid == tk.end) {
            if (cnt > 4) mid = tk.begin + cnt / 2;
            else { nd.left = tk.begin; nd.count = cnt; s.nodes[tk.node] = nd; continue; }
        }
        uint32_t l = (uint32_t)s.nodes.size();
        s.nodes.push_back(BNode{});
        s.nodes.push_back(BNode{});
        nd.left = l;
        nd.count = 0;
        s.nodes[tk.node] = nd;
        stack.push_back({l, tk.begin, mid});
        stack.push_back({l + 1, mid, tk.end});
    }
}

// Moller-Trumbore, FP32, without the reciprocal: the barycentric tests compare the
// numerators u*det and v*det against det (sign-aware), and t = t_num / det is
// divided (correctly rounded) only for hits inside the triangle.  Cross-product
// components are a product and one fused multiply-add, dot products a product and
// two (std::fma is correctly rounded, as the GPU's fmaf).  The CUDA trace kernel
// evaluates the same operation sequence on the same per-triangle (v0, v1-v0,
// v2-v0) values, so t is bit-identical.  Inlined into the traversal routines,
// which are built twice (GCC target clones): with the host's FMA instruction where
// the CPU has one, else through libm's fmaf; both give the same correctly rounded
// results.
__attribute__((always_inline)) inline bool mt32(const float o[3], const float d[3], const float* v0, const float* e1,
                                                const float* e2, float& t) {
    float px = std::fma(d[1], e2[2], -(d[2] * e2[1]));
    float py = std::fma(d[2], e2[0], -(d[0] * e2[2]));
    float pz = std::fma(d[0], e2[1], -(d[1] * e2[0]));
    float det = std::fma(e1[0], px, std::fma(e1[1], py, e1[2] * pz));
    if (det == 0.0f) return false;
    float sx = o[0] - v0[0], sy = o[1] - v0[1], sz = o[2] - v0[2];
    float un = std::fma(sx, px, std::fma(sy, py, sz * pz));
    float qx = std::fma(sy, e1[2], -(sz * e1[1]));
    float qy = std::fma(sz, e1[0], -(sx * e1[2]));
    float qz = std::fma(sx, e1[1], -(sy * e1[0]));
    float vn = std::fma(d[0], qx, std::fma(d[1], qy, d[2] * qz));
    float uv = un + vn;
    bool inside = det > 0.0f ? (un >= 0.0f && vn >= 0.0f && uv <= det) : (un <= 0.0f && vn <= 0.0f && uv >= det);
    if (!inside) return false;
    t = std::fma(e2[0], qx, std::fma(e2[1], qy, e2[2] * qz)) / det;
    return true;
}

inline bool mt64(const double o[3], const double d[3], const double v0[3], const double e1[3],
                        const double e2[3], double& t) {
    double px = d[1] * e2[2] - d[2] * e2[1], py = d[2] * e2[0] - d[0] * e2[2], pz = d[0] * e2[1] - d[1] * e2[0];
    double det = e1[0] * px + e1[1] * py + e1[2] * pz;
    if (det == 0.0) return false;
    double inv = 1.0 / det;
    double sx = o[0] - v0[0], sy = o[1] - v0[1], sz = o[2] - v0[2];
    double u = (sx * px + sy * py + sz * pz) * inv;
    if (!(u >= 0.0 && u <= 1.0)) return false;
    double qx = sy * e1[2] - sz * e1[1], qy = sz * e1[0] - sx * e1[2], qz = sx * e1[1] - sy * e1[0];
    double v = (d[0] * qx + d[1] * qy + d[2] * qz) * inv;
    if (!(v >= 0.0 && u + v <= 1.0)) return false;
    t = (e2[0] * qx + e2[1] * qy + e2[2] * qz) * inv;
    return true;
}

// Slab test with the far distance widened by a few ulps so that rounding never
// culls a box whose triangles the exact test would hit.
inline bool box_hit(const BNode& b, const float o[3], const float inv[3], float tmin, float tmax) {
    // the current best t is widened too: a box reaching an equal-t hit must be
    // opened so ties resolve to the lowest triangle index wherever they lie
    float t0 = tmin, t1 = tmax * 1.0000005f;
    for (int k = 0; k < 3; ++k) {
        float a = (b.lo[k] - o[k]) * inv[k], c = (b.hi[k] - o[k]) * inv[k];
        float n = std::min(a, c), f = std::max(a, c);
        if (n != n) n = -INFINITY;  // 0*inf
        if (f != f) f = INFINITY;
        t0 = std::max(t0, n);
        t1 = std::min(t1, f * 1.0000004f);
    }
    return t0 <= t1;
}

// Closest hit over [tmin, tmax]; ties in t go to the lower triangle index.
__attribute__((target_clones("fma", "default"))) static bool closest32(const Scene& s, const float o[3],
                                                                      const float d[3], float tmin, float tmax,
                                                                      float& tb, uint32_t& pb) {
    float inv[3] = {1.0f / d[0], 1.0f / d[1], 1.0f / d[2]};
    tb = tmax;
    pb = 0xffffffffu;
    uint32_t st[128];
    int sp = 0;
    st[sp++] = 0;
    while (sp) {
        const BNode& nd = s.nodes[st[--sp]];
        if (!box_hit(nd, o, inv, tmin, tb)) continue;
        if (nd.count) {
            for (uint32_t i = 0; i < nd.count; ++i) {
                uint32_t p = s.primOrder[nd.left + i];
                float t;
                if (mt32(o, d, &s.triV0[3 * (size_t)p], &s.triE1[3 * (size_t)p], &s.triE2[3 * (size_t)p], t) &&
                    t >= tmin && t <= tmax && (t < tb || (t == tb && p < pb))) {
                    tb = t;
                    pb = p;
                }
            }
        } else {
            st[sp++] = nd.left;
            st[sp++] = nd.left + 1;
        }
    }
    return pb != 0xffffffffu;
}

// FP64 slab test against the FP32 box (which bounds the FP32 vertices exactly),
// widened by a relative 1e-9 plus an absolute 1e-12 on both ends: far more than the
// ~1e-16 relative rounding of the double arithmetic, so no box whose triangles the
// exact test hits is ever culled.
inline bool box_hit64(const BNode& b, const double o[3], const double inv[3], double tmin, double tmax) {
    double t0 = tmin, t1 = tmax;
    for (int k = 0; k < 3; ++k) {
        double a = ((double)b.lo[k] - o[k]) * inv[k], c = ((double)b.hi[k] - o[k]) * inv[k];
        double n = std::min(a, c), f = std::max(a, c);
        if (n != n) n = -INFINITY;  // 0*inf
        if (f != f) f = INFINITY;
        t0 = std::max(t0, n);
        t1 = std::min(t1, f);
    }
    return t0 - (std::fabs(t0) * 1e-9 + 1e-12) <= t1 + (std::fabs(t1) * 1e-9 + 1e-12);
}

// Exact-reference closest hit: the FP64 Moller-Trumbore of every triangle a ray can
// reach, found by walking the CPU BVH with the widened FP64 slab test above (the
// result equals testing all triangles, without the O(triangles) cost per ray).
// Ties in t go to the lower triangle index.
static bool closest64(const Scene& s, const double o[3], const double d[3], double tmin, double tmax, double& tb,
                      uint32_t& pb) {
    double inv[3] = {1.0 / d[0], 1.0 / d[1], 1.0 / d[2]};
    tb = tmax;
    pb = 0xffffffffu;
    uint32_t st[128];
    int sp = 0;
    st[sp++] = 0;
    while (sp) {
        const BNode& nd = s.nodes[st[--sp]];
        if (!box_hit64(nd, o, inv, tmin, tb)) continue;
        if (nd.count) {
            for (uint32_t i = 0; i < nd.count; ++i) {
                uint32_t p = s.primOrder[nd.left + i];
                // edges recomputed in double from the vertices (the FP32 edge arrays are rounded)
                V3f va = s.vert(s.idx[3 * (size_t)p]), vb = s.vert(s.idx[3 * (size_t)p + 1]),
                    vc = s.vert(s.idx[3 * (size_t)p + 2]);
                double v0[3] = {va.x, va.y, va.z};
                double e1[3] = {(double)vb.x - va.x, (double)vb.y - va.y, (double)vb.z - va.z};
                double e2[3] = {(double)vc.x - va.x, (double)vc.y - va.y, (double)vc.z - va.z};
                double t;
                if (mt64(o, d, v0, e1, e2, t) && t >= tmin && t <= tmax && (t < tb || (t == tb && p < pb))) {
                    tb = t;
                    pb = p;
                }
            }
        } else {
            st[sp++] = nd.left;
            st[sp++] = nd.left + 1;
        }
    }
    return pb != 0xffffffffu;
}

__attribute__((target_clones("fma", "default"))) static bool occluded32(const Scene& s, const float o[3],
                                                                       const float d[3], float tmin, float tmax) {
    float inv[3] = {1.0f / d[0], 1.0f / d[1], 1.0f / d[2]};
    uint32_t st[128];
    int sp = 0;
    st[sp++] = 0;
    while (sp) {
        const BNode& nd = s.nodes[st[--sp]];
        if (!box_hit(nd, o, inv, tmin, tmax)) continue;
        if (nd.count) {
            for (uint32_t i = 0; i < nd.count; ++i) {
                uint32_t p = s.primOrder[nd.left + i];
                float t;
                if (mt32(o, d, &s.triV0[3 * (size_t)p], &s.triE1[3 * (size_t)p], &s.triE2[3 * (size_t)p], t) &&
                    t >= tmin && t <= tmax)
                    return true;
            }
        } else {
            st[sp++] = nd.left;
            st[sp++] = nd.left + 1;
        }
    }
    return false;
}

// ---------------------------------------------------------------------------
// Camera basis (types.h:41-50 via GLM: normalize = v * (1/sqrt(dot))), tan(fovY/2)
// on the host (renderer.cpp:153).
struct CamBasis {
    V3f pos, fwd, right, up;
    float tanHalf, aspect, focal, lens;
};
inline V3f glm_normalize(V3f v) {
    float r = 1.0f / std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    return {v.x * r, v.y * r, v.z * r};
}
inline CamBasis cam_basis(const orc_camera& c) {
    CamBasis b;
    b.pos = {c.position[0], c.position[1], c.position[2]};
    V3f tg{c.target[0], c.target[1], c.target[2]}, up{c.up[0], c.up[1], c.up[2]};
    b.fwd = glm_normalize(tg - b.pos);
    b.right = glm_normalize(cross(b.fwd, up));
    b.up = glm_normalize(cross(b.right, b.fwd));
    b.tanHalf = std::tan(c.fovY * 0.5f);
    b.aspect = c.aspect;
    b.focal = c.focalDistance;
    b.lens = c.lensRadius;
    return b;
}


// Builds the oracle scene from the C descriptor: copies buffers, builds the light
// list/CDF and the BVH.
inline Scene* scene_from_desc(const orc_scene_desc* d) {
    Scene* s = new Scene();
    s->nt = d->numTriangles;
    s->vtx.assign(d->vertices, d->vertices + 3 * (size_t)d->numVertices);
    if (d->normals) { s->nrm.assign(d->normals, d->normals + 3 * (size_t)d->numVertices); s->hasNormals = true; }
    if (d->uvs) { s->uv.assign(d->uvs, d->uvs + 2 * (size_t)d->numVertices); s->hasUVs = true; }
    s->idx.assign(d->indices, d->indices + 3 * (size_t)d->numTriangles);
    s->triMat.assign(d->triMaterial, d->triMaterial + d->numTriangles);
    s->mats.assign(d->materials, d->materials + d->numMaterials);
    for (uint32_t i = 0; i < d->numTextures; ++i) {
        Tex t;
        t.w = d->textures[i].width;
        t.h = d->textures[i].height;
        if (d->textures[i].rgba) t.px.assign(d->textures[i].rgba, d->textures[i].rgba + 4 * (size_t)t.w * t.h);
        s->tex.push_back(std::move(t));
    }
    for (int k = 0; k < 3; ++k) s->env[k] = d->envRadiance[k];
    build_light_cdf(*s);
    build_bvh(*s);
    return s;
}

}  // namespace orc
