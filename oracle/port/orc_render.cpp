// CPU oracle -- test infrastructure only.  Only tests/, the smoke check and the
// CPU-baseline leg of bench.py load this; the product never links it.
//
// Restates libWR's render path on the CPU (reference paths below are inside
// trianglestrip/OfflineRenderer):
//   * Scene::finalize light list + power CDF          libWR/src/internal/scene.cpp:423-491
//   * camera basis                                     libWR/include/wr/types.h:41-50,
//                                                      libWR/src/internal/renderer.cpp:144-156
//   * raygen / closest-hit / miss programs             libWR/kernels/trace.cu:17-323
//   * shade dispatch + material shaders                libWR/kernels/shade.cu:24-85,
//                                                      libWR/kernels/materials/*.cuh
//   * the host wavefront loop (per-path view)          libWR/src/internal/renderer.cpp:190-313
// OptiX traversal is replaced by a CPU binned-SAH BVH with a Moller-Trumbore test
// whose FP32 arithmetic is the same formula the CUDA trace kernel evaluates; the
// FP64 modes of orc_closest are the exact reference: mode 1 tests every triangle in
// double precision, mode 2 walks the BVH with conservatively widened FP64 boxes
// (the same answer in O(log n) per ray, for multi-million-triangle scenes).
#include "orc_geom.h"

#include <atomic>
#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// Camera ray for (pixel, sample): trace.cu:54-125.
static void camera_ray(const CamBasis& cb, uint32_t w, uint32_t h, uint32_t pixel, uint32_t sample,
                       uint32_t user_seed, V3f& o, V3f& d, uint32_t& seed) {
    uint32_t px = pixel % w, py = pixel / w;
    seed = path_seed(pixel, sample, user_seed);
    uint32_t js = seed;
    float r1 = lcg_randf(js);
    float r2 = lcg_randf(js);
    float nx = (2.0f * ((float)px + r1) / (float)w - 1.0f) * cb.aspect;
    float ny = 1.0f - 2.0f * ((float)py + r2) / (float)h;
    V3f dir = normalize(cb.fwd + cb.right * nx * cb.tanHalf + cb.up * ny * cb.tanHalf);
    if (cb.lens > 0.0f && cb.focal > 0.0f) {
        float r3 = lcg_randf(js);
        float r4 = lcg_randf(js);
        float th = 2.0f * 3.14159265f * r3;
        float rad = std::sqrt(r4) * cb.lens;
        float ct = std::cos(th), sn = std::sin(th);
        V3f off{cb.right.x * rad * ct + cb.up.x * rad * sn, cb.right.y * rad * ct + cb.up.y * rad * sn,
                cb.right.z * rad * ct + cb.up.z * rad * sn};
        V3f fp{cb.pos.x + dir.x * cb.focal, cb.pos.y + dir.y * cb.focal, cb.pos.z + dir.z * cb.focal};
        o = {cb.pos.x + off.x, cb.pos.y + off.y, cb.pos.z + off.z};
        d = normalize(mk(fp.x - o.x, fp.y - o.y, fp.z - o.z));
    } else {
        o = cb.pos;
        d = dir;
    }
}

// ---------------------------------------------------------------------------
struct Hit {
    V3f pos, n, ng;
    float u, v;
    uint32_t mat, prim;
};

struct Path {
    V3f o, d, thr, rad, shadowC, savedD;
    uint32_t pixel, depth, seed, stage, dim, neeDone;
    float tmin, tmax, prevPdf;
    bool firstHit, prevDelta;
};

struct Ctx {
    const Scene* s;
    const orc_render_params* p;
    float* accum;   // float3 per pixel (sums)
    float* albedo;  // may be null
    float* normal;
    uint64_t ext = 0, shd = 0;
};

static inline V3f albedo_of(const Scene& s, const orc_material& m, float u, float v) {
    if (m.albedoTextureId != 0 && m.albedoTextureId <= s.tex.size()) {
        const Tex& t = s.tex[m.albedoTextureId - 1];
        if (t.px.empty()) return {1, 1, 1};
        float c[4];
        tex_fetch(t.px.data(), t.w, t.h, u, v, c);
        return {c[0], c[1], c[2]};
    }
    return {m.albedo[0], m.albedo[1], m.albedo[2]};
}

static inline void add3(float* buf, uint32_t px, V3f v) {
    buf[3 * px] += v.x;
    buf[3 * px + 1] += v.y;
    buf[3 * px + 2] += v.z;
}

// material_common.cuh:31-36
static inline void terminate(Ctx& c, Path& r) {
    V3f cl = clamp_fireflies(r.rad, c.p->fireflyClamp);
    add3(c.accum, r.pixel, cl);
    r.stage = kStageDone;
}
static inline bool apply_rr(Ctx& c, Path& r, bool delta) {
    V3f nt;
    float xi = rnd_dim(r.seed, r.dim++);
    if (!russian_roulette(r.thr, r.depth, c.p->rrStartDepth, xi, nt, delta)) {
        terminate(c, r);
        return false;
    }
    r.thr = nt;
    return true;
}
static inline void next_bounce(Ctx& c, Path& r, const Hit& h, V3f nd) {
    r.d = nd;
    r.o = offset_origin(h.pos, h.n, nd);
    r.tmin = 0.0f;
    r.tmax = 1e20f;
    r.depth++;
    r.stage = kStageTrace;
    if (r.depth >= c.p->maxBounces) terminate(c, r);
}
// Two uniforms consumed by one call (lambertian.cuh:534-535,613-614;
// ggx_material.cuh:79-80,168-169).  Which argument receives the earlier dimension
// is the compiler's argument-evaluation order.
static inline void draw2(Path& r, uint32_t order, float& a, float& b) {
    float x = rnd_dim(r.seed, r.dim++);
    float y = rnd_dim(r.seed, r.dim++);
    if (order == 0) { a = x; b = y; } else { a = y; b = x; }
}

static inline void light_vertices(const Scene& s, uint32_t tri, V3f& a, V3f& b, V3f& cc) {
    a = s.vert(s.idx[3 * tri]);
    b = s.vert(s.idx[3 * tri + 1]);
    cc = s.vert(s.idx[3 * tri + 2]);
}

// lambertian.cuh:8-147
static void shade_lambert(Ctx& c, Path& r, const Hit& h, const orc_material& m) {
    const Scene& s = *c.s;
    uint32_t nE = (uint32_t)s.emissive.size();
    if (c.p->useNEE && nE > 0 && !r.neeDone) {
        float lu = rnd_dim(r.seed, r.dim++);
        uint32_t li = cdf_lower_bound(lu, s.cdf.data(), nE);
        uint32_t tri = s.emissive[li];
        V3f a, b, cc;
        light_vertices(s, tri, a, b, cc);
        float u1, u2;
        draw2(r, c.p->drawOrder, u1, u2);
        V3f ln;
        float la;
        V3f lp = sample_triangle(u1, u2, a, b, cc, ln, la);
        V3f tl{lp.x - h.pos.x, lp.y - h.pos.y, lp.z - h.pos.z};
        float d2 = dot(tl, tl);
        float dist = std::sqrt(d2);
        tl = {tl.x / dist, tl.y / dist, tl.z / dist};
        float ct = dot(h.n, tl);
        float cl = -dot(ln, tl);
        if (ct > 0.0f && cl > 0.0f) {
            const orc_material& lm = s.mats[s.triMat[tri]];
            float pa = 1.0f / ((float)nE * la);
            float lpdf = pa * d2 / std::fmax(cl, 1e-8f);
            float bpdf = cosine_pdf(ct);
            float w = power_heuristic(lpdf, bpdf);
            V3f al = albedo_of(s, m, h.u, h.v);
            V3f f{al.x / kPiT<float>() * ct, al.y / kPiT<float>() * ct, al.z / kPiT<float>() * ct};
            V3f con{r.thr.x * f.x * lm.emission[0] * w / lpdf, r.thr.y * f.y * lm.emission[1] * w / lpdf,
                    r.thr.z * f.z * lm.emission[2] * w / lpdf};
            if (std::isfinite(con.x) && std::isfinite(con.y) && std::isfinite(con.z) && con.x >= 0.0f &&
                con.y >= 0.0f && con.z >= 0.0f) {
                r.shadowC = con;
                r.savedD = r.d;
                r.d = tl;
                r.o = offset_origin(h.pos, h.n, tl);
                r.tmin = 1e-5f;
                r.tmax = dist - 1e-5f;
                r.neeDone = 1;
                r.stage = kStageShadow;
                return;
            }
        }
    }
    r.neeDone = 0;
    V3f tg, bt;
    frame(h.n, tg, bt);
    float u1, u2, pdf;
    draw2(r, c.p->drawOrder, u1, u2);
    V3f loc = cosine_hemisphere(u1, u2, pdf);
    V3f wd = to_world(loc, h.n, tg, bt);
    V3f al = albedo_of(s, m, h.u, h.v);
    r.thr = r.thr * al;
    r.prevPdf = pdf;
    r.prevDelta = false;
    if (!apply_rr(c, r, false)) return;
    next_bounce(c, r, h, wd);
}

// glass.cuh:10-140 and ggx_transmission.cuh:12-107 (identical behaviour)
static void shade_dielectric(Ctx& c, Path& r, const Hit& h, const orc_material& m) {
    V3f wo = -r.d;
    float ci = dot(wo, h.n);
    float ei = 1.0f, et = m.ior;
    V3f n = h.n;
    if (ci < 0.0f) { ci = -ci; n = -n; ei = m.ior; et = 1.0f; }
    float F = fresnel_dielectric(ci, ei, et);
    float xi = rnd_dim(r.seed, r.dim++);
    V3f al = albedo_of(*c.s, m, h.u, h.v);
    if (xi < F) {
        r.d = r.d - n * (2.0f * dot(r.d, n));
        r.thr = {r.thr.x * al.x, r.thr.y * al.y, r.thr.z * al.z};
    } else {
        float eta = ei / et;
        float s2 = eta * eta * (1.0f - ci * ci);
        if (s2 >= 1.0f) {
            r.d = r.d - n * (2.0f * dot(r.d, n));
            r.thr = {r.thr.x * al.x, r.thr.y * al.y, r.thr.z * al.z};
        } else {
            float ct = std::sqrt(std::fmax(0.0f, 1.0f - s2));
            V3f rf = eta * r.d + n * (eta * ci - ct);
            r.d = rf;
            r.thr = {r.thr.x * al.x, r.thr.y * al.y, r.thr.z * al.z};
            float k = shading_correction(rf, h.n, h.ng);
            r.thr = {r.thr.x * k, r.thr.y * k, r.thr.z * k};
        }
    }
    r.prevDelta = true;
    if (!apply_rr(c, r, true)) return;
    next_bounce(c, r, h, r.d);
}

// ggx_material.cuh:10-213
static void shade_ggx(Ctx& c, Path& r, const Hit& h, const orc_material& m) {
    const Scene& s = *c.s;
    V3f wo = -r.d;
    V3f alb{m.albedo[0], m.albedo[1], m.albedo[2]};
    uint32_t nE = (uint32_t)s.emissive.size();
    if (c.p->useNEE && nE > 0) {
        float lu = rnd_dim(r.seed, r.dim++);
        uint32_t li = cdf_lower_bound(lu, s.cdf.data(), nE);
        uint32_t tri = s.emissive[li];
        V3f a, b, cc;
        light_vertices(s, tri, a, b, cc);
        float u1, u2;
        draw2(r, c.p->drawOrder, u1, u2);
        V3f ln;
        float la;
        V3f lp = sample_triangle(u1, u2, a, b, cc, ln, la);
        V3f tl{lp.x - h.pos.x, lp.y - h.pos.y, lp.z - h.pos.z};
        float d2 = dot(tl, tl);
        float dist = std::sqrt(d2);
        tl = {tl.x / dist, tl.y / dist, tl.z / dist};
        float ct = dot(h.n, tl);
        float cl = -dot(ln, tl);
        if (ct > 0.0f && cl > 0.0f) {
            const orc_material& lm = s.mats[s.triMat[tri]];
            float pa = 1.0f / ((float)nE * la);
            float lpdf = pa * d2 / std::fmax(cl, 1e-8f);
            V3f f = ggx_eval(wo, tl, h.n, alb, m.roughness, m.metallic, m.ior);
            float bpdf = ggx_pdf(wo, tl, h.n, m.roughness);
            float w = power_heuristic(lpdf, bpdf);
            V3f con{r.thr.x * f.x * lm.emission[0] * ct * w / lpdf, r.thr.y * f.y * lm.emission[1] * ct * w / lpdf,
                    r.thr.z * f.z * lm.emission[2] * ct * w / lpdf};
            if (std::isfinite(con.x) && std::isfinite(con.y) && std::isfinite(con.z) && con.x >= 0.0f &&
                con.y >= 0.0f && con.z >= 0.0f)
                r.rad = {r.rad.x + con.x, r.rad.y + con.y, r.rad.z + con.z};
        }
    }
    V3f tg, bt;
    frame(h.n, tg, bt);
    V3f wi{0, 0, 0};
    float pdf = 0.0f, u0, u1;
    draw2(r, c.p->drawOrder, u0, u1);
    ggx_sample(wo, h.n, tg, bt, m.roughness, u0, u1, wi, pdf);
    float ct = dot(h.n, wi);
    if (pdf < 1e-5f || ct <= 0.0f) { terminate(c, r); return; }
    V3f f = ggx_eval(wo, wi, h.n, alb, m.roughness, m.metallic, m.ior);
    if (!std::isfinite(f.x) || !std::isfinite(f.y) || !std::isfinite(f.z)) { terminate(c, r); return; }
    r.thr = {r.thr.x * f.x * ct / pdf, r.thr.y * f.y * ct / pdf, r.thr.z * f.z * ct / pdf};
    r.prevPdf = pdf;
    r.prevDelta = false;
    if (!apply_rr(c, r, false)) return;
    next_bounce(c, r, h, wi);
}

// Hit record and first-hit guides / emission (trace.cu:155-319).
static void closest_hit_program(Ctx& c, Path& r, float t, uint32_t prim, Hit& h) {
    const Scene& s = *c.s;
    V3f hp{r.o.x + t * r.d.x, r.o.y + t * r.d.y, r.o.z + t * r.d.z};
    uint32_t i0 = s.idx[3 * prim], i1 = s.idx[3 * prim + 1], i2 = s.idx[3 * prim + 2];
    V3f a = s.vert(i0), b = s.vert(i1), cc = s.vert(i2);
    V3f e1 = b - a, e2 = cc - a;
    V3f gn = normalize(cross(e1, e2));
    V3f vp = hp - a;
    float d00 = dot(e1, e1), d01 = dot(e1, e2), d11 = dot(e2, e2), d20 = dot(vp, e1), d21 = dot(vp, e2);
    float den = d00 * d11 - d01 * d01;
    float bv = (d11 * d20 - d01 * d21) / std::fmax(den, 1e-8f);
    float bw = (d00 * d21 - d01 * d20) / std::fmax(den, 1e-8f);
    float bu = 1.0f - bv - bw;
    V3f sn = gn;
    if (s.hasNormals) {
        V3f n0{s.nrm[3 * i0], s.nrm[3 * i0 + 1], s.nrm[3 * i0 + 2]};
        V3f n1{s.nrm[3 * i1], s.nrm[3 * i1 + 1], s.nrm[3 * i1 + 2]};
        V3f n2{s.nrm[3 * i2], s.nrm[3 * i2 + 1], s.nrm[3 * i2 + 2]};
        if (len(n0) > 1e-6f && len(n1) > 1e-6f && len(n2) > 1e-6f) {
            sn = normalize(bu * n0 + bv * n1 + bw * n2);
            if (dot(sn, gn) < 0.0f) sn = -sn;
        }
    }
    V3f ng = dot(gn, r.d) > 0.0f ? -gn : gn;
    V3f snf = dot(sn, r.d) > 0.0f ? -sn : sn;
    h.pos = hp;
    h.n = snf;
    h.ng = ng;
    h.mat = s.triMat[prim];
    h.prim = prim;
    if (s.hasUVs) {
        h.u = bu * s.uv[2 * i0] + bv * s.uv[2 * i1] + bw * s.uv[2 * i2];
        h.v = bu * s.uv[2 * i0 + 1] + bv * s.uv[2 * i1 + 1] + bw * s.uv[2 * i2 + 1];
    } else {
        h.u = h.v = 0.0f;
    }
    uint32_t nm = (uint32_t)s.mats.size();
    if (r.firstHit) {
        if (h.mat < nm) {
            V3f al = albedo_of(s, s.mats[h.mat], h.u, h.v);
            if (c.albedo) add3(c.albedo, r.pixel, al);
            if (c.normal) add3(c.normal, r.pixel, ng);
        }
        r.firstHit = false;
    }
    if (h.mat < nm) {
        const orc_material& m = s.mats[h.mat];
        if (m.type == kEmissive) {
            float w = 1.0f;
            uint32_t nE = (uint32_t)s.emissive.size();
            if (c.p->useNEE && r.depth > 0 && !r.prevDelta && nE > 0) {
                float area = 0.5f * len(cross(e1, e2));
                float d2 = t * t;
                float cl = std::fabs(dot(ng, r.d));
                float pa = 1.0f / ((float)nE * area);
                float lpdf = pa * d2 / std::fmax(cl, 1e-8f);
                w = power_heuristic(r.prevPdf, lpdf);
            }
            V3f em{m.emission[0], m.emission[1], m.emission[2]};
            r.rad = r.rad + r.thr * em * w;
        }
    }
}

// Normal-map perturbation of the shading normal (utils/normal_map.cuh:12-60).
static V3f normal_mapped(const Scene& s, const orc_material& m, const Hit& h) {
    if (m.normalTextureId > 0 && m.normalTextureId <= s.tex.size()) {
        const Tex& t = s.tex[m.normalTextureId - 1];
        float c[4] = {0.5f, 0.5f, 1.0f, 1.0f};
        if (!t.px.empty()) tex_fetch(t.px.data(), t.w, t.h, h.u, h.v, c);
        V3f tg, bt;
        frame(h.n, tg, bt);
        V3f q{c[0] * 2.0f - 1.0f, c[1] * 2.0f - 1.0f, c[2] * 2.0f - 1.0f};
        V3f w{tg.x * q.x + bt.x * q.y + h.n.x * q.z, tg.y * q.x + bt.y * q.y + h.n.y * q.z,
              tg.z * q.x + bt.z * q.y + h.n.z * q.z};
        return normalize(w);
    }
    return h.n;
}

// One path through at most maxIterations wavefront iterations (renderer.cpp:213);
// a path still alive afterwards is dropped without accumulating, as the host loop
// does when it exits.
static void run_path(Ctx& c, const CamBasis& cb, uint32_t pixel, uint32_t sample) {
    const Scene& s = *c.s;
    const orc_render_params& p = *c.p;
    Path r{};
    Hit h{};
    r.stage = kStageTrace;
    r.depth = 0;
    uint32_t iters = p.maxIterations ? p.maxIterations : 8;
    for (uint32_t it = 0; it < iters; ++it) {
        if (r.stage == kStageShadow) {
            float o[3] = {r.o.x, r.o.y, r.o.z}, d[3] = {r.d.x, r.d.y, r.d.z};
            c.shd++;
            if (!occluded32(s, o, d, r.tmin, r.tmax)) r.rad = r.rad + r.shadowC;
            r.d = r.savedD;
            r.stage = kStageShade;
        } else if (r.stage == kStageTrace) {
            if (r.depth == 0 && it == 0) {
                camera_ray(cb, p.width, p.height, pixel, sample, p.seed, r.o, r.d, r.seed);
                r.thr = {1, 1, 1};
                r.rad = {0, 0, 0};
                r.pixel = pixel;
                r.tmin = 0.0001f;
                r.tmax = 1e20f;
                r.firstHit = true;
                r.prevPdf = 1.0f;
                r.prevDelta = true;
                r.dim = 0;
                r.neeDone = 0;
            }
            float o[3] = {r.o.x, r.o.y, r.o.z}, d[3] = {r.d.x, r.d.y, r.d.z};
            float t;
            uint32_t prim;
            c.ext++;
            if (!closest32(s, o, d, r.tmin, r.tmax, t, prim)) {
                V3f env{s.env[0], s.env[1], s.env[2]};
                r.rad = r.rad + r.thr * env;
                terminate(c, r);
                return;
            }
            closest_hit_program(c, r, t, prim, h);
            r.stage = kStageShade;
        }
        if (r.stage == kStageShade) {
            if (h.mat >= s.mats.size()) return;  // shade.cu:35-38: terminated, nothing accumulated
            const orc_material& m = s.mats[h.mat];
            Hit eh = h;
            if (m.normalTextureId > 0) eh.n = normal_mapped(s, m, h);
            switch (m.type) {
                case kEmissive: terminate(c, r); break;
                case kLambert: shade_lambert(c, r, eh, m); break;
                case kGlass:
                case kGGXT: shade_dielectric(c, r, eh, m); break;
                case kGGX: shade_ggx(c, r, eh, m); break;
                default: terminate(c, r); break;
            }
        }
        if (r.stage == kStageDone) return;
    }
}

}  // namespace orc

using namespace orc;

template <class T>
static void bsdf_one(const float* in, double* out) {
    V3<T> wo{T(in[0]), T(in[1]), T(in[2])}, wi{T(in[3]), T(in[4]), T(in[5])}, n{T(in[6]), T(in[7]), T(in[8])};
    V3<T> al{T(in[9]), T(in[10]), T(in[11])};
    T rough = T(in[12]), metal = T(in[13]), ior = T(in[14]), u0 = T(in[15]), u1 = T(in[16]), u2 = T(in[17]);
    uint32_t depth = (uint32_t)in[18];
    float rr = in[19];
    V3<T> e = ggx_eval(wo, wi, n, al, rough, metal, ior);
    out[0] = e.x; out[1] = e.y; out[2] = e.z;
    T gp = ggx_pdf(wo, wi, n, rough);
    out[3] = gp;
    V3<T> tg, bt;
    frame(n, tg, bt);
    V3<T> sw{0, 0, 0};
    T sp = 0;
    ggx_sample(wo, n, tg, bt, rough, u0, u1, sw, sp);
    bool ok = sp > T(0) || sp != sp;
    if (!ok) sw = {0, 0, 0};
    out[4] = sw.x; out[5] = sw.y; out[6] = sw.z; out[7] = sp; out[8] = ok ? 1.0 : 0.0;
    out[9] = fresnel_dielectric(std::fabs(dot(wo, n)), T(1), ior);
    T cp;
    V3<T> ch = cosine_hemisphere(u0, u1, cp);
    out[10] = ch.x; out[11] = ch.y; out[12] = ch.z; out[13] = cp;
    T cpdf = cosine_pdf(dot(n, wi));
    out[14] = power_heuristic(gp, cpdf);
    out[15] = cpdf;
    V3<T> nt{0, 0, 0};
    bool sv = russian_roulette(al, depth, rr, u2, nt, metal > T(0.5f));
    out[16] = sv ? 1.0 : 0.0;
    out[17] = nt.x; out[18] = nt.y; out[19] = nt.z;
    out[20] = tg.x; out[21] = tg.y; out[22] = tg.z; out[23] = bt.x; out[24] = bt.y; out[25] = bt.z;
    V3<T> ln;
    T la;
    V3<T> pp = sample_triangle(u0, u1, wo, wi, n, ln, la);
    out[26] = pp.x; out[27] = pp.y; out[28] = pp.z; out[29] = la; out[30] = ln.x; out[31] = ln.y; out[32] = ln.z;
    out[33] = shading_correction(wi, n, normalize(wo));
}


extern "C" {

void* orc_scene_create(const orc_scene_desc* d) { return scene_from_desc(d); }

void orc_scene_destroy(void* s) { delete (Scene*)s; }
uint32_t orc_scene_num_emissive(void* s) { return (uint32_t)((Scene*)s)->emissive.size(); }
void orc_scene_light_cdf(void* sp, uint32_t* tris, float* cdf) {
    Scene* s = (Scene*)sp;
    for (size_t i = 0; i < s->emissive.size(); ++i) { tris[i] = s->emissive[i]; cdf[i] = s->cdf[i]; }
}

void orc_render(void* sp, const orc_camera* cam, const orc_render_params* p, float* rgb, float* albedo,
                float* normal, int threads, orc_stats* stats) {
    const Scene* s = (const Scene*)sp;
    uint32_t np = p->width * p->height;
    uint32_t pb = p->pixelBegin, pe = p->pixelEnd ? p->pixelEnd : np;
    std::vector<float> accum(3 * (size_t)np, 0.0f);
    if (albedo) std::memset(albedo, 0, sizeof(float) * 3 * (size_t)np);
    if (normal) std::memset(normal, 0, sizeof(float) * 3 * (size_t)np);
    CamBasis cb = cam_basis(*cam);
    uint64_t ext = 0, shd = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel reduction(+ : ext, shd)
#endif
    {
        Ctx c{s, p, accum.data(), albedo, normal};
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
        for (int64_t px = pb; px < (int64_t)pe; ++px)
            for (uint32_t k = 0; k < p->spp; ++k) run_path(c, cb, (uint32_t)px, p->sampleBegin + k);
        ext += c.ext;
        shd += c.shd;
    }
    float inv = 1.0f / (float)p->spp;
    if (rgb)
        for (size_t i = 0; i < 3 * (size_t)np; ++i) rgb[i] = accum[i] * inv;
    if (stats) {
        stats->extensionRays = ext;
        stats->shadowRays = shd;
        stats->paths = (uint64_t)(pe - pb) * p->spp;
    }
}

void orc_closest(void* sp, const float* rays, uint32_t n, int mode, float* out_t, uint32_t* out_prim,
                 int threads) {
    const Scene* s = (const Scene*)sp;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 256)
#endif
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const float* r = rays + 8 * i;
        float o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
        if (mode == 0) {
            float t;
            uint32_t p;
            closest32(*s, o, d, r[3], r[7], t, p);
            out_t[i] = (p == 0xffffffffu) ? INFINITY : t;
            out_prim[i] = p;
        } else if (mode == 2) {
            double od[3] = {o[0], o[1], o[2]}, dd[3] = {d[0], d[1], d[2]};
            double t;
            uint32_t p;
            closest64(*s, od, dd, r[3], r[7], t, p);
            out_t[i] = (p == 0xffffffffu) ? INFINITY : (float)t;
            out_prim[i] = p;
        } else {
            double od[3] = {o[0], o[1], o[2]}, dd[3] = {d[0], d[1], d[2]};
            double tb = r[7];
            uint32_t pb = 0xffffffffu;
            for (uint32_t t = 0; t < s->nt; ++t) {
                V3f a = s->vert(s->idx[3 * t]), b = s->vert(s->idx[3 * t + 1]), c = s->vert(s->idx[3 * t + 2]);
                double v0[3] = {a.x, a.y, a.z};
                double e1[3] = {(double)b.x - a.x, (double)b.y - a.y, (double)b.z - a.z};
                double e2[3] = {(double)c.x - a.x, (double)c.y - a.y, (double)c.z - a.z};
                double th;
                if (mt64(od, dd, v0, e1, e2, th) && th >= r[3] && th <= r[7] && (th < tb || (th == tb && t < pb))) {
                    tb = th;
                    pb = t;
                }
            }
            out_t[i] = (pb == 0xffffffffu) ? INFINITY : (float)tb;
            out_prim[i] = pb;
        }
    }
}

void orc_occluded(void* sp, const float* rays, uint32_t n, uint32_t* out, int threads) {
    const Scene* s = (const Scene*)sp;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 256)
#endif
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const float* r = rays + 8 * i;
        float o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
        out[i] = occluded32(*s, o, d, r[3], r[7]) ? 1u : 0u;
    }
}

void orc_camera_rays(const orc_camera* cam, uint32_t w, uint32_t h, const uint32_t* pixels, const uint32_t* samples,
                     uint32_t n, uint32_t seed, float* out) {
    CamBasis cb = cam_basis(*cam);
    for (uint32_t i = 0; i < n; ++i) {
        V3f o, d;
        uint32_t sd;
        camera_ray(cb, w, h, pixels[i], samples[i], seed, o, d, sd);
        float* q = out + 8 * (size_t)i;
        q[0] = o.x; q[1] = o.y; q[2] = o.z; q[3] = 0.0001f;
        q[4] = d.x; q[5] = d.y; q[6] = d.z; q[7] = 1e20f;
    }
}

// BSDF batch.  Input record (20 floats): wo[3] wi[3] n[3] albedo[3] rough metal ior
// u0 u1 u2 depth rrStart.  Output record (34 doubles):
//  0-2 ggx_eval  3 ggx_pdf  4-6 ggx_sample wi  7 ggx_sample pdf  8 ggx_sample ok
//  9 fresnel_dielectric(|wo.n|, 1, ior)  10-12 cosine_hemisphere(u0,u1)  13 its pdf
//  14 power_heuristic(ggx_pdf, cosine_pdf(n.wi))  15 cosine_pdf(n.wi)
//  16 RR survive (xi=u2, thr=albedo, delta = metal>0.5)  17-19 RR throughput
//  20-22 frame tangent(n)  23-25 bitangent  26-28 sample_triangle(u0,u1; wo,wi,n)
//  29 its area  30-32 its normal  33 shading_correction(wi, n, normalize(wo))
void orc_bsdf_batch(const float* in, uint32_t n, int prec, double* out) {
    cr_elementary() = prec == 2;
    for (uint32_t i = 0; i < n; ++i) {
        if (prec == 0 || prec == 2) bsdf_one<float>(in + 20 * (size_t)i, out + 34 * (size_t)i);
        else bsdf_one<double>(in + 20 * (size_t)i, out + 34 * (size_t)i);
    }
    cr_elementary() = 0;
}

void orc_rng_batch(const uint32_t* seeds, const uint32_t* dims, uint32_t n, uint32_t* hash, float* u) {
    for (uint32_t i = 0; i < n; ++i) {
        hash[i] = pcg_hash_dim(seeds[i], dims[i]);
        u[i] = rnd_dim(seeds[i], dims[i]);
    }
}

void orc_cdf_batch(const float* cdf, uint32_t ncdf, const float* u, uint32_t n, uint32_t* out) {
    for (uint32_t i = 0; i < n; ++i) out[i] = cdf_lower_bound(u[i], cdf, ncdf);
}

void orc_tonemap(const float* rgb, uint32_t npix, uint8_t* out) {
    for (size_t i = 0; i < 3 * (size_t)npix; ++i) out[i] = aces_byte(rgb[i]);
}

void orc_texture_batch(const orc_texture* t, const float* uv, uint32_t n, float* out) {
    for (uint32_t i = 0; i < n; ++i) tex_fetch(t->rgba, t->width, t->height, uv[2 * i], uv[2 * i + 1], out + 4 * (size_t)i);
}

uint32_t orc_compact(const uint32_t* stage, const uint32_t* idx, uint32_t n, uint32_t* out) {
    uint32_t c = 0;
    for (uint32_t i = 0; i < n; ++i)
        if (stage[idx[i]] != kStageDone) out[c++] = idx[i];
    return c;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Independent CPU reader of the library's 8-wide BVH format (test infrastructure):
// decodes the exported nodes / leaf triangles and traverses them to count node
// visits and triangle tests per ray, and returns the closest hit for comparison.
namespace {
struct Node8 {
    float p[3];
    int e[3];
    uint32_t imask, childBase, triBase;
    uint8_t meta[8], qlo[3][8], qhi[3][8];
};
Node8 decode8(const uint32_t* w) {
    Node8 n;
    for (int k = 0; k < 3; ++k) std::memcpy(&n.p[k], &w[k], 4);
    for (int k = 0; k < 3; ++k) n.e[k] = (int)((w[3] >> (8 * k)) & 0xff) - 127;
    n.imask = w[3] >> 24;
    n.childBase = w[4];
    n.triBase = w[5];
    for (int s = 0; s < 8; ++s) n.meta[s] = (uint8_t)(w[6 + s / 4] >> (8 * (s % 4)));
    const uint32_t* q = w + 8;  // qlox(2) qloy(2) qloz(2) qhix(2) qhiy(2) qhiz(2)
    for (int a = 0; a < 3; ++a)
        for (int s = 0; s < 8; ++s) {
            n.qlo[a][s] = (uint8_t)(q[2 * a + s / 4] >> (8 * (s % 4)));
            n.qhi[a][s] = (uint8_t)(q[6 + 2 * a + s / 4] >> (8 * (s % 4)));
        }
    return n;
}
}  // namespace

extern "C" {

// Checks structural invariants; returns 0 if all hold, else a code (1 bad index,
// 2 triangle outside its child box, 3 triangle referenced not exactly once).
// out[0] = max depth, out[1] = internal child slots, out[2] = leaf child slots.
int orc_bvh8_validate(const uint32_t* nodes, uint32_t nn, const float* tris, uint32_t nt, uint32_t* out) {
    std::vector<uint32_t> seen(nt, 0);
    std::vector<std::pair<uint32_t, uint32_t>> stack{{0, 1}};
    uint32_t maxd = 0, ni = 0, nl = 0;
    while (!stack.empty()) {
        auto [idx, depth] = stack.back();
        stack.pop_back();
        if (idx >= nn) return 1;
        maxd = std::max(maxd, depth);
        Node8 n = decode8(nodes + 20 * (size_t)idx);
        uint32_t rank = 0;
        for (int s = 0; s < 8; ++s) {
            bool empty = n.qlo[0][s] > n.qhi[0][s];
            if (empty) continue;
            double lo[3], hi[3];
            for (int a = 0; a < 3; ++a) {
                double sc = std::ldexp(1.0, n.e[a]);
                lo[a] = n.p[a] + n.qlo[a][s] * sc;
                hi[a] = n.p[a] + n.qhi[a][s] * sc;
            }
            if ((n.imask >> s) & 1u) {
                stack.push_back({n.childBase + rank, depth + 1});
                ++rank;
                ++ni;
            } else {
                ++nl;
                uint32_t cnt = (n.meta[s] >> 5) + 1, off = n.meta[s] & 31;
                for (uint32_t k = 0; k < cnt; ++k) {
                    uint32_t ti = n.triBase + off + k;
                    if (ti >= nt) return 1;
                    const float* t = tris + 12 * (size_t)ti;
                    uint32_t prim;
                    std::memcpy(&prim, &t[3], 4);
                    if (prim >= nt) return 1;
                    seen[prim]++;
                    double v[3][3];
                    for (int a = 0; a < 3; ++a) {
                        v[0][a] = t[a];
                        v[1][a] = (double)t[a] + t[4 + a];
                        v[2][a] = (double)t[a] + t[8 + a];
                    }
                    for (int j = 0; j < 3; ++j)
                        for (int a = 0; a < 3; ++a)
                            if (v[j][a] < lo[a] - 1e-6 * (1 + std::fabs(lo[a])) ||
                                v[j][a] > hi[a] + 1e-6 * (1 + std::fabs(hi[a])))
                                return 2;
                }
            }
        }
    }
    for (uint32_t c : seen)
        if (c != 1) return 3;
    out[0] = maxd;
    out[1] = ni;
    out[2] = nl;
    return 0;
}

// Closest hit through the exported BVH (same traversal order as the GPU) with
// per-ray node-visit and triangle-test counts.
void orc_bvh8_trace(const uint32_t* nodes, uint32_t nn, const float* tris, uint32_t nt, const float* rays, uint32_t n,
                    float* out_t, uint32_t* out_prim, uint32_t* visits, uint32_t* tests) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 256)
#endif
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const float* r = rays + 8 * i;
        float o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
        float inv[3] = {1.0f / d[0], 1.0f / d[1], 1.0f / d[2]};
        uint32_t octinv = ((d[0] < 0) | ((d[1] < 0) << 1) | ((d[2] < 0) << 2)) ^ 7u;
        float tb = r[7];
        uint32_t pb = 0xffffffffu, nv = 0, ntst = 0;
        std::vector<uint32_t> stack{0};
        while (!stack.empty()) {
            uint32_t idx = stack.back();
            stack.pop_back();
            if (idx >= nn) break;
            ++nv;
            Node8 nd = decode8(nodes + 20 * (size_t)idx);
            struct Hit { uint32_t key, slot; };
            std::vector<Hit> hits;
            uint32_t rank = 0;
            uint32_t ranks[8];
            for (int s = 0; s < 8; ++s) { ranks[s] = rank; if ((nd.imask >> s) & 1u) ++rank; }
            for (int s = 0; s < 8; ++s) {
                if (nd.qlo[0][s] > nd.qhi[0][s]) continue;
                float t0 = r[3], t1 = tb * 1.0000005f;
                for (int a = 0; a < 3; ++a) {
                    double sc = std::ldexp(1.0, nd.e[a]);
                    float lo = (float)(nd.p[a] + nd.qlo[a][s] * sc), hi = (float)(nd.p[a] + nd.qhi[a][s] * sc);
                    float x = (lo - o[a]) * inv[a], y = (hi - o[a]) * inv[a];
                    float mn = std::min(x, y), mx = std::max(x, y);
                    if (mn != mn) mn = -INFINITY;
                    if (mx != mx) mx = INFINITY;
                    t0 = std::max(t0, mn);
                    t1 = std::min(t1, mx * 1.0000005f);
                }
                if (t0 > t1) continue;
                if ((nd.imask >> s) & 1u) {
                    hits.push_back({(uint32_t)s ^ octinv, nd.childBase + ranks[s]});
                } else {
                    uint32_t cnt = (nd.meta[s] >> 5) + 1, off = nd.meta[s] & 31;
                    for (uint32_t k = 0; k < cnt; ++k) {
                        const float* t = tris + 12 * (size_t)(nd.triBase + off + k);
                        float th;
                        ++ntst;
                        if (mt32(o, d, t, t + 4, t + 8, th) && th >= r[3] && th <= r[7]) {
                            uint32_t prim;
                            std::memcpy(&prim, &t[3], 4);
                            if (th < tb || (th == tb && prim < pb)) { tb = th; pb = prim; }
                        }
                    }
                }
            }
            std::sort(hits.begin(), hits.end(), [](const Hit& a, const Hit& b) { return a.key > b.key; });
            for (auto& h : hits) stack.push_back(h.slot);  // lowest key popped first
        }
        out_t[i] = pb == 0xffffffffu ? INFINITY : tb;
        out_prim[i] = pb;
        visits[i] = nv;
        tests[i] = ntst;
    }
}

}  // extern "C"
