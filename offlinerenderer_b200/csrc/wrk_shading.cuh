// Device shading / sampling / RNG math for the wavefront renderer.
//
// Restates the formulas of libWR's kernels (paths inside trianglestrip/
// OfflineRenderer): vector_math.cuh, sampling.cuh, ggx.cuh, utils/fresnel.cuh,
// utils/ray_offset.cuh, materials/material_common.cuh.  The expression order
// follows the reference's so that, built with --fmad=false, every FP32 result
// rounds the way the reference's arithmetic does; normalize() uses the correctly
// rounded __frsqrt_rn in place of the approximate rsqrtf.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace wrk {

// float pi: sampling.cuh:6-8 / material_common.cuh:9 (both the same float).
constexpr float kPi = 3.14159265358979323846f;

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 neg(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 mul(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 mul(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 mul(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length(float3 v) { return sqrtf(dot(v, v)); }
__device__ __forceinline__ float3 normalize(float3 v) { return mul(v, __frsqrt_rn(dot(v, v))); }
__device__ __forceinline__ bool finite3(float3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

// ---- RNG (sampling.cuh:17-38, utils/atomic_ops.cuh:16-19) ----
__device__ __forceinline__ uint32_t pcg_hash(uint32_t s) {
    uint32_t st = s * 747796405u + 2891336453u;
    uint32_t w = ((st >> ((st >> 28u) + 4u)) ^ st) * 277803737u;
    return (w >> 22u) ^ w;
}
__device__ __forceinline__ uint32_t pcg_hash_dim(uint32_t s, uint32_t d) {
    uint32_t st = s * 747796405u + 2891336453u + d * 1013904223u;
    uint32_t w = ((st >> ((st >> 28u) + 4u)) ^ st) * 277803737u;
    return (w >> 22u) ^ w;
}
__device__ __forceinline__ float rnd_dim(uint32_t s, uint32_t d) { return float(pcg_hash_dim(s, d)) / 4294967296.0f; }
__device__ __forceinline__ float lcg_randf(uint32_t& s) {
    s = s * 1664525u + 1013904223u;
    return (float)(s >> 8) / 16777216.0f;
}
// Per-path seed keyed by (pixel, sample): trace.cu:58 with slot == pixel.
__device__ __forceinline__ uint32_t path_seed(uint32_t pixel, uint32_t sample, uint32_t user_seed) {
    uint32_t s = (pixel * 1664525u + sample * 1013904223u) ^ 0x9e3779b9u;
    if (user_seed != 0u) s ^= pcg_hash(user_seed);
    return s;
}

// ---- frames and warps (sampling.cuh:44-110) ----
__device__ __forceinline__ void frame(float3 n, float3& t, float3& b) {
    float3 up = fabsf(n.y) < 0.999f ? f3(0, 1, 0) : f3(1, 0, 0);
    t = normalize(cross(up, n));
    b = cross(n, t);
}
__device__ __forceinline__ float3 to_world(float3 v, float3 n, float3 t, float3 b) {
    return f3(t.x * v.x + b.x * v.y + n.x * v.z, t.y * v.x + b.y * v.y + n.y * v.z, t.z * v.x + b.z * v.y + n.z * v.z);
}
// sin / cos / pow of the sampling and Fresnel formulas, correctly rounded: computed
// in double precision and rounded once to float.  The sampled directions and the
// VNDF pdf are sensitive to the last bit of these values (the GGX D term near its
// peak multiplies an error of the half-vector by ~1/a^2), so the device rounds them
// the one reproducible way; the oracle's matching mode does the same on the host.
__device__ __forceinline__ void sincos_cr(float x, float& s, float& c) {
    double sd, cd;
    sincos((double)x, &sd, &cd);
    s = (float)sd;
    c = (float)cd;
}
// x^5 (the Schlick Fresnel power) in double: x^2 is exact, x^4 and x^5 carry one
// double rounding each, so the float rounding is the correctly rounded x^5 except
// when x^5 lies within ~2^-52 (relative) of a float rounding boundary.
__device__ __forceinline__ float pow5_cr(float x) {
    const double x2 = (double)x * (double)x;
    return (float)(x2 * x2 * (double)x);
}
__device__ __forceinline__ float3 cosine_hemisphere(float u1, float u2, float& pdf) {
    float r = sqrtf(u1);
    float th = 2.0f * kPi * u2;
    float z = sqrtf(fmaxf(0.0f, 1.0f - u1));
    pdf = z / kPi;
    float sn, cs;
    sincos_cr(th, sn, cs);
    return f3(r * cs, r * sn, z);
}
__device__ __forceinline__ float cosine_pdf(float c) { return fmaxf(0.0f, c / kPi); }
__device__ __forceinline__ float3 sample_triangle(float u1, float u2, float3 a, float3 b, float3 c, float3& nrm,
                                                  float& area) {
    float su = sqrtf(u1);
    float b0 = 1.0f - su, b1 = su * (1.0f - u2), b2 = su * u2;
    float3 p = f3(a.x * b0 + b.x * b1 + c.x * b2, a.y * b0 + b.y * b1 + c.y * b2, a.z * b0 + b.z * b1 + c.z * b2);
    float3 cr = cross(sub(b, a), sub(c, a));
    area = 0.5f * length(cr);
    nrm = normalize(cr);
    return p;
}
// Lower bound of u in the light CDF (sampling.cuh:116-135); integer result.
__device__ __forceinline__ uint32_t cdf_lower_bound(float u, const float* __restrict__ cdf, uint32_t n) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t m = (lo + hi) >> 1;
        if (__ldg(cdf + m) < u) lo = m + 1; else hi = m;
    }
    return min(lo, n - 1);
}
__device__ __forceinline__ float power_heuristic(float a, float b) {
    float a2 = a * a, b2 = b * b;
    return a2 / (a2 + b2);
}
// sampling.cuh:162-193
__device__ __forceinline__ bool russian_roulette(float3 thr, uint32_t depth, float rr_start, float xi, float3& out,
                                                 bool delta) {
    if ((float)depth < rr_start) { out = thr; return true; }
    float lum = 0.2126f * thr.x + 0.7152f * thr.y + 0.0722f * thr.z;
    float df = 1.0f / (1.0f + 0.1f * ((float)depth - rr_start));
    float q = fmaxf(delta ? 0.5f : 0.05f, fminf(0.95f, lum * df));
    if (xi < q) { out = f3(thr.x / q, thr.y / q, thr.z / q); return true; }
    return false;
}
__device__ __forceinline__ float3 clamp_fireflies(float3 r, float maxl) {
    if (maxl <= 0.0f) return r;
    float lum = 0.2126f * r.x + 0.7152f * r.y + 0.0722f * r.z;
    if (lum > maxl) { float s = maxl / lum; return f3(r.x * s, r.y * s, r.z * s); }
    return r;
}

// ---- dielectric Fresnel, shading correction, ray offset ----
__device__ __forceinline__ float fresnel_dielectric(float ci, float ei, float et) {
    float s2 = ei / et * ei / et * (1.0f - ci * ci);
    if (s2 > 1.0f) return 1.0f;
    float ct = sqrtf(1.0f - s2);
    float rs = (ei * ci - et * ct) / (ei * ci + et * ct);
    float rp = (et * ci - ei * ct) / (et * ci + ei * ct);
    return (rs * rs + rp * rp) * 0.5f;
}
__device__ __forceinline__ float shading_correction(float3 wi, float3 ns, float3 ng) {
    float cs = fabsf(dot(wi, ns)), cg = fabsf(dot(wi, ng));
    if (cs < 1e-6f || cg < 1e-6f) return 1.0f;
    return cg / cs;
}
__device__ __forceinline__ float3 offset_origin(float3 p, float3 n, float3 d) {
    float3 od = dot(d, n) > 0.0f ? n : neg(n);
    const float e = 1e-4f;
    return f3(p.x + od.x * e, p.y + od.y * e, p.z + od.z * e);
}

// ---- GGX (ggx.cuh:18-63, 113-317) ----
__device__ __forceinline__ float ggx_D(float noh, float a) {
    float a2 = a * a, c2 = noh * noh;
    float den = c2 * (a2 - 1.0f) + 1.0f;
    return a2 / (kPi * den * den);
}
__device__ __forceinline__ float ggx_G1(float nov, float a) {
    float a2 = a * a, c2 = nov * nov;
    return 2.0f * nov / (nov + sqrtf(a2 + (1.0f - a2) * c2));
}
__device__ __forceinline__ float3 ggx_eval(float3 wo, float3 wi, float3 n, float3 alb, float rough, float metal,
                                           float ior) {
    float nov = fmaxf(0.0f, dot(n, wo)), nol = fmaxf(0.0f, dot(n, wi));
    if (nov < 1e-5f || nol < 1e-5f) return f3(0, 0, 0);
    float3 h = normalize(f3(wo.x + wi.x, wo.y + wi.y, wo.z + wi.z));
    float noh = fmaxf(0.0f, dot(n, h)), voh = fmaxf(0.0f, dot(wo, h));
    float a = rough * rough;
    float D = ggx_D(noh, a);
    float G = ggx_G1(nov, a) * ggx_G1(nol, a);
    float f0 = (ior - 1.0f) / (ior + 1.0f);
    f0 = f0 * f0;
    float3 F0 = f3(f0 * (1.0f - metal) + alb.x * metal, f0 * (1.0f - metal) + alb.y * metal,
                   f0 * (1.0f - metal) + alb.z * metal);
    float fw = pow5_cr(1.0f - voh);
    float3 F = f3(F0.x + (1.0f - F0.x) * fw, F0.y + (1.0f - F0.y) * fw, F0.z + (1.0f - F0.z) * fw);
    float den = 4.0f * nov * nol;
    float3 spec = f3(D * G * F.x / den, D * G * F.y / den, D * G * F.z / den);
    float3 kd = f3((1.0f - F.x) * (1.0f - metal), (1.0f - F.y) * (1.0f - metal), (1.0f - F.z) * (1.0f - metal));
    float3 diff = f3(kd.x * alb.x / kPi, kd.y * alb.y / kPi, kd.z * alb.z / kPi);
    return f3(diff.x + spec.x, diff.y + spec.y, diff.z + spec.z);
}
__device__ __forceinline__ float ggx_pdf(float3 wo, float3 wi, float3 n, float rough) {
    float nov = fmaxf(0.0f, dot(n, wo)), nol = fmaxf(0.0f, dot(n, wi));
    if (nov < 1e-5f || nol < 1e-5f) return 0.0f;
    float3 h = normalize(f3(wo.x + wi.x, wo.y + wi.y, wo.z + wi.z));
    float noh = fmaxf(0.0f, dot(n, h)), voh = fmaxf(0.0f, dot(wo, h));
    if (voh < 1e-5f) return 0.0f;
    float a = rough * rough;
    return ggx_G1(nov, a) * ggx_D(noh, a) / (4.0f * nov);
}
// Visible-normal sampling; pdf = 0 on failure (wi then untouched / below the surface).
__device__ __forceinline__ void ggx_sample(float3 wo, float3 n, float3 tg, float3 bt, float rough, float u0,
                                           float u1, float3& wi, float& pdf) {
    float a = rough * rough;
    float3 v = f3(dot(wo, tg), dot(wo, bt), dot(wo, n));
    float3 sv = normalize(f3(a * v.x, a * v.y, v.z));
    float d2 = sqrtf(sv.x * sv.x + sv.y * sv.y);
    float3 t1, t2;
    if (d2 > 1e-6f) {
        float r = 1.0f / d2;
        t1 = f3(sv.y * r, -sv.x * r, 0.0f);
        t2 = f3(t1.y * sv.z, -t1.x * sv.z, d2);
    } else {
        t1 = f3(1, 0, 0);
        t2 = f3(0, 1, 0);
    }
    float ia = 1.0f / (1.0f + sv.z);
    float r = sqrtf(u0);
    bool lower = u1 < ia;
    float phi = kPi * (lower ? u1 / ia : 1.0f + (u1 - ia) / (1.0f - ia));
    float sp, cp;
    sincos_cr(phi, sp, cp);
    float p1 = r * cp;
    float p2 = r * sp * (lower ? 1.0f : sv.z);
    float sq = sqrtf(fmaxf(0.0f, 1.0f - (p1 * p1 + p2 * p2)));
    float3 m = f3(p1 * t1.x + p2 * t2.x + sq * sv.x, p1 * t1.y + p2 * t2.y + sq * sv.y, p1 * t1.z + p2 * t2.z + sq * sv.z);
    m = normalize(f3(a * m.x, a * m.y, m.z));
    float3 h = f3(tg.x * m.x + bt.x * m.y + n.x * m.z, tg.y * m.x + bt.y * m.y + n.y * m.z,
                  tg.z * m.x + bt.z * m.y + n.z * m.z);
    float voh = dot(wo, h);
    if (voh <= 0.0f) { pdf = 0.0f; return; }
    wi = f3(2.0f * voh * h.x - wo.x, 2.0f * voh * h.y - wo.y, 2.0f * voh * h.z - wo.z);
    if (dot(n, wi) <= 0.0f) { pdf = 0.0f; return; }
    float nov = fmaxf(0.0f, dot(n, wo)), noh = fmaxf(0.0f, dot(n, h));
    pdf = ggx_G1(nov, a) * ggx_D(noh, a) / (4.0f * nov);
}

// ---- texture: RGBA8, wrap, bilinear with 8-bit weight fractions, normalized float ----
__device__ __forceinline__ float4 tex_fetch(const uint8_t* __restrict__ px, uint32_t w, uint32_t h, float u, float v) {
    float uw = u - floorf(u), vw = v - floorf(v);
    float x = uw * (float)w - 0.5f, y = vw * (float)h - 0.5f;
    float fx = floorf(x), fy = floorf(y);
    float ax = rintf((x - fx) * 256.0f) * (1.0f / 256.0f);
    float ay = rintf((y - fy) * 256.0f) * (1.0f / 256.0f);
    int ix = (int)fx, iy = (int)fy;
    int x0 = ((ix % (int)w) + (int)w) % (int)w, y0 = ((iy % (int)h) + (int)h) % (int)h;
    int x1 = (x0 + 1) % (int)w, y1 = (y0 + 1) % (int)h;
    uchar4 t00 = __ldg(reinterpret_cast<const uchar4*>(px) + (size_t)y0 * w + x0);
    uchar4 t10 = __ldg(reinterpret_cast<const uchar4*>(px) + (size_t)y0 * w + x1);
    uchar4 t01 = __ldg(reinterpret_cast<const uchar4*>(px) + (size_t)y1 * w + x0);
    uchar4 t11 = __ldg(reinterpret_cast<const uchar4*>(px) + (size_t)y1 * w + x1);
    float bx = 1.0f - ax, by = 1.0f - ay;
    float4 o;
#define WRK_LERP(c)                                                                                        \
    ((float)t00.c / 255.0f * bx + (float)t10.c / 255.0f * ax) * by +                                      \
        ((float)t01.c / 255.0f * bx + (float)t11.c / 255.0f * ax) * ay
    o.x = WRK_LERP(x);
    o.y = WRK_LERP(y);
    o.z = WRK_LERP(z);
    o.w = WRK_LERP(w);
#undef WRK_LERP
    return o;
}

// ---- environment map: directionToUV + a float4 texture with linear filtering,
//      normalized coordinates, wrap in u and clamp in v
//      (libWR/kernels/utils/environment_sampling.cuh:10-52, scene.cpp:325-331) ----
__device__ __forceinline__ float3 env_lookup(const float4* __restrict__ map, uint32_t w, uint32_t h, float3 d) {
    d = normalize(d);
    float phi = atan2f(d.z, d.x);
    float theta = acosf(fmaxf(-1.0f, fminf(1.0f, d.y)));
    float u = (phi + 3.14159265f) / (2.0f * 3.14159265f);
    float v = theta / 3.14159265f;
    float x = (u - floorf(u)) * (float)w - 0.5f;
    float y = fminf(fmaxf(v, 0.0f), 1.0f) * (float)h - 0.5f;
    float fx = floorf(x), fy = floorf(y);
    float ax = rintf((x - fx) * 256.0f) * (1.0f / 256.0f), ay = rintf((y - fy) * 256.0f) * (1.0f / 256.0f);
    int ix = (int)fx, iy = (int)fy;
    int x0 = ((ix % (int)w) + (int)w) % (int)w, x1 = (x0 + 1) % (int)w;
    int y0 = min(max(iy, 0), (int)h - 1), y1 = min(max(iy + 1, 0), (int)h - 1);
    float4 t00 = __ldg(map + (size_t)y0 * w + x0), t10 = __ldg(map + (size_t)y0 * w + x1);
    float4 t01 = __ldg(map + (size_t)y1 * w + x0), t11 = __ldg(map + (size_t)y1 * w + x1);
    float bx = 1.0f - ax, by = 1.0f - ay;
    return f3((t00.x * bx + t10.x * ax) * by + (t01.x * bx + t11.x * ax) * ay,
              (t00.y * bx + t10.y * ax) * by + (t01.y * bx + t11.y * ax) * ay,
              (t00.z * bx + t10.z * ax) * by + (t01.z * bx + t11.z * ax) * ay);
}

// ---- ACES filmic + gamma (libWR/test/helpers/image.cpp:14-49) ----
__device__ __forceinline__ uint8_t aces_byte(float lin) {
    float x = lin * 2.2f;
    float v = (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
    v = fminf(fmaxf(v, 0.0f), 1.0f);
    if (v != v) v = 0.0f;
    // pow in double, rounded once to float: equals the correctly rounded powf.
    float g = 1.0f / 2.2f;
    float p = (float)pow((double)v, (double)g);
    return (uint8_t)(p * 255.0f);
}

}  // namespace wrk
