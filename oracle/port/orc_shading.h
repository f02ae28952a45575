// CPU oracle -- test infrastructure only. Nothing in the product links this file.
//
// Restatement, in plain C++, of libWR's shading / sampling / RNG formulas so that
// the CUDA renderer can be checked against it.  Every function is a template over
// the scalar type T: instantiated with float it reproduces the reference's FP32
// arithmetic operation for operation (same operand order, no FMA contraction --
// build with -ffp-contract=off); instantiated with double it is the FP64
// transcription used for the 1e-5 relative per-kernel checks.
//
// Reference files cited below are paths inside trianglestrip/OfflineRenderer.
#pragma once
#include <cmath>
#include <cstdint>
#include <algorithm>

namespace orc {

// float pi as the reference's kernels use it: M_PI is defined as the float literal
// 3.14159265358979323846f (libWR/kernels/sampling.cuh:6-8, ggx.cuh:5-7) and
// kPi = 3.14159265f (materials/material_common.cuh:9); both round to the same float.
template <class T> constexpr T kPiT() { return T(3.14159265358979323846f); }

// Elementary functions of the FP32 restatement.  By default glibc's sinf / cosf /
// powf, as the reference's shading headers get them when built on the host (the
// bit-exact pin against that build).  With cr_elementary() set, the correctly
// rounded value -- computed in double and rounded once to float -- which is what
// the device library evaluates; the GPU parity tests use that mode so the device
// and the restatement round alike.  The double instantiation is unaffected.
inline int& cr_elementary() {
    static thread_local int mode = 0;
    return mode;
}
template <class T> inline T esin(T x) { return std::sin(x); }
template <class T> inline T ecos(T x) { return std::cos(x); }
template <class T> inline T epow(T x, T y) { return std::pow(x, y); }
template <> inline float esin<float>(float x) { return cr_elementary() ? (float)std::sin((double)x) : std::sin(x); }
template <> inline float ecos<float>(float x) { return cr_elementary() ? (float)std::cos((double)x) : std::cos(x); }
template <> inline float epow<float>(float x, float y) {
    return cr_elementary() ? (float)std::pow((double)x, (double)y) : std::pow(x, y);
}

template <class T> struct V3 {
    T x, y, z;
};
template <class T> inline V3<T> mk(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
// libWR/kernels/vector_math.cuh:32-35: division by a scalar goes through its reciprocal.
template <class T> inline V3<T> divs(V3<T> a, T s) { T r = T(1) / s; return a * r; }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> inline T len(V3<T> v) { return std::sqrt(dot(v, v)); }

// 1/sqrt(x) correctly rounded.  The reference uses the device rsqrtf (approximate);
// the CUDA renderer uses __frsqrt_rn, which is correctly rounded, and so does this.
inline float rsqrt_cr(float x) { return (float)(1.0 / std::sqrt((double)x)); }
inline double rsqrt_cr(double x) { return 1.0 / std::sqrt(x); }
// vector_math.cuh:49-52
template <class T> inline V3<T> normalize(V3<T> v) { T r = rsqrt_cr(dot(v, v)); return v * r; }

// ---------------------------------------------------------------------------
// RNG (libWR/kernels/sampling.cuh:17-38, utils/atomic_ops.cuh:16-19). Integer, bit-exact.
inline uint32_t pcg_hash(uint32_t s) {
    uint32_t st = s * 747796405u + 2891336453u;
    uint32_t w = ((st >> ((st >> 28u) + 4u)) ^ st) * 277803737u;
    return (w >> 22u) ^ w;
}
inline uint32_t pcg_hash_dim(uint32_t s, uint32_t dim) {
    uint32_t st = s * 747796405u + 2891336453u + dim * 1013904223u;
    uint32_t w = ((st >> ((st >> 28u) + 4u)) ^ st) * 277803737u;
    return (w >> 22u) ^ w;
}
inline float rnd_dim(uint32_t s, uint32_t dim) { return float(pcg_hash_dim(s, dim)) / 4294967296.0f; }
inline float lcg_randf(uint32_t& s) {
    s = s * 1664525u + 1013904223u;
    return (float)(s >> 8) / 16777216.0f;
}
// Path seed: trace.cu:58 with the pixel as the slot (renderer.cpp:195-198).  A
// non-zero user seed (an extension; 0 keeps the reference formula) is folded in by
// XOR with its PCG hash.
inline uint32_t path_seed(uint32_t pixel, uint32_t sample, uint32_t user_seed) {
    uint32_t s = (pixel * 1664525u + sample * 1013904223u) ^ 0x9e3779b9u;
    if (user_seed != 0u) s ^= pcg_hash(user_seed);
    return s;
}

// ---------------------------------------------------------------------------
// Frames and warps (sampling.cuh:44-110)
template <class T> inline void frame(V3<T> n, V3<T>& t, V3<T>& b) {
    V3<T> up = std::fabs(n.y) < T(0.999f) ? mk<T>(0, 1, 0) : mk<T>(1, 0, 0);
    t = normalize(cross(up, n));
    b = cross(n, t);
}
template <class T> inline V3<T> to_world(V3<T> v, V3<T> n, V3<T> t, V3<T> b) {
    return {t.x * v.x + b.x * v.y + n.x * v.z, t.y * v.x + b.y * v.y + n.y * v.z,
            t.z * v.x + b.z * v.y + n.z * v.z};
}
template <class T> inline V3<T> cosine_hemisphere(T u1, T u2, T& pdf) {
    T r = std::sqrt(u1);
    T th = T(2) * kPiT<T>() * u2;
    T z = std::sqrt(std::fmax(T(0), T(1) - u1));
    pdf = z / kPiT<T>();
    return {r * ecos(th), r * esin(th), z};
}
template <class T> inline T cosine_pdf(T c) { return std::fmax(T(0), c / kPiT<T>()); }
template <class T>
inline V3<T> sample_triangle(T u1, T u2, V3<T> a, V3<T> b, V3<T> c, V3<T>& nrm, T& area) {
    T su = std::sqrt(u1);
    T b0 = T(1) - su, b1 = su * (T(1) - u2), b2 = su * u2;
    V3<T> p{a.x * b0 + b.x * b1 + c.x * b2, a.y * b0 + b.y * b1 + c.y * b2, a.z * b0 + b.z * b1 + c.z * b2};
    V3<T> cr = cross(b - a, c - a);
    area = T(0.5f) * len(cr);
    nrm = normalize(cr);
    return p;
}
// sampling.cuh:116-135: first index whose CDF value is >= u, clamped to n-1.
inline uint32_t cdf_lower_bound(float u, const float* cdf, uint32_t n) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t m = (lo + hi) / 2;
        if (cdf[m] < u) lo = m + 1; else hi = m;
    }
    return std::min(lo, n - 1);
}
template <class T> inline T power_heuristic(T a, T b) { T a2 = a * a, b2 = b * b; return a2 / (a2 + b2); }

// Russian roulette (sampling.cuh:162-193). Returns survive; writes the new throughput.
template <class T>
inline bool russian_roulette(V3<T> thr, uint32_t depth, float rr_start, T xi, V3<T>& out, bool delta) {
    if ((float)depth < rr_start) { out = thr; return true; }
    T lum = T(0.2126f) * thr.x + T(0.7152f) * thr.y + T(0.0722f) * thr.z;
    T df = T(1) / (T(1) + T(0.1f) * (T((float)depth) - T(rr_start)));
    T q = std::fmax(T(delta ? 0.5f : 0.05f), std::fmin(T(0.95f), lum * df));
    if (xi < q) { out = {thr.x / q, thr.y / q, thr.z / q}; return true; }
    return false;
}
template <class T> inline V3<T> clamp_fireflies(V3<T> r, T maxl) {
    if (maxl <= T(0)) return r;
    T lum = T(0.2126f) * r.x + T(0.7152f) * r.y + T(0.0722f) * r.z;
    if (lum > maxl) { T s = maxl / lum; return {r.x * s, r.y * s, r.z * s}; }
    return r;
}

// ---------------------------------------------------------------------------
// Dielectric Fresnel (utils/fresnel.cuh:8-16)
template <class T> inline T fresnel_dielectric(T ci, T ei, T et) {
    T s2 = ei / et * ei / et * (T(1) - ci * ci);
    if (s2 > T(1)) return T(1);
    T ct = std::sqrt(T(1) - s2);
    T rs = (ei * ci - et * ct) / (ei * ci + et * ct);
    T rp = (et * ci - ei * ct) / (et * ci + ei * ct);
    return (rs * rs + rp * rp) * T(0.5f);
}
// material_common.cuh:14-29
template <class T> inline T shading_correction(V3<T> wi, V3<T> ns, V3<T> ng) {
    T cs = std::fabs(dot(wi, ns)), cg = std::fabs(dot(wi, ng));
    if (cs < T(1e-6f) || cg < T(1e-6f)) return T(1);
    return cg / cs;
}
// utils/ray_offset.cuh:9-21
template <class T> inline V3<T> offset_origin(V3<T> p, V3<T> n, V3<T> d) {
    V3<T> od = dot(d, n) > T(0) ? n : -n;
    const T e = T(1e-4f);
    return {p.x + od.x * e, p.y + od.y * e, p.z + od.z * e};
}

// ---------------------------------------------------------------------------
// GGX (libWR/kernels/ggx.cuh)
template <class T> inline T ggx_D(T noh, T a) {
    T a2 = a * a, c2 = noh * noh;
    T den = c2 * (a2 - T(1)) + T(1);
    return a2 / (kPiT<T>() * den * den);
}
template <class T> inline T ggx_G1(T nov, T a) {
    T a2 = a * a, c2 = nov * nov;
    return T(2) * nov / (nov + std::sqrt(a2 + (T(1) - a2) * c2));
}
template <class T> inline V3<T> schlick3(T voh, V3<T> f0) {
    T f = epow(T(1) - voh, T(5));
    return {f0.x + (T(1) - f0.x) * f, f0.y + (T(1) - f0.y) * f, f0.z + (T(1) - f0.z) * f};
}
template <class T> inline V3<T> mix_f0(V3<T> alb, T metal, T ior) {
    T f = (ior - T(1)) / (ior + T(1));
    f = f * f;
    return {f * (T(1) - metal) + alb.x * metal, f * (T(1) - metal) + alb.y * metal,
            f * (T(1) - metal) + alb.z * metal};
}
// ggx.cuh:113-176: diffuse + Cook-Torrance; caller multiplies by cos.
template <class T>
inline V3<T> ggx_eval(V3<T> wo, V3<T> wi, V3<T> n, V3<T> alb, T rough, T metal, T ior) {
    T nov = std::fmax(T(0), dot(n, wo)), nol = std::fmax(T(0), dot(n, wi));
    if (nov < T(1e-5f) || nol < T(1e-5f)) return {0, 0, 0};
    V3<T> h = normalize(mk(wo.x + wi.x, wo.y + wi.y, wo.z + wi.z));
    T noh = std::fmax(T(0), dot(n, h)), voh = std::fmax(T(0), dot(wo, h));
    T a = rough * rough;
    T D = ggx_D(noh, a);
    T G = ggx_G1(nov, a) * ggx_G1(nol, a);
    V3<T> F = schlick3(voh, mix_f0(alb, metal, ior));
    T den = T(4) * nov * nol;
    V3<T> spec{D * G * F.x / den, D * G * F.y / den, D * G * F.z / den};
    V3<T> kd{(T(1) - F.x) * (T(1) - metal), (T(1) - F.y) * (T(1) - metal), (T(1) - F.z) * (T(1) - metal)};
    V3<T> diff{kd.x * alb.x / kPiT<T>(), kd.y * alb.y / kPiT<T>(), kd.z * alb.z / kPiT<T>()};
    return {diff.x + spec.x, diff.y + spec.y, diff.z + spec.z};
}
// ggx.cuh:182-215
template <class T> inline T ggx_pdf(V3<T> wo, V3<T> wi, V3<T> n, T rough) {
    T nov = std::fmax(T(0), dot(n, wo)), nol = std::fmax(T(0), dot(n, wi));
    if (nov < T(1e-5f) || nol < T(1e-5f)) return T(0);
    V3<T> h = normalize(mk(wo.x + wi.x, wo.y + wi.y, wo.z + wi.z));
    T noh = std::fmax(T(0), dot(n, h)), voh = std::fmax(T(0), dot(wo, h));
    if (voh < T(1e-5f)) return T(0);
    T a = rough * rough;
    return ggx_G1(nov, a) * ggx_D(noh, a) / (T(4) * nov);
}
// ggx.cuh:222-317: visible-normal sampling (Heitz 2018 form).  Returns false (pdf 0)
// when the half vector faces away or the reflected direction is below the surface.
template <class T>
inline bool ggx_sample(V3<T> wo, V3<T> n, V3<T> tg, V3<T> bt, T rough, T u0, T u1, V3<T>& wi, T& pdf) {
    T a = rough * rough;
    V3<T> v{dot(wo, tg), dot(wo, bt), dot(wo, n)};
    V3<T> sv = normalize(mk(a * v.x, a * v.y, v.z));
    T d2 = std::sqrt(sv.x * sv.x + sv.y * sv.y);
    V3<T> t1, t2;
    if (d2 > T(1e-6f)) {
        T r = T(1) / d2;
        t1 = {sv.y * r, -sv.x * r, T(0)};
        t2 = {t1.y * sv.z, -t1.x * sv.z, d2};
    } else {
        t1 = {1, 0, 0};
        t2 = {0, 1, 0};
    }
    T ia = T(1) / (T(1) + sv.z);
    T r = std::sqrt(u0);
    bool lower = u1 < ia;
    T phi = kPiT<T>() * (lower ? u1 / ia : T(1) + (u1 - ia) / (T(1) - ia));
    T sp = esin(phi), cp = ecos(phi);
    T p1 = r * cp;
    T p2 = r * sp * (lower ? T(1) : sv.z);
    T sq = std::sqrt(std::fmax(T(0), T(1) - (p1 * p1 + p2 * p2)));
    V3<T> m{p1 * t1.x + p2 * t2.x + sq * sv.x, p1 * t1.y + p2 * t2.y + sq * sv.y, p1 * t1.z + p2 * t2.z + sq * sv.z};
    m = normalize(mk(a * m.x, a * m.y, m.z));
    V3<T> h{tg.x * m.x + bt.x * m.y + n.x * m.z, tg.y * m.x + bt.y * m.y + n.y * m.z,
            tg.z * m.x + bt.z * m.y + n.z * m.z};
    T voh = dot(wo, h);
    if (voh <= T(0)) { pdf = T(0); return false; }
    wi = {T(2) * voh * h.x - wo.x, T(2) * voh * h.y - wo.y, T(2) * voh * h.z - wo.z};
    if (dot(n, wi) <= T(0)) { pdf = T(0); return false; }
    T nov = std::fmax(T(0), dot(n, wo)), noh = std::fmax(T(0), dot(n, h));
    pdf = ggx_G1(nov, a) * ggx_D(noh, a) / (T(4) * nov);
    return true;
}

// ---------------------------------------------------------------------------
// ACES filmic tone map + gamma, as the reference's image writer applies it
// (libWR/test/helpers/image.cpp:14-49): x*2.2 -> Narkowicz ACES fit clamped to
// [0,1] -> pow(x, 1/2.2) -> *255 truncated to a byte.
inline float aces_fit(float x) {
    float v = (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
    return std::min(std::max(v, 0.0f), 1.0f);
}
inline uint8_t aces_byte(float lin) {
    float g = 1.0f / 2.2f;
    float t = aces_fit(lin * 2.2f);
    return (uint8_t)(std::pow(t, g) * 255.0f);
}

}  // namespace orc
