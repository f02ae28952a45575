// The ray-triangle test of the traversal kernels (trace.cu), shared with the
// Lambert shade (render.cu), which answers the shadow queries whose light triangle
// blocks the ray itself.
#pragma once
#include "wrk_internal.h"

namespace wrk {

struct Ray {
    float ox, oy, oz, dx, dy, dz, tmin, tmax;
};

// Moller-Trumbore without the reciprocal: barycentric numerators are compared
// with det (sign-aware) and t is divided only for hits inside the triangle.  Each
// cross-product component is one product and one FMA, each dot product one product
// and two FMAs (correctly rounded intrinsics, in the CPU oracle's exact order).
__device__ __forceinline__ bool mt_rn(const Ray& r, float4 a, float4 b, float4 c, float& t) {
    float px = __fmaf_rn(r.dy, c.z, -__fmul_rn(r.dz, c.y));
    float py = __fmaf_rn(r.dz, c.x, -__fmul_rn(r.dx, c.z));
    float pz = __fmaf_rn(r.dx, c.y, -__fmul_rn(r.dy, c.x));
    float det = __fmaf_rn(b.x, px, __fmaf_rn(b.y, py, __fmul_rn(b.z, pz)));
    float sx = __fsub_rn(r.ox, a.x), sy = __fsub_rn(r.oy, a.y), sz = __fsub_rn(r.oz, a.z);
    float un = __fmaf_rn(sx, px, __fmaf_rn(sy, py, __fmul_rn(sz, pz)));
    float qx = __fmaf_rn(sy, b.z, -__fmul_rn(sz, b.y));
    float qy = __fmaf_rn(sz, b.x, -__fmul_rn(sx, b.z));
    float qz = __fmaf_rn(sx, b.y, -__fmul_rn(sy, b.x));
    float vn = __fmaf_rn(r.dx, qx, __fmaf_rn(r.dy, qy, __fmul_rn(r.dz, qz)));
    float uv = __fadd_rn(un, vn);
    bool inside = det > 0.0f ? (un >= 0.0f && vn >= 0.0f && uv <= det)
                             : (det < 0.0f && un <= 0.0f && vn <= 0.0f && uv >= det);
    if (!inside) return false;
    t = __fdiv_rn(__fmaf_rn(c.x, qx, __fmaf_rn(c.y, qy, __fmul_rn(c.z, qz))), det);
    return true;
}

// Does the ray hit the light triangle of light record `lr` (v0, v1, v2 in its first
// three float4s) within [tmin, tmax]?  The triangle is rebuilt as the BVH builder
// writes it (v0, v1 - v0, v2 - v0 with correctly rounded subtractions), so the
// answer is the one the traversal's triangle test gives for the same triangle.
__device__ __forceinline__ bool light_blocks(const float4* lr, const Ray& r) {
    const float4 l0 = __ldg(lr), l1 = __ldg(lr + 1), l2 = __ldg(lr + 2);
    const float4 a = make_float4(l0.x, l0.y, l0.z, 0.0f);
    const float4 b = make_float4(__fsub_rn(l1.x, l0.x), __fsub_rn(l1.y, l0.y), __fsub_rn(l1.z, l0.z), 0.0f);
    const float4 c = make_float4(__fsub_rn(l2.x, l0.x), __fsub_rn(l2.y, l0.y), __fsub_rn(l2.z, l0.z), 0.0f);
    float th;
    return mt_rn(r, a, b, c, th) && th >= r.tmin && th <= r.tmax;
}

}  // namespace wrk
