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

// Does the ray hit scene triangle `prim` within [tmin, tmax]?  The triangle record
// is rebuilt from the scene's vertices exactly as the BVH builder writes it (v0,
// v1 - v0, v2 - v0 with correctly rounded subtractions), so the answer is the one
// the traversal's triangle test gives for the same triangle.
__device__ __forceinline__ bool light_blocks(const DevScene& s, const Ray& r, uint32_t prim) {
    const uint32_t i0 = __ldg(s.idx + 3 * prim), i1 = __ldg(s.idx + 3 * prim + 1), i2 = __ldg(s.idx + 3 * prim + 2);
    const float ax = __ldg(s.vtx + 3 * i0), ay = __ldg(s.vtx + 3 * i0 + 1), az = __ldg(s.vtx + 3 * i0 + 2);
    const float bx = __ldg(s.vtx + 3 * i1), by = __ldg(s.vtx + 3 * i1 + 1), bz = __ldg(s.vtx + 3 * i1 + 2);
    const float cx = __ldg(s.vtx + 3 * i2), cy = __ldg(s.vtx + 3 * i2 + 1), cz = __ldg(s.vtx + 3 * i2 + 2);
    const float4 a = make_float4(ax, ay, az, 0.0f);
    const float4 b = make_float4(__fsub_rn(bx, ax), __fsub_rn(by, ay), __fsub_rn(bz, az), 0.0f);
    const float4 c = make_float4(__fsub_rn(cx, ax), __fsub_rn(cy, ay), __fsub_rn(cz, az), 0.0f);
    float th;
    return mt_rn(r, a, b, c, th) && th >= r.tmin && th <= r.tmax;
}

}  // namespace wrk
