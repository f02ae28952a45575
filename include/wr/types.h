// wr::Vec3 and wr::Camera -- public math types of the drop-in C++ API
// (libWR/include/wr/types.h:1-53 in trianglestrip/OfflineRenderer).
//
// libWR's public types are GLM's: Vec3 = glm::vec3 (types.h:10), with Vec4 / Mat3 /
// Mat4 beside it and Camera's view / projection helpers built on glm::lookAt and
// glm::perspective.  When GLM's headers are on the include path this header uses
// exactly those types, so a libWR application that does GLM math on wr::Vec3 or
// calls glm::radians compiles unchanged.  Without GLM (define WR_NO_GLM to force
// this) it falls back to a small 12-byte Vec3 with the members, constructors and
// arithmetic libWR code uses, and a Camera with the same fields and basis helpers
// (the matrix helpers need GLM and are left out).
//
// Either way libwrk.so never sees the type: every member of the C++ API that takes
// or returns a Vec3 (or a Camera / RenderParams, which hold them) is defined inline
// in these headers and hands plain floats to the library, so one build of
// libwrk.so serves callers compiled with or without GLM.
#pragma once
#include <cmath>

#if !defined(WR_NO_GLM) && defined(__has_include)
#if __has_include(<glm/glm.hpp>)
#define WR_HAS_GLM 1
#endif
#endif

#ifdef WR_HAS_GLM
#include <glm/glm.hpp>
#include <glm/gtc/matrix_transform.hpp>
#include <glm/gtc/type_ptr.hpp>

namespace wr {

using Vec3 = glm::vec3;
using Vec4 = glm::vec4;
using Mat3 = glm::mat3;
using Mat4 = glm::mat4;

// Camera configuration (libWR/include/wr/types.h:16-51): fovY in radians, vertical.
struct Camera {
    Vec3 position{0.0f, 0.0f, 0.0f};
    Vec3 target{0.0f, 0.0f, -1.0f};
    Vec3 up{0.0f, 1.0f, 0.0f};
    float fovY{glm::radians(45.0f)};
    float aspect{1.0f};
    float focalDistance{0.0f};  // 0 = infinite focus (no depth of field)
    float lensRadius{0.0f};     // 0 = pinhole

    Mat4 getViewMatrix() const { return glm::lookAt(position, target, up); }
    Mat4 getProjectionMatrix(float nearPlane = 0.1f, float farPlane = 100.0f) const {
        return glm::perspective(fovY, aspect, nearPlane, farPlane);
    }
    Vec3 getForward() const { return glm::normalize(target - position); }
    Vec3 getRight() const { return glm::normalize(glm::cross(getForward(), up)); }
    Vec3 getUp() const { return glm::normalize(glm::cross(getRight(), getForward())); }
};

}  // namespace wr

#else  // no GLM

namespace wr {

struct Vec3 {
    float x = 0.0f, y = 0.0f, z = 0.0f;
    constexpr Vec3() = default;
    constexpr Vec3(float x_, float y_, float z_) : x(x_), y(y_), z(z_) {}
    constexpr explicit Vec3(float s) : x(s), y(s), z(s) {}
    constexpr Vec3 operator+(const Vec3& o) const { return {x + o.x, y + o.y, z + o.z}; }
    constexpr Vec3 operator-(const Vec3& o) const { return {x - o.x, y - o.y, z - o.z}; }
    constexpr Vec3 operator-() const { return {-x, -y, -z}; }
    constexpr Vec3 operator*(float s) const { return {x * s, y * s, z * s}; }
    constexpr Vec3 operator*(const Vec3& o) const { return {x * o.x, y * o.y, z * o.z}; }
    constexpr Vec3 operator/(float s) const { return {x / s, y / s, z / s}; }
    constexpr bool operator==(const Vec3& o) const { return x == o.x && y == o.y && z == o.z; }
};

inline constexpr Vec3 operator*(float s, const Vec3& v) { return {s * v.x, s * v.y, s * v.z}; }
inline float dot(const Vec3& a, const Vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec3 cross(const Vec3& a, const Vec3& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// v * (1/sqrt(dot(v,v))), the rounding GLM's normalize has.
inline Vec3 normalize(const Vec3& v) {
    float r = 1.0f / std::sqrt(dot(v, v));
    return {v.x * r, v.y * r, v.z * r};
}
// glm::radians for float.
inline float radians(float degrees) { return degrees * 0.01745329251994329576923690768489f; }

// Camera configuration (libWR/include/wr/types.h:16-51): fovY in radians, vertical.
struct Camera {
    Vec3 position{0.0f, 0.0f, 0.0f};
    Vec3 target{0.0f, 0.0f, -1.0f};
    Vec3 up{0.0f, 1.0f, 0.0f};
    float fovY{radians(45.0f)};
    float aspect{1.0f};
    float focalDistance{0.0f};  // 0 = infinite focus (no depth of field)
    float lensRadius{0.0f};     // 0 = pinhole

    Vec3 getForward() const { return normalize(target - position); }
    Vec3 getRight() const { return normalize(cross(getForward(), up)); }
    Vec3 getUp() const { return normalize(cross(getRight(), getForward())); }
};

}  // namespace wr

#endif

namespace wr {
static_assert(sizeof(Vec3) == 3 * sizeof(float), "Vec3 must be three packed floats (render output layout)");
}  // namespace wr
