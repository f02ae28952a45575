// wr::Vec3 and wr::Camera -- public math types of the drop-in C++ API.
// libWR (trianglestrip/OfflineRenderer, libWR/include/wr/types.h:10-51) uses
// glm::vec3 as wr::Vec3; this header provides a GLM-free Vec3 with the members and
// constructors libWR code uses (Vec3(x,y,z), .x/.y/.z, arithmetic) and the same
// Camera fields and basis helpers.
#pragma once
#include <cmath>

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
static_assert(sizeof(Vec3) == 12, "Vec3 must be three packed floats (render output layout)");

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

// Camera configuration (libWR/include/wr/types.h:16-51).
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
