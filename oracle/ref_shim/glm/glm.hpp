// Minimal stand-in for the parts of GLM (a header-only third-party library,
// unpinned in the reference's vcpkg.json) that the reference's geometry code
// uses: glm::vec3 (construction, +, -, scalar *) and glm::cross.  Written for
// this project from the vector-algebra definitions; used only to compile the
// reference's own voxelize.cpp / stl_loader.cpp into the checker under
// oracle/_ref.  The cross product keeps GLM's documented operand order.
#pragma once

#include <cmath>   // GLM's headers bring <cmath> in; the reference relies on it

namespace glm {

struct vec3 {
    float x, y, z;
    vec3() : x(0.0f), y(0.0f), z(0.0f) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
};

inline vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator*(float s, const vec3& v) { return vec3(s * v.x, s * v.y, s * v.z); }
inline vec3 operator*(const vec3& v, float s) { return vec3(v.x * s, v.y * s, v.z * s); }

inline vec3 cross(const vec3& a, const vec3& b) {
    return vec3(a.y * b.z - b.y * a.z,
                a.z * b.x - b.z * a.x,
                a.x * b.y - b.x * a.y);
}

}  // namespace glm
