/* Minimal stand-in for the parts of glm that the reference's SphBase.h/.cpp
 * name (glm::vec3/vec4/mat3/mat4, translate, rotate, inverse).  Only the
 * reference's ice/"candidate" code touches these, and that code is never run
 * by the oracle harness; the stand-in exists so those translation units
 * compile.  Test infrastructure only. */
#ifndef ORACLE_GLM_SHIM_H_
#define ORACLE_GLM_SHIM_H_
#include <cmath>
namespace glm {
struct vec3 {
    float x, y, z;
    vec3() : x(0), y(0), z(0) {}
    explicit vec3(float a) : x(a), y(a), z(a) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    float& operator[](int i) { return (&x)[i]; }
    const float& operator[](int i) const { return (&x)[i]; }
};
struct vec4 {
    float x, y, z, w;
    vec4() : x(0), y(0), z(0), w(0) {}
    vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    float& operator[](int i) { return (&x)[i]; }
    const float& operator[](int i) const { return (&x)[i]; }
};
struct mat3 {
    vec3 c[3];
    mat3() { for (int i = 0; i < 3; ++i) { c[i] = vec3(0); c[i][i] = 1; } }
    explicit mat3(float d) { for (int i = 0; i < 3; ++i) { c[i] = vec3(0); c[i][i] = d; } }
    vec3& operator[](int i) { return c[i]; }
    const vec3& operator[](int i) const { return c[i]; }
};
struct mat4 {
    vec4 c[4];
    mat4() { for (int i = 0; i < 4; ++i) { c[i] = vec4(0, 0, 0, 0); c[i][i] = 1; } }
    explicit mat4(float d) { for (int i = 0; i < 4; ++i) { c[i] = vec4(0, 0, 0, 0); c[i][i] = d; } }
    vec4& operator[](int i) { return c[i]; }
    const vec4& operator[](int i) const { return c[i]; }
};
inline vec3 operator*(const mat3& m, const vec3& v) {
    vec3 r;
    for (int i = 0; i < 3; ++i) r[i] = m[0][i] * v[0] + m[1][i] * v[1] + m[2][i] * v[2];
    return r;
}
inline vec4 operator*(const mat4& m, const vec4& v) {
    vec4 r;
    for (int i = 0; i < 4; ++i)
        r[i] = m[0][i] * v[0] + m[1][i] * v[1] + m[2][i] * v[2] + m[3][i] * v[3];
    return r;
}
inline mat4 operator*(const mat4& a, const mat4& b) {
    mat4 r(0.f);
    for (int j = 0; j < 4; ++j) r[j] = a * b[j];
    return r;
}
inline mat4 translate(const mat4& m, const vec3& t) {
    mat4 r = m;
    for (int i = 0; i < 4; ++i) r[3][i] = m[0][i] * t[0] + m[1][i] * t[1] + m[2][i] * t[2] + m[3][i];
    return r;
}
inline mat4 translate(const vec3& t) { return translate(mat4(), t); }
inline mat4 rotate(const mat4& m, float a, const vec3& axis) {
    float n = std::sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
    float x = axis[0] / n, y = axis[1] / n, z = axis[2] / n, c = std::cos(a), s = std::sin(a), t = 1 - c;
    mat4 R;
    R[0] = vec4(t * x * x + c, t * x * y + s * z, t * x * z - s * y, 0);
    R[1] = vec4(t * x * y - s * z, t * y * y + c, t * y * z + s * x, 0);
    R[2] = vec4(t * x * z + s * y, t * y * z - s * x, t * z * z + c, 0);
    return m * R;
}
inline mat4 scale(const vec3& s) { mat4 r; r[0][0] = s[0]; r[1][1] = s[1]; r[2][2] = s[2]; return r; }
inline mat3 inverse(const mat3& m) {
    float a = m[0][0], b = m[1][0], c = m[2][0], d = m[0][1], e = m[1][1], f = m[2][1],
          g = m[0][2], h = m[1][2], k = m[2][2];
    float det = a * (e * k - f * h) - b * (d * k - f * g) + c * (d * h - e * g);
    mat3 r;
    r[0][0] = (e * k - f * h) / det; r[1][0] = (c * h - b * k) / det; r[2][0] = (b * f - c * e) / det;
    r[0][1] = (f * g - d * k) / det; r[1][1] = (a * k - c * g) / det; r[2][1] = (c * d - a * f) / det;
    r[0][2] = (d * h - e * g) / det; r[1][2] = (b * g - a * h) / det; r[2][2] = (a * e - b * d) / det;
    return r;
}
}  // namespace glm
#endif
