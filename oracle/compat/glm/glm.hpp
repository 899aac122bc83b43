/* Minimal stand-in for glm (absent): the vector/matrix types the reference's
 * hot-path headers name, with field access only.  Test infrastructure only. */
#pragma once
namespace glm {
struct vec2 { float x, y; vec2(float a = 0, float b = 0) : x(a), y(b) {} };
struct vec3 { float x, y, z; vec3(float a = 0, float b = 0, float c = 0) : x(a), y(b), z(c) {} };
struct vec4 { float x, y, z, w; vec4(float a = 0, float b = 0, float c = 0, float d = 0) : x(a), y(b), z(c), w(d) {}
              float& operator[](int i) { return (&x)[i]; } const float& operator[](int i) const { return (&x)[i]; } };
struct mat4 { vec4 c[4]; vec4& operator[](int i) { return c[i]; } const vec4& operator[](int i) const { return c[i]; } };
}
