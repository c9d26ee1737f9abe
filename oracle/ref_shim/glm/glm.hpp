// Minimal glm subset for compiling the reference renderer's kernel sources
// on the host (see oracle/ref_shim/sycl/sycl.hpp).  TEST INFRASTRUCTURE
// ONLY.  The kernels use glm::radians; the shared data-structure header
// converts between glm vectors/matrices (column-major, m[column][row]) and
// its own row-major matrices.
#pragma once

namespace glm {

template <typename T>
constexpr T radians(T degrees) {
  return degrees * static_cast<T>(0.01745329251994329576923690768489);
}

struct vec2 {
  float x = 0, y = 0;
  vec2() = default;
  vec2(float a, float b) : x(a), y(b) {}
  float& operator[](int i) { return i == 0 ? x : y; }
  float operator[](int i) const { return i == 0 ? x : y; }
};
struct vec3 {
  float x = 0, y = 0, z = 0;
  vec3() = default;
  explicit vec3(float a) : x(a), y(a), z(a) {}
  vec3(float a, float b, float c) : x(a), y(b), z(c) {}
  float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
struct vec4 {
  float x = 0, y = 0, z = 0, w = 0;
  vec4() = default;
  vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
  float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};
struct mat3 {
  vec3 c[3];
  mat3() : c{vec3(1, 0, 0), vec3(0, 1, 0), vec3(0, 0, 1)} {}
  vec3& operator[](int i) { return c[i]; }
  const vec3& operator[](int i) const { return c[i]; }
};
struct mat4 {
  vec4 c[4];
  mat4() : c{vec4(1, 0, 0, 0), vec4(0, 1, 0, 0), vec4(0, 0, 1, 0), vec4(0, 0, 0, 1)} {}
  vec4& operator[](int i) { return c[i]; }
  const vec4& operator[](int i) const { return c[i]; }
};

}  // namespace glm
