// Minimal stand-in for the handful of glm functions that the reference's CSG
// front end (vulkan/src/csg/*.cpp) calls. glm is not installed in this image.
// Test infrastructure only: it lets oracle/Makefile compile the reference's own
// tape compiler so that the product's compiler can be pinned against it.
//
// Semantics follow glm's documented definitions: sin/cos/exp/sqrt forward to
// <cmath>; min(x, y) = (y < x) ? y : x and max(x, y) = (x < y) ? y : x.
#pragma once
#include <cmath>

namespace glm {
template <typename T> inline T sin(T x) { return std::sin(x); }
template <typename T> inline T cos(T x) { return std::cos(x); }
template <typename T> inline T exp(T x) { return std::exp(x); }
template <typename T> inline T sqrt(T x) { return std::sqrt(x); }
template <typename T> inline T tan(T x) { return std::tan(x); }
template <typename T> inline T min(T x, T y) { return (y < x) ? y : x; }
template <typename T> inline T max(T x, T y) { return (x < y) ? y : x; }
template <typename T> inline T pow(T x, T y) { return std::pow(x, y); }
}  // namespace glm
