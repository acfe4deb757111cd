// Stand-in for glm/gtc/constants.hpp: only pi<T>() is used by the reference.
#pragma once
#include "../glm.hpp"

namespace glm {
template <typename T> constexpr T pi() { return static_cast<T>(3.14159265358979323846264338327950288); }
}  // namespace glm
