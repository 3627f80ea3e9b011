// Test infrastructure only: the make_vec* builders of GLM's documented
// <glm/gtc/type_ptr.hpp> API (a vector from consecutive components in memory),
// for compiling the reference's kernels as a checker.  Not GLM's source.
#ifndef TG_ORACLE_GLM_SHIM_TYPE_PTR_HPP
#define TG_ORACLE_GLM_SHIM_TYPE_PTR_HPP

#include "../glm.hpp"

namespace glm {

template <typename T>
TGG_QUAL vec<2, T> make_vec2(const T* p) { return vec<2, T>(p[0], p[1]); }
template <typename T>
TGG_QUAL vec<3, T> make_vec3(const T* p) { return vec<3, T>(p[0], p[1], p[2]); }
template <typename T>
TGG_QUAL vec<4, T> make_vec4(const T* p) { return vec<4, T>(p[0], p[1], p[2], p[3]); }

template <length_t L, typename T, qualifier Q>
TGG_QUAL T* value_ptr(vec<L, T, Q>& v) { return &v[0]; }
template <length_t L, typename T, qualifier Q>
TGG_QUAL const T* value_ptr(const vec<L, T, Q>& v) { return &v[0]; }

}  // namespace glm

#endif
