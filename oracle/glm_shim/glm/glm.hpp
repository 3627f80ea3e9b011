// Test infrastructure only: a small stand-in for the GLM vector/matrix header,
// used to compile the reference's own CUDA kernels as a checker.
//
// The reference includes <glm/glm.hpp> from an un-vendored git submodule
// (textured_gaussians/cuda/csrc/third_party/glm, empty in the mounted tree;
// upstream github.com/icaven/glm, pinned commit unknown).  Its kernels use a
// narrow slice of GLM's documented public API: the templates vec<L,T> and
// mat<C,R,T> (C columns of R rows, column-major, m[i] is column i), element-wise
// vector arithmetic, matrix products, and the free functions dot, cross,
// length, transpose, outerProduct and two-argument atan.  This header restates
// that documented behaviour in plain code of its own; it is not GLM's source.
//
// Semantics kept from GLM's documentation:
//  * default construction leaves the components unset (a trivial constructor,
//    so the types may sit in shared memory);
//  * a vector converts implicitly to a vector of the same length and another
//    component type, and explicitly to a shorter one;
//  * vec<L,T>(s) broadcasts s; mat<C,R,T>(s) puts s on the diagonal;
//  * mat<C,R,T>(x0, ..., xk) takes its scalars column by column;
//  * M * v contracts over the columns (sum_i M[i] * v[i]); v * M is the row
//    vector times M; A * B for A = mat<C1,R> and B = mat<C2,C1> is mat<C2,R>.
#ifndef TG_ORACLE_GLM_SHIM_GLM_HPP
#define TG_ORACLE_GLM_SHIM_GLM_HPP

#include <cmath>
#include <cstddef>
#include <type_traits>

#if defined(__CUDACC__)
#define TGG_QUAL __host__ __device__ __forceinline__
#else
#define TGG_QUAL inline
#endif

namespace glm {

typedef int length_t;
enum qualifier { defaultp = 0, packed_highp = 0, highp = 0 };

template <length_t L, typename T, qualifier Q = defaultp>
struct vec;

// ---------------------------------------------------------------- vectors ---

template <typename T, qualifier Q>
struct vec<2, T, Q> {
    typedef T value_type;
    union { T x; T r; T s; };
    union { T y; T g; T t; };

    vec() = default;
    TGG_QUAL explicit vec(T v) : x(v), y(v) {}
    TGG_QUAL vec(T a, T b) : x(a), y(b) {}
    template <typename A, typename B>
    TGG_QUAL vec(A a, B b) : x(static_cast<T>(a)), y(static_cast<T>(b)) {}
    template <typename U, qualifier P>
    TGG_QUAL vec(const vec<2, U, P>& o) : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)) {}
    template <typename U, qualifier P>
    TGG_QUAL explicit vec(const vec<3, U, P>& o) : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)) {}
    template <typename U, qualifier P>
    TGG_QUAL explicit vec(const vec<4, U, P>& o) : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)) {}

    static constexpr length_t length() { return 2; }
    TGG_QUAL T& operator[](length_t i) { return i == 0 ? x : y; }
    TGG_QUAL const T& operator[](length_t i) const { return i == 0 ? x : y; }
};

template <typename T, qualifier Q>
struct vec<3, T, Q> {
    typedef T value_type;
    union { T x; T r; T s; };
    union { T y; T g; T t; };
    union { T z; T b; T p; };

    vec() = default;
    TGG_QUAL explicit vec(T v) : x(v), y(v), z(v) {}
    TGG_QUAL vec(T a, T b, T c) : x(a), y(b), z(c) {}
    template <typename A, typename B, typename C>
    TGG_QUAL vec(A a, B b, C c) : x(static_cast<T>(a)), y(static_cast<T>(b)), z(static_cast<T>(c)) {}
    template <typename A, typename B, qualifier P>
    TGG_QUAL vec(const vec<2, A, P>& xy, B c) : x(static_cast<T>(xy.x)), y(static_cast<T>(xy.y)), z(static_cast<T>(c)) {}
    template <typename A, typename B, qualifier P>
    TGG_QUAL vec(A a, const vec<2, B, P>& yz) : x(static_cast<T>(a)), y(static_cast<T>(yz.x)), z(static_cast<T>(yz.y)) {}
    template <typename U, qualifier P>
    TGG_QUAL vec(const vec<3, U, P>& o)
        : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)), z(static_cast<T>(o.z)) {}
    template <typename U, qualifier P>
    TGG_QUAL explicit vec(const vec<4, U, P>& o)
        : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)), z(static_cast<T>(o.z)) {}

    static constexpr length_t length() { return 3; }
    TGG_QUAL T& operator[](length_t i) { return i == 0 ? x : (i == 1 ? y : z); }
    TGG_QUAL const T& operator[](length_t i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

template <typename T, qualifier Q>
struct vec<4, T, Q> {
    typedef T value_type;
    union { T x; T r; T s; };
    union { T y; T g; T t; };
    union { T z; T b; T p; };
    union { T w; T a; T q; };

    vec() = default;
    TGG_QUAL explicit vec(T v) : x(v), y(v), z(v), w(v) {}
    TGG_QUAL vec(T a_, T b_, T c_, T d_) : x(a_), y(b_), z(c_), w(d_) {}
    template <typename A, typename B, typename C, typename D>
    TGG_QUAL vec(A a_, B b_, C c_, D d_)
        : x(static_cast<T>(a_)), y(static_cast<T>(b_)), z(static_cast<T>(c_)), w(static_cast<T>(d_)) {}
    template <typename A, typename B, qualifier P>
    TGG_QUAL vec(const vec<3, A, P>& xyz, B d_)
        : x(static_cast<T>(xyz.x)), y(static_cast<T>(xyz.y)), z(static_cast<T>(xyz.z)), w(static_cast<T>(d_)) {}
    template <typename A, typename B, typename C, qualifier P>
    TGG_QUAL vec(const vec<2, A, P>& xy, B c_, C d_)
        : x(static_cast<T>(xy.x)), y(static_cast<T>(xy.y)), z(static_cast<T>(c_)), w(static_cast<T>(d_)) {}
    template <typename U, qualifier P>
    TGG_QUAL vec(const vec<4, U, P>& o)
        : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)), z(static_cast<T>(o.z)), w(static_cast<T>(o.w)) {}

    static constexpr length_t length() { return 4; }
    TGG_QUAL T& operator[](length_t i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    TGG_QUAL const T& operator[](length_t i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};

// Element-wise operators, written once for every length.
#define TGG_VEC_BINOP(OP)                                                                   \
    template <length_t L, typename T, qualifier Q>                                          \
    TGG_QUAL vec<L, T, Q> operator OP(const vec<L, T, Q>& a, const vec<L, T, Q>& b) {       \
        vec<L, T, Q> r;                                                                     \
        for (length_t i = 0; i < L; ++i) r[i] = a[i] OP b[i];                               \
        return r;                                                                           \
    }                                                                                       \
    template <length_t L, typename T, qualifier Q>                                          \
    TGG_QUAL vec<L, T, Q> operator OP(const vec<L, T, Q>& a, T s) {                         \
        vec<L, T, Q> r;                                                                     \
        for (length_t i = 0; i < L; ++i) r[i] = a[i] OP s;                                  \
        return r;                                                                           \
    }                                                                                       \
    template <length_t L, typename T, qualifier Q>                                          \
    TGG_QUAL vec<L, T, Q> operator OP(T s, const vec<L, T, Q>& a) {                         \
        vec<L, T, Q> r;                                                                     \
        for (length_t i = 0; i < L; ++i) r[i] = s OP a[i];                                  \
        return r;                                                                           \
    }                                                                                       \
    template <length_t L, typename T, qualifier Q>                                          \
    TGG_QUAL vec<L, T, Q>& operator OP##=(vec<L, T, Q>& a, const vec<L, T, Q>& b) {         \
        for (length_t i = 0; i < L; ++i) a[i] = a[i] OP b[i];                               \
        return a;                                                                           \
    }                                                                                       \
    template <length_t L, typename T, qualifier Q, typename U>                              \
    TGG_QUAL vec<L, T, Q>& operator OP##=(vec<L, T, Q>& a, U s) {                           \
        for (length_t i = 0; i < L; ++i) a[i] = a[i] OP static_cast<T>(s);                  \
        return a;                                                                           \
    }

TGG_VEC_BINOP(+)
TGG_VEC_BINOP(-)
TGG_VEC_BINOP(*)
TGG_VEC_BINOP(/)
#undef TGG_VEC_BINOP

template <length_t L, typename T, qualifier Q>
TGG_QUAL vec<L, T, Q> operator-(const vec<L, T, Q>& a) {
    vec<L, T, Q> r;
    for (length_t i = 0; i < L; ++i) r[i] = -a[i];
    return r;
}
template <length_t L, typename T, qualifier Q>
TGG_QUAL vec<L, T, Q> operator+(const vec<L, T, Q>& a) { return a; }

template <length_t L, typename T, qualifier Q>
TGG_QUAL bool operator==(const vec<L, T, Q>& a, const vec<L, T, Q>& b) {
    for (length_t i = 0; i < L; ++i)
        if (!(a[i] == b[i])) return false;
    return true;
}
template <length_t L, typename T, qualifier Q>
TGG_QUAL bool operator!=(const vec<L, T, Q>& a, const vec<L, T, Q>& b) { return !(a == b); }

// --------------------------------------------------------------- matrices ---

// C columns, each a vec<R,T>.
template <length_t C, length_t R, typename T, qualifier Q = defaultp>
struct mat {
    typedef vec<R, T, Q> col_type;
    typedef T value_type;
    col_type value[C];

    mat() = default;
    // s on the diagonal, zero elsewhere
    TGG_QUAL explicit mat(T s) {
        for (length_t i = 0; i < C; ++i)
            for (length_t j = 0; j < R; ++j) value[i][j] = (i == j) ? s : T(0);
    }
    // C column vectors
    TGG_QUAL mat(const col_type& c0, const col_type& c1) {
        static_assert(C == 2, "two columns");
        value[0] = c0; value[1] = c1;
    }
    TGG_QUAL mat(const col_type& c0, const col_type& c1, const col_type& c2) {
        static_assert(C == 3, "three columns");
        value[0] = c0; value[1] = c1; value[2] = c2;
    }
    TGG_QUAL mat(const col_type& c0, const col_type& c1, const col_type& c2, const col_type& c3) {
        static_assert(C == 4, "four columns");
        value[0] = c0; value[1] = c1; value[2] = c2; value[3] = c3;
    }
    // C*R scalars, column by column
    template <typename... A, typename = typename std::enable_if<sizeof...(A) == C * R>::type>
    TGG_QUAL mat(A... s) {
        const T v[C * R] = {static_cast<T>(s)...};
        for (length_t i = 0; i < C; ++i)
            for (length_t j = 0; j < R; ++j) value[i][j] = v[i * R + j];
    }
    template <typename U, qualifier P>
    TGG_QUAL explicit mat(const mat<C, R, U, P>& o) {
        for (length_t i = 0; i < C; ++i) value[i] = col_type(o[i]);
    }

    static constexpr length_t length() { return C; }
    TGG_QUAL col_type& operator[](length_t i) { return value[i]; }
    TGG_QUAL const col_type& operator[](length_t i) const { return value[i]; }

    TGG_QUAL mat& operator+=(const mat& o) {
        for (length_t i = 0; i < C; ++i) value[i] += o.value[i];
        return *this;
    }
    TGG_QUAL mat& operator-=(const mat& o) {
        for (length_t i = 0; i < C; ++i) value[i] -= o.value[i];
        return *this;
    }
    template <typename U>
    TGG_QUAL mat& operator*=(U s) {
        for (length_t i = 0; i < C; ++i) value[i] *= static_cast<T>(s);
        return *this;
    }
    template <typename U>
    TGG_QUAL mat& operator/=(U s) {
        for (length_t i = 0; i < C; ++i) value[i] /= static_cast<T>(s);
        return *this;
    }
};

template <length_t C, length_t R, typename T, qualifier Q>
TGG_QUAL mat<C, R, T, Q> operator+(const mat<C, R, T, Q>& a, const mat<C, R, T, Q>& b) {
    mat<C, R, T, Q> r;
    for (length_t i = 0; i < C; ++i) r[i] = a[i] + b[i];
    return r;
}
template <length_t C, length_t R, typename T, qualifier Q>
TGG_QUAL mat<C, R, T, Q> operator-(const mat<C, R, T, Q>& a, const mat<C, R, T, Q>& b) {
    mat<C, R, T, Q> r;
    for (length_t i = 0; i < C; ++i) r[i] = a[i] - b[i];
    return r;
}
template <length_t C, length_t R, typename T, qualifier Q>
TGG_QUAL mat<C, R, T, Q> operator-(const mat<C, R, T, Q>& a) {
    mat<C, R, T, Q> r;
    for (length_t i = 0; i < C; ++i) r[i] = -a[i];
    return r;
}
template <length_t C, length_t R, typename T, qualifier Q>
TGG_QUAL mat<C, R, T, Q> operator*(const mat<C, R, T, Q>& a, T s) {
    mat<C, R, T, Q> r;
    for (length_t i = 0; i < C; ++i) r[i] = a[i] * s;
    return r;
}
template <length_t C, length_t R, typename T, qualifier Q>
TGG_QUAL mat<C, R, T, Q> operator*(T s, const mat<C, R, T, Q>& a) {
    mat<C, R, T, Q> r;
    for (length_t i = 0; i < C; ++i) r[i] = s * a[i];
    return r;
}
template <length_t C, length_t R, typename T, qualifier Q>
TGG_QUAL mat<C, R, T, Q> operator/(const mat<C, R, T, Q>& a, T s) {
    mat<C, R, T, Q> r;
    for (length_t i = 0; i < C; ++i) r[i] = a[i] / s;
    return r;
}

// M * v: sum over columns, row by row, in column order.
template <length_t C, length_t R, typename T, qualifier Q>
TGG_QUAL vec<R, T, Q> operator*(const mat<C, R, T, Q>& m, const vec<C, T, Q>& v) {
    vec<R, T, Q> r;
    for (length_t j = 0; j < R; ++j) {
        T acc = m[0][j] * v[0];
        for (length_t i = 1; i < C; ++i) acc = acc + m[i][j] * v[i];
        r[j] = acc;
    }
    return r;
}
// v * M: the row vector v (length R) times M; component i is dot(v, M[i]).
template <length_t C, length_t R, typename T, qualifier Q>
TGG_QUAL vec<C, T, Q> operator*(const vec<R, T, Q>& v, const mat<C, R, T, Q>& m) {
    vec<C, T, Q> r;
    for (length_t i = 0; i < C; ++i) {
        T acc = m[i][0] * v[0];
        for (length_t j = 1; j < R; ++j) acc = acc + m[i][j] * v[j];
        r[i] = acc;
    }
    return r;
}
// A (K columns of R rows) * B (C columns of K rows) -> C columns of R rows.
template <length_t K, length_t R, length_t C, typename T, qualifier Q>
TGG_QUAL mat<C, R, T, Q> operator*(const mat<K, R, T, Q>& a, const mat<C, K, T, Q>& b) {
    mat<C, R, T, Q> r;
    for (length_t i = 0; i < C; ++i) r[i] = a * b[i];
    return r;
}

// --------------------------------------------------------------- functions ---

template <length_t L, typename T, qualifier Q>
TGG_QUAL T dot(const vec<L, T, Q>& a, const vec<L, T, Q>& b) {
    T acc = a[0] * b[0];
    for (length_t i = 1; i < L; ++i) acc = acc + a[i] * b[i];
    return acc;
}
template <typename T>
TGG_QUAL T dot(T a, T b) { return a * b; }

template <typename T, qualifier Q>
TGG_QUAL vec<3, T, Q> cross(const vec<3, T, Q>& a, const vec<3, T, Q>& b) {
    return vec<3, T, Q>(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}

template <length_t L, typename T, qualifier Q>
TGG_QUAL T length(const vec<L, T, Q>& v) {
    using std::sqrt;
    return sqrt(dot(v, v));
}

template <length_t L, typename T, qualifier Q>
TGG_QUAL vec<L, T, Q> normalize(const vec<L, T, Q>& v) {
    using std::sqrt;
    return v * (T(1) / sqrt(dot(v, v)));
}

template <length_t C, length_t R, typename T, qualifier Q>
TGG_QUAL mat<R, C, T, Q> transpose(const mat<C, R, T, Q>& m) {
    mat<R, C, T, Q> r;
    for (length_t i = 0; i < C; ++i)
        for (length_t j = 0; j < R; ++j) r[j][i] = m[i][j];
    return r;
}

// outerProduct(c, r): the matrix c * r^T, i.e. column i is c * r[i].
template <length_t LC, length_t LR, typename T, qualifier Q>
TGG_QUAL mat<LR, LC, T, Q> outerProduct(const vec<LC, T, Q>& c, const vec<LR, T, Q>& r) {
    mat<LR, LC, T, Q> m;
    for (length_t i = 0; i < LR; ++i) m[i] = c * r[i];
    return m;
}

template <typename T>
TGG_QUAL T atan(T y, T x) {
    using std::atan2;
    return atan2(y, x);
}
template <typename T>
TGG_QUAL T atan(T y_over_x) {
    using std::atan;
    return atan(y_over_x);
}

// The float aliases GLM provides.
typedef vec<2, float> vec2;
typedef vec<3, float> vec3;
typedef vec<4, float> vec4;
typedef mat<2, 2, float> mat2;
typedef mat<3, 3, float> mat3;
typedef mat<4, 4, float> mat4;
typedef mat<3, 2, float> mat3x2;
typedef mat<2, 3, float> mat2x3;

}  // namespace glm

#endif
