// Minimal stand-in for the parts of Kokkos 5.1.1's SIMD API that the DUMMEST
// reference engine uses.  TEST INFRASTRUCTURE ONLY: it exists so that the
// reference sources (whose Kokkos submodule is absent) compile into the CPU
// oracle under oracle/_ref.  Nothing in the shipped library includes it.
//
// Surface provided (the complete list the reference engine and its unit test
// touch): simd<float> (8 lanes, AVX2) and simd<double> (4 lanes, AVX2) with
// size(), broadcast / native-vector / default constructors, *=, unary -,
// + - * (vector-vector and scalar-vector), simd_mask with < and ==,
// condition(), simd_unchecked_load / simd_unchecked_store, simd_flag_default,
// and the elementwise Kokkos::fma / max / abs / exp / log / exp2 / log2.
//
// Arithmetic is plain IEEE elementwise, exactly as the Kokkos AVX2 backend
// issues it (one vector instruction per operator; fma maps to vfmadd).
#pragma once

#include <immintrin.h>
#include <cmath>
#include <cstddef>

#if !defined(__AVX2__) || !defined(__FMA__)
#error "the oracle is built for the reference's portable x86-64-v3 ABI (AVX2 + FMA)"
#endif

namespace Kokkos {
namespace Experimental {

struct simd_flag_default_t {};
inline constexpr simd_flag_default_t simd_flag_default{};

template <typename T> class simd;
template <typename T> class simd_mask;

template <> class simd_mask<float> {
public:
    __m256 m;
    simd_mask() = default;
    explicit simd_mask(__m256 v) : m(v) {}
};

template <> class simd_mask<double> {
public:
    __m256d m;
    simd_mask() = default;
    explicit simd_mask(__m256d v) : m(v) {}
};

template <> class simd<float> {
public:
    using value_type = float;
    using native = __m256;
    __m256 v;
    static constexpr int size() { return 8; }
    simd() = default;
    simd(float x) : v(_mm256_set1_ps(x)) {}
    simd(double x) : v(_mm256_set1_ps((float)x)) {}
    simd(int x) : v(_mm256_set1_ps((float)x)) {}
    simd(__m256 x) : v(x) {}
    explicit operator __m256() const { return v; }
    simd &operator*=(const simd &o) { v = _mm256_mul_ps(v, o.v); return *this; }
    simd &operator+=(const simd &o) { v = _mm256_add_ps(v, o.v); return *this; }
    simd operator-() const { return simd(_mm256_sub_ps(_mm256_setzero_ps(), v)); }
};

template <> class simd<double> {
public:
    using value_type = double;
    using native = __m256d;
    __m256d v;
    static constexpr int size() { return 4; }
    simd() = default;
    simd(double x) : v(_mm256_set1_pd(x)) {}
    simd(float x) : v(_mm256_set1_pd((double)x)) {}
    simd(int x) : v(_mm256_set1_pd((double)x)) {}
    simd(__m256d x) : v(x) {}
    explicit operator __m256d() const { return v; }
    simd &operator*=(const simd &o) { v = _mm256_mul_pd(v, o.v); return *this; }
    simd &operator+=(const simd &o) { v = _mm256_add_pd(v, o.v); return *this; }
    simd operator-() const { return simd(_mm256_sub_pd(_mm256_setzero_pd(), v)); }
};

// float lanes
inline simd<float> operator+(simd<float> a, simd<float> b) { return _mm256_add_ps(a.v, b.v); }
inline simd<float> operator-(simd<float> a, simd<float> b) { return _mm256_sub_ps(a.v, b.v); }
inline simd<float> operator*(simd<float> a, simd<float> b) { return _mm256_mul_ps(a.v, b.v); }
inline simd<float> operator*(float a, simd<float> b) { return _mm256_mul_ps(_mm256_set1_ps(a), b.v); }
inline simd<float> operator*(simd<float> a, float b) { return _mm256_mul_ps(a.v, _mm256_set1_ps(b)); }
inline simd<float> operator+(float a, simd<float> b) { return _mm256_add_ps(_mm256_set1_ps(a), b.v); }
inline simd<float> operator+(simd<float> a, float b) { return _mm256_add_ps(a.v, _mm256_set1_ps(b)); }
inline simd_mask<float> operator<(simd<float> a, simd<float> b) {
    return simd_mask<float>(_mm256_cmp_ps(a.v, b.v, _CMP_LT_OQ));
}
inline simd_mask<float> operator==(simd<float> a, simd<float> b) {
    return simd_mask<float>(_mm256_cmp_ps(a.v, b.v, _CMP_EQ_OQ));
}
inline simd<float> condition(const simd_mask<float> &m, simd<float> a, simd<float> b) {
    return _mm256_blendv_ps(b.v, a.v, m.m);
}

// double lanes
inline simd<double> operator+(simd<double> a, simd<double> b) { return _mm256_add_pd(a.v, b.v); }
inline simd<double> operator-(simd<double> a, simd<double> b) { return _mm256_sub_pd(a.v, b.v); }
inline simd<double> operator*(simd<double> a, simd<double> b) { return _mm256_mul_pd(a.v, b.v); }
inline simd<double> operator*(double a, simd<double> b) { return _mm256_mul_pd(_mm256_set1_pd(a), b.v); }
inline simd<double> operator*(simd<double> a, double b) { return _mm256_mul_pd(a.v, _mm256_set1_pd(b)); }
inline simd<double> operator+(double a, simd<double> b) { return _mm256_add_pd(_mm256_set1_pd(a), b.v); }
inline simd<double> operator+(simd<double> a, double b) { return _mm256_add_pd(a.v, _mm256_set1_pd(b)); }
inline simd_mask<double> operator<(simd<double> a, simd<double> b) {
    return simd_mask<double>(_mm256_cmp_pd(a.v, b.v, _CMP_LT_OQ));
}
inline simd_mask<double> operator==(simd<double> a, simd<double> b) {
    return simd_mask<double>(_mm256_cmp_pd(a.v, b.v, _CMP_EQ_OQ));
}
inline simd<double> condition(const simd_mask<double> &m, simd<double> a, simd<double> b) {
    return _mm256_blendv_pd(b.v, a.v, m.m);
}

template <typename V> inline V simd_unchecked_load(const typename V::value_type *p);
template <> inline simd<float> simd_unchecked_load<simd<float>>(const float *p) { return _mm256_loadu_ps(p); }
template <> inline simd<double> simd_unchecked_load<simd<double>>(const double *p) { return _mm256_loadu_pd(p); }
template <typename V, typename Flag> inline V simd_unchecked_load(const typename V::value_type *p, Flag) {
    return simd_unchecked_load<V>(p);
}

inline void simd_unchecked_store(const simd<float> &v, float *p, simd_flag_default_t) { _mm256_storeu_ps(p, v.v); }
inline void simd_unchecked_store(const simd<double> &v, double *p, simd_flag_default_t) { _mm256_storeu_pd(p, v.v); }

}  // namespace Experimental

using Experimental::simd;

inline Experimental::simd<float> fma(Experimental::simd<float> a, Experimental::simd<float> b,
                                     Experimental::simd<float> c) {
    return _mm256_fmadd_ps(a.v, b.v, c.v);
}
inline Experimental::simd<double> fma(Experimental::simd<double> a, Experimental::simd<double> b,
                                      Experimental::simd<double> c) {
    return _mm256_fmadd_pd(a.v, b.v, c.v);
}
inline Experimental::simd<float> max(Experimental::simd<float> a, Experimental::simd<float> b) {
    return _mm256_max_ps(a.v, b.v);
}
inline Experimental::simd<double> max(Experimental::simd<double> a, Experimental::simd<double> b) {
    return _mm256_max_pd(a.v, b.v);
}
inline Experimental::simd<float> abs(Experimental::simd<float> a) {
    return _mm256_andnot_ps(_mm256_set1_ps(-0.0f), a.v);
}
inline Experimental::simd<double> abs(Experimental::simd<double> a) {
    return _mm256_andnot_pd(_mm256_set1_pd(-0.0), a.v);
}

// Elementwise libm on each lane (the engine only uses these off the hot path).
template <typename T, typename F> inline Experimental::simd<T> lanewise_(Experimental::simd<T> a, F f) {
    constexpr int n = Experimental::simd<T>::size();
    alignas(32) T buf[n];
    Experimental::simd_unchecked_store(a, buf, Experimental::simd_flag_default);
    for (int k = 0; k < n; ++k) buf[k] = f(buf[k]);
    return Experimental::simd_unchecked_load<Experimental::simd<T>>(buf);
}
inline Experimental::simd<float> exp(Experimental::simd<float> a) { return lanewise_(a, [](float x) { return std::exp(x); }); }
inline Experimental::simd<double> exp(Experimental::simd<double> a) { return lanewise_(a, [](double x) { return std::exp(x); }); }
inline Experimental::simd<float> log(Experimental::simd<float> a) { return lanewise_(a, [](float x) { return std::log(x); }); }
inline Experimental::simd<double> log(Experimental::simd<double> a) { return lanewise_(a, [](double x) { return std::log(x); }); }
inline Experimental::simd<float> exp2(Experimental::simd<float> a) { return lanewise_(a, [](float x) { return std::exp2(x); }); }
inline Experimental::simd<double> exp2(Experimental::simd<double> a) { return lanewise_(a, [](double x) { return std::exp2(x); }); }
inline Experimental::simd<float> log2(Experimental::simd<float> a) { return lanewise_(a, [](float x) { return std::log2(x); }); }
inline Experimental::simd<double> log2(Experimental::simd<double> a) { return lanewise_(a, [](double x) { return std::log2(x); }); }

}  // namespace Kokkos
