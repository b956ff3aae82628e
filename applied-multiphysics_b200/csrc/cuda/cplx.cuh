// Complex FP64 scalar for the complex-symmetric LDL^T (A = A^T, no conjugation anywhere, as the reference's
// ComplexSupernodalLDLT, ldlt.mjs:648-864): a plain pair (re, im), 16-byte aligned so that one entry is one 16-byte
// access, with the arithmetic the templated factor kernels use. Products and quotients are written out as the
// reference writes them: (a + ib)(c + id) = (ac - bd) + i(ad + bc), 1 / d = (dr - i di) / (dr^2 + di^2).
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

namespace amp {

struct __align__(16) cplx {
  double re, im;
  cplx() = default;  // trivial, so that shared-memory arrays of it need no initialisation
  __host__ __device__ constexpr cplx(double r, double i = 0.0) : re(r), im(i) {}
};

__host__ __device__ __forceinline__ cplx operator+(cplx a, cplx b) { return cplx(a.re + b.re, a.im + b.im); }
__host__ __device__ __forceinline__ cplx operator-(cplx a, cplx b) { return cplx(a.re - b.re, a.im - b.im); }
__host__ __device__ __forceinline__ cplx operator-(cplx a) { return cplx(-a.re, -a.im); }
__host__ __device__ __forceinline__ cplx operator*(cplx a, cplx b) {
  return cplx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__host__ __device__ __forceinline__ cplx operator/(cplx a, cplx d) {
  const double den = d.re * d.re + d.im * d.im, ir = d.re / den, ii = -d.im / den;
  return cplx(a.re * ir - a.im * ii, a.re * ii + a.im * ir);
}
__host__ __device__ __forceinline__ cplx &operator+=(cplx &a, cplx b) { return a = a + b; }
__host__ __device__ __forceinline__ cplx &operator-=(cplx &a, cplx b) { return a = a - b; }
__host__ __device__ __forceinline__ cplx &operator*=(cplx &a, cplx b) { return a = a * b; }
__host__ __device__ __forceinline__ bool operator==(cplx a, cplx b) { return a.re == b.re && a.im == b.im; }

template <class T>
struct is_cplx : std::false_type {};
template <>
struct is_cplx<cplx> : std::true_type {};
// real type of a scalar: the type of its magnitude and of the pivot threshold
template <class T>
struct real_of {
  using type = T;
};
template <>
struct real_of<cplx> {
  using type = double;
};
// type of the CSR values a factor of scalar type T assembles from (FP64 real, or complex)
template <class T>
using value_of = typename std::conditional<is_cplx<T>::value, cplx, double>::type;

}  // namespace amp
