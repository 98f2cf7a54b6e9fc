// dem_math.cuh — 2-D vector/matrix algebra for the device (MathVector.h,
// MathMatrix2d.h of the reference), templated on the arithmetic type.  The
// library is compiled with -fmad=false so that every FP64 operation rounds
// separately, as the reference's x86-64 build does; the FP32 routines of the
// mixed-precision path use explicit fma where they want one.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace xdem {

template <class R>
struct vec2 {
  R x, y;
};
template <class R>
struct mat2 {
  R xx, xy, yx, yy;
};

template <class R>
__host__ __device__ __forceinline__ vec2<R> V(R x, R y) {
  return vec2<R>{x, y};
}
template <class R>
__host__ __device__ __forceinline__ vec2<R> operator+(vec2<R> a, vec2<R> b) {
  return V<R>(a.x + b.x, a.y + b.y);
}
template <class R>
__host__ __device__ __forceinline__ vec2<R> operator-(vec2<R> a, vec2<R> b) {
  return V<R>(a.x - b.x, a.y - b.y);
}
template <class R>
__host__ __device__ __forceinline__ vec2<R> operator-(vec2<R> a) {
  return V<R>(-a.x, -a.y);
}
template <class R>
__host__ __device__ __forceinline__ vec2<R> operator*(vec2<R> a, R f) {
  return V<R>(a.x * f, a.y * f);
}
template <class R>
__host__ __device__ __forceinline__ vec2<R> operator/(vec2<R> a, R f) {
  return V<R>(a.x / f, a.y / f);
}
template <class R>
__host__ __device__ __forceinline__ R dot(vec2<R> a, vec2<R> b) {
  return a.x * b.x + a.y * b.y;
}
template <class R>
__host__ __device__ __forceinline__ R cross(vec2<R> a, vec2<R> b) {
  return a.x * b.y - a.y * b.x;
}
// vector2d::cross(omega) (MathVector.h:202-205)
template <class R>
__host__ __device__ __forceinline__ vec2<R> crossw(vec2<R> a, R w) {
  return V<R>(-w * a.y, w * a.x);
}
template <class R>
__host__ __device__ __forceinline__ R len2(vec2<R> a) {
  return a.x * a.x + a.y * a.y;
}
template <class R>
__device__ __forceinline__ R len(vec2<R> a) {
  return sqrt(len2(a));
}
// getUnitVector (MathVector.h:169-178)
template <class R>
__device__ __forceinline__ vec2<R> unit(vec2<R> a) {
  R l2 = len2(a);
  if (l2 != R(0)) return a / R(sqrt(l2));
  return V<R>(R(0), R(0));
}
// normalize (MathVector.h:180-190): zero length raises a status bit
template <class R>
__device__ __forceinline__ vec2<R> normalize(vec2<R> a, uint32_t& st) {
  R l2 = len2(a);
  if (l2 != R(0)) return a / R(sqrt(l2));
  st |= 1u << 4;  // XDEM_ERR_ZERO_VECTOR
  return a;
}

template <class R>
__host__ __device__ __forceinline__ mat2<R> M(R xx, R xy, R yx, R yy) {
  return mat2<R>{xx, xy, yx, yy};
}
template <class R>
__host__ __device__ __forceinline__ mat2<R> operator+(mat2<R> a, mat2<R> b) {
  return M<R>(a.xx + b.xx, a.xy + b.xy, a.yx + b.yx, a.yy + b.yy);
}
template <class R>
__host__ __device__ __forceinline__ mat2<R> operator-(mat2<R> a, mat2<R> b) {
  return M<R>(a.xx - b.xx, a.xy - b.xy, a.yx - b.yx, a.yy - b.yy);
}
template <class R>
__host__ __device__ __forceinline__ mat2<R> operator*(mat2<R> a, R f) {
  return M<R>(a.xx * f, a.xy * f, a.yx * f, a.yy * f);
}
template <class R>
__host__ __device__ __forceinline__ mat2<R> operator/(mat2<R> a, R f) {
  return M<R>(a.xx / f, a.xy / f, a.yx / f, a.yy / f);
}
template <class R>
__host__ __device__ __forceinline__ vec2<R> operator*(mat2<R> a, vec2<R> v) {
  return V<R>(a.xx * v.x + a.xy * v.y, a.yx * v.x + a.yy * v.y);
}
// matrix2d::operator*(matrix2d) exactly as written in MathMatrix2d.h:85-91
// (its yy entry reads other.yx(); every right operand on the path is
// symmetric, so the product equals the mathematical one bit for bit)
template <class R>
__host__ __device__ __forceinline__ mat2<R> matmul_ref(mat2<R> a, mat2<R> o) {
  return M<R>(a.xx * o.xx + a.xy * o.yx, a.xx * o.xy + a.xy * o.yy, a.yx * o.xx + a.yy * o.yx,
              a.yx * o.yx + a.yy * o.yy);
}
template <class R>
__host__ __device__ __forceinline__ mat2<R> dyad(vec2<R> a, vec2<R> b) {
  return M<R>(a.x * b.x, a.x * b.y, a.y * b.x, a.y * b.y);
}
template <class R>
__host__ __device__ __forceinline__ R det(mat2<R> a) {
  return a.xx * a.yy - a.xy * a.yx;
}
// matrix2d::inv (MathMatrix2d.h:137-140)
template <class R>
__host__ __device__ __forceinline__ mat2<R> inv(mat2<R> a) {
  return M<R>(a.yy, -a.xy, -a.yx, a.xx) / det(a);
}
// std::isnormal: finite, non-zero and not subnormal (false for NaN)
__host__ __device__ __forceinline__ bool is_normal(double x) {
  double a = fabs(x);
  return a >= 2.2250738585072014e-308 && a <= 1.7976931348623157e308;
}
// int abs(int) applied to a double, as the reference's matrix2d::eigen does
// (MathMatrix2d.h:122 is compiled where only int abs(int) is declared): the
// conversion truncates toward zero; NaN and out-of-range values become
// INT_MIN as on x86-64, and abs(INT_MIN) stays INT_MIN
__host__ __device__ __forceinline__ int trunc_abs(double x) {
  if (!(fabs(x) < 2147483648.0)) return (-2147483647 - 1);
  int i = (int)x;
  return i < 0 ? -i : i;
}
// std::min(a, b)
template <class R>
__host__ __device__ __forceinline__ R std_min(R a, R b) {
  return (b < a) ? b : a;
}

}  // namespace xdem
