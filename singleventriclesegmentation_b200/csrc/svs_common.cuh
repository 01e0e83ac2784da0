// Shared device helpers of libsvsflow: boundary folding, 1D Catmull-Rom, 3D sampling in the
// three interpolation modes, and host-side status handling.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "svsflow.h"

namespace svs {

// ------------------------------------------------------------------------------- host status
void set_error(const std::string& msg);
svs_status fail(svs_status code, const std::string& msg);
// Checks the launch that was just issued (cudaGetLastError) and counts it.
svs_status check_launch(const char* what, uint64_t launches = 1);
svs_status check_cuda(cudaError_t e, const char* what);
void count_launches(uint64_t n);

#define SVS_REQUIRE(cond, msg)                                              \
  do {                                                                      \
    if (!(cond)) return ::svs::fail(SVS_ERR_INVALID_ARG, std::string(msg)); \
  } while (0)

inline unsigned ceil_div(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

// ----------------------------------------------------------------------------- device helpers

// Index folding of boundary.cuh:25-46 (a single fold), followed by a clamp so that no sample is
// ever read outside the array: the reference reads out of bounds when a sample lies more than
// one volume length outside (boundary.cuh:33-46). The fold is a switch, not the reference's
// device function-pointer table (boundary.cuh:54), so it inlines.
__device__ __forceinline__ int fold(int i, int n, int bdry) {
  int f;
  if (bdry == SVS_BOUNDARY_MIRROR) f = i < 0 ? -i - 1 : (i > n - 1 ? 2 * n - 1 - i : i);
  else if (bdry == SVS_BOUNDARY_NEAREST) f = i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
  else f = i < 0 ? -i : (i > n - 1 ? 2 * n - 2 - i : i);
  return min(max(f, 0), n - 1);
}

// The helpers below are templates on the value type T (float, or double for the FP64 forms of
// the per-operator entry points); the float instantiations are the arithmetic of the reference's
// float path.
__device__ __forceinline__ float tfloor(float v) { return floorf(v); }
__device__ __forceinline__ double tfloor(double v) { return floor(v); }

// 1D Catmull-Rom through 4 samples in the reference's coefficient form
// (interpolation_cubicHermiteSpline.cuh:20-56), evaluated at buffer coordinate w + 1.
template <typename T>
__device__ __forceinline__ T hermite4(T b0, T b1, T b2, T b3, T w) {
  const T local = w + T(1);
  const int kf = (int)tfloor(local);
  T out;
  if (kf == 1) {
    const T pf = b1, dpf = (b2 - b0) / 2, pc = b2, dpc = (b3 - b1) / 2;
    const T a = 2 * pf - 2 * pc + dpf + dpc;
    const T b = -3 * pf + 3 * pc - 2 * dpf - dpc;
    const T t = local - T(1);
    out = t * (t * (t * a + b) + dpf) + pf;
  } else {
    // w + 1 rounded up to 2.0 (w within half an ulp of 1): the reference then shifts its
    // window by one and reads a zero past the buffer end; at t = 0 this returns b2.
    const T pf = b2, dpf = (b3 - b1) / 2, pc = b3, dpc = (T(0) - b2) / 2;
    const T a = 2 * pf - 2 * pc + dpf + dpc;
    const T b = -3 * pf + 3 * pc - 2 * dpf - dpc;
    const T t = local - T(2);
    out = t * (t * (t * a + b) + dpf) + pf;
  }
  return out;
}

// Strided accessor of one component of a [NZ,NY,NX,stride] field.
template <typename T>
struct FieldRefT {
  const T* __restrict__ p;
  int nz, ny, nx, stride;
  __device__ __forceinline__ T at(int z, int y, int x) const {
    return __ldg(p + ((size_t)((size_t)z * ny + y) * nx + x) * stride);
  }
};
using FieldRef = FieldRefT<float>;

// Grid coordinate -> (floor index, fraction), the reference's floorf(c/h) and c/h - floor.
template <typename T>
__device__ __forceinline__ void split_coord(T c, T h, int& i, T& w) {
  const T g = c / h;
  i = (int)tfloor(g);
  w = g - (T)i;
}

// Tricubic sample (interpolation_cubicHermiteSpline.cuh:482-525, and the vector/matrix/CNN
// variants :645-791 that differ only in addressing).
template <typename T>
__device__ __forceinline__ T sample_cubic(const FieldRefT<T>& f, T cz, T cy, T cx, T hz, T hy, T hx, int bdry) {
  int ix, iy, iz;
  T wx, wy, wz;
  split_coord(cx, hx, ix, wx);
  split_coord(cy, hy, iy, wy);
  split_coord(cz, hz, iz, wz);
  int xs[4];
#pragma unroll
  for (int d = 0; d < 4; ++d) xs[d] = fold(ix + d - 1, f.nx, bdry);
  T bz[4];
#pragma unroll
  for (int dz = 0; dz < 4; ++dz) {
    const int zz = fold(iz + dz - 1, f.nz, bdry);
    T by[4];
#pragma unroll
    for (int dy = 0; dy < 4; ++dy) {
      const int yy = fold(iy + dy - 1, f.ny, bdry);
      by[dy] = hermite4(f.at(zz, yy, xs[0]), f.at(zz, yy, xs[1]), f.at(zz, yy, xs[2]), f.at(zz, yy, xs[3]), wx);
    }
    bz[dz] = hermite4(by[0], by[1], by[2], by[3], wy);
  }
  return hermite4(bz[0], bz[1], bz[2], bz[3], wz);
}

// Trilinear sample, interpolation_linear.cuh:250-295 (the 8 terms in the reference's order).
template <typename T>
__device__ __forceinline__ T sample_linear(const FieldRefT<T>& f, T cz, T cy, T cx, T hz, T hy, T hx, int bdry) {
  int ix, iy, iz;
  T wx, wy, wz;
  split_coord(cx, hx, ix, wx);
  split_coord(cy, hy, iy, wy);
  split_coord(cz, hz, iz, wz);
  const int x0 = fold(ix, f.nx, bdry), x1 = fold(ix + 1, f.nx, bdry);
  const int y0 = fold(iy, f.ny, bdry), y1 = fold(iy + 1, f.ny, bdry);
  const int z0 = fold(iz, f.nz, bdry), z1 = fold(iz + 1, f.nz, bdry);
  T out = (1 - wz) * (1 - wy) * (1 - wx) * f.at(z0, y0, x0);
  out += wz * (1 - wy) * (1 - wx) * f.at(z1, y0, x0);
  out += (1 - wz) * (1 - wy) * wx * f.at(z0, y0, x1);
  out += wz * (1 - wy) * wx * f.at(z1, y0, x1);
  out += (1 - wz) * wy * (1 - wx) * f.at(z0, y1, x0);
  out += wz * wy * (1 - wx) * f.at(z1, y1, x0);
  out += (1 - wz) * wy * wx * f.at(z0, y1, x1);
  out += wz * wy * wx * f.at(z1, y1, x1);
  return out;
}

// Nearest-node sample, interpolation_nearest.cuh:250-294 (ties go to the ceiling node).
template <typename T>
__device__ __forceinline__ int nearest_axis(T c, T h, int n, int bdry) {
  const T g = c / h;
  const int f = (int)tfloor(g);
  const T df = g - (T)f;
  const T dc = (T)(f + 1) - g;
  return fold(df < dc ? f : f + 1, n, bdry);
}
template <typename T>
__device__ __forceinline__ T sample_nearest(const FieldRefT<T>& f, T cz, T cy, T cx, T hz, T hy, T hx, int bdry) {
  return f.at(nearest_axis(cz, hz, f.nz, bdry), nearest_axis(cy, hy, f.ny, bdry), nearest_axis(cx, hx, f.nx, bdry));
}

template <typename T>
__device__ __forceinline__ T sample(const FieldRefT<T>& f, T cz, T cy, T cx, T hz, T hy, T hx, int interp, int bdry) {
  if (interp == SVS_INTERPOLATE_CUBIC_HERMITESPLINE) return sample_cubic(f, cz, cy, cx, hz, hy, hx, bdry);
  if (interp == SVS_INTERPOLATE_LINEAR) return sample_linear(f, cz, cy, cx, hz, hy, hx, bdry);
  return sample_nearest(f, cz, cy, cx, hz, hy, hx, bdry);
}

// Forward difference along one axis (differentialOps.cu:540-655): MIRROR is zero on both
// faces, NEAREST and REFLECT take one-sided half differences there. The reference evaluates
// 0.5*(a-b)/h in double (0.5 is a double literal) and rounds to float; 0.5f*(a-b) is exact, so
// the float quotient below is the same correctly rounded value (barring double-rounding ties).
template <typename T>
__device__ __forceinline__ T fwd_axis(T prev, T cur, T next, int i, int n, int bdry, T h) {
  T d;
  if (bdry == SVS_BOUNDARY_MIRROR) {
    if (i > 0 && i < n - 1) d = next - prev;
    else return T(0);
  } else {
    d = (i > 0) ? ((i < n - 1) ? next - prev : cur - prev) : next - cur;
  }
  return (T(0.5) * d) / h;
}

// Adjoint difference along one axis (differentialOps.cu:658-1039), rounded to T per axis.
template <typename T>
__device__ __forceinline__ T adj_axis(T prev, T cur, T next, int i, int n, int bdry) {
  if (bdry == SVS_BOUNDARY_MIRROR) {
    if (i > 1) return (i < n - 2) ? T(0.5) * (prev - next) : T(0.5) * prev;
    return T(-0.5) * next;
  }
  if (i > 0) return (i < n - 1) ? T(0.5) * (prev - next) : T(0.5) * (prev + cur);
  return T(0.5) * (-cur - next);
}

}  // namespace svs
