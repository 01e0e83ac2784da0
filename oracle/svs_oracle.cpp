// Oracle: a CPU restatement (C++17 / OpenMP) of the reference's 3D TV-L1 optical-flow path and
// of its tricubic mask propagation. TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check
// and the CPU-baseline leg of the bench call it as the checker. The product never links it.
//
// Every function names the reference file:line it restates (paths relative to the reference
// project root). Each operator is templated on the scalar type: the float instantiation follows
// the reference's float evaluation order (this file is compiled with -ffp-contract=off, so no
// multiply-add is fused behind the source's back); the double instantiation is a true-double
// oracle (double sqrt/exp/pow/floor instead of the reference's float intrinsics).
//
// Parity pinning: the reference has no tests and no golden vectors. This oracle is pinned by
// fixtures produced by the reference's own CUDA extension (built from its sources for sm_100a)
// on seeded inputs; see tests/golden/.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum { BDRY_NEAREST = 0, BDRY_MIRROR = 1, BDRY_REFLECT = 2 };
enum { INTERP_NEAREST = 0, INTERP_LINEAR = 1, INTERP_CUBIC = 2 };

// Index folding, boundary.cuh:25-46 (one fold only, exactly as the reference).
inline int fold(int i, int n, int bdry) {
  switch (bdry) {
    case BDRY_NEAREST: return i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
    case BDRY_MIRROR: return i < 0 ? -i - 1 : (i > n - 1 ? 2 * n - 1 - i : i);
    default: return i < 0 ? -i : (i > n - 1 ? 2 * n - 2 - i : i);
  }
}
// The oracle never reads outside the array: after the single fold it clamps. The reference
// reads out of bounds when a sample lies more than one volume length outside (boundary.cuh:33-46).
inline int fold_safe(int i, int n, int bdry) {
  int f = fold(i, n, bdry);
  return f < 0 ? 0 : (f > n - 1 ? n - 1 : f);
}

template <class T> inline T floor_t(T x) { return std::floor(x); }
template <> inline float floor_t<float>(float x) { return std::floor(x); }
template <class T> inline T sqrt_t(T x) { return std::sqrt(x); }
template <class T> inline T exp_t(T x) { return std::exp(x); }
template <class T> inline T pow_t(T x, T y) { return std::pow(x, y); }

// 1D Catmull-Rom on a 4-sample buffer, interpolation_cubicHermiteSpline.cuh:20-56.
// `local` is (w + 1) with w in [0,1): the reference evaluates at buffer coordinate w+1.
template <class T> inline T hermite_local(const T* buf, T local) {
  const int kf = (int)floor_t<T>(local);
  const int kc = kf + 1, kf1 = kf - 1, kc1 = kc + 1;
  T uf = (kf >= 0 && kf < 4) ? buf[kf] : T(0);
  T uf1 = (kf1 >= 0 && kf1 < 4) ? buf[kf1] : T(0);
  T uc = (kc >= 0 && kc < 4) ? buf[kc] : T(0);
  T uc1 = (kc1 >= 0 && kc1 < 4) ? buf[kc1] : T(0);
  const T pf = uf, dpf = (uc - uf1) / 2, pc = uc, dpc = (uc1 - uf) / 2;
  const T a = 2 * pf - 2 * pc + dpf + dpc;
  const T b = -3 * pf + 3 * pc - 2 * dpf - dpc;
  const T c = dpf, d = pf;
  const T w = local - (T)kf;
  return w * (w * (w * a + b) + c) + d;
}

// Strided view of one scalar component of a [NZ,NY,NX,C] field (C = 1 for a scalar field).
template <class T> struct Field {
  const T* p; int nz, ny, nx, stride, off;
  inline T at(int z, int y, int x) const {
    return p[(((size_t)z * ny + y) * nx + x) * stride + off];
  }
};

// Tricubic Hermite sample at grid coordinate (cz,cy,cx) given in physical units with spacings h,
// interpolation_cubicHermiteSpline.cuh:482-525 (scalar), :645-689 (vector), :695-739 (matrix),
// :747-791 (CNN): all four share this arithmetic and differ only in addressing.
template <class T>
T sample_cubic(const Field<T>& f, T cz, T cy, T cx, float hz, float hy, float hx, int bdry) {
  const T gx = cx / (T)hx, gy = cy / (T)hy, gz = cz / (T)hz;
  const int ixf = (int)floor_t<T>(gx), iyf = (int)floor_t<T>(gy), izf = (int)floor_t<T>(gz);
  const T wx = gx - (T)ixf, wy = gy - (T)iyf, wz = gz - (T)izf;
  T bz[4], by[4], bx[4];
  for (int dz = -1; dz < 3; ++dz) {
    const int zz = fold_safe(izf + dz, f.nz, bdry);
    for (int dy = -1; dy < 3; ++dy) {
      const int yy = fold_safe(iyf + dy, f.ny, bdry);
      for (int dx = -1; dx < 3; ++dx) bx[dx + 1] = f.at(zz, yy, fold_safe(ixf + dx, f.nx, bdry));
      by[dy + 1] = hermite_local<T>(bx, wx + 1);
    }
    bz[dz + 1] = hermite_local<T>(by, wy + 1);
  }
  return hermite_local<T>(bz, wz + 1);
}

// Trilinear sample, interpolation_linear.cuh:250-295 (scalar; the vector, matrix and CNN
// variants at :369-515 share the arithmetic): the 8 corner terms are accumulated in the
// reference's order (fff, z, x, xz, y, yz, xy, xyz).
template <class T>
T sample_linear(const Field<T>& f, T cz, T cy, T cx, float hz, float hy, float hx, int bdry) {
  const T gx = cx / (T)hx, gy = cy / (T)hy, gz = cz / (T)hz;
  const int ixf = (int)floor_t<T>(gx), iyf = (int)floor_t<T>(gy), izf = (int)floor_t<T>(gz);
  const T wx = gx - (T)ixf, wy = gy - (T)iyf, wz = gz - (T)izf;
  const int x0 = fold_safe(ixf, f.nx, bdry), x1 = fold_safe(ixf + 1, f.nx, bdry);
  const int y0 = fold_safe(iyf, f.ny, bdry), y1 = fold_safe(iyf + 1, f.ny, bdry);
  const int z0 = fold_safe(izf, f.nz, bdry), z1 = fold_safe(izf + 1, f.nz, bdry);
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

// Nearest-node sample, interpolation_nearest.cuh:250-294: per axis, the floor node unless the
// ceiling node is strictly closer or equally close (ties go to the ceiling).
template <class T> inline int nearest_axis(T c, float h, int n, int bdry) {
  const T g = c / (T)h;
  const int f = (int)floor_t<T>(g);
  const float df = (float)(g - (T)f);
  const float dc = (float)((T)(f + 1) - g);
  return fold_safe(df < dc ? f : f + 1, n, bdry);
}
template <class T>
T sample_nearest(const Field<T>& f, T cz, T cy, T cx, float hz, float hy, float hx, int bdry) {
  return f.at(nearest_axis(cz, hz, f.nz, bdry), nearest_axis(cy, hy, f.ny, bdry),
              nearest_axis(cx, hx, f.nx, bdry));
}

template <class T>
inline T sample(const Field<T>& f, T cz, T cy, T cx, float hz, float hy, float hx, int interp,
                int bdry) {
  if (interp == INTERP_CUBIC) return sample_cubic(f, cz, cy, cx, hz, hy, hx, bdry);
  if (interp == INTERP_LINEAR) return sample_linear(f, cz, cy, cx, hz, hy, hx, bdry);
  return sample_nearest(f, cz, cy, cx, hz, hy, hx, bdry);
}

inline size_t vox(int nz, int ny, int nx) { return (size_t)nz * ny * nx; }

// ---------------------------------------------------------------------------------------------
// Central-difference gradient and its adjoint ("backward"), differentialOps.cu:540-1039.
// The reference evaluates each difference as a double expression (0.5 is a double literal) and
// rounds the result to the field type; the forward divides by h in double, the adjoint divides
// the rounded per-axis term by h in the field type and sums x + y + z left to right.
// ---------------------------------------------------------------------------------------------

// One axis of the forward gradient at index i along an axis of length n and stride s.
// MIRROR (differentialOps.cu:579-615, :824-863): zero on both faces.
// NEAREST and REFLECT (:540-576, :619-655, :782-822, :866-907): one-sided half differences.
template <class T> inline T fwd_axis(const T* q, ptrdiff_t s, int i, int n, int bdry, float h) {
  if (bdry == BDRY_MIRROR) {
    if (i > 0 && i < n - 1) return (T)(0.5 * (double)(q[s] - q[-s]) / (double)h);
    return T(0);
  }
  if (i > 0) {
    if (i < n - 1) return (T)(0.5 * (double)(q[s] - q[-s]) / (double)h);
    return (T)(0.5 * (double)(q[0] - q[-s]) / (double)h);
  }
  return (T)(0.5 * (double)(q[s] - q[0]) / (double)h);
}

// One axis of the adjoint at index i.
// MIRROR (:699-737, :953-994): i>1 && i<N-2: 0.5(p[i-1]-p[i+1]); i>1: 0.5 p[i-1]; else -0.5 p[i+1].
// NEAREST and REFLECT (:658-697, :741-779, :909-951, :998-1039):
//   0<i<N-1: 0.5(p[i-1]-p[i+1]); i=N-1: 0.5(p[i-1]+p[i]); i=0: 0.5(-p[i]-p[i+1]).
template <class T> inline T adj_axis(const T* q, ptrdiff_t s, int i, int n, int bdry) {
  if (bdry == BDRY_MIRROR) {
    if (i > 1) {
      if (i < n - 2) return (T)(0.5 * (double)(q[-s] - q[s]));
      return (T)(0.5 * (double)q[-s]);
    }
    return (T)(-0.5 * (double)q[s]);
  }
  if (i > 0) {
    if (i < n - 1) return (T)(0.5 * (double)(q[-s] - q[s]));
    return (T)(0.5 * (double)(q[-s] + q[0]));
  }
  return (T)(0.5 * (double)(-q[0] - q[s]));
}

// Gradient of each component of a C-component field: in [Z,Y,X,C] -> out [Z,Y,X,C,3],
// components (d/dx, d/dy, d/dz). C = 1 is the scalar gradient (out [Z,Y,X,3]).
template <class T>
void nabla_fwd_vf(const T* b, int nz, int ny, int nx, int C, float hz, float hy, float hx,
                  int bdry, T* out) {
  const ptrdiff_t sx = C, sy = (ptrdiff_t)nx * C, sz = (ptrdiff_t)nx * ny * C;
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const size_t i = (((size_t)z * ny + y) * nx + x) * C;
        for (int c = 0; c < C; ++c) {
          const T* q = b + i + c;
          T* o = out + (i + c) * 3;
          o[0] = fwd_axis(q, sx, x, nx, bdry, hx);
          o[1] = fwd_axis(q, sy, y, ny, bdry, hy);
          o[2] = fwd_axis(q, sz, z, nz, bdry, hz);
        }
      }
}

// Adjoint for a C x 3 field: in [Z,Y,X,C,3] -> out [Z,Y,X,C]. C = 1 is the scalar adjoint.
template <class T>
void nabla_bwd_vf(const T* p, int nz, int ny, int nx, int C, float hz, float hy, float hx,
                  int bdry, T* out) {
  const ptrdiff_t sx = 3 * C, sy = (ptrdiff_t)nx * 3 * C, sz = (ptrdiff_t)nx * ny * 3 * C;
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const size_t i = ((size_t)z * ny + y) * nx + x;
        for (int c = 0; c < C; ++c) {
          const T* q = p + (i * C + c) * 3;
          const T dx = adj_axis(q + 0, sx, x, nx, bdry), dy = adj_axis(q + 1, sy, y, ny, bdry),
                  dz = adj_axis(q + 2, sz, z, nz, bdry);
          out[i * C + c] = dx / (T)hx + dy / (T)hy + dz / (T)hz;
        }
      }
}

// ---------------------------------------------------------------------------------------------
// Anisotropic operator, anisotropicDifferentialOps.cu:89-175.
// ---------------------------------------------------------------------------------------------
template <class T>
void aniso_tangents(const T* g, size_t n, float alpha, float beta, T* s, T* nrm, T* t1, T* t2) {
#pragma omp parallel for schedule(static)
  for (ptrdiff_t i = 0; i < (ptrdiff_t)n; ++i) {
    const T* gi = g + 3 * i;
    T nsq = 0;
    for (int d = 0; d < 3; ++d) nsq += gi[d] * gi[d];
    const T norm = sqrt_t<T>(nsq);
    T* ni = nrm + 3 * i; T* a = t1 + 3 * i; T* b = t2 + 3 * i;
    if (norm > 0) {
      s[i] = exp_t<T>(-(T)alpha * pow_t<T>(norm, (T)beta));
      for (int d = 0; d < 3; ++d) ni[d] = gi[d] / norm;
      if (ni[2] > 0.5) { a[0] = ni[2]; a[1] = 0; a[2] = -ni[0]; }
      else { a[0] = ni[1]; a[1] = -ni[0]; a[2] = 0; }
      b[0] = ni[1] * a[2] - ni[2] * a[1];
      b[1] = ni[2] * a[0] - ni[0] * a[2];
      b[2] = ni[0] * a[1] - ni[1] * a[0];
    } else {
      s[i] = 0;
      for (int d = 0; d < 3; ++d) { ni[d] = 0; a[d] = 0; b[d] = 0; }
    }
  }
}

// out[c][d] = s*(n.in_c)*n[d] + (t1.in_c)*t1[d]; the reference's t2 term carries a factor that is
// never accumulated (tangent2Fac = 0, anisotropicDifferentialOps.cu:160-172) and adds nothing.
template <class T>
void aniso_apply(const T* in, size_t n, const T* s, const T* nrm, const T* t1, T* out) {
#pragma omp parallel for schedule(static)
  for (ptrdiff_t i = 0; i < (ptrdiff_t)n; ++i) {
    const T* ni = nrm + 3 * i; const T* a = t1 + 3 * i;
    for (int c = 0; c < 3; ++c) {
      const T* g = in + 9 * i + 3 * c;
      T nf = 0, tf = 0;
      for (int d = 0; d < 3; ++d) { nf += ni[d] * g[d]; tf += a[d] * g[d]; }
      T* o = out + 9 * i + 3 * c;
      for (int d = 0; d < 3; ++d) {
        T v = s[i] * nf * ni[d];
        v += tf * a[d];
        o[d] = v;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Proximal operators, opticalFlowOps.cu:123-175 (primal) and :179-208 (dual).
// ---------------------------------------------------------------------------------------------
template <class T>
void prox_primal(const T* pv, size_t n, float tau, float lam, const T* rho, const T* g, T* out) {
  const float factor = tau * lam;  // opticalFlowOps.cu:440
#pragma omp parallel for schedule(static)
  for (ptrdiff_t i = 0; i < (ptrdiff_t)n; ++i) {
    const T r = rho[i];
    const T* gi = g + 3 * i;
    T g2 = 0;
    for (int c = 0; c < 3; ++c) g2 += gi[c] * gi[c];
    T delta[3];
    if (r < -(T)factor * g2) { for (int c = 0; c < 3; ++c) delta[c] = (T)factor * gi[c]; }
    else if (r > (T)factor * g2) { for (int c = 0; c < 3; ++c) delta[c] = -(T)factor * gi[c]; }
    else if ((double)g2 > 1e-10) { for (int c = 0; c < 3; ++c) delta[c] = -r * gi[c] / g2; }
    else { for (int c = 0; c < 3; ++c) delta[c] = 0; }
    for (int c = 0; c < 3; ++c) out[3 * i + c] = pv[3 * i + c] + delta[c];
  }
}

template <class T> void prox_dual(const T* dv, size_t n, float wtv, T* out) {
#pragma omp parallel for schedule(static)
  for (ptrdiff_t i = 0; i < (ptrdiff_t)n; ++i) {
    for (int c = 0; c < 3; ++c) {
      const T* q = dv + 9 * i + 3 * c;
      T nsq = 0;
      for (int d = 0; d < 3; ++d) nsq += q[d] * q[d];
      const T den = std::max(T(1), sqrt_t<T>(nsq) / (T)wtv);
      for (int d = 0; d < 3; ++d) out[9 * i + 3 * c + d] = q[d] / den;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Warping and resampling.
// ---------------------------------------------------------------------------------------------

// I(x + phi(x)) for a C-component field, warpingOps.cu:572-596 (C=1) and :632-660.
template <class T>
void warp_field(const T* u, int nz, int ny, int nx, int C, const T* phi, float hz, float hy,
                float hx, int interp, int bdry, T* out) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const size_t i = ((size_t)z * ny + y) * nx + x;
        const T cx = (T)x * (T)hx + phi[3 * i + 0];
        const T cy = (T)y * (T)hy + phi[3 * i + 1];
        const T cz = (T)z * (T)hz + phi[3 * i + 2];
        for (int c = 0; c < C; ++c) {
          Field<T> f{u, nz, ny, nx, C, c};
          out[i * C + c] = sample<T>(f, cz, cy, cx, hz, hy, hx, interp, bdry);
        }
      }
}


// Warping3D.backward (warpingOps.cu:598-630 cubic, :384-412 trilinear, :172-200 nearest):
// grad_u[j] += grad_out(v) * weight_j(v) on the folded stencil node j; grad_phi(v) =
// grad_out(v) * d interpolant / d coordinate / h (interpolation_cubicHermiteSpline.cuh:527-636,
// interpolation_linear.cuh:298-366, interpolation_nearest.cuh:296-356). Sequential (the
// scatter is a sum; a sequential order makes the oracle deterministic).
template <class T> inline void cr_weights(T w, T W[4]) {
  const T w2 = w * w, w3 = w2 * w;
  W[0] = -w3 / 2 + w2 - w / 2;
  W[1] = (3 * w3) / 2 - (5 * w2) / 2 + 1;
  W[2] = -(3 * w3) / 2 + 2 * w2 + w / 2;
  W[3] = w3 / 2 - w2 / 2;
}
template <class T> inline T cr_dvalue(const T* b, T w) {
  const T pf = b[1], dpf = (b[2] - b[0]) / 2, pc = b[2], dpc = (b[3] - b[1]) / 2;
  const T a = 2 * pf - 2 * pc + dpf + dpc;
  const T bb = -3 * pf + 3 * pc - 2 * dpf - dpc;
  return 3 * w * w * a + 2 * bb * w + dpf;
}
template <class T>
void warp_backward(const T* u, int nz, int ny, int nx, const T* phi, const T* gout, float hz,
                   float hy, float hx, int interp, int bdry, T* grad_u, T* grad_phi) {
  const size_t n = vox(nz, ny, nx);
  std::fill(grad_u, grad_u + n, T(0));
  Field<T> f{u, nz, ny, nx, 1, 0};
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const size_t v = ((size_t)z * ny + y) * nx + x;
        const T cx = (T)x * (T)hx + phi[3 * v], cy = (T)y * (T)hy + phi[3 * v + 1],
                cz = (T)z * (T)hz + phi[3 * v + 2];
        const T g = gout[v];
        T gpx = 0, gpy = 0, gpz = 0;
        const T gx = cx / (T)hx, gy = cy / (T)hy, gz = cz / (T)hz;
        const int ixf = (int)floor_t<T>(gx), iyf = (int)floor_t<T>(gy), izf = (int)floor_t<T>(gz);
        T wx = gx - (T)ixf, wy = gy - (T)iyf, wz = gz - (T)izf;
        if (interp == INTERP_CUBIC) {
          wx = (wx + 1) - 1; wy = (wy + 1) - 1; wz = (wz + 1) - 1;
          T Wx[4], Wy[4], Wz[4];
          cr_weights(wx, Wx); cr_weights(wy, Wy); cr_weights(wz, Wz);
          T bz[4];
          for (int dz = 0; dz < 4; ++dz) {
            const int zz = fold_safe(izf + dz - 1, nz, bdry);
            T by[4];
            for (int dy = 0; dy < 4; ++dy) {
              const int yy = fold_safe(iyf + dy - 1, ny, bdry);
              T r[4];
              int xs[4];
              for (int dx = 0; dx < 4; ++dx) { xs[dx] = fold_safe(ixf + dx - 1, nx, bdry); r[dx] = f.at(zz, yy, xs[dx]); }
              by[dy] = hermite_local<T>(r, wx + 1);
              const T gzy = g * Wz[dz] * Wy[dy];
              gpx += cr_dvalue(r, wx) * gzy;
              for (int dx = 0; dx < 4; ++dx) grad_u[((size_t)zz * ny + yy) * nx + xs[dx]] += Wx[dx] * gzy;
            }
            bz[dz] = hermite_local<T>(by, wy + 1);
            gpy += cr_dvalue(by, wy) * (g * Wz[dz]);
          }
          gpz = cr_dvalue(bz, wz) * g;
          gpx /= (T)hx; gpy /= (T)hy; gpz /= (T)hz;
        } else if (interp == INTERP_LINEAR) {
          const int x0 = fold_safe(ixf, nx, bdry), x1 = fold_safe(ixf + 1, nx, bdry);
          const int y0 = fold_safe(iyf, ny, bdry), y1 = fold_safe(iyf + 1, ny, bdry);
          const int z0 = fold_safe(izf, nz, bdry), z1 = fold_safe(izf + 1, nz, bdry);
          const T fff = f.at(z0, y0, x0), ffc = f.at(z1, y0, x0), fcf = f.at(z0, y1, x0),
                  fcc = f.at(z1, y1, x0), cff = f.at(z0, y0, x1), cfc = f.at(z1, y0, x1),
                  ccf = f.at(z0, y1, x1), ccc = f.at(z1, y1, x1);
          auto add = [&](int zz, int yy, int xx, T w) { grad_u[((size_t)zz * ny + yy) * nx + xx] += w * g; };
          add(z0, y0, x0, (1 - wz) * (1 - wy) * (1 - wx));
          add(z0, y1, x0, (1 - wz) * wy * (1 - wx));
          add(z0, y0, x1, (1 - wz) * (1 - wy) * wx);
          add(z0, y1, x1, (1 - wz) * wy * wx);
          add(z1, y0, x0, wz * (1 - wy) * (1 - wx));
          add(z1, y1, x0, wz * wy * (1 - wx));
          add(z1, y0, x1, wz * (1 - wy) * wx);
          add(z1, y1, x1, wz * wy * wx);
          gpx = ((1 - wz) * (1 - wy) * (cff - fff) + (1 - wz) * wy * (ccf - fcf) + wz * (1 - wy) * (cfc - ffc) + wz * wy * (ccc - fcc)) / (T)hx * g;
          gpy = ((1 - wz) * (1 - wx) * (fcf - fff) + (1 - wz) * wx * (ccf - cff) + wz * (1 - wx) * (fcc - ffc) + wz * wx * (ccc - cfc)) / (T)hy * g;
          gpz = ((1 - wy) * (1 - wx) * (ffc - fff) + (1 - wy) * wx * (cfc - cff) + wy * (1 - wx) * (fcc - fcf) + wy * wx * (ccc - ccf)) / (T)hz * g;
        } else {
          const int xx = nearest_axis(cx, hx, nx, bdry), yy = nearest_axis(cy, hy, ny, bdry),
                    zz = nearest_axis(cz, hz, nz, bdry);
          grad_u[((size_t)zz * ny + yy) * nx + xx] += g;
        }
        grad_phi[3 * v] = gpx; grad_phi[3 * v + 1] = gpy; grad_phi[3 * v + 2] = gpz;
      }
}

// Resampling between meshes (restriction and prolongation), prolongationOps.cu:533-625:
// target node i maps to source coordinate (i*h_t)*L_s/L_t.
template <class T>
void prolongate(const T* u, int nz, int ny, int nx, int C, float lz, float ly, float lx, int tz,
                int ty, int tx, float tlz, float tly, float tlx, int interp, int bdry, T* out) {
  const float hz = lz / (nz - 1), hy = ly / (ny - 1), hx = lx / (nx - 1);
  const float thz = tlz / (tz - 1), thy = tly / (ty - 1), thx = tlx / (tx - 1);
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < tz; ++z)
    for (int y = 0; y < ty; ++y)
      for (int x = 0; x < tx; ++x) {
        const T cx = (T)x * (T)thx * (T)lx / (T)tlx;
        const T cy = (T)y * (T)thy * (T)ly / (T)tly;
        const T cz = (T)z * (T)thz * (T)lz / (T)tlz;
        const size_t i = ((size_t)z * ty + y) * tx + x;
        for (int c = 0; c < C; ++c) {
          Field<T> f{u, nz, ny, nx, C, c};
          out[i * C + c] = sample<T>(f, cz, cy, cx, hz, hy, hx, interp, bdry);
        }
      }
}

// Batched volume warp for masks, warpingOpsCNN.cu:97-128: m [B,C,Z,Y,X], phi [B,Z,Y,X,3].
template <class T>
void warp_cnn(const T* m, int B, int C, int nz, int ny, int nx, const T* phi, float hz, float hy,
              float hx, int interp, int bdry, T* out) {
  const size_t nv = vox(nz, ny, nx);
  for (int b = 0; b < B; ++b) {
    const T* ph = phi + (size_t)b * nv * 3;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
          const size_t i = ((size_t)z * ny + y) * nx + x;
          const T cx = (T)x * (T)hx + ph[3 * i + 0];
          const T cy = (T)y * (T)hy + ph[3 * i + 1];
          const T cz = (T)z * (T)hz + ph[3 * i + 2];
          for (int c = 0; c < C; ++c) {
            Field<T> f{m + ((size_t)b * C + c) * nv, nz, ny, nx, 1, 0};
            out[((size_t)b * C + c) * nv + i] = sample<T>(f, cz, cy, cx, hz, hy, hx, interp, bdry);
          }
        }
  }
}

// ---------------------------------------------------------------------------------------------
// Pre/post filters, svs/utils/flow_utils.py.
// ---------------------------------------------------------------------------------------------

// 3D convolution with a (2r+1)^3 kernel and zero padding r, flow_utils.py:94-112 (F.conv3d).
// The kernel weights are passed in (computed by the caller exactly as flow_utils.py:74-91 does).
template <class T>
void conv3d_zero(const T* in, int nz, int ny, int nx, const float* w, int r, T* out) {
  const int k = 2 * r + 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        double acc = 0;
        for (int a = 0; a < k; ++a) {
          const int zz = z + a - r; if (zz < 0 || zz >= nz) continue;
          for (int b = 0; b < k; ++b) {
            const int yy = y + b - r; if (yy < 0 || yy >= ny) continue;
            for (int c = 0; c < k; ++c) {
              const int xx = x + c - r; if (xx < 0 || xx >= nx) continue;
              acc += (double)w[(a * k + b) * k + c] * (double)in[((size_t)zz * ny + yy) * nx + xx];
            }
          }
        }
        out[((size_t)z * ny + y) * nx + x] = (T)acc;
      }
}

// ks^3 median per component of a [Z,Y,X,C] field with scipy's 'reflect' mode (half-sample
// symmetric = MIRROR fold), flow_utils.py:115-132 (scipy.ndimage.median_filter, size
// (ks,ks,ks,1)): the value of rank ks^3//2 among the window.
template <class T>
void median3(const T* in, int nz, int ny, int nx, int C, int ks, T* out) {
  const int r = ks / 2, n = ks * ks * ks;
#pragma omp parallel
  {
    std::vector<T> win(n);
#pragma omp for collapse(2) schedule(static)
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
          for (int c = 0; c < C; ++c) {
            int m = 0;
            for (int a = -r; a <= r; ++a)
              for (int b = -r; b <= r; ++b)
                for (int d = -r; d <= r; ++d) {
                  const int zz = fold_safe(z + a, nz, BDRY_MIRROR);
                  const int yy = fold_safe(y + b, ny, BDRY_MIRROR);
                  const int xx = fold_safe(x + d, nx, BDRY_MIRROR);
                  win[m++] = in[(((size_t)zz * ny + yy) * nx + xx) * C + c];
                }
            std::nth_element(win.begin(), win.begin() + n / 2, win.end());
            out[(((size_t)z * ny + y) * nx + x) * C + c] = win[n / 2];
          }
  }
}

}  // namespace

// =============================================================================================
// Solver driver: svs/modules/flow/tvl13d.py:69-255.
// =============================================================================================
extern "C" {

struct svso_params {
  int num_scales, max_warps, max_iters;
  float weight_matching, weight_tv;
  int pd_type;  // 1 or 2
  double sigma, tau, theta, gamma;
  int use_aniso; float alpha, beta;
  int use_blur; float blur_sigma;
  int interp, bdry;
  int length_type;  // 0 = numDofs (L = N-1), 1 = fixed
  float len_z, len_y, len_x;
};
}

namespace {

struct Mesh { int nz, ny, nx; float lz, ly, lx, hz, hy, hx; };

Mesh make_mesh(const svso_params& P, int nz, int ny, int nx) {
  Mesh m{nz, ny, nx, 0, 0, 0, 0, 0, 0};
  if (P.length_type == 0) { m.lz = (float)(nz - 1); m.ly = (float)(ny - 1); m.lx = (float)(nx - 1); }
  else { m.lz = P.len_z; m.ly = P.len_y; m.lx = P.len_x; }
  // coreDefines.h:72-75: h = L / (N - 1) in float
  m.hz = m.lz / (nz - 1); m.hy = m.ly / (ny - 1); m.hx = m.lx / (nx - 1);
  return m;
}

// One pyramid level, tvl13d.py:164-255.
template <class T>
void solve_level(const svso_params& P, const Mesh& M, const T* I0, const T* I1, std::vector<T>& u,
                 std::vector<T>& p) {
  const size_t n = vox(M.nz, M.ny, M.nx);
  std::vector<T> g(3 * n), s(n, 0), nrm(3 * n, 0), t1(3 * n, 0), t2(3 * n, 0);
  nabla_fwd_vf<T>(I1, M.nz, M.ny, M.nx, 1, M.hz, M.hy, M.hx, P.bdry, g.data());
  if (P.use_aniso) aniso_tangents<T>(g.data(), n, P.alpha, P.beta, s.data(), nrm.data(), t1.data(), t2.data());
  std::vector<T> I1w(n), gw(3 * n), rho_c(n), rho(n), zg(9 * n), Dz(9 * n), dv(9 * n), Dp(9 * n),
      div(3 * n), pv(3 * n);
  for (int w = 0; w < P.max_warps; ++w) {
    warp_field<T>(I1, M.nz, M.ny, M.nx, 1, u.data(), M.hz, M.hy, M.hx, P.interp, P.bdry, I1w.data());
    warp_field<T>(g.data(), M.nz, M.ny, M.nx, 3, u.data(), M.hz, M.hy, M.hx, P.interp, P.bdry, gw.data());
    // rho_c = I1w - sum(u * gw, dim=3) - I0   (tvl13d.py:201)
#pragma omp parallel for schedule(static)
    for (ptrdiff_t i = 0; i < (ptrdiff_t)n; ++i) {
      const T sum = u[3 * i] * gw[3 * i] + u[3 * i + 1] * gw[3 * i + 1] + u[3 * i + 2] * gw[3 * i + 2];
      rho_c[i] = I1w[i] - sum - I0[i];
    }
    double sigma = P.sigma, tau = P.tau, gamma = P.gamma;  // reset per warp, tvl13d.py:208-211
    for (int it = 0; it < P.max_iters; ++it) {
      // dual step, tvl13d.py:215-224 (z = u: no over-relaxation)
      nabla_fwd_vf<T>(u.data(), M.nz, M.ny, M.nx, 3, M.hz, M.hy, M.hx, P.bdry, zg.data());
      const T* Dzp = zg.data();
      if (P.use_aniso) { aniso_apply<T>(zg.data(), n, s.data(), nrm.data(), t1.data(), Dz.data()); Dzp = Dz.data(); }
      const T sg = (T)(float)sigma;
#pragma omp parallel for schedule(static)
      for (ptrdiff_t i = 0; i < (ptrdiff_t)(9 * n); ++i) dv[i] = p[i] + sg * Dzp[i];
      prox_dual<T>(dv.data(), n, P.weight_tv, p.data());
      if (P.weight_tv == 0.f) std::fill(p.begin(), p.end(), T(0));
      // primal step, tvl13d.py:226-237
#pragma omp parallel for schedule(static)
      for (ptrdiff_t i = 0; i < (ptrdiff_t)n; ++i) {
        const T sum = u[3 * i] * gw[3 * i] + u[3 * i + 1] * gw[3 * i + 1] + u[3 * i + 2] * gw[3 * i + 2];
        rho[i] = rho_c[i] + sum;
      }
      const T* Dpp = p.data();
      if (P.use_aniso) { aniso_apply<T>(p.data(), n, s.data(), nrm.data(), t1.data(), Dp.data()); Dpp = Dp.data(); }
      nabla_bwd_vf<T>(Dpp, M.nz, M.ny, M.nx, 3, M.hz, M.hy, M.hx, P.bdry, div.data());
      const T tf = (T)(float)tau;
#pragma omp parallel for schedule(static)
      for (ptrdiff_t i = 0; i < (ptrdiff_t)(3 * n); ++i) pv[i] = u[i] - tf * div[i];
      prox_primal<T>(pv.data(), n, (float)tau, P.weight_matching, rho.data(), gw.data(), u.data());
      // step sizes, tvl13d.py:240-249 (host float64)
      if (P.pd_type == 2) {
        const double theta = 1.0 / std::sqrt(1.0 + 2.0 * gamma * tau);
        tau *= theta;
        sigma /= theta;
      }
    }
  }
}

// tvl13d.py:122-162 with generate_pyramid (:69-120). blur_w: (2r+1)^3 weights or null.
template <class T>
int compute(const svso_params& P, const T* I0in, const T* I1in, int nz, int ny, int nx,
            const float* blur_w, int blur_r, const T* u_in, const T* p_in, T* u_out, T* p_out) {
  if (P.num_scales < 1 || nz < 3 || ny < 3 || nx < 3) return 1;
  std::vector<Mesh> meshes;
  meshes.push_back(make_mesh(P, nz, ny, nx));
  int cz = nz, cy = ny, cx = nx;
  for (int s = 1; s < P.num_scales; ++s) {
    cz = (cz + 1) / 2; cy = (cy + 1) / 2; cx = (cx + 1) / 2;  // math.ceil(0.5*N)
    if (cz < 3 || cy < 3 || cx < 3) return 1;
    meshes.push_back(make_mesh(P, cz, cy, cx));
  }
  const size_t n0 = vox(nz, ny, nx);
  std::vector<std::vector<T>> I0s(P.num_scales), I1s(P.num_scales), us(P.num_scales), ps(P.num_scales);
  I0s[0].assign(I0in, I0in + n0);
  I1s[0].assign(I1in, I1in + n0);
  if (P.use_blur && blur_w) {
    std::vector<T> tmp(n0);
    conv3d_zero<T>(I0s[0].data(), nz, ny, nx, blur_w, blur_r, tmp.data()); I0s[0] = tmp;
    conv3d_zero<T>(I1s[0].data(), nz, ny, nx, blur_w, blur_r, tmp.data()); I1s[0] = tmp;
  }
  us[0].assign(3 * n0, T(0)); ps[0].assign(9 * n0, T(0));
  if (u_in) us[0].assign(u_in, u_in + 3 * n0);
  if (p_in) ps[0].assign(p_in, p_in + 9 * n0);
  for (int s = 1; s < P.num_scales; ++s) {
    const Mesh& a = meshes[s - 1]; const Mesh& b = meshes[s];
    const size_t nb = vox(b.nz, b.ny, b.nx);
    I0s[s].resize(nb); I1s[s].resize(nb);
    prolongate<T>(I0s[s - 1].data(), a.nz, a.ny, a.nx, 1, a.lz, a.ly, a.lx, b.nz, b.ny, b.nx, b.lz, b.ly, b.lx, P.interp, P.bdry, I0s[s].data());
    prolongate<T>(I1s[s - 1].data(), a.nz, a.ny, a.nx, 1, a.lz, a.ly, a.lx, b.nz, b.ny, b.nx, b.lz, b.ly, b.lx, P.interp, P.bdry, I1s[s].data());
    us[s].assign(3 * nb, T(0)); ps[s].assign(9 * nb, T(0));
  }
  for (int s = P.num_scales - 1; s >= 0; --s) {
    solve_level<T>(P, meshes[s], I0s[s].data(), I1s[s].data(), us[s], ps[s]);
    if (s == 0) break;
    const Mesh& c = meshes[s]; const Mesh& f = meshes[s - 1];
    const size_t nf = vox(f.nz, f.ny, f.nx);
    us[s - 1].resize(3 * nf); ps[s - 1].resize(9 * nf);
    prolongate<T>(us[s].data(), c.nz, c.ny, c.nx, 3, c.lz, c.ly, c.lx, f.nz, f.ny, f.nx, f.lz, f.ly, f.lx, P.interp, P.bdry, us[s - 1].data());
    // tvl13d.py:151-153: python float (double) ratio, applied to a float32 tensor
    const T kx = (T)(float)((double)f.lx / (double)c.lx);
    const T ky = (T)(float)((double)f.ly / (double)c.ly);
    const T kz = (T)(float)((double)f.lz / (double)c.lz);
    for (size_t i = 0; i < nf; ++i) { us[s - 1][3 * i] *= kx; us[s - 1][3 * i + 1] *= ky; us[s - 1][3 * i + 2] *= kz; }
    prolongate<T>(ps[s].data(), c.nz, c.ny, c.nx, 9, c.lz, c.ly, c.lx, f.nz, f.ny, f.nx, f.lz, f.ly, f.lx, P.interp, P.bdry, ps[s - 1].data());
  }
  std::copy(us[0].begin(), us[0].end(), u_out);
  if (p_out) std::copy(ps[0].begin(), ps[0].end(), p_out);
  return 0;
}

}  // namespace

// =============================================================================================
// C ABI of the oracle (consumed by oracle/oracle.py through ctypes).
// =============================================================================================
extern "C" {

int svso_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void svso_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

#define DEF_OPS(T, SFX)                                                                              \
  void svso_nabla_fwd_vf_##SFX(const T* b, int nz, int ny, int nx, int C, float hz, float hy, float hx, \
                               int bdry, T* o) {                                                     \
    nabla_fwd_vf<T>(b, nz, ny, nx, C, hz, hy, hx, bdry, o); }                                        \
  void svso_nabla_bwd_vf_##SFX(const T* p, int nz, int ny, int nx, int C, float hz, float hy, float hx, \
                               int bdry, T* o) {                                                     \
    nabla_bwd_vf<T>(p, nz, ny, nx, C, hz, hy, hx, bdry, o); }                                        \
  void svso_aniso_tangents_##SFX(const T* g, size_t n, float a, float b, T* s, T* nr, T* t1, T* t2) { \
    aniso_tangents<T>(g, n, a, b, s, nr, t1, t2); }                                                  \
  void svso_aniso_apply_##SFX(const T* in, size_t n, const T* s, const T* nr, const T* t1, T* o) {   \
    aniso_apply<T>(in, n, s, nr, t1, o); }                                                           \
  void svso_prox_primal_##SFX(const T* pv, size_t n, float tau, float lam, const T* rho, const T* g, T* o) { \
    prox_primal<T>(pv, n, tau, lam, rho, g, o); }                                                    \
  void svso_prox_dual_##SFX(const T* dv, size_t n, float w, T* o) { prox_dual<T>(dv, n, w, o); }     \
  void svso_warp_##SFX(const T* u, int nz, int ny, int nx, int C, const T* phi, float hz, float hy, float hx, \
                       int interp, int bdry, T* o) {                                                  \
    warp_field<T>(u, nz, ny, nx, C, phi, hz, hy, hx, interp, bdry, o); }                             \
  void svso_prolongate_##SFX(const T* u, int nz, int ny, int nx, int C, float lz, float ly, float lx, \
                             int tz, int ty, int tx, float tlz, float tly, float tlx, int interp, int bdry, T* o) { \
    prolongate<T>(u, nz, ny, nx, C, lz, ly, lx, tz, ty, tx, tlz, tly, tlx, interp, bdry, o); }       \
  void svso_warp_cnn_##SFX(const T* m, int B, int C, int nz, int ny, int nx, const T* phi, float hz, float hy, \
                           float hx, int interp, int bdry, T* o) {                                    \
    warp_cnn<T>(m, B, C, nz, ny, nx, phi, hz, hy, hx, interp, bdry, o); }                            \
  void svso_warp_backward_##SFX(const T* u, int nz, int ny, int nx, const T* phi, const T* g, float hz, \
                                float hy, float hx, int interp, int bdry, T* gu, T* gp) {            \
    warp_backward<T>(u, nz, ny, nx, phi, g, hz, hy, hx, interp, bdry, gu, gp); }                    \
  void svso_conv3d_##SFX(const T* in, int nz, int ny, int nx, const float* w, int r, T* o) {          \
    conv3d_zero<T>(in, nz, ny, nx, w, r, o); }                                                       \
  void svso_median3_##SFX(const T* in, int nz, int ny, int nx, int C, int ks, T* o) {                 \
    median3<T>(in, nz, ny, nx, C, ks, o); }                                                          \
  int svso_tvl1_compute_##SFX(const svso_params* P, const T* I0, const T* I1, int nz, int ny, int nx, \
                              const float* blur_w, int blur_r, const T* u_in, const T* p_in, T* u_out, T* p_out) { \
    return compute<T>(*P, I0, I1, nz, ny, nx, blur_w, blur_r, u_in, p_in, u_out, p_out); }

DEF_OPS(float, f32)
DEF_OPS(double, f64)

// Dice and symmetric Hausdorff distance between two binary masks, as the reference's
// svs/modules/flow/warping.py:245-270 obtains them from monai (compute_dice,
// compute_hausdorff_distance; include_background=False on a single channel keeps that channel):
// dice = 2|A and B| / (|A| + |B|) (NaN when both are empty); edges = mask minus its erosion by the
// 6-neighbour cross with zero border; HD = max of the two directed max-min Euclidean edge
// distances in voxel units (inf when exactly one edge set is empty, NaN when both are).
double svso_dice(const uint8_t* a, const uint8_t* b, size_t n) {
  size_t inter = 0, sa = 0, sb = 0;
  for (size_t i = 0; i < n; ++i) { sa += a[i] != 0; sb += b[i] != 0; inter += (a[i] && b[i]); }
  if (sa + sb == 0) return std::numeric_limits<double>::quiet_NaN();
  return 2.0 * (double)inter / (double)(sa + sb);
}

static void edges_of(const uint8_t* m, int nz, int ny, int nx, std::vector<int>& pts) {
  auto at = [&](int z, int y, int x) -> int {
    if (z < 0 || y < 0 || x < 0 || z >= nz || y >= ny || x >= nx) return 0;
    return m[((size_t)z * ny + y) * nx + x] != 0;
  };
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        if (!at(z, y, x)) continue;
        const bool interior = at(z - 1, y, x) && at(z + 1, y, x) && at(z, y - 1, x) &&
                              at(z, y + 1, x) && at(z, y, x - 1) && at(z, y, x + 1);
        if (!interior) { pts.push_back(z); pts.push_back(y); pts.push_back(x); }
      }
}

static double directed_hd(const std::vector<int>& a, const std::vector<int>& b) {
  double worst = 0;
  const ptrdiff_t na = (ptrdiff_t)a.size() / 3, nb = (ptrdiff_t)b.size() / 3;
#pragma omp parallel for reduction(max : worst) schedule(static)
  for (ptrdiff_t i = 0; i < na; ++i) {
    long best = std::numeric_limits<long>::max();
    for (ptrdiff_t j = 0; j < nb; ++j) {
      const long dz = a[3 * i] - b[3 * j], dy = a[3 * i + 1] - b[3 * j + 1], dx = a[3 * i + 2] - b[3 * j + 2];
      best = std::min(best, dz * dz + dy * dy + dx * dx);
    }
    worst = std::max(worst, std::sqrt((double)best));
  }
  return worst;
}

double svso_hausdorff(const uint8_t* a, const uint8_t* b, int nz, int ny, int nx) {
  std::vector<int> ea, eb;
  edges_of(a, nz, ny, nx, ea);
  edges_of(b, nz, ny, nx, eb);
  if (ea.empty() && eb.empty()) return std::numeric_limits<double>::quiet_NaN();
  if (ea.empty() || eb.empty()) return std::numeric_limits<double>::infinity();
  return std::max(directed_hd(ea, eb), directed_hd(eb, ea));
}

}  // extern "C"
