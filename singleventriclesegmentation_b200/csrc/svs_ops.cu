// Per-operator kernels of libsvsflow: one entry point per op of the reference's
// opticalFlow_cuda_ext.opticalFlow module (3D subset). These back the drop-in Python module and
// the per-op parity tests; the fused solver (svs_solver.cu) does not call them.
//
// Layout: one thread per output voxel over a flat 1D grid (x fastest), so neighbouring threads
// touch neighbouring addresses. Each kernel writes every output element (no zero-fill pass,
// unlike the reference's torch::zeros + kernel).
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <string>
#include <vector>

#include "svs_common.cuh"

namespace svs {

namespace {
thread_local std::string g_last_error;
std::atomic<uint64_t>* launch_counter() {
  static std::atomic<uint64_t> c{0};
  return &c;
}
}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }
svs_status fail(svs_status code, const std::string& msg) {
  set_error(msg);
  return code;
}
void count_launches(uint64_t n) { launch_counter()->fetch_add(n, std::memory_order_relaxed); }
svs_status check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SVS_OK;
  const svs_status code = (e == cudaErrorMemoryAllocation) ? SVS_ERR_OUT_OF_MEMORY : SVS_ERR_CUDA;
  return fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}
svs_status check_launch(const char* what, uint64_t launches) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SVS_ERR_LAUNCH, std::string(what) + ": " + cudaGetErrorString(e));
  count_launches(launches);
  return SVS_OK;
}

namespace {

constexpr int kThreads = 256;

inline bool valid_dims(int nz, int ny, int nx) { return nz > 0 && ny > 0 && nx > 0; }
inline bool valid_bdry(int b) { return b >= 0 && b <= 2; }
inline bool valid_interp(int i) { return i >= 0 && i <= 2; }

// Rounded addition without contraction in the value type (the float path of the reference sums
// dx/hx + dy/hy + dz/hz as separate float additions).
__device__ __forceinline__ float tadd_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double tadd_rn(double a, double b) { return __dadd_rn(a, b); }

// Every kernel below is a template on the value type T: float for the reference's float path,
// double for the FP64 entry points (the reference dispatches both, AT_DISPATCH_FLOATING_TYPES).
// ---------------------------------------------------------------------------------- gradients
// Nabla3D_CD.forward/.forwardVectorField: differentialOps.cu:540-655 and :782-907.
template <typename T>
__global__ void nabla_fwd_kernel(const T* __restrict__ b, int nz, int ny, int nx, int C,
                                 T hz, T hy, T hx, int bdry, T* __restrict__ out) {
  const int64_t n = (int64_t)nz * ny * nx * C;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = t / C;
    const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((int64_t)nx * ny));
    const int64_t sx = C, sy = (int64_t)nx * C, sz = (int64_t)nx * ny * C;
    const T c = b[t];
    const T xm = x > 0 ? b[t - sx] : T(0), xp = x < nx - 1 ? b[t + sx] : T(0);
    const T ym = y > 0 ? b[t - sy] : T(0), yp = y < ny - 1 ? b[t + sy] : T(0);
    const T zm = z > 0 ? b[t - sz] : T(0), zp = z < nz - 1 ? b[t + sz] : T(0);
    out[3 * t + 0] = fwd_axis(xm, c, xp, x, nx, bdry, hx);
    out[3 * t + 1] = fwd_axis(ym, c, yp, y, ny, bdry, hy);
    out[3 * t + 2] = fwd_axis(zm, c, zp, z, nz, bdry, hz);
  }
}

// Nabla3D_CD.backward/.backwardVectorField: differentialOps.cu:658-779 and :909-1039.
// out = dx/hx + dy/hy + dz/hz summed left to right in T.
template <typename T>
__global__ void nabla_bwd_kernel(const T* __restrict__ p, int nz, int ny, int nx, int C,
                                 T hz, T hy, T hx, int bdry, T* __restrict__ out) {
  const int64_t n = (int64_t)nz * ny * nx * C;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = t / C;
    const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((int64_t)nx * ny));
    const int64_t sx = 3 * C, sy = (int64_t)nx * 3 * C, sz = (int64_t)nx * ny * 3 * C;
    const T* q = p + 3 * t;
    const T dx = adj_axis(x > 0 ? q[-sx] : T(0), q[0], x < nx - 1 ? q[sx] : T(0), x, nx, bdry);
    const T dy = adj_axis(y > 0 ? q[1 - sy] : T(0), q[1], y < ny - 1 ? q[1 + sy] : T(0), y, ny, bdry);
    const T dz = adj_axis(z > 0 ? q[2 - sz] : T(0), q[2], z < nz - 1 ? q[2 + sz] : T(0), z, nz, bdry);
    out[t] = tadd_rn(tadd_rn(dx / hx, dy / hy), dz / hz);
  }
}

// --------------------------------------------------------------------------------- anisotropy
// computeTangentVecs: anisotropicDifferentialOps.cu:89-141.
template <typename T>
__global__ void aniso_tangents_kernel(const T* __restrict__ g, int64_t n, T alpha,
                                      T beta, T* __restrict__ s, T* __restrict__ nrm,
                                      T* __restrict__ t1, T* __restrict__ t2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T g0 = g[3 * i], g1 = g[3 * i + 1], g2 = g[3 * i + 2];
    const T nsq = g0 * g0 + g1 * g1 + g2 * g2;
    const T norm = sqrt(nsq);
    if (norm > T(0)) {
      s[i] = exp(-alpha * pow(norm, beta));
      const T n0 = g0 / norm, n1 = g1 / norm, n2 = g2 / norm;
      T a0, a1, a2;
      if (n2 > T(0.5)) { a0 = n2; a1 = T(0); a2 = -n0; }
      else { a0 = n1; a1 = -n0; a2 = T(0); }
      nrm[3 * i] = n0; nrm[3 * i + 1] = n1; nrm[3 * i + 2] = n2;
      t1[3 * i] = a0; t1[3 * i + 1] = a1; t1[3 * i + 2] = a2;
      t2[3 * i] = n1 * a2 - n2 * a1;
      t2[3 * i + 1] = n2 * a0 - n0 * a2;
      t2[3 * i + 2] = n0 * a1 - n1 * a0;
    } else {
      s[i] = T(0);
#pragma unroll
      for (int d = 0; d < 3; ++d) nrm[3 * i + d] = t1[3 * i + d] = t2[3 * i + d] = T(0);
    }
  }
}

// forwardVectorField (== backwardVectorField): anisotropicDifferentialOps.cu:143-175.
template <typename T>
__global__ void aniso_apply_kernel(const T* __restrict__ in, int64_t n,
                                   const T* __restrict__ s, const T* __restrict__ nrm,
                                   const T* __restrict__ t1, T* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T si = s[i];
    const T n0 = nrm[3 * i], n1 = nrm[3 * i + 1], n2 = nrm[3 * i + 2];
    const T a0 = t1[3 * i], a1 = t1[3 * i + 1], a2 = t1[3 * i + 2];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T* b = in + 9 * i + 3 * c;
      const T b0 = b[0], b1 = b[1], b2 = b[2];
      const T nf = n0 * b0 + n1 * b1 + n2 * b2;
      const T tf = a0 * b0 + a1 * b1 + a2 * b2;
      const T k = si * nf;
      T* o = out + 9 * i + 3 * c;
      o[0] = k * n0 + tf * a0;
      o[1] = k * n1 + tf * a1;
      o[2] = k * n2 + tf * a2;
    }
  }
}

// ------------------------------------------------------------------------------------- proxes
// proxPrimal: opticalFlowOps.cu:123-175.
template <typename T>
__global__ void prox_primal_kernel(const T* __restrict__ pv, int64_t n, T factor,
                                   const T* __restrict__ rho, const T* __restrict__ g,
                                   T* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T r = rho[i];
    const T g0 = g[3 * i], g1 = g[3 * i + 1], g2 = g[3 * i + 2];
    const T g2s = g0 * g0 + g1 * g1 + g2 * g2;
    T d0, d1, d2;
    if (r < -factor * g2s) { d0 = factor * g0; d1 = factor * g1; d2 = factor * g2; }
    else if (r > factor * g2s) { d0 = -factor * g0; d1 = -factor * g1; d2 = -factor * g2; }
    else if ((double)g2s > 1e-10) { d0 = -r * g0 / g2s; d1 = -r * g1 / g2s; d2 = -r * g2 / g2s; }
    else { d0 = d1 = d2 = T(0); }
    out[3 * i] = pv[3 * i] + d0;
    out[3 * i + 1] = pv[3 * i + 1] + d1;
    out[3 * i + 2] = pv[3 * i + 2] + d2;
  }
}

// proxDual: opticalFlowOps.cu:179-208, p_c / max(1, |p_c| / weight_tv) per flow component.
template <typename T>
__global__ void prox_dual_kernel(const T* __restrict__ dv, int64_t n3, T wtv,
                                 T* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n3;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T q0 = dv[3 * i], q1 = dv[3 * i + 1], q2 = dv[3 * i + 2];
    const T den = fmax(T(1), sqrt(q0 * q0 + q1 * q1 + q2 * q2) / wtv);
    out[3 * i] = q0 / den;
    out[3 * i + 1] = q1 / den;
    out[3 * i + 2] = q2 / den;
  }
}

// -------------------------------------------------------------------------------- resampling
// Warping3D.forward/.forwardVectorField: warpingOps.cu:572-660 (and nearest/trilinear siblings).
template <typename T>
__global__ void warp_kernel(const T* __restrict__ u, int nz, int ny, int nx, int C,
                            const T* __restrict__ phi, T hz, T hy, T hx,
                            int interp, int bdry, T* __restrict__ out) {
  const int64_t n = (int64_t)nz * ny * nx;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((int64_t)nx * ny));
    const T cx = (T)x * hx + phi[3 * v];
    const T cy = (T)y * hy + phi[3 * v + 1];
    const T cz = (T)z * hz + phi[3 * v + 2];
    for (int c = 0; c < C; ++c) {
      FieldRefT<T> f{u + c, nz, ny, nx, C};
      out[v * C + c] = sample(f, cz, cy, cx, hz, hy, hx, interp, bdry);
    }
  }
}

// WarpingCNN3D.forward: warpingOpsCNN.cu:97-128, grid over (b, voxel), loop over channels.
template <typename T>
__global__ void warp_cnn_kernel(const T* __restrict__ m, int B, int C, int nz, int ny, int nx,
                                const T* __restrict__ phi, T hz, T hy, T hx,
                                int interp, int bdry, T* __restrict__ out) {
  const int64_t nv = (int64_t)nz * ny * nx;
  const int64_t n = nv * B;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(t / nv);
    const int64_t v = t - (int64_t)b * nv;
    const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((int64_t)nx * ny));
    const T* ph = phi + (size_t)b * nv * 3;
    const T cx = (T)x * hx + ph[3 * v];
    const T cy = (T)y * hy + ph[3 * v + 1];
    const T cz = (T)z * hz + ph[3 * v + 2];
    for (int c = 0; c < C; ++c) {
      FieldRefT<T> f{m + ((size_t)b * C + c) * nv, nz, ny, nx, 1};
      out[((size_t)b * C + c) * nv + v] = sample(f, cz, cy, cx, hz, hy, hx, interp, bdry);
    }
  }
}

// Prolongation3D: prolongationOps.cu:533-625. Target node i -> source coordinate (i*h_t)*L_s/L_t.
template <typename T>
__global__ void prolongate_kernel(const T* __restrict__ u, int nz, int ny, int nx, int C,
                                  T lz, T ly, T lx, T hz, T hy, T hx,
                                  int tz, int ty, int tx, T tlz, T tly, T tlx,
                                  T thz, T thy, T thx, int interp, int bdry,
                                  T* __restrict__ out) {
  const int64_t n = (int64_t)tz * ty * tx;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(v % tx), y = (int)((v / tx) % ty), z = (int)(v / ((int64_t)tx * ty));
    const T cx = (T)x * thx * lx / tlx;
    const T cy = (T)y * thy * ly / tly;
    const T cz = (T)z * thz * lz / tlz;
    for (int c = 0; c < C; ++c) {
      FieldRefT<T> f{u + c, nz, ny, nx, C};
      out[v * C + c] = sample(f, cz, cy, cx, hz, hy, hx, interp, bdry);
    }
  }
}


// ------------------------------------------------------------------------------ warp backward
// Catmull-Rom basis weights at fraction w (the d_out_d_p_* of
// interpolation_cubicHermiteSpline.cuh:132-136) and the derivative of the 1D cubic with respect
// to w in the reference's coefficient form 3w^2 a + 2 w b + c (:196-198).
template <typename T>
__device__ __forceinline__ void cr_weights(T w, T W[4]) {
  const T w2 = w * w, w3 = w2 * w;
  W[0] = -w3 / 2 + w2 - w / 2;
  W[1] = (3 * w3) / 2 - (5 * w2) / 2 + 1;
  W[2] = -(3 * w3) / 2 + 2 * w2 + w / 2;
  W[3] = w3 / 2 - w2 / 2;
}
template <typename T>
__device__ __forceinline__ T cr_dvalue(T b0, T b1, T b2, T b3, T w) {
  const T pf = b1, dpf = (b2 - b0) / 2, pc = b2, dpc = (b3 - b1) / 2;
  const T a = 2 * pf - 2 * pc + dpf + dpc;
  const T b = -3 * pf + 3 * pc - 2 * dpf - dpc;
  return 3 * w * w * a + 2 * b * w + dpf;
}

// Warping3D.backward for one voxel: grad_phi is the gradient of the interpolant at the sample
// point times grad_out / h; grad_u receives grad_out times each stencil weight (atomic adds on the
// folded node, warpingOps.cu:598-630 / interpolation_cubicHermiteSpline.cuh:527-636, trilinear
// interpolation_linear.cuh:298-366, nearest interpolation_nearest.cuh:296-356).
template <typename T>
__global__ void warp_backward_kernel(const T* __restrict__ u, int nz, int ny, int nx,
                                     const T* __restrict__ phi, const T* __restrict__ gout,
                                     T hz, T hy, T hx, int interp, int bdry,
                                     T* __restrict__ grad_u, T* __restrict__ grad_phi) {
  const int64_t n = (int64_t)nz * ny * nx;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((int64_t)nx * ny));
    const T cx = (T)x * hx + phi[3 * v];
    const T cy = (T)y * hy + phi[3 * v + 1];
    const T cz = (T)z * hz + phi[3 * v + 2];
    const T g = gout[v];
    T gpx = T(0), gpy = T(0), gpz = T(0);
    FieldRefT<T> f{u, nz, ny, nx, 1};
    if (interp == SVS_INTERPOLATE_CUBIC_HERMITESPLINE) {
      int ix, iy, iz;
      T wx, wy, wz;
      split_coord(cx, hx, ix, wx);
      split_coord(cy, hy, iy, wy);
      split_coord(cz, hz, iz, wz);
      wx = (wx + T(1)) - T(1);
      wy = (wy + T(1)) - T(1);
      wz = (wz + T(1)) - T(1);
      T Wx[4], Wy[4], Wz[4];
      cr_weights(wx, Wx);
      cr_weights(wy, Wy);
      cr_weights(wz, Wz);
      int xs[4], ys[4], zs[4];
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        xs[d] = fold(ix + d - 1, nx, bdry);
        ys[d] = fold(iy + d - 1, ny, bdry);
        zs[d] = fold(iz + d - 1, nz, bdry);
      }
      T bz[4];
#pragma unroll
      for (int dz = 0; dz < 4; ++dz) {
        T by[4];
#pragma unroll
        for (int dy = 0; dy < 4; ++dy) {
          const T r0 = f.at(zs[dz], ys[dy], xs[0]), r1 = f.at(zs[dz], ys[dy], xs[1]);
          const T r2 = f.at(zs[dz], ys[dy], xs[2]), r3 = f.at(zs[dz], ys[dy], xs[3]);
          by[dy] = hermite4(r0, r1, r2, r3, wx);
          const T gzy = g * Wz[dz] * Wy[dy];
          gpx += cr_dvalue(r0, r1, r2, r3, wx) * gzy;
          T* row = grad_u + ((size_t)zs[dz] * ny + ys[dy]) * nx;
#pragma unroll
          for (int dx = 0; dx < 4; ++dx) atomicAdd(row + xs[dx], Wx[dx] * gzy);
        }
        bz[dz] = hermite4(by[0], by[1], by[2], by[3], wy);
        gpy += cr_dvalue(by[0], by[1], by[2], by[3], wy) * (g * Wz[dz]);
      }
      gpz = cr_dvalue(bz[0], bz[1], bz[2], bz[3], wz) * g;
      gpx /= hx;
      gpy /= hy;
      gpz /= hz;
    } else if (interp == SVS_INTERPOLATE_LINEAR) {
      int ix, iy, iz;
      T wx, wy, wz;
      split_coord(cx, hx, ix, wx);
      split_coord(cy, hy, iy, wy);
      split_coord(cz, hz, iz, wz);
      const int x0 = fold(ix, nx, bdry), x1 = fold(ix + 1, nx, bdry);
      const int y0 = fold(iy, ny, bdry), y1 = fold(iy + 1, ny, bdry);
      const int z0 = fold(iz, nz, bdry), z1 = fold(iz + 1, nz, bdry);
      const T fff = f.at(z0, y0, x0), ffc = f.at(z1, y0, x0), fcf = f.at(z0, y1, x0),
                  fcc = f.at(z1, y1, x0), cff = f.at(z0, y0, x1), cfc = f.at(z1, y0, x1),
                  ccf = f.at(z0, y1, x1), ccc = f.at(z1, y1, x1);
      auto add = [&](int zz, int yy, int xx, T w) { atomicAdd(grad_u + ((size_t)zz * ny + yy) * nx + xx, w * g); };
      add(z0, y0, x0, (1 - wz) * (1 - wy) * (1 - wx));
      add(z0, y1, x0, (1 - wz) * wy * (1 - wx));
      add(z0, y0, x1, (1 - wz) * (1 - wy) * wx);
      add(z0, y1, x1, (1 - wz) * wy * wx);
      add(z1, y0, x0, wz * (1 - wy) * (1 - wx));
      add(z1, y1, x0, wz * wy * (1 - wx));
      add(z1, y0, x1, wz * (1 - wy) * wx);
      add(z1, y1, x1, wz * wy * wx);
      gpx = ((1 - wz) * (1 - wy) * (cff - fff) + (1 - wz) * wy * (ccf - fcf) + wz * (1 - wy) * (cfc - ffc) + wz * wy * (ccc - fcc)) / hx * g;
      gpy = ((1 - wz) * (1 - wx) * (fcf - fff) + (1 - wz) * wx * (ccf - cff) + wz * (1 - wx) * (fcc - ffc) + wz * wx * (ccc - cfc)) / hy * g;
      gpz = ((1 - wy) * (1 - wx) * (ffc - fff) + (1 - wy) * wx * (cfc - cff) + wy * (1 - wx) * (fcc - fcf) + wy * wx * (ccc - ccf)) / hz * g;
    } else {
      const int xx = nearest_axis(cx, hx, nx, bdry), yy = nearest_axis(cy, hy, ny, bdry),
                zz = nearest_axis(cz, hz, nz, bdry);
      atomicAdd(grad_u + ((size_t)zz * ny + yy) * nx + xx, g);
    }
    grad_phi[3 * v] = gpx;
    grad_phi[3 * v + 1] = gpy;
    grad_phi[3 * v + 2] = gpz;
  }
}

unsigned grid_for(int64_t n) {
  const int64_t blocks = (n + kThreads - 1) / kThreads;
  return (unsigned)(blocks < 148 * 64 ? (blocks > 0 ? blocks : 1) : 148 * 64);
}

}  // namespace
}  // namespace svs

using namespace svs;

namespace svs {
namespace {

// Entry-point bodies, templated on the value type (float: svs_*, double: svs_*_f64).
template <typename T>
svs_status nabla_forward(const char* nm, const T* b, int nz, int ny, int nx, int C, T hz, T hy, T hx, int boundary,
                         T* out, cudaStream_t stream) {
  SVS_REQUIRE(b && out, std::string(nm) + ": null pointer");
  SVS_REQUIRE(valid_dims(nz, ny, nx) && C > 0, std::string(nm) + ": bad sizes");
  SVS_REQUIRE(valid_bdry(boundary), std::string(nm) + ": bad boundary type");
  const int64_t n = (int64_t)nz * ny * nx * C;
  nabla_fwd_kernel<T><<<grid_for(n), kThreads, 0, stream>>>(b, nz, ny, nx, C, hz, hy, hx, boundary, out);
  return check_launch(nm);
}

template <typename T>
svs_status nabla_backward(const char* nm, const T* p, int nz, int ny, int nx, int C, T hz, T hy, T hx, int boundary,
                          T* out, cudaStream_t stream) {
  SVS_REQUIRE(p && out, std::string(nm) + ": null pointer");
  SVS_REQUIRE(valid_dims(nz, ny, nx) && C > 0, std::string(nm) + ": bad sizes");
  SVS_REQUIRE(valid_bdry(boundary), std::string(nm) + ": bad boundary type");
  // The MIRROR adjoint reads index i+1 at i = 1 (differentialOps.cu:711-717): it needs N >= 3.
  SVS_REQUIRE(boundary != SVS_BOUNDARY_MIRROR || (nz >= 3 && ny >= 3 && nx >= 3),
              std::string(nm) + ": the MIRROR adjoint needs at least 3 nodes per axis");
  const int64_t n = (int64_t)nz * ny * nx * C;
  nabla_bwd_kernel<T><<<grid_for(n), kThreads, 0, stream>>>(p, nz, ny, nx, C, hz, hy, hx, boundary, out);
  return check_launch(nm);
}

template <typename T>
svs_status aniso_tangents(const char* nm, const T* g, int64_t n, T alpha, T beta, T* s, T* normals, T* t1, T* t2,
                          cudaStream_t stream) {
  if (n == 0) return SVS_OK;
  SVS_REQUIRE(g && s && normals && t1 && t2, std::string(nm) + ": null pointer");
  SVS_REQUIRE(n >= 0, std::string(nm) + ": bad size");
  aniso_tangents_kernel<T><<<grid_for(n), kThreads, 0, stream>>>(g, n, alpha, beta, s, normals, t1, t2);
  return check_launch(nm);
}

template <typename T>
svs_status aniso_apply(const char* nm, const T* in, int64_t n, const T* s, const T* normals, const T* t1, T* out,
                       cudaStream_t stream) {
  if (n == 0) return SVS_OK;
  SVS_REQUIRE(in && s && normals && t1 && out, std::string(nm) + ": null pointer");
  SVS_REQUIRE(n >= 0, std::string(nm) + ": bad size");
  aniso_apply_kernel<T><<<grid_for(n), kThreads, 0, stream>>>(in, n, s, normals, t1, out);
  return check_launch(nm);
}

template <typename T>
svs_status prox_primal(const char* nm, const T* primal, int64_t n, T tau, T weight_matching, const T* rho,
                       const T* i1w_grad, T* out, cudaStream_t stream) {
  if (n == 0) return SVS_OK;
  SVS_REQUIRE(primal && rho && i1w_grad && out, std::string(nm) + ": null pointer");
  SVS_REQUIRE(n >= 0, std::string(nm) + ": bad size");
  const T factor = tau * weight_matching;  // opticalFlowOps.cu:440
  prox_primal_kernel<T><<<grid_for(n), kThreads, 0, stream>>>(primal, n, factor, rho, i1w_grad, out);
  return check_launch(nm);
}

template <typename T>
svs_status prox_dual(const char* nm, const T* dual, int64_t n, T weight_tv, T* out, cudaStream_t stream) {
  if (n == 0) return SVS_OK;
  SVS_REQUIRE(dual && out, std::string(nm) + ": null pointer");
  SVS_REQUIRE(n >= 0, std::string(nm) + ": bad size");
  prox_dual_kernel<T><<<grid_for(3 * n), kThreads, 0, stream>>>(dual, 3 * n, weight_tv, out);
  return check_launch(nm);
}

template <typename T>
svs_status warp3d(const char* nm, const T* u, int nz, int ny, int nx, int C, const T* phi, T hz, T hy, T hx,
                  int interpolation, int boundary, T* out, cudaStream_t stream) {
  SVS_REQUIRE(u && phi && out, std::string(nm) + ": null pointer");
  SVS_REQUIRE(valid_dims(nz, ny, nx) && C > 0, std::string(nm) + ": bad sizes");
  SVS_REQUIRE(valid_bdry(boundary) && valid_interp(interpolation), std::string(nm) + ": bad mode");
  const int64_t n = (int64_t)nz * ny * nx;
  warp_kernel<T><<<grid_for(n), kThreads, 0, stream>>>(u, nz, ny, nx, C, phi, hz, hy, hx, interpolation, boundary, out);
  return check_launch(nm);
}

template <typename T>
svs_status warp3d_backward(const char* nm, const T* u, int nz, int ny, int nx, const T* phi, const T* grad_out,
                           T hz, T hy, T hx, int interpolation, int boundary, T* grad_u, T* grad_phi,
                           cudaStream_t stream) {
  SVS_REQUIRE(u && phi && grad_out && grad_u && grad_phi, std::string(nm) + ": null pointer");
  SVS_REQUIRE(valid_dims(nz, ny, nx), std::string(nm) + ": bad sizes");
  SVS_REQUIRE(valid_bdry(boundary) && valid_interp(interpolation), std::string(nm) + ": bad mode");
  const int64_t n = (int64_t)nz * ny * nx;
  svs_status st = check_cuda(cudaMemsetAsync(grad_u, 0, n * sizeof(T), stream), nm);
  if (st) return st;
  warp_backward_kernel<T><<<grid_for(n), kThreads, 0, stream>>>(u, nz, ny, nx, phi, grad_out, hz, hy, hx,
                                                                 interpolation, boundary, grad_u, grad_phi);
  return check_launch(nm);
}

template <typename T>
svs_status warp_cnn3d(const char* nm, const T* m, int B, int C, int nz, int ny, int nx, const T* phi, T hz, T hy,
                      T hx, int interpolation, int boundary, T* out, cudaStream_t stream) {
  SVS_REQUIRE(m && phi && out, std::string(nm) + ": null pointer");
  SVS_REQUIRE(valid_dims(nz, ny, nx) && B > 0 && C > 0, std::string(nm) + ": bad sizes");
  SVS_REQUIRE(valid_bdry(boundary) && valid_interp(interpolation), std::string(nm) + ": bad mode");
  const int64_t n = (int64_t)nz * ny * nx * B;
  warp_cnn_kernel<T><<<grid_for(n), kThreads, 0, stream>>>(m, B, C, nz, ny, nx, phi, hz, hy, hx, interpolation,
                                                            boundary, out);
  return check_launch(nm);
}

template <typename T>
svs_status prolongate3d(const char* nm, const T* u, int nz, int ny, int nx, int C, T lz, T ly, T lx, int tz, int ty,
                        int tx, T tlz, T tly, T tlx, int interpolation, int boundary, T* out, cudaStream_t stream) {
  SVS_REQUIRE(u && out, std::string(nm) + ": null pointer");
  SVS_REQUIRE(valid_dims(nz, ny, nx) && valid_dims(tz, ty, tx) && C > 0, std::string(nm) + ": bad sizes");
  SVS_REQUIRE(nz > 1 && ny > 1 && nx > 1 && tz > 1 && ty > 1 && tx > 1,
              std::string(nm) + ": meshes need at least 2 nodes per axis (h = L/(N-1))");
  SVS_REQUIRE(valid_bdry(boundary) && valid_interp(interpolation), std::string(nm) + ": bad mode");
  // MeshInfo3D, coreDefines.h:72-75: h = L / (N - 1) in the value type.
  const T hz = lz / (T)(nz - 1), hy = ly / (T)(ny - 1), hx = lx / (T)(nx - 1);
  const T thz = tlz / (T)(tz - 1), thy = tly / (T)(ty - 1), thx = tlx / (T)(tx - 1);
  const int64_t n = (int64_t)tz * ty * tx;
  prolongate_kernel<T><<<grid_for(n), kThreads, 0, stream>>>(u, nz, ny, nx, C, lz, ly, lx, hz, hy, hx, tz, ty, tx, tlz,
                                                              tly, tlx, thz, thy, thx, interpolation, boundary, out);
  return check_launch(nm);
}

}  // namespace
}  // namespace svs

extern "C" {

const char* svs_last_error(void) { return svs::g_last_error.c_str(); }
int svs_version(void) { return 1; }
uint64_t svs_launch_count(void) { return launch_counter()->load(); }

svs_status svs_nabla3d_forward(const float* b, int nz, int ny, int nx, int C, float hz, float hy, float hx, int boundary, float* out, svs_stream_t stream) {
  return nabla_forward<float>("svs_nabla3d_forward", b, nz, ny, nx, C, hz, hy, hx, boundary, out, stream);
}

svs_status svs_nabla3d_forward_f64(const double* b, int nz, int ny, int nx, int C, double hz, double hy, double hx, int boundary, double* out, svs_stream_t stream) {
  return nabla_forward<double>("svs_nabla3d_forward_f64", b, nz, ny, nx, C, hz, hy, hx, boundary, out, stream);
}

svs_status svs_nabla3d_backward(const float* p, int nz, int ny, int nx, int C, float hz, float hy, float hx, int boundary, float* out, svs_stream_t stream) {
  return nabla_backward<float>("svs_nabla3d_backward", p, nz, ny, nx, C, hz, hy, hx, boundary, out, stream);
}

svs_status svs_nabla3d_backward_f64(const double* p, int nz, int ny, int nx, int C, double hz, double hy, double hx, int boundary, double* out, svs_stream_t stream) {
  return nabla_backward<double>("svs_nabla3d_backward_f64", p, nz, ny, nx, C, hz, hy, hx, boundary, out, stream);
}

svs_status svs_aniso3d_tangents(const float* g, int64_t n, float alpha, float beta, float* s, float* normals, float* t1, float* t2, svs_stream_t stream) {
  return aniso_tangents<float>("svs_aniso3d_tangents", g, n, alpha, beta, s, normals, t1, t2, stream);
}

svs_status svs_aniso3d_tangents_f64(const double* g, int64_t n, double alpha, double beta, double* s, double* normals, double* t1, double* t2, svs_stream_t stream) {
  return aniso_tangents<double>("svs_aniso3d_tangents_f64", g, n, alpha, beta, s, normals, t1, t2, stream);
}

svs_status svs_aniso3d_apply(const float* in, int64_t n, const float* s, const float* normals, const float* t1, const float* t2, float* out, svs_stream_t stream) {
  return ((void)t2, aniso_apply<float>("svs_aniso3d_apply", in, n, s, normals, t1, out, stream));
}

svs_status svs_aniso3d_apply_f64(const double* in, int64_t n, const double* s, const double* normals, const double* t1, const double* t2, double* out, svs_stream_t stream) {
  return ((void)t2, aniso_apply<double>("svs_aniso3d_apply_f64", in, n, s, normals, t1, out, stream));
}

svs_status svs_tvl1_prox_primal(const float* primal, int64_t n, float tau, float weight_matching, const float* rho, const float* i1w_grad, float* out, svs_stream_t stream) {
  return prox_primal<float>("svs_tvl1_prox_primal", primal, n, tau, weight_matching, rho, i1w_grad, out, stream);
}

svs_status svs_tvl1_prox_primal_f64(const double* primal, int64_t n, double tau, double weight_matching, const double* rho, const double* i1w_grad, double* out, svs_stream_t stream) {
  return prox_primal<double>("svs_tvl1_prox_primal_f64", primal, n, tau, weight_matching, rho, i1w_grad, out, stream);
}

svs_status svs_tvl1_prox_dual(const float* dual, int64_t n, float sigma, float weight_tv, float* out, svs_stream_t stream) {
  return ((void)sigma, prox_dual<float>("svs_tvl1_prox_dual", dual, n, weight_tv, out, stream));
}

svs_status svs_tvl1_prox_dual_f64(const double* dual, int64_t n, double sigma, double weight_tv, double* out, svs_stream_t stream) {
  return ((void)sigma, prox_dual<double>("svs_tvl1_prox_dual_f64", dual, n, weight_tv, out, stream));
}

svs_status svs_warp3d(const float* u, int nz, int ny, int nx, int C, const float* phi, float hz, float hy, float hx, int interpolation, int boundary, float* out, svs_stream_t stream) {
  return warp3d<float>("svs_warp3d", u, nz, ny, nx, C, phi, hz, hy, hx, interpolation, boundary, out, stream);
}

svs_status svs_warp3d_f64(const double* u, int nz, int ny, int nx, int C, const double* phi, double hz, double hy, double hx, int interpolation, int boundary, double* out, svs_stream_t stream) {
  return warp3d<double>("svs_warp3d_f64", u, nz, ny, nx, C, phi, hz, hy, hx, interpolation, boundary, out, stream);
}

svs_status svs_warp3d_backward(const float* u, int nz, int ny, int nx, const float* phi, const float* grad_out, float hz, float hy, float hx, int interpolation, int boundary, float* grad_u, float* grad_phi, svs_stream_t stream) {
  return warp3d_backward<float>("svs_warp3d_backward", u, nz, ny, nx, phi, grad_out, hz, hy, hx, interpolation, boundary, grad_u, grad_phi, stream);
}

svs_status svs_warp3d_backward_f64(const double* u, int nz, int ny, int nx, const double* phi, const double* grad_out, double hz, double hy, double hx, int interpolation, int boundary, double* grad_u, double* grad_phi, svs_stream_t stream) {
  return warp3d_backward<double>("svs_warp3d_backward_f64", u, nz, ny, nx, phi, grad_out, hz, hy, hx, interpolation, boundary, grad_u, grad_phi, stream);
}

svs_status svs_warp_cnn3d(const float* m, int B, int C, int nz, int ny, int nx, const float* phi, float hz, float hy, float hx, int interpolation, int boundary, float* out, svs_stream_t stream) {
  return warp_cnn3d<float>("svs_warp_cnn3d", m, B, C, nz, ny, nx, phi, hz, hy, hx, interpolation, boundary, out, stream);
}

svs_status svs_warp_cnn3d_f64(const double* m, int B, int C, int nz, int ny, int nx, const double* phi, double hz, double hy, double hx, int interpolation, int boundary, double* out, svs_stream_t stream) {
  return warp_cnn3d<double>("svs_warp_cnn3d_f64", m, B, C, nz, ny, nx, phi, hz, hy, hx, interpolation, boundary, out, stream);
}

svs_status svs_prolongate3d(const float* u, int nz, int ny, int nx, int C, float lz, float ly, float lx, int tz, int ty, int tx, float tlz, float tly, float tlx, int interpolation, int boundary, float* out, svs_stream_t stream) {
  return prolongate3d<float>("svs_prolongate3d", u, nz, ny, nx, C, lz, ly, lx, tz, ty, tx, tlz, tly, tlx, interpolation, boundary, out, stream);
}

svs_status svs_prolongate3d_f64(const double* u, int nz, int ny, int nx, int C, double lz, double ly, double lx, int tz, int ty, int tx, double tlz, double tly, double tlx, int interpolation, int boundary, double* out, svs_stream_t stream) {
  return prolongate3d<double>("svs_prolongate3d_f64", u, nz, ny, nx, C, lz, ly, lx, tz, ty, tx, tlz, tly, tlx, interpolation, boundary, out, stream);
}

}  // extern "C"
