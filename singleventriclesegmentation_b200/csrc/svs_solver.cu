// Fused batched TV-L1 solver of libsvsflow: TVL13DOpticalFlow.compute
// (svs/modules/flow/tvl13d.py:122-255) for many independent frame pairs at once.
//
// Data layout in HBM (per pair and pyramid level, n = NZ*NY*NX voxels): every field is PLANAR
// (component-major: comp c of voxel v at [c*n + v]) so that a warp's 32 consecutive x-voxels
// read 32 consecutive elements of each component.
//   float : I0, I1 (level images), ig = (I1, grad I1) interleaved, one float4 per voxel (the
//           four fields the linearisation samples at the same 64 taps, one 16-byte load each)
//   S     : D (6 planes, the symmetric anisotropic tensor s n n^T + t1 t1^T packed
//           d00 d01 d02 d11 d12 d22), rc (rho_c), gw (warped gradient, 3 planes),
//           u[2] (3 planes each, ping-pong), p[2] (9 planes each, ping-pong)
// S is float, bf16 or fp16 storage; all arithmetic is float.
//
// Kernels per solve: blur (level 0), restrict (levels 1..L-1), and per level: prepare (grad I1
// and D), then per warp: linearise (I1(x+u), grad I1(x+u), rho_c), then per iteration ONE
// iterate kernel that does the dual step and the primal step of tvl13d.py:213-253 together.
// The iterate kernel marches along z through a TX x TY column tile: for each plane it computes
// the new dual field on the tile plus a one-voxel x/y halo (recomputed, so no grid-wide
// dependency between the two half steps) and the new flow on the plane below. The only
// per-iteration HBM traffic is read u, p, D, rc, gw and write u, p: 34 values per voxel.
// The whole batched solve is captured once into a CUDA graph.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "svs_common.cuh"
#include "svs_iterate.cuh"

namespace svs {
namespace {

// Iterate-kernel variants compiled into the library (id 1..N; 0 = automatic).
enum TileForm { kPlain = 0, kTma = 1, kSplit = 2 };
struct TileShape {
  int tx, ty, dist;  // dist: TMA prefetch distance in planes (0 for the plain-load form)
  int form;
  int split;         // index into kSplitShapes (split-role form)
};
constexpr TileShape split_entry(int i) {
  return {kSplitShapes[i].tx, kSplitShapes[i].ty, kSplitShapes[i].dist, kSplit, i};
}
constexpr TileShape kTileShapes[] = {
    {32, 8, 2, kTma, 0},   {32, 8, 3, kTma, 0},   {64, 4, 2, kTma, 0},   {16, 16, 2, kTma, 0},
    {32, 16, 2, kTma, 0},  {32, 8, 0, kPlain, 0}, {32, 4, 0, kPlain, 0}, {16, 16, 0, kPlain, 0},
    split_entry(0),        split_entry(1),        split_entry(2),        split_entry(3),
    split_entry(4),        split_entry(5),        split_entry(6),        split_entry(7),
    split_entry(8),        split_entry(9),        split_entry(10),       split_entry(11),
    split_entry(12),       split_entry(13),       split_entry(14),       split_entry(15),
    split_entry(16),       split_entry(17),       split_entry(18),       split_entry(19),
    split_entry(20),       split_entry(21),       split_entry(22),       split_entry(23),
    split_entry(24)};
constexpr bool split_table_complete() {
  int n = 0;
  for (const TileShape& t : kTileShapes) n += t.form == kSplit;
  return n == kNumSplitShapes;
}
static_assert(split_table_complete(), "every compiled split-role shape has a variant id");
constexpr int kNumTileShapes = sizeof(kTileShapes) / sizeof(kTileShapes[0]);

// ------------------------------------------------------------------------------ small kernels
// grid: (ceil(max voxels / 256), pairs). Desc array offset selects the level.

// Gaussian pre-blur of both frames, flow_utils.py:94-112 (zero padding, (2r+1)^3 taps).
struct BlurW {
  float w[729];  // up to 9^3 taps (sigma < 2)
};
__global__ void blur_pair_kernel(const Desc* __restrict__ descs, float* const* __restrict__ raw,
                                 int r, const __grid_constant__ BlurW W, int use_blur) {
  const Desc d = descs[blockIdx.y];
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v >= d.n) return;
  const float* in0 = raw[2 * blockIdx.y];
  const float* in1 = raw[2 * blockIdx.y + 1];
  float* out0 = const_cast<float*>(d.I0);
  float* out1 = const_cast<float*>(d.I1);
  if (!use_blur) {
    out0[v] = in0[v];
    out1[v] = in1[v];
    return;
  }
  const int x = (int)(v % d.nx), y = (int)((v / d.nx) % d.ny), z = (int)(v / ((int64_t)d.nx * d.ny));
  const int k = 2 * r + 1;
  float a0 = 0.f, a1 = 0.f;
  for (int a = 0; a < k; ++a) {
    const int zz = z + a - r;
    if (zz < 0 || zz >= d.nz) continue;
    for (int b = 0; b < k; ++b) {
      const int yy = y + b - r;
      if (yy < 0 || yy >= d.ny) continue;
      const size_t row = ((size_t)zz * d.ny + yy) * d.nx;
      const float* wr = W.w + (a * k + b) * k;
      for (int c = 0; c < k; ++c) {
        const int xx = x + c - r;
        if (xx < 0 || xx >= d.nx) continue;
        a0 = fmaf(wr[c], __ldg(in0 + row + xx), a0);
        a1 = fmaf(wr[c], __ldg(in1 + row + xx), a1);
      }
    }
  }
  out0[v] = a0;
  out1[v] = a1;
}

// Restriction of I0, I1 from level l-1 (fine) to level l, prolongationOps.cu:533-559 with the
// source coordinate (i*h_c)*L_f/L_c.
__global__ void restrict_kernel(const Desc* __restrict__ fine, const Desc* __restrict__ coarse,
                                int interp, int bdry) {
  const Desc f = fine[blockIdx.y], c = coarse[blockIdx.y];
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v >= c.n) return;
  const int x = (int)(v % c.nx), y = (int)((v / c.nx) % c.ny), z = (int)(v / ((int64_t)c.nx * c.ny));
  const float cx = (float)x * c.hx * f.lx / c.lx;
  const float cy = (float)y * c.hy * f.ly / c.ly;
  const float cz = (float)z * c.hz * f.lz / c.lz;
  FieldRef r0{f.I0, f.nz, f.ny, f.nx, 1}, r1{f.I1, f.nz, f.ny, f.nx, 1};
  const_cast<float*>(c.I0)[v] = sample(r0, cz, cy, cx, f.hz, f.hy, f.hx, interp, bdry);
  const_cast<float*>(c.I1)[v] = sample(r1, cz, cy, cx, f.hz, f.hy, f.hx, interp, bdry);
}

// Per-level preparation, tvl13d.py:179-192: grad I1 (differentialOps.cu:540-655), stored with I1
// as one float4 per voxel, the
// anisotropic tensor from s, n, t1 (anisotropicDifferentialOps.cu:89-141) packed as the
// symmetric matrix s n n^T + t1 t1^T (d00 d01 d02 d11 d12 d22), and (first level only) zero u, p.
// Without anisotropy D is the identity (tvl13d.py:218-219, 231-232 skip the operator).
template <typename SU, typename SP>
__global__ void prepare_kernel(const Desc* __restrict__ descs, int use_aniso, float alpha,
                               float beta, int bdry, int zero_state, int src) {
  const Desc d = descs[blockIdx.y];
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v >= d.n) return;
  const int x = (int)(v % d.nx), y = (int)((v / d.nx) % d.ny), z = (int)(v / ((int64_t)d.nx * d.ny));
  const float* I = d.I1;
  const int64_t sy = d.nx, sz = (int64_t)d.nx * d.ny;
  const float c = I[v];
  const float g0 = fwd_axis(x > 0 ? I[v - 1] : 0.f, c, x < d.nx - 1 ? I[v + 1] : 0.f, x, d.nx, bdry, d.hx);
  const float g1 = fwd_axis(y > 0 ? I[v - sy] : 0.f, c, y < d.ny - 1 ? I[v + sy] : 0.f, y, d.ny, bdry, d.hy);
  const float g2 = fwd_axis(z > 0 ? I[v - sz] : 0.f, c, z < d.nz - 1 ? I[v + sz] : 0.f, z, d.nz, bdry, d.hz);
  reinterpret_cast<float4*>(d.ig)[v] = make_float4(c, g0, g1, g2);
  float D[6] = {1.f, 0.f, 0.f, 1.f, 0.f, 1.f};
  if (use_aniso) {
    const float norm = sqrtf(g0 * g0 + g1 * g1 + g2 * g2);
    if (norm > 0.f) {
      const float s = expf(-alpha * powf(norm, beta));
      const float n0 = g0 / norm, n1 = g1 / norm, n2 = g2 / norm;
      float a0, a1, a2;
      if (n2 > 0.5f) { a0 = n2; a1 = 0.f; a2 = -n0; }
      else { a0 = n1; a1 = -n0; a2 = 0.f; }
      D[0] = s * n0 * n0 + a0 * a0;
      D[1] = s * n0 * n1 + a0 * a1;
      D[2] = s * n0 * n2 + a0 * a2;
      D[3] = s * n1 * n1 + a1 * a1;
      D[4] = s * n1 * n2 + a1 * a2;
      D[5] = s * n2 * n2 + a2 * a2;
    } else {
      for (int i = 0; i < 6; ++i) D[i] = 0.f;
    }
  }
  const long long o = pidx(d, z, y, x);
  SP* Dp = reinterpret_cast<SP*>(d.D);
#pragma unroll
  for (int i = 0; i < 6; ++i) Store<SP>::st(Dp + i * d.cs + o, D[i]);
  if (zero_state) {
    SU* u = reinterpret_cast<SU*>(d.u[src]);
    SP* p = reinterpret_cast<SP*>(d.p[src]);
    for (int i = 0; i < 3; ++i) Store<SU>::st(u + i * d.cs + o, 0.f);
    for (int i = 0; i < 9; ++i) Store<SP>::st(p + i * d.cs + o, 0.f);
  }
}

// Tricubic sample of four interleaved fields (I1 and grad I1, one float4 per voxel) at one
// coordinate, one 16-byte load per tap (warpingOps.cu:572-596 and :632-660 sample each field
// separately, with the same weights and order).
__device__ __forceinline__ void sample_cubic4(const float4* __restrict__ IG, int nz, int ny, int nx, float cz,
                                              float cy, float cx, float hz, float hy, float hx, int bdry,
                                              float out[4]) {
  int ix, iy, iz;
  float wx, wy, wz;
  split_coord(cx, hx, ix, wx);
  split_coord(cy, hy, iy, wy);
  split_coord(cz, hz, iz, wz);
  int xs[4], ys[4];
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    xs[d] = fold(ix + d - 1, nx, bdry);
    ys[d] = fold(iy + d - 1, ny, bdry);
  }
  float bz[4][4];
#pragma unroll
  for (int dz = 0; dz < 4; ++dz) {
    const int zz = fold(iz + dz - 1, nz, bdry);
    float by[4][4];
#pragma unroll
    for (int dy = 0; dy < 4; ++dy) {
      const float4* R = IG + ((int64_t)zz * ny + ys[dy]) * nx;
      const float4 t0 = __ldg(R + xs[0]), t1 = __ldg(R + xs[1]), t2 = __ldg(R + xs[2]), t3 = __ldg(R + xs[3]);
      by[0][dy] = hermite4(t0.x, t1.x, t2.x, t3.x, wx);
      by[1][dy] = hermite4(t0.y, t1.y, t2.y, t3.y, wx);
      by[2][dy] = hermite4(t0.z, t1.z, t2.z, t3.z, wx);
      by[3][dy] = hermite4(t0.w, t1.w, t2.w, t3.w, wx);
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) bz[f][dz] = hermite4(by[f][0], by[f][1], by[f][2], by[f][3], wy);
  }
#pragma unroll
  for (int f = 0; f < 4; ++f) out[f] = hermite4(bz[f][0], bz[f][1], bz[f][2], bz[f][3], wz);
}

// Per-warp linearisation, tvl13d.py:196-201: I1w = I1(x+u), gw = (grad I1)(x+u),
// rho_c = I1w - u.gw - I0.
template <typename SU, typename SP>
__global__ void linearise_kernel(const Desc* __restrict__ descs, int src, int interp, int bdry) {
  const Desc d = descs[blockIdx.y];
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v >= d.n || (d.stop && *d.stop)) return;
  const int x = (int)(v % d.nx), y = (int)((v / d.nx) % d.ny), z = (int)(v / ((int64_t)d.nx * d.ny));
  const long long o = pidx(d, z, y, x);
  const SU* u = reinterpret_cast<const SU*>(d.u[src]);
  const float u0 = Store<SU>::ld(u + o), u1 = Store<SU>::ld(u + d.cs + o), u2 = Store<SU>::ld(u + 2 * d.cs + o);
  const float cx = (float)x * d.hx + u0;
  const float cy = (float)y * d.hy + u1;
  const float cz = (float)z * d.hz + u2;
  float s[4];
  if (interp == SVS_INTERPOLATE_CUBIC_HERMITESPLINE) {
    sample_cubic4(reinterpret_cast<const float4*>(d.ig), d.nz, d.ny, d.nx, cz, cy, cx, d.hz, d.hy, d.hx, bdry, s);
  } else {
    for (int f = 0; f < 4; ++f) {
      FieldRef r{d.ig + f, d.nz, d.ny, d.nx, 4};
      s[f] = sample(r, cz, cy, cx, d.hz, d.hy, d.hx, interp, bdry);
    }
  }
  const float dot = u0 * s[1] + u1 * s[2] + u2 * s[3];
  const float rc = s[0] - dot - d.I0[v];
  SP* gw = reinterpret_cast<SP*>(d.gw);
  Store<SP>::st(reinterpret_cast<SP*>(d.rc) + o, rc);
  Store<SP>::st(gw + o, s[1]);
  Store<SP>::st(gw + d.cs + o, s[2]);
  Store<SP>::st(gw + 2 * d.cs + o, s[3]);
}

// Coarse -> fine transfer of u (scaled by L_f/L_c per axis, tvl13d.py:151-153) and p
// (tvl13d.py:158), prolongationOps.cu:561-625; writes the fine level's buffer 0.
template <typename SU, typename SP>
__global__ void prolong_kernel(const Desc* __restrict__ coarse, const Desc* __restrict__ fine,
                               int src, int interp, int bdry) {
  const Desc c = coarse[blockIdx.y], f = fine[blockIdx.y];
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v >= f.n) return;
  const int x = (int)(v % f.nx), y = (int)((v / f.nx) % f.ny), z = (int)(v / ((int64_t)f.nx * f.ny));
  const float cx = (float)x * f.hx * c.lx / f.lx;
  const float cy = (float)y * f.hy * c.ly / f.ly;
  const float cz = (float)z * f.hz * c.lz / f.lz;
  // python float (double) ratios applied to a float32 tensor
  const float kx = (float)((double)f.lx / (double)c.lx);
  const float ky = (float)((double)f.ly / (double)c.ly);
  const float kz = (float)((double)f.lz / (double)c.lz);
  const SU* uc = reinterpret_cast<const SU*>(c.u[src]);
  const SP* pc = reinterpret_cast<const SP*>(c.p[src]);
  SU* uf = reinterpret_cast<SU*>(f.u[0]);
  SP* pf = reinterpret_cast<SP*>(f.p[0]);
  const long long of = pidx(f, z, y, x);
  int ix, iy, iz;
  float wx, wy, wz;
  split_coord(cx, c.hx, ix, wx);
  split_coord(cy, c.hy, iy, wy);
  split_coord(cz, c.hz, iz, wz);
  for (int comp = 0; comp < 12; ++comp) {
    const SU* FU = uc + comp * c.cs;
    const SP* FP = pc + (comp - 3) * c.cs;
    auto at = [&](int zz, int yy, int xx) {
      const long long o = pidx(c, zz, yy, xx);
      return comp < 3 ? Store<SU>::ld(FU + o) : Store<SP>::ld(FP + o);
    };
    float val;
    if (interp == SVS_INTERPOLATE_CUBIC_HERMITESPLINE) {
      float bz[4];
      for (int dz = 0; dz < 4; ++dz) {
        const int zz = fold(iz + dz - 1, c.nz, bdry);
        float by[4];
        for (int dy = 0; dy < 4; ++dy) {
          const int yy = fold(iy + dy - 1, c.ny, bdry);
          by[dy] = hermite4(at(zz, yy, fold(ix - 1, c.nx, bdry)), at(zz, yy, fold(ix, c.nx, bdry)),
                            at(zz, yy, fold(ix + 1, c.nx, bdry)), at(zz, yy, fold(ix + 2, c.nx, bdry)), wx);
        }
        bz[dz] = hermite4(by[0], by[1], by[2], by[3], wy);
      }
      val = hermite4(bz[0], bz[1], bz[2], bz[3], wz);
    } else if (interp == SVS_INTERPOLATE_LINEAR) {
      const int x0 = fold(ix, c.nx, bdry), x1 = fold(ix + 1, c.nx, bdry);
      const int y0 = fold(iy, c.ny, bdry), y1 = fold(iy + 1, c.ny, bdry);
      const int z0 = fold(iz, c.nz, bdry), z1 = fold(iz + 1, c.nz, bdry);
      val = (1 - wz) * (1 - wy) * (1 - wx) * at(z0, y0, x0);
      val += wz * (1 - wy) * (1 - wx) * at(z1, y0, x0);
      val += (1 - wz) * (1 - wy) * wx * at(z0, y0, x1);
      val += wz * (1 - wy) * wx * at(z1, y0, x1);
      val += (1 - wz) * wy * (1 - wx) * at(z0, y1, x0);
      val += wz * wy * (1 - wx) * at(z1, y1, x0);
      val += (1 - wz) * wy * wx * at(z0, y1, x1);
      val += wz * wy * wx * at(z1, y1, x1);
    } else {
      val = at(nearest_axis(cz, c.hz, c.nz, bdry), nearest_axis(cy, c.hy, c.ny, bdry),
               nearest_axis(cx, c.hx, c.nx, bdry));
    }
    if (comp < 3) {
      const float k = comp == 0 ? kx : (comp == 1 ? ky : kz);
      Store<SU>::st(uf + comp * f.cs + of, val * k);
    } else {
      Store<SP>::st(pf + (comp - 3) * f.cs + of, val);
    }
  }
}

// Cubic coarse -> fine transfer as three separable passes through shared memory: x (reading the
// coarse field), then y, then z. Every output is the same nesting of hermite4 calls on the same
// values as in prolong_kernel (x innermost, then y, then z; folded tap indices), so the result is
// bitwise the same, but a block of PFX x PFY x PFZ fine voxels reads each coarse value it needs
// about once per component instead of 64 times per output. Valid when every coarse axis has at
// most as many nodes as the fine one (the pyramid's halving): a block then needs at most PF + 4
// coarse rows per axis.
constexpr int PFX = 32, PFY = 8, PFZ = 8;
template <typename SU, typename SP>
__global__ void __launch_bounds__(PFX * PFY)
prolong_cubic_kernel(const Desc* __restrict__ coarse, const Desc* __restrict__ fine, int src, int bdry) {
  __shared__ float A[PFZ + 4][PFY + 4][PFX];  // x pass at coarse (z, y) rows
  __shared__ float Bz[PFZ + 4][PFY][PFX];     // y pass at coarse z rows
  __shared__ int tix[PFX], tiy[PFY], tiz[PFZ];
  __shared__ float twx[PFX], twy[PFY], twz[PFZ];
  const Desc c = coarse[blockIdx.y], f = fine[blockIdx.y];
  const int nbx = (f.nx + PFX - 1) / PFX, nby = (f.ny + PFY - 1) / PFY, nbz = (f.nz + PFZ - 1) / PFZ;
  if ((int)blockIdx.x >= nbx * nby * nbz) return;
  const int x0 = (blockIdx.x % nbx) * PFX, y0 = ((blockIdx.x / nbx) % nby) * PFY, z0 = (blockIdx.x / (nbx * nby)) * PFZ;
  const int nxb = min(PFX, f.nx - x0), nyb = min(PFY, f.ny - y0), nzb = min(PFZ, f.nz - z0);
  const int tid = threadIdx.x;
  // per-axis taps and weights of the block's fine nodes, as prolong_kernel computes them
  if (tid < PFX) {
    float w = 0.f;
    int i = 0;
    if (tid < nxb) split_coord((float)(x0 + tid) * f.hx * c.lx / f.lx, c.hx, i, w);
    tix[tid] = i;
    twx[tid] = w;
  } else if (tid < PFX + PFY) {
    const int k = tid - PFX;
    float w = 0.f;
    int i = 0;
    if (k < nyb) split_coord((float)(y0 + k) * f.hy * c.ly / f.ly, c.hy, i, w);
    tiy[k] = i;
    twy[k] = w;
  } else if (tid < PFX + PFY + PFZ) {
    const int k = tid - PFX - PFY;
    float w = 0.f;
    int i = 0;
    if (k < nzb) split_coord((float)(z0 + k) * f.hz * c.lz / f.lz, c.hz, i, w);
    tiz[k] = i;
    twz[k] = w;
  }
  __syncthreads();
  // coarse rows the block needs: [i(first) - 1, i(last) + 2] per axis (taps are monotone in the
  // fine index); at most PF + 4 rows when the coarse axis is no finer than the fine one
  const int ylo = tiy[0] - 1, zlo = tiz[0] - 1;
  const int nyr = min(tiy[nyb - 1] + 3 - ylo, PFY + 4), nzr = min(tiz[nzb - 1] + 3 - zlo, PFZ + 4);
  const float kx = (float)((double)f.lx / (double)c.lx);
  const float ky = (float)((double)f.ly / (double)c.ly);
  const float kz = (float)((double)f.lz / (double)c.lz);
  const SU* uc = reinterpret_cast<const SU*>(c.u[src]);
  const SP* pc = reinterpret_cast<const SP*>(c.p[src]);
  SU* uf = reinterpret_cast<SU*>(f.u[0]);
  SP* pf = reinterpret_cast<SP*>(f.p[0]);
  const int xf = tid % PFX, yf = tid / PFX;
  for (int comp = 0; comp < 12; ++comp) {
    const SU* FU = uc + comp * c.cs;
    const SP* FP = pc + (comp - 3) * c.cs;
    // x pass: A[z row][y row][fine x]
    for (int e = tid; e < nzr * nyr * PFX; e += PFX * PFY) {
      const int xi = e % PFX, yr = (e / PFX) % nyr, zr = e / (PFX * nyr);
      if (xi >= nxb) continue;
      const int zz = fold(zlo + zr, c.nz, bdry), yy = fold(ylo + yr, c.ny, bdry);
      const long long row = pidx(c, zz, yy, 0);
      const int ix = tix[xi];
      long long o[4];
#pragma unroll
      for (int d = 0; d < 4; ++d) o[d] = row + fold(ix + d - 1, c.nx, bdry);
      float v[4];
      if (comp < 3) {
#pragma unroll
        for (int d = 0; d < 4; ++d) v[d] = Store<SU>::ld(FU + o[d]);
      } else {
#pragma unroll
        for (int d = 0; d < 4; ++d) v[d] = Store<SP>::ld(FP + o[d]);
      }
      A[zr][yr][xi] = hermite4(v[0], v[1], v[2], v[3], twx[xi]);
    }
    __syncthreads();
    // y pass: Bz[z row][fine y][fine x]
    for (int e = tid; e < nzr * PFY * PFX; e += PFX * PFY) {
      const int xi = e % PFX, yi = (e / PFX) % PFY, zr = e / (PFX * PFY);
      if (xi >= nxb || yi >= nyb) continue;
      const int r = tiy[yi] - 1 - ylo;
      Bz[zr][yi][xi] = hermite4(A[zr][r][xi], A[zr][r + 1][xi], A[zr][r + 2][xi], A[zr][r + 3][xi], twy[yi]);
    }
    __syncthreads();
    // z pass and store: thread (yf, xf) writes its column of the block
    if (xf < nxb && yf < nyb) {
      const float k = comp == 0 ? kx : (comp == 1 ? ky : kz);
      for (int zi = 0; zi < nzb; ++zi) {
        const int r = tiz[zi] - 1 - zlo;
        const float val = hermite4(Bz[r][yf][xf], Bz[r + 1][yf][xf], Bz[r + 2][yf][xf], Bz[r + 3][yf][xf], twz[zi]);
        const long long of = pidx(f, z0 + zi, y0 + yf, x0 + xf);
        if (comp < 3) Store<SU>::st(uf + comp * f.cs + of, val * k);
        else Store<SP>::st(pf + (comp - 3) * f.cs + of, val);
      }
    }
    __syncthreads();
  }
}

// Level 0 planar state -> the caller's AoS layouts: u [Z,Y,X,3], p [Z,Y,X,3,3].
// Residuals (optional): the root-mean-square change of each pair's flow over one warp,
// sqrt(sum (u_w - u_{w-1})^2 / (3N)), summed in FP64 (warp shuffles, one atomic per block). The
// reference computes per-iteration norms of the changes and never uses them (tvl13d.py:240-253);
// here they are per warp and may stop a converged pair for the rest of the level.
__global__ void residual_reset_kernel(int* __restrict__ stop, double* __restrict__ acc, int np) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < np) {
    stop[i] = 0;
    acc[i] = 0.0;
  }
}

// snaps[pair] holds the flow at the end of the previous warp ([3][n] float); copy_only = 1 at
// the start of a level takes the snapshot without accumulating.
template <typename SU>
__global__ void residual_kernel(const Desc* __restrict__ descs, int src, float* const* __restrict__ snaps,
                                double* __restrict__ acc, int copy_only) {
  const Desc d = descs[blockIdx.y];
  if (*d.stop) return;  // uniform over the block
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double sum = 0.0;
  if (v < d.n) {
    const int x = (int)(v % d.nx), y = (int)((v / d.nx) % d.ny), z = (int)(v / ((int64_t)d.nx * d.ny));
    const long long o = pidx(d, z, y, x);
    const SU* u = reinterpret_cast<const SU*>(d.u[src]);
    float* snap = snaps[blockIdx.y];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float now = Store<SU>::ld(u + c * d.cs + o);
      const double diff = (double)now - (double)snap[c * d.n + v];
      sum += diff * diff;
      snap[c * d.n + v] = now;
    }
  }
  if (copy_only) return;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off);
  __shared__ double part[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) part[wid] = sum;
  __syncthreads();
  if (wid == 0) {
    sum = lane < (int)(blockDim.x >> 5) ? part[lane] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off);
    if (lane == 0) atomicAdd(acc + blockIdx.y, sum);
  }
}

// Log the warp's residual of every pair (-1 if the pair had stopped) and apply the stop rule.
__global__ void residual_finish_kernel(const Desc* __restrict__ descs, double* __restrict__ acc,
                                       float* __restrict__ log, int levels, int warps, int level, int w,
                                       float tol, int np) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const Desc& d = descs[i];
  float* slot = log + ((size_t)i * levels + level) * warps + w;
  if (*d.stop) {
    *slot = -1.f;
    return;
  }
  const double r = sqrt(acc[i] / (3.0 * (double)d.n));
  *slot = (float)r;
  acc[i] = 0.0;
  if (tol > 0.f && r < (double)tol) *d.stop = 1;
}

template <typename SU, typename SP>
__global__ void finalize_kernel(const Desc* __restrict__ descs, int src, float* const* __restrict__ u_out,
                                float* const* __restrict__ p_out) {
  const Desc d = descs[blockIdx.y];
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v >= d.n) return;
  const int x = (int)(v % d.nx), y = (int)((v / d.nx) % d.ny), z = (int)(v / ((int64_t)d.nx * d.ny));
  const long long o = pidx(d, z, y, x);
  const SU* u = reinterpret_cast<const SU*>(d.u[src]);
  float* uo = u_out[blockIdx.y];
  for (int c = 0; c < 3; ++c) uo[3 * v + c] = Store<SU>::ld(u + c * d.cs + o);
  float* po = p_out[blockIdx.y];
  if (po) {
    const SP* p = reinterpret_cast<const SP*>(d.p[src]);
    for (int c = 0; c < 9; ++c) po[9 * v + c] = Store<SP>::ld(p + c * d.cs + o);
  }
}

// Optional warm start (num_scales == 1 only: otherwise the reference overwrites u and p,
// tvl13d.py:150, 158): AoS caller fields -> level-0 planar buffer 0.
template <typename SU, typename SP>
__global__ void warm_start_kernel(const Desc* __restrict__ descs, const float* const* __restrict__ u_in,
                                  const float* const* __restrict__ p_in) {
  const Desc d = descs[blockIdx.y];
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v >= d.n) return;
  const int x = (int)(v % d.nx), y = (int)((v / d.nx) % d.ny), z = (int)(v / ((int64_t)d.nx * d.ny));
  const long long o = pidx(d, z, y, x);
  const float* ui = u_in[blockIdx.y];
  const float* pi = p_in[blockIdx.y];
  SU* u = reinterpret_cast<SU*>(d.u[0]);
  SP* p = reinterpret_cast<SP*>(d.p[0]);
  for (int c = 0; c < 3; ++c) Store<SU>::st(u + c * d.cs + o, ui ? ui[3 * v + c] : 0.f);
  for (int c = 0; c < 9; ++c) Store<SP>::st(p + c * d.cs + o, pi ? pi[9 * v + c] : 0.f);
}

}  // namespace
}  // namespace svs

// =============================================================================================
// Host side: plan (device state, tile lists, TMA descriptors), the enqueue sequence, CUDA graph.
// =============================================================================================
struct svs_plan {
  svs_tvl1_params prm{};
  int num_pairs = 0;
  int capacity = 0;                        // pairs the device tables hold (svs_tvl1_plan_retarget)
  int levels = 0;
  std::vector<int> dims;                   // level-0 dims, 3 per pair
  std::vector<svs::Desc> h_descs;          // [levels][pairs]
  svs::Desc* d_descs = nullptr;
  svs::TMaps* d_maps = nullptr;            // [levels][pairs], for the tile shape in use
  std::vector<std::vector<svs::Tile>> h_tiles;  // per level
  std::vector<svs::Tile*> d_tiles;
  std::vector<int> level_tile;             // tile id used per level
  std::vector<std::vector<int>> pair_used; // tile id used per level and pair (groups included)
  std::vector<int> level_tile_req;         // per-level request (0 = use tile_id)
  std::vector<int> level_chunks_req;       // per-level z chunks per column (0 = the wave model)
  int tile_id = 0;                         // requested for all levels (0 = automatic)
  int tiles_built_for = -1;
  int tile_epoch = 0;                      // bumped on every tile request change
  void* arena = nullptr;
  size_t arena_bytes = 0;
  int* d_status = nullptr;                 // device error bits (SVS_DEV_*)
  float** d_raw = nullptr;                 // [2*pairs] raw input frames (device)
  float** d_uout = nullptr;                // [pairs] AoS u results
  float** d_pout = nullptr;                // [pairs] AoS p results (or null entries)
  float** d_umed = nullptr;                // [pairs] median outputs
  const float** d_uinit = nullptr;         // [pairs] warm start (num_scales == 1)
  const float** d_pinit = nullptr;
  std::vector<float*> raw, uout, pout, umed;
  std::vector<const float*> uinit, pinit;
  std::vector<float> sig_sched, tau_sched;  // per iteration inside one warp
  svs::BlurW blur{};
  int blur_r = 0;
  bool want_p = false;
  bool warm = false;
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t graph_kernels = 0;
  int graph_tile = -1;
  bool graph_warm = false;
  bool graph_want_p = false;
  // pairs whose variant differs from their level's (svs_tvl1_plan_set_pair_tile): per level, one
  // group per variant; the groups of a level run as parallel branches of the graph
  struct TileGroup {
    int tid = 0;
    std::vector<svs::Tile> h;
    svs::Tile* d = nullptr;
  };
  std::vector<std::vector<TileGroup>> extra;  // [level]
  std::vector<std::vector<int>> pair_tile_req;  // [level][pair], 0 = the level's variant
  const std::vector<char>* pair_mask = nullptr; // during set-up: the pairs a dispatch or tile build covers
  const svs::Tile* launch_tiles = nullptr;      // launch override (a group's tiles)
  unsigned launch_count = 0;
  bool launch_override = false;
  std::vector<cudaStream_t> side;               // one per group of the widest level
  std::vector<cudaEvent_t> events;              // fork + one join per side stream
  // residuals (svs_tvl1_plan_set_residuals)
  bool res_on = false;
  float res_tol = 0.f;
  int* d_stop = nullptr;                   // [pairs]
  double* d_acc = nullptr;                 // [pairs]
  float* d_reslog = nullptr;               // [pairs][levels][max_warps]
  float** d_snaps = nullptr;               // [pairs] -> [3][n0] floats
  std::vector<float*> snaps;
  // bounded pipeline waits (svs_tvl1_plan_set_stall_test)
  unsigned wait_us = 2000000;
  int stall_level = -1, stall_cta = -1, stall_plane = -1;
  // persistent iteration loop (svs_tvl1_plan_set_persistent): one cooperative launch per warp
  bool persistent = false;
  std::vector<char> level_persist;         // per level: the persistent form is used
  float* d_sig = nullptr;                  // [max_outer_iterations] schedule on the device
  float* d_tau = nullptr;
  unsigned* d_gridbar = nullptr;           // grid-barrier arrival counter
};

namespace svs {
namespace {

// Storage of the flow (u) and of the other iteration fields (p, D, rc, gw).
size_t flow_bytes(int storage) { return (storage == SVS_STORAGE_BF16 || storage == SVS_STORAGE_F16) ? 2 : 4; }
size_t field_bytes(int storage) { return storage == SVS_STORAGE_F32 ? 4 : 2; }
CUtensorMapDataType map_type(int bytes, bool bf16) {
  return bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                    : (bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16);
}
bool is_bf16(int storage) { return storage == SVS_STORAGE_BF16 || storage == SVS_STORAGE_BF16_FLOW32; }

// ---------------------------------------------------------------------- TMA tensor maps
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// A 4D map (x, y, z, component) over one pitched planar field, box {bx, by, 1, bc}.
bool encode_field(CUtensorMap* m, int es_bytes, bool bf16, const void* base, const Desc& d, int comps, int bx,
                  int by) {
  auto fn = encode_fn();
  if (!fn) return false;
  const CUtensorMapDataType dt = map_type(es_bytes, bf16);
  const cuuint64_t es = (cuuint64_t)es_bytes;
  cuuint64_t gdim[4] = {(cuuint64_t)d.nx, (cuuint64_t)d.ny, (cuuint64_t)d.nz, (cuuint64_t)comps};
  cuuint64_t gstride[3] = {(cuuint64_t)d.pitch * es, (cuuint64_t)d.pitch * d.ny * es, (cuuint64_t)d.cs * es};
  cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 1u, (cuuint32_t)comps};
  cuuint32_t estride[4] = {1, 1, 1, 1};
  const CUresult r = fn(m, dt, 4, const_cast<void*>(base), gdim, gstride, box, estride,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Tensor maps of every pair of a level, boxes {ux, uy} for u, {px, py} for p and D, tile {tx, ty}
// for rc and gw.
bool encode_maps(svs_plan& P, std::vector<TMaps>& maps, int level, int ux, int uy, int px, int py, int tx,
                 int ty) {
  const bool bf = is_bf16(P.prm.storage);
  const int esu = (int)flow_bytes(P.prm.storage), esp = (int)field_bytes(P.prm.storage);
  for (int i = 0; i < P.num_pairs; ++i) {
    if (P.pair_mask && !(*P.pair_mask)[i]) continue;
    const size_t k = (size_t)level * P.num_pairs + i;
    const Desc& d = P.h_descs[k];
    TMaps& m = maps[k];
    bool ok = encode_field(&m.u[0], esu, bf, d.u[0], d, 3, ux, uy) &&
              encode_field(&m.u[1], esu, bf, d.u[1], d, 3, ux, uy) &&
              encode_field(&m.p[0], esp, bf, d.p[0], d, 9, px, py) &&
              encode_field(&m.p[1], esp, bf, d.p[1], d, 9, px, py) &&
              encode_field(&m.D, esp, bf, d.D, d, 6, px, py) &&
              encode_field(&m.rc, esp, bf, d.rc, d, 1, tx, ty) &&
              encode_field(&m.gw, esp, bf, d.gw, d, 3, tx, ty);
    if (!ok) return false;
  }
  return true;
}

template <typename SU, typename SP, int TX, int TY, int DIST>
bool tma_prepare(svs_plan& P, std::vector<TMaps>& maps, int level) {
  using G = TmaGeom<SU, SP, TX, TY, DIST>;
  if (G::SMEM > 227 * 1024) return false;
  if (cudaFuncSetAttribute(iterate_tma_kernel<SU, SP, TX, TY, DIST, false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM) != cudaSuccess ||
      cudaFuncSetAttribute(iterate_tma_kernel<SU, SP, TX, TY, DIST, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return encode_maps(P, maps, level, G::UXB, G::UYB, G::PXB, G::PYB, TX, TY);
}

// Dispatch over the compiled variants. `op` 0: prepare (attributes + maps), 1: launch.
template <typename SU, typename SP>
bool iter_variant(svs_plan& P, std::vector<TMaps>* maps, int level, int tid, int op, const IterArgs* a,
                  cudaStream_t s) {
  const unsigned nt = P.launch_override ? P.launch_count : (unsigned)P.h_tiles[level].size();
  const Tile* tl = P.launch_override ? P.launch_tiles : (P.d_tiles.empty() ? nullptr : P.d_tiles[level]);
  if (op == 1 && nt == 0) return true;  // nothing of this level runs this variant
  // the MIRROR boundary (the solver's default) gets two-term stencils; other boundaries the
  // general three-term form
  const bool gen = P.prm.boundary != SVS_BOUNDARY_MIRROR;
#define SVS_TMA_CASE(ID, TX, TY, DS)                                                                      \
  case ID:                                                                                                \
    if (op == 0) return tma_prepare<SU, SP, TX, TY, DS>(P, *maps, level);                                \
    if (gen)                                                                                              \
      iterate_tma_kernel<SU, SP, TX, TY, DS, true><<<nt, (TX + 2) * (TY + 2), TmaGeom<SU, SP, TX, TY, DS>::SMEM, s>>>( \
          tl, P.d_descs, P.d_maps, *a, P.d_status);                                                       \
    else                                                                                                  \
      iterate_tma_kernel<SU, SP, TX, TY, DS, false><<<nt, (TX + 2) * (TY + 2), TmaGeom<SU, SP, TX, TY, DS>::SMEM, s>>>( \
          tl, P.d_descs, P.d_maps, *a, P.d_status);                                                       \
    return true;
#define SVS_PLAIN_CASE(ID, TX, TY)                                                                   \
  case ID:                                                                                           \
    if (op == 0) return true;                                                                        \
    if (gen) iterate_kernel<SU, SP, TX, TY, true><<<nt, (TX + 2) * (TY + 2), 0, s>>>(tl, P.d_descs, *a); \
    else iterate_kernel<SU, SP, TX, TY, false><<<nt, (TX + 2) * (TY + 2), 0, s>>>(tl, P.d_descs, *a); \
    return true;
  switch (tid) {
    SVS_TMA_CASE(1, 32, 8, 2)
    SVS_TMA_CASE(2, 32, 8, 3)
    SVS_TMA_CASE(3, 64, 4, 2)
    SVS_TMA_CASE(4, 16, 16, 2)
    SVS_TMA_CASE(5, 32, 16, 2)
    SVS_PLAIN_CASE(6, 32, 8)
    SVS_PLAIN_CASE(7, 32, 4)
    SVS_PLAIN_CASE(8, 16, 16)
    default: return false;
  }
#undef SVS_TMA_CASE
#undef SVS_PLAIN_CASE
}

bool iter_dispatch(svs_plan& P, std::vector<TMaps>* maps, int level, int tid, int op, const IterArgs* a,
                   cudaStream_t s) {
  const TileShape& ts = kTileShapes[tid - 1];
  if (ts.form == kSplit) {
    const unsigned nt = P.launch_override ? P.launch_count : (unsigned)P.h_tiles[level].size();
    const Tile* tl = P.launch_override ? P.launch_tiles : (P.d_tiles.empty() ? nullptr : P.d_tiles[level]);
    if (op == 1 && nt == 0) return true;
    const bool gen = P.prm.boundary != SVS_BOUNDARY_MIRROR;
    int box[4] = {0, 0, 0, 0};
    if (!split_variant(P.prm.storage, ts.split, op, gen, nt, tl, P.d_descs, P.d_maps, a, P.d_status, s, box))
      return false;
    return op != 0 || encode_maps(P, *maps, level, box[0], box[1], box[2], box[3], ts.tx, ts.ty);
  }
  switch (P.prm.storage) {
    case SVS_STORAGE_BF16: return iter_variant<__nv_bfloat16, __nv_bfloat16>(P, maps, level, tid, op, a, s);
    case SVS_STORAGE_F16: return iter_variant<__half, __half>(P, maps, level, tid, op, a, s);
    case SVS_STORAGE_BF16_FLOW32: return iter_variant<float, __nv_bfloat16>(P, maps, level, tid, op, a, s);
    case SVS_STORAGE_F16_FLOW32: return iter_variant<float, __half>(P, maps, level, tid, op, a, s);
    default: return iter_variant<float, float>(P, maps, level, tid, op, a, s);
  }
}

constexpr int split_id(int tx, int ty, int dist, int v, int opt = 0) {
  for (int i = 0; i < kNumTileShapes; ++i)
    if (kTileShapes[i].form == kSplit && kTileShapes[i].tx == tx && kTileShapes[i].ty == ty &&
        kTileShapes[i].dist == dist && kSplitShapes[kTileShapes[i].split].v == v &&
        !kSplitShapes[kTileShapes[i].split].as && kSplitShapes[kTileShapes[i].split].opt == opt &&
        kSplitShapes[kTileShapes[i].split].smask == kAllStorages)
      return i + 1;
  return 0;
}
constexpr int kAutoF32 = split_id(32, 16, 3, 2), kAuto16 = split_id(16, 16, 3, 1),
              kAuto16W40 = split_id(40, 8, 3, 2, kRowPairs | kNoSel), kAuto16Narrow = split_id(32, 8, 3, 1);
static_assert(kAutoF32 > 0 && kAuto16 > 0 && kAuto16W40 > 0 && kAuto16Narrow > 0,
              "automatic variants are compiled");

// Automatic choice per level from the level's sizes (nz, ny, nx per pair), the storage mode and
// the SM count; host arithmetic only. Returns the level's variant; pair_tid[i] is pair i's own
// variant where it differs (0: the level's).
//
// Levels whose column tiles do not fill the GPU twice over (measured on B200 with batches of 80^3
// pairs, levels 80^3, 40^3 and 20^3): split-role pipelines with prefetch distance 3. 4-byte
// fields: 32x16 tiles of voxel pairs (one CTA per SM). 2-byte fields: 40x8 tiles of voxel pairs
// when every width is a multiple of 40 (no idle lanes; interior lanes placed in row pairs, which
// halves the shared-memory bank conflicts), 32x8 tiles of single voxels for widths up to 32, 16x16
// tiles of single voxels otherwise.
//
// 2-byte fields at levels that fill the GPU at least twice (the iteration time is then the work of
// all tiles, not the latency of one z march): each pair takes the variant with the least work,
// column tiles x planes x the variant's time per column-tile plane at full occupancy (measured on
// B200 at level 0 of 68-128 pairs of 64^3-128^3); the variant with the most work becomes the
// level's, the others run as groups of pairs (parallel branches of the graph).
//
// The plain-load 32x8 form if TMA descriptors cannot be built. The autotuner measures instead of
// assuming.
struct AutoCost {
  int tid;
  float ns;  // per column-tile plane
};
// f16-flow32 and bf16-flow32: 40x8 voxel pairs in row pairs 5.96-6.32 ns (320 voxels), 32x8
// voxel pairs 5.05-5.28 ns (256 voxels), 16x16 single voxels 5.90-6.09 ns (256 voxels): per voxel
// the first two are alike (~19-20 ps) and the third 15% slower
constexpr AutoCost kAutoCosts16[] = {{kAuto16W40, 6.13f}, {split_id(32, 8, 3, 2), 5.20f}, {kAuto16, 6.00f}};
constexpr int kAutoWaves = 2;  // waves of 40x8 column tiles (two CTAs per SM) for the per-pair choice

int auto_choice(int storage, int n, const int* dims, int sms, int* pair_tid) {
  for (int i = 0; i < n; ++i) pair_tid[i] = 0;
  if (storage == SVS_STORAGE_F32) return kAutoF32;
  bool all40 = true;
  int widest = 0;
  long long cols = 0;
  for (int i = 0; i < n; ++i) {
    const int ny = dims[3 * i + 1], nx = dims[3 * i + 2];
    all40 = all40 && nx % 40 == 0;
    widest = std::max(widest, nx);
    cols += (long long)ceil_div(nx, 40) * ceil_div(ny, 8);
  }
  const int base = all40 ? kAuto16W40 : widest <= 32 ? kAuto16Narrow : kAuto16;
  if (n < 1 || cols < (long long)kAutoWaves * 2 * std::max(sms, 1)) return base;
  std::vector<double> work(kNumTileShapes + 1, 0.0);
  for (int i = 0; i < n; ++i) {
    const int nz = dims[3 * i], ny = dims[3 * i + 1], nx = dims[3 * i + 2];
    double best = -1.0;
    for (const AutoCost& c : kAutoCosts16) {
      const TileShape& ts = kTileShapes[c.tid - 1];
      const double w = (double)ceil_div(nx, ts.tx) * ceil_div(ny, ts.ty) * nz * c.ns;
      if (best < 0 || w < best) {
        best = w;
        pair_tid[i] = c.tid;
      }
    }
    work[pair_tid[i]] += best;
  }
  const int main_tid = (int)(std::max_element(work.begin(), work.end()) - work.begin());
  for (int i = 0; i < n; ++i)
    if (pair_tid[i] == main_tid) pair_tid[i] = 0;
  return main_tid;
}

int auto_level(const svs_plan& P, int level, std::vector<int>& pair_tid) {
  std::vector<int> dims(3 * (size_t)P.num_pairs);
  for (int i = 0; i < P.num_pairs; ++i) {
    const Desc& d = P.h_descs[(size_t)level * P.num_pairs + i];
    dims[3 * i] = d.nz;
    dims[3 * i + 1] = d.ny;
    dims[3 * i + 2] = d.nx;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  pair_tid.assign(P.num_pairs, 0);
  return auto_choice(P.prm.storage, P.num_pairs, dims.data(), sms, pair_tid.data());
}

// z chunks per column for a split-role variant. The launch's CTAs are dispatched in tile-list
// order onto the resident slots (SMs x CTAs per SM from the occupancy calculator). Columns fill
// whole waves of `main_c` chunks each; the `tail_cols` columns that would leave the last wave
// part-empty come after them, cut into `tail_c` chunks, so the tail spreads over all slots. The
// plan minimises the makespan in plane steps, sum over the two phases of waves x (planes per chunk
// + kFillPlanes), where kFillPlanes stands for the pipeline start of a chunk (the first DIST
// planes and the extra dual plane below z0). Chunks go down to one plane: a single 80^3 pair runs
// a level-1 iteration (40^3, five 40x8 column tiles) 1.7x faster as 200 one-plane chunks than as
// 25 eight-plane chunks.
constexpr int kFillPlanes = 3;
struct ChunkPlan {
  int main_c = 1, tail_c = 1;
  long long tail_cols = 0;  // the last tail_cols columns of the tile list use tail_c
};
// The plan for `xy_tiles` columns of up to `nz` planes on `slots` resident CTA slots.
ChunkPlan chunk_plan(long long xy_tiles, int nz, long long slots) {
  ChunkPlan best;
  if (xy_tiles <= 0 || nz <= 0 || slots <= 0) return best;
  long long best_cost = -1;
  for (int cm = 1; cm <= nz; ++cm) {
    // columns whose chunks fill whole waves; the rest form the tail
    const long long main_cols = std::min(xy_tiles, (xy_tiles * cm / slots) * slots / cm);
    const long long t_main = ceil_div(main_cols * cm, slots) * (ceil_div(nz, cm) + kFillPlanes);
    const long long rest = xy_tiles - main_cols;
    for (int ct = cm; ct <= nz; ++ct) {
      const long long t_tail = rest ? ceil_div(rest * ct, slots) * (ceil_div(nz, ct) + kFillPlanes) : 0;
      if (best_cost < 0 || t_main + t_tail < best_cost) {
        best_cost = t_main + t_tail;
        best = ChunkPlan{cm, rest ? ct : cm, rest};
      }
      if (!rest) break;
    }
  }
  return best;
}

ChunkPlan split_chunks(const svs_plan& P, int level, int tid, long long xy_tiles) {
  ChunkPlan best;
  int dev = 0, sms = 148, per_sm = 0, nz = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int box[4] = {0, 0, 0, 0};
  const TileShape& ts = kTileShapes[tid - 1];
  if (!split_variant(P.prm.storage, ts.split, 2, P.prm.boundary != SVS_BOUNDARY_MIRROR, 0, nullptr, nullptr,
                     nullptr, nullptr, nullptr, nullptr, box) ||
      xy_tiles <= 0)
    return best;
  per_sm = std::max(1, box[0]);
  for (int i = 0; i < P.num_pairs; ++i)
    if (!P.pair_mask || (*P.pair_mask)[i]) nz = std::max(nz, P.h_descs[(size_t)level * P.num_pairs + i].nz);
  return chunk_plan(xy_tiles, nz, (long long)sms * per_sm);
}

// Tiles of the level's pairs (those in P.pair_mask when set) for variant tid, into `out_opt` or
// the level's own list.
void build_tiles(svs_plan& P, int level, int tid, std::vector<Tile>* out_opt = nullptr) {
  const TileShape ts = kTileShapes[tid - 1];
  std::vector<Tile>& out = out_opt ? *out_opt : P.h_tiles[level];
  out.clear();
  auto in = [&](int i) { return !P.pair_mask || (*P.pair_mask)[i]; };
  long long xy_tiles = 0;
  for (int i = 0; i < P.num_pairs; ++i) {
    if (!in(i)) continue;
    const Desc& d = P.h_descs[(size_t)level * P.num_pairs + i];
    xy_tiles += (long long)ceil_div(d.nx, ts.tx) * ceil_div(d.ny, ts.ty);
  }
  // split-role variants: chunks from the wave model above (the tail columns after the others);
  // other forms: z is split into chunks only when the level has too few column tiles to fill the
  // GPU; a per-level request overrides both with one count for every column
  const int req_c = level < (int)P.level_chunks_req.size() ? P.level_chunks_req[level] : 0;
  ChunkPlan cp;
  if (req_c > 0) {
    cp.main_c = req_c;
  } else if (ts.form == kSplit) {
    cp = split_chunks(P, level, tid, xy_tiles);
  } else {
    const long long target = 148LL * 2;
    if (xy_tiles < target) cp.main_c = (int)((target + xy_tiles - 1) / xy_tiles);
  }
  const bool plain_cap = req_c <= 0 && ts.form != kSplit;  // at least 8 planes per chunk
  std::vector<Tile> tail;
  long long col = 0;
  for (int i = 0; i < P.num_pairs; ++i) {
    if (!in(i)) continue;
    const Desc& d = P.h_descs[(size_t)level * P.num_pairs + i];
    const long long ncols = (long long)ceil_div(d.nx, ts.tx) * ceil_div(d.ny, ts.ty);
    // within a pair, chunk by chunk (the columns of one z range next to each other)
    for (int part = 0; part < 2; ++part) {
      int chunks = part ? cp.tail_c : cp.main_c;
      chunks = std::max(1, std::min(chunks, plain_cap ? std::max(1, d.nz / 8) : d.nz));
      const int zc = (d.nz + chunks - 1) / chunks;
      for (int z0 = 0; z0 < d.nz; z0 += zc) {
        long long c = col;
        for (int y0 = 0; y0 < d.ny; y0 += ts.ty)
          for (int x0 = 0; x0 < d.nx; x0 += ts.tx, ++c) {
            if ((c >= xy_tiles - cp.tail_cols) != (part == 1)) continue;
            const int z1 = std::min(d.nz, z0 + zc);
            (part ? tail : out).push_back(Tile{level * P.num_pairs + i, x0, y0, z0 | (z1 << 16)});
          }
      }
    }
    col += ncols;
  }
  out.insert(out.end(), tail.begin(), tail.end());
}

// (Re)build tile lists and TMA descriptors for the requested tile id.
svs_status setup_tiles(svs_plan& P) {
  const int want = P.tile_id;
  P.h_tiles.assign(P.levels, {});
  P.level_tile.assign(P.levels, 0);
  P.pair_used.assign(P.levels, {});
  for (auto& lv : P.extra)
    for (auto& grp : lv) cudaFree(grp.d);
  P.extra.assign(P.levels, {});
  std::vector<TMaps> maps((size_t)P.levels * P.num_pairs);
  std::memset(maps.data(), 0, maps.size() * sizeof(TMaps));
  for (int l = 0; l < P.levels; ++l) {
    const int req = (l < (int)P.level_tile_req.size() && P.level_tile_req[l] > 0) ? P.level_tile_req[l] : want;
    std::vector<int> autop;
    int tid = req > 0 ? req : auto_level(P, l, autop);
    // per-pair requests (and, without a level request, the automatic per-pair choices) that
    // differ from the level's variant form groups of their own
    std::vector<int> own(P.num_pairs, 0);
    if (l < (int)P.pair_tile_req.size())
      for (int i = 0; i < P.num_pairs; ++i) own[i] = P.pair_tile_req[l][i];
    if (req <= 0 && !autop.empty()) {
      // an automatic group whose variant cannot be set up (shared memory or TMA descriptor
      // limits) leaves every pair with the level's variant
      bool usable = true;
      for (const AutoCost& c : kAutoCosts16) {
        std::vector<char> gm(P.num_pairs, 0);
        bool any = false;
        for (int i = 0; i < P.num_pairs; ++i) any |= gm[i] = !own[i] && autop[i] == c.tid;
        if (!any) continue;
        P.pair_mask = &gm;
        usable = usable && iter_dispatch(P, &maps, l, c.tid, 0, nullptr, nullptr);
      }
      P.pair_mask = nullptr;
      for (int i = 0; i < P.num_pairs && usable; ++i)
        if (!own[i]) own[i] = autop[i];
    }
    std::vector<char> mask(P.num_pairs, 1);
    for (int i = 0; i < P.num_pairs; ++i) mask[i] = own[i] == 0 || own[i] == tid;
    P.pair_mask = &mask;
    // attributes and tensor maps first: the tile builder asks the occupancy calculator
    if (!iter_dispatch(P, &maps, l, tid, 0, nullptr, nullptr)) {
      if (req > 0) {
        P.pair_mask = nullptr;
        return fail(SVS_ERR_UNSUPPORTED, "tile variant not usable for this plan (shared memory or TMA descriptor limits)");
      }
      tid = 6;  // plain-load 32x8
      for (int i = 0; i < P.num_pairs; ++i) mask[i] = own[i] == 0 || own[i] == tid;
    }
    build_tiles(P, l, tid);
    P.level_tile[l] = tid;
    for (int i = 0; i < P.num_pairs; ++i) {
      if (mask[i]) continue;
      const int g = own[i];
      bool seen = false;
      for (auto& grp : P.extra[l]) seen |= grp.tid == g;
      if (seen) continue;
      std::vector<char> gm(P.num_pairs, 0);
      for (int j = 0; j < P.num_pairs; ++j) gm[j] = own[j] == g && !mask[j];
      P.pair_mask = &gm;
      if (!iter_dispatch(P, &maps, l, g, 0, nullptr, nullptr)) {
        P.pair_mask = nullptr;
        return fail(SVS_ERR_UNSUPPORTED, "pair tile variant not usable for this plan (shared memory or TMA descriptor limits)");
      }
      svs_plan::TileGroup grp;
      grp.tid = g;
      build_tiles(P, l, g, &grp.h);
      P.extra[l].push_back(std::move(grp));
    }
    P.pair_mask = nullptr;
    P.pair_used[l].assign(P.num_pairs, tid);
    for (int i = 0; i < P.num_pairs; ++i)
      if (!mask[i]) P.pair_used[l][i] = own[i];
  }
  // persistent iteration loop: levels whose pairs share one split-role variant that has the form
  P.level_persist.assign(P.levels, 0);
  for (int l = 0; l < P.levels && P.persistent; ++l) {
    const TileShape& ts = kTileShapes[P.level_tile[l] - 1];
    P.level_persist[l] = P.extra[l].empty() && ts.form == kSplit && !P.h_tiles[l].empty() &&
                         split_persist(P.prm.storage, ts.split, 0, P.prm.boundary != SVS_BOUNDARY_MIRROR, 0, nullptr,
                                       nullptr, nullptr, nullptr, nullptr, nullptr);
  }
  for (auto* p : P.d_tiles) cudaFree(p);
  P.d_tiles.assign(P.levels, nullptr);
  size_t widest = 0;
  for (int l = 0; l < P.levels; ++l) {
    const size_t bytes = P.h_tiles[l].size() * sizeof(Tile);
    svs_status st = check_cuda(cudaMalloc(&P.d_tiles[l], std::max<size_t>(bytes, sizeof(Tile))), "tile list");
    if (!st && bytes) st = check_cuda(cudaMemcpy(P.d_tiles[l], P.h_tiles[l].data(), bytes, cudaMemcpyHostToDevice), "tile list");
    for (auto& grp : P.extra[l]) {
      const size_t gb = grp.h.size() * sizeof(Tile);
      if (!st) st = check_cuda(cudaMalloc(&grp.d, gb), "tile list");
      if (!st) st = check_cuda(cudaMemcpy(grp.d, grp.h.data(), gb, cudaMemcpyHostToDevice), "tile list");
    }
    if (st) return st;
    widest = std::max(widest, P.extra[l].size());
  }
  while (P.side.size() < widest) {
    cudaStream_t st_ = nullptr;
    svs_status st = check_cuda(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "group stream");
    if (st) return st;
    P.side.push_back(st_);
  }
  while (P.events.size() < widest + 1) {
    cudaEvent_t e = nullptr;
    svs_status st = check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "group event");
    if (st) return st;
    P.events.push_back(e);
  }
  return check_cuda(cudaMemcpy(P.d_maps, maps.data(), maps.size() * sizeof(TMaps), cudaMemcpyHostToDevice), "tensor maps");
}

// Blocks of prolong_cubic_kernel for the largest pair of a (fine) level.
unsigned prolong_blocks(const svs_plan& P, int level) {
  long long m = 0;
  for (int i = 0; i < P.num_pairs; ++i) {
    const Desc& d = P.h_descs[(size_t)level * P.num_pairs + i];
    m = std::max(m, (long long)ceil_div(d.nx, PFX) * ceil_div(d.ny, PFY) * ceil_div(d.nz, PFZ));
  }
  return (unsigned)m;
}

// Every pair's level `level` has at most as many nodes per axis as level-1 (prolong_cubic_kernel).
bool coarse_within(const svs_plan& P, int level) {
  for (int i = 0; i < P.num_pairs; ++i) {
    const Desc& c = P.h_descs[(size_t)level * P.num_pairs + i];
    const Desc& f = P.h_descs[(size_t)(level - 1) * P.num_pairs + i];
    if (c.nx > f.nx || c.ny > f.ny || c.nz > f.nz) return false;
  }
  return true;
}

long long max_voxels(const svs_plan& P, int level) {
  long long m = 0;
  for (int i = 0; i < P.num_pairs; ++i) m = std::max(m, P.h_descs[(size_t)level * P.num_pairs + i].n);
  return m;
}

IterArgs iter_args(const svs_plan& P, int it, int cur) {
  IterArgs a;
  a.sigma = P.sig_sched.empty() ? (float)P.prm.sigma : P.sig_sched[it];
  a.tau = P.tau_sched.empty() ? (float)P.prm.tau : P.tau_sched[it];
  a.factor = a.tau * P.prm.weight_matching;  // opticalFlowOps.cu:440
  a.wtv = P.prm.weight_tv;
  a.src = cur;
  a.bdry = P.prm.boundary;
  a.wait_us = P.wait_us;
  a.stall_cta = -1;
  a.stall_plane = -1;
  return a;
}

// Groups of pairs with their own variant (svs_tvl1_plan_set_pair_tile) run on side streams:
// fork after the level's linearisation, one launch per group and iteration, join before the next.
size_t level_groups(const svs_plan& P, int l) { return l < (int)P.extra.size() ? P.extra[l].size() : 0; }
void fork_groups(svs_plan& P, int l, cudaStream_t s) {
  if (!level_groups(P, l)) return;
  cudaEventRecord(P.events[0], s);
  for (size_t g = 0; g < level_groups(P, l); ++g) cudaStreamWaitEvent(P.side[g], P.events[0], 0);
}
void join_groups(svs_plan& P, int l, cudaStream_t s) {
  for (size_t g = 0; g < level_groups(P, l); ++g) {
    cudaEventRecord(P.events[1 + g], P.side[g]);
    cudaStreamWaitEvent(s, P.events[1 + g], 0);
  }
}
// One iteration of level l over all its pairs; returns the launches issued.
int level_iteration(svs_plan& P, int l, const IterArgs& a_in, cudaStream_t s) {
  IterArgs a = a_in;
  if (l == P.stall_level) {
    a.stall_cta = P.stall_cta;
    a.stall_plane = P.stall_plane;
  }
  iter_dispatch(P, nullptr, l, P.level_tile[l], 1, &a, s);
  for (size_t g = 0; g < level_groups(P, l); ++g) {
    const svs_plan::TileGroup& grp = P.extra[l][g];
    P.launch_override = true;
    P.launch_tiles = grp.d;
    P.launch_count = (unsigned)grp.h.size();
    iter_dispatch(P, nullptr, l, grp.tid, 1, &a_in, P.side[g]);
    P.launch_override = false;
  }
  return 1 + (int)level_groups(P, l);
}

// The whole batched solve as a sequence of launches on stream s. Returns the number of kernel
// launches issued or -1 after a launch error.
template <typename SU, typename SP>
long long enqueue_solve(svs_plan& P, cudaStream_t s) {
  const svs_tvl1_params& q = P.prm;
  const int L = P.levels, np = P.num_pairs;
  long long launches = 0;
  auto grid = [&](int level) { return dim3(ceil_div(max_voxels(P, level), 256), np); };
  const Desc* D = P.d_descs;
  blur_pair_kernel<<<grid(0), 256, 0, s>>>(D, P.d_raw, P.blur_r, P.blur, q.use_gaussian_blur);
  ++launches;
  for (int l = 1; l < L; ++l) {
    restrict_kernel<<<grid(l), 256, 0, s>>>(D + (size_t)(l - 1) * np, D + (size_t)l * np, q.interpolation, q.boundary);
    ++launches;
  }
  if (P.warm && L == 1) {
    warm_start_kernel<SU, SP><<<grid(0), 256, 0, s>>>(D, P.d_uinit, P.d_pinit);
    ++launches;
  }
  int cur = 0;
  for (int l = L - 1; l >= 0; --l) {
    const int zero = (l == L - 1) && !(P.warm && L == 1);
    prepare_kernel<SU, SP><<<grid(l), 256, 0, s>>>(D + (size_t)l * np, q.use_anisotropic_diff, q.alpha, q.beta, q.boundary, zero, cur);
    ++launches;
    if (P.res_on) {
      residual_reset_kernel<<<ceil_div(np, 128), 128, 0, s>>>(P.d_stop, P.d_acc, np);
      residual_kernel<SU><<<grid(l), 256, 0, s>>>(D + (size_t)l * np, cur, P.d_snaps, P.d_acc, 1);
      launches += 2;
    }
    for (int w = 0; w < q.max_warps; ++w) {
      linearise_kernel<SU, SP><<<grid(l), 256, 0, s>>>(D + (size_t)l * np, cur, q.interpolation, q.boundary);
      ++launches;
      if (l < (int)P.level_persist.size() && P.level_persist[l] && q.max_outer_iterations > 0) {
        // every iteration of the warp in one cooperative launch (grid barrier between them)
        PersistArgs pa;
        pa.sig = P.d_sig;
        pa.tau = P.d_tau;
        pa.wm = P.prm.weight_matching;
        pa.wtv = P.prm.weight_tv;
        pa.src0 = cur;
        pa.bdry = P.prm.boundary;
        pa.iters = q.max_outer_iterations;
        pa.wait_us = P.wait_us;
        pa.stall_cta = l == P.stall_level ? P.stall_cta : -1;
        pa.stall_plane = l == P.stall_level ? P.stall_plane : -1;
        pa.counter = P.d_gridbar;
        cudaMemsetAsync(P.d_gridbar, 0, sizeof(unsigned), s);
        const TileShape& ts = kTileShapes[P.level_tile[l] - 1];
        if (!split_persist(P.prm.storage, ts.split, 1, q.boundary != SVS_BOUNDARY_MIRROR,
                           (unsigned)P.h_tiles[l].size(), P.d_tiles[l], P.d_descs, P.d_maps, &pa, P.d_status, s))
          return -1;
        ++launches;
        cur ^= q.max_outer_iterations & 1;
      } else {
        fork_groups(P, l, s);
        for (int it = 0; it < q.max_outer_iterations; ++it) {
          const IterArgs a = iter_args(P, it, cur);
          launches += level_iteration(P, l, a, s);
          cur ^= 1;
        }
        join_groups(P, l, s);
      }
      if (P.res_on) {
        residual_kernel<SU><<<grid(l), 256, 0, s>>>(D + (size_t)l * np, cur, P.d_snaps, P.d_acc, 0);
        residual_finish_kernel<<<ceil_div(np, 128), 128, 0, s>>>(D + (size_t)l * np, P.d_acc, P.d_reslog, L,
                                                                 q.max_warps, l, w, P.res_tol, np);
        launches += 2;
      }
    }
    if (l > 0) {
      if (q.interpolation == SVS_INTERPOLATE_CUBIC_HERMITESPLINE && coarse_within(P, l))
        prolong_cubic_kernel<SU, SP><<<dim3(prolong_blocks(P, l - 1), np), PFX * PFY, 0, s>>>(
            D + (size_t)l * np, D + (size_t)(l - 1) * np, cur, q.boundary);
      else
        prolong_kernel<SU, SP><<<grid(l - 1), 256, 0, s>>>(D + (size_t)l * np, D + (size_t)(l - 1) * np, cur,
                                                          q.interpolation, q.boundary);
      ++launches;
      cur = 0;
    }
  }
  float** uo = q.median_kernel > 1 ? P.d_umed : P.d_uout;
  finalize_kernel<SU, SP><<<grid(0), 256, 0, s>>>(D, cur, uo, P.d_pout);
  ++launches;
  if (cudaPeekAtLastError() != cudaSuccess) return -1;
  if (q.median_kernel > 1) {
    for (int i = 0; i < np; ++i) {
      const Desc& d = P.h_descs[i];
      if (svs_median3d(P.umed[i], d.nz, d.ny, d.nx, 3, q.median_kernel, P.uout[i], s) != SVS_OK) return -1;
      ++launches;
    }
  }
  return launches;
}

long long enqueue(svs_plan& P, cudaStream_t s) {
  switch (P.prm.storage) {
    case SVS_STORAGE_BF16: return enqueue_solve<__nv_bfloat16, __nv_bfloat16>(P, s);
    case SVS_STORAGE_F16: return enqueue_solve<__half, __half>(P, s);
    case SVS_STORAGE_BF16_FLOW32: return enqueue_solve<float, __nv_bfloat16>(P, s);
    case SVS_STORAGE_F16_FLOW32: return enqueue_solve<float, __half>(P, s);
    default: return enqueue_solve<float, float>(P, s);
  }
}

template <typename T> T* carve(char*& cur, size_t count) {
  T* p = reinterpret_cast<T*>(cur);
  cur += (count * sizeof(T) + 255) / 256 * 256;
  return p;
}

// Mesh sizes per level (tvl13d.py:91-99, ceil halving), spacings (coreDefines.h:72-75) and the
// device bytes of a batch of `n` pairs with level-0 sizes dims[3i..3i+2]; descs gets
// [levels][n] descriptors without device pointers.
svs_status layout_batch(const svs_plan& P, int n, const int* dims, std::vector<Desc>& descs, size_t& bytes) {
  const svs_tvl1_params& prm = P.prm;
  descs.assign((size_t)P.levels * n, Desc{});
  bytes = 0;
  const size_t ub = flow_bytes(prm.storage), sb = field_bytes(prm.storage);
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  for (int i = 0; i < n; ++i) {
    int nz = dims[3 * i], ny = dims[3 * i + 1], nx = dims[3 * i + 2];
    if (nz >= 65535 || ny >= 65535 || nx >= 65535) return fail(SVS_ERR_INVALID_ARG, "plan: volume dimension too large");
    for (int l = 0; l < P.levels; ++l) {
      if (l > 0) { nz = (nz + 1) / 2; ny = (ny + 1) / 2; nx = (nx + 1) / 2; }
      if (nz < 3 || ny < 3 || nx < 3)
        return fail(SVS_ERR_INVALID_ARG, "plan: every pyramid level needs at least 3 nodes per axis");
      Desc& d = descs[(size_t)l * n + i];
      std::memset(&d, 0, sizeof(d));
      d.nz = nz; d.ny = ny; d.nx = nx;
      d.pitch = (nx + 7) / 8 * 8;
      d.n = (long long)nz * ny * nx;
      d.cs = (long long)d.pitch * ny * nz;
      if (prm.length_type == 0) { d.lz = (float)(nz - 1); d.ly = (float)(ny - 1); d.lx = (float)(nx - 1); }
      else { d.lz = prm.length_z; d.ly = prm.length_y; d.lx = prm.length_x; }
      d.hz = d.lz / (float)(nz - 1); d.hy = d.ly / (float)(ny - 1); d.hx = d.lx / (float)(nx - 1);
      const size_t nv = (size_t)d.n, cs = (size_t)d.cs;
      bytes += 2 * al(nv * 4) + al(4 * nv * 4);                      // I0, I1, ig
      bytes += al(6 * cs * sb) + al(cs * sb) + al(3 * cs * sb);      // D, rc, gw
      bytes += 2 * al(3 * cs * ub) + 2 * al(9 * cs * sb);            // u[2], p[2]
      if (9 * cs >= (size_t)1 << 31) return fail(SVS_ERR_INVALID_ARG, "plan: volume too large for 32-bit field offsets");
      if (l == 0) bytes += 2 * al(nv * 4) + 2 * al(3 * nv * 4) + al(9 * nv * 4);  // raw x2, uout, umed, pout
    }
  }
  bytes += 4096;
  return SVS_OK;
}

// Device pointers of P.h_descs ([levels][num_pairs]) and the per-pair buffers, carved from the arena.
void carve_batch(svs_plan& P) {
  const int n = P.num_pairs;
  const size_t ub = flow_bytes(P.prm.storage), sb = field_bytes(P.prm.storage);
  char* cur = reinterpret_cast<char*>(P.arena);
  P.raw.assign(2 * n, nullptr); P.uout.assign(n, nullptr); P.pout.assign(n, nullptr); P.umed.assign(n, nullptr);
  P.uinit.assign(n, nullptr); P.pinit.assign(n, nullptr);
  for (int l = 0; l < P.levels; ++l)
    for (int i = 0; i < n; ++i) {
      Desc& d = P.h_descs[(size_t)l * n + i];
      const size_t nv = (size_t)d.n, cs = (size_t)d.cs;
      d.I0 = carve<float>(cur, nv);
      d.I1 = carve<float>(cur, nv);
      d.ig = carve<float>(cur, 4 * nv);
      d.D = carve<char>(cur, 6 * cs * sb);
      d.rc = carve<char>(cur, cs * sb);
      d.gw = carve<char>(cur, 3 * cs * sb);
      d.u[0] = carve<char>(cur, 3 * cs * ub);
      d.u[1] = carve<char>(cur, 3 * cs * ub);
      d.p[0] = carve<char>(cur, 9 * cs * sb);
      d.p[1] = carve<char>(cur, 9 * cs * sb);
      if (l == 0) {
        P.raw[2 * i] = carve<float>(cur, nv);
        P.raw[2 * i + 1] = carve<float>(cur, nv);
        P.uout[i] = carve<float>(cur, 3 * nv);
        P.umed[i] = carve<float>(cur, 3 * nv);
        P.pout[i] = carve<float>(cur, 9 * nv);
      }
    }
}

}  // namespace
}  // namespace svs

using namespace svs;

extern "C" {

int svs_tvl1_num_tiles(void) { return kNumTileShapes; }

svs_status svs_tvl1_tile_info(int tile_id, int* tx, int* ty, int* dist, int* form, int* lane_voxels) {
  SVS_REQUIRE(tile_id >= 1 && tile_id <= kNumTileShapes, "svs_tvl1_tile_info: unknown tile id");
  const TileShape& t = kTileShapes[tile_id - 1];
  if (tx) *tx = t.tx;
  if (ty) *ty = t.ty;
  if (dist) *dist = t.dist;
  if (form) *form = t.form;
  if (lane_voxels) *lane_voxels = t.form == kSplit ? kSplitShapes[t.split].v : 1;
  return SVS_OK;
}

svs_status svs_tvl1_tile_occupancy(int storage, int tile_id, int general_boundary, int* ctas_per_sm) {
  SVS_REQUIRE(tile_id >= 1 && tile_id <= kNumTileShapes, "svs_tvl1_tile_occupancy: unknown tile id");
  SVS_REQUIRE(storage >= SVS_STORAGE_F32 && storage <= SVS_STORAGE_F16_FLOW32, "svs_tvl1_tile_occupancy: unknown storage");
  SVS_REQUIRE(ctas_per_sm, "svs_tvl1_tile_occupancy: null output");
  const TileShape& t = kTileShapes[tile_id - 1];
  SVS_REQUIRE(t.form == kSplit, "svs_tvl1_tile_occupancy: split-role variants only");
  const bool gen = general_boundary != 0;
  int box[4] = {0, 0, 0, 0};
  // op 0 sets the kernels' shared-memory attribute, which the occupancy query (op 2) needs
  if (!split_variant(storage, t.split, 0, gen, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, box))
    return fail(SVS_ERR_UNSUPPORTED, "svs_tvl1_tile_occupancy: variant not compiled for this storage, or its shared memory does not fit");
  if (!split_variant(storage, t.split, 2, gen, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, box))
    return fail(SVS_ERR_CUDA, "svs_tvl1_tile_occupancy: occupancy query failed");
  *ctas_per_sm = box[0];
  return SVS_OK;
}

svs_status svs_tvl1_plan_create(const svs_tvl1_params* prm, int num_pairs, const int* dims,
                                svs_plan** out) {
  SVS_REQUIRE(prm && dims && out, "svs_tvl1_plan_create: null pointer");
  SVS_REQUIRE(num_pairs > 0, "svs_tvl1_plan_create: num_pairs must be positive");
  SVS_REQUIRE(prm->num_scales >= 1 && prm->num_scales <= 8, "svs_tvl1_plan_create: num_scales out of range");
  SVS_REQUIRE(prm->max_warps >= 0 && prm->max_outer_iterations >= 0, "svs_tvl1_plan_create: negative iteration count");
  SVS_REQUIRE(prm->primaldual_algorithm_type == 1 || prm->primaldual_algorithm_type == 2,
              "svs_tvl1_plan_create: primaldual_algorithm_type must be 1 or 2");
  SVS_REQUIRE(prm->boundary >= 0 && prm->boundary <= 2, "svs_tvl1_plan_create: bad boundary type");
  SVS_REQUIRE(prm->interpolation >= 0 && prm->interpolation <= 2, "svs_tvl1_plan_create: bad interpolation type");
  SVS_REQUIRE(prm->storage >= 0 && prm->storage <= 4, "svs_tvl1_plan_create: bad storage type");
  SVS_REQUIRE(prm->weight_tv >= 0.f, "svs_tvl1_plan_create: weight_tv must be >= 0");
  SVS_REQUIRE(prm->median_kernel == 0 || prm->median_kernel == 1 || prm->median_kernel == 3 ||
                  prm->median_kernel == 5 || prm->median_kernel == 7,
              "svs_tvl1_plan_create: median kernel must be 0, 1, 3, 5 or 7");
  svs_plan* P = new svs_plan();
  P->prm = *prm;
  P->levels = prm->num_scales;
  size_t bytes = 0;
  svs_status st = layout_batch(*P, num_pairs, dims, P->h_descs, bytes);
  if (st) { delete P; return st; }
  P->num_pairs = num_pairs;
  P->capacity = num_pairs;
  P->dims.assign(dims, dims + 3 * num_pairs);
  st = check_cuda(cudaMalloc(&P->arena, bytes), "svs_tvl1_plan_create: device state");
  if (st) { delete P; return st; }
  P->arena_bytes = bytes;
  // zero the whole arena once: pitch padding and planes never written stay zero
  st = check_cuda(cudaMemset(P->arena, 0, bytes), "svs_tvl1_plan_create");
  if (st) { svs_tvl1_plan_destroy(P); return st; }
  carve_batch(*P);
  auto upload = [&](void** dptr, const void* src, size_t sz) -> svs_status {
    svs_status s2 = check_cuda(cudaMalloc(dptr, sz), "svs_tvl1_plan_create");
    if (s2) return s2;
    return check_cuda(cudaMemcpy(*dptr, src, sz, cudaMemcpyHostToDevice), "svs_tvl1_plan_create");
  };
  st = upload((void**)&P->d_descs, P->h_descs.data(), P->h_descs.size() * sizeof(Desc));
  if (!st) st = upload((void**)&P->d_raw, P->raw.data(), P->raw.size() * sizeof(float*));
  if (!st) st = upload((void**)&P->d_uout, P->uout.data(), P->uout.size() * sizeof(float*));
  if (!st) st = upload((void**)&P->d_umed, P->umed.data(), P->umed.size() * sizeof(float*));
  std::vector<float*> nop(num_pairs, nullptr);
  if (!st) st = upload((void**)&P->d_pout, nop.data(), nop.size() * sizeof(float*));
  if (!st) st = upload((void**)&P->d_uinit, P->uinit.data(), P->uinit.size() * sizeof(float*));
  if (!st) st = upload((void**)&P->d_pinit, P->pinit.data(), P->pinit.size() * sizeof(float*));
  if (!st) st = check_cuda(cudaMalloc((void**)&P->d_maps, (size_t)P->levels * num_pairs * sizeof(TMaps)), "svs_tvl1_plan_create");
  if (!st) st = check_cuda(cudaMalloc((void**)&P->d_status, sizeof(int)), "svs_tvl1_plan_create");
  if (!st) st = check_cuda(cudaMemset(P->d_status, 0, sizeof(int)), "svs_tvl1_plan_create");
  if (st) { svs_tvl1_plan_destroy(P); return st; }
  // step-size schedule within a warp (tvl13d.py:208-211 reset, :240-249 update, host float64),
  // each value rounded to float as torch and pybind do.
  {
    double sg = prm->sigma, ta = prm->tau;
    for (int it = 0; it < prm->max_outer_iterations; ++it) {
      P->sig_sched.push_back((float)sg);
      P->tau_sched.push_back((float)ta);
      if (prm->primaldual_algorithm_type == 2) {
        const double th = 1.0 / std::sqrt(1.0 + 2.0 * prm->gamma * ta);
        ta *= th;
        sg /= th;
      }
    }
  }
  // Gaussian kernel weights, flow_utils.py:74-91 and :106-107, in float32
  if (prm->use_gaussian_blur) {
    const double sgm = prm->gaussian_blur_sigma;
    int ks = (int)(sgm * 5);
    if (ks % 2 == 0) ks += 1;
    if (ks > 9 || ks < 1) { svs_tvl1_plan_destroy(P); return fail(SVS_ERR_INVALID_ARG, "svs_tvl1_plan_create: gaussian_blur_sigma out of range (kernel size <= 9)"); }
    // torch.linspace(-ks//2, ks//2 + 1, ks) with Python floor division
    const int lo = -((ks + 1) / 2), hi = ks / 2 + 1;
    std::vector<float> t(ks), g(ks), k1(ks);
    for (int i = 0; i < ks; ++i) t[i] = (ks == 1) ? (float)lo : (float)(lo + (double)(hi - lo) * i / (ks - 1));
    float gs = 0.f;
    for (int i = 0; i < ks; ++i) {
      const float a = t[i] / (float)sgm;
      g[i] = std::exp(-(a * a) / 2.0f);
      gs += g[i];
    }
    for (int i = 0; i < ks; ++i) k1[i] = g[i] / gs;
    float tot = 0.f;
    std::vector<float> k3((size_t)ks * ks * ks);
    for (int a = 0; a < ks; ++a)
      for (int b = 0; b < ks; ++b)
        for (int c = 0; c < ks; ++c) { k3[(a * ks + b) * ks + c] = k1[a] * k1[b] * k1[c]; tot += k3[(a * ks + b) * ks + c]; }
    for (size_t i = 0; i < k3.size(); ++i) P->blur.w[i] = k3[i] / tot;
    P->blur_r = ks / 2;
  }
  // the schedule again on the device, for the persistent iteration loop, and its barrier counter
  const size_t nsch = std::max<size_t>(1, P->sig_sched.size());
  st = check_cuda(cudaMalloc((void**)&P->d_sig, nsch * sizeof(float)), "svs_tvl1_plan_create");
  if (!st) st = check_cuda(cudaMalloc((void**)&P->d_tau, nsch * sizeof(float)), "svs_tvl1_plan_create");
  if (!st) st = check_cuda(cudaMalloc((void**)&P->d_gridbar, sizeof(unsigned)), "svs_tvl1_plan_create");
  if (!st && !P->sig_sched.empty())
    st = check_cuda(cudaMemcpy(P->d_sig, P->sig_sched.data(), P->sig_sched.size() * sizeof(float), cudaMemcpyHostToDevice),
                    "svs_tvl1_plan_create");
  if (!st && !P->tau_sched.empty())
    st = check_cuda(cudaMemcpy(P->d_tau, P->tau_sched.data(), P->tau_sched.size() * sizeof(float), cudaMemcpyHostToDevice),
                    "svs_tvl1_plan_create");
  if (!st) st = check_cuda(cudaStreamCreateWithFlags(&P->cap_stream, cudaStreamNonBlocking), "svs_tvl1_plan_create");
  if (st) { svs_tvl1_plan_destroy(P); return st; }
  *out = P;
  return SVS_OK;
}

svs_status svs_tvl1_plan_destroy(svs_plan* P) {
  if (!P) return SVS_OK;
  if (P->exec) cudaGraphExecDestroy(P->exec);
  if (P->cap_stream) cudaStreamDestroy(P->cap_stream);
  for (auto* t : P->d_tiles) cudaFree(t);
  cudaFree(P->d_descs); cudaFree(P->d_raw); cudaFree(P->d_uout); cudaFree(P->d_umed);
  cudaFree(P->d_pout); cudaFree(P->d_uinit); cudaFree(P->d_pinit); cudaFree(P->d_maps);
  cudaFree(P->d_status);
  cudaFree(P->d_sig); cudaFree(P->d_tau); cudaFree(P->d_gridbar);
  for (auto& lv : P->extra)
    for (auto& grp : lv) cudaFree(grp.d);
  for (cudaStream_t st_ : P->side) cudaStreamDestroy(st_);
  for (cudaEvent_t e : P->events) cudaEventDestroy(e);
  cudaFree(P->d_stop);
  cudaFree(P->d_acc);
  cudaFree(P->d_reslog);
  cudaFree(P->d_snaps);
  for (float* p : P->snaps) cudaFree(p);
  cudaFree(P->arena);
  delete P;
  return SVS_OK;
}

size_t svs_tvl1_plan_device_bytes(const svs_plan* P) { return P ? P->arena_bytes : 0; }

svs_status svs_tvl1_plan_set_tile(svs_plan* P, int tile_id) {
  SVS_REQUIRE(P, "svs_tvl1_plan_set_tile: null plan");
  SVS_REQUIRE(tile_id >= 0 && tile_id <= kNumTileShapes, "svs_tvl1_plan_set_tile: unknown tile id");
  P->tile_id = tile_id;
  ++P->tile_epoch;
  return SVS_OK;
}

svs_status svs_tvl1_plan_set_level_tile(svs_plan* P, int level, int tile_id) {
  SVS_REQUIRE(P, "svs_tvl1_plan_set_level_tile: null plan");
  SVS_REQUIRE(level >= 0 && level < P->levels, "svs_tvl1_plan_set_level_tile: bad level");
  SVS_REQUIRE(tile_id >= 0 && tile_id <= kNumTileShapes, "svs_tvl1_plan_set_level_tile: unknown tile id");
  if ((int)P->level_tile_req.size() < P->levels) P->level_tile_req.resize(P->levels, 0);
  P->level_tile_req[level] = tile_id;
  ++P->tile_epoch;
  return SVS_OK;
}

svs_status svs_tvl1_plan_set_level_chunks(svs_plan* P, int level, int chunks) {
  SVS_REQUIRE(P, "svs_tvl1_plan_set_level_chunks: null plan");
  SVS_REQUIRE(level >= 0 && level < P->levels, "svs_tvl1_plan_set_level_chunks: bad level");
  SVS_REQUIRE(chunks >= 0, "svs_tvl1_plan_set_level_chunks: chunks must be >= 0");
  if ((int)P->level_chunks_req.size() < P->levels) P->level_chunks_req.resize(P->levels, 0);
  P->level_chunks_req[level] = chunks;
  ++P->tile_epoch;
  return SVS_OK;
}

svs_status svs_tvl1_plan_set_pair_tile(svs_plan* P, int level, int pair, int tile_id) {
  SVS_REQUIRE(P, "svs_tvl1_plan_set_pair_tile: null plan");
  SVS_REQUIRE(level >= 0 && level < P->levels, "svs_tvl1_plan_set_pair_tile: bad level");
  SVS_REQUIRE(pair >= 0 && pair < P->num_pairs, "svs_tvl1_plan_set_pair_tile: bad pair");
  SVS_REQUIRE(tile_id >= 0 && tile_id <= kNumTileShapes, "svs_tvl1_plan_set_pair_tile: unknown tile id");
  if ((int)P->pair_tile_req.size() < P->levels) P->pair_tile_req.resize(P->levels, std::vector<int>(P->num_pairs, 0));
  P->pair_tile_req[level][pair] = tile_id;
  ++P->tile_epoch;
  return SVS_OK;
}

svs_status svs_tvl1_plan_set_residuals(svs_plan* P, int record, float stop_tol) {
  SVS_REQUIRE(P, "svs_tvl1_plan_set_residuals: null plan");
  SVS_REQUIRE(stop_tol >= 0.f, "svs_tvl1_plan_set_residuals: stop_tol must be >= 0");
  SVS_REQUIRE(stop_tol == 0.f || P->prm.max_outer_iterations % 2 == 0,
              "svs_tvl1_plan_set_residuals: stopping needs an even max_outer_iterations (the iteration "
              "state alternates between two buffers)");
  const bool on = record != 0 || stop_tol > 0.f;
  const int np = P->num_pairs;
  if (on && !P->d_stop) {
    svs_status st = check_cuda(cudaMalloc(&P->d_stop, np * sizeof(int)), "residuals");
    if (!st) st = check_cuda(cudaMalloc(&P->d_acc, np * sizeof(double)), "residuals");
    const size_t nlog = (size_t)np * P->levels * std::max(1, P->prm.max_warps);
    if (!st) st = check_cuda(cudaMalloc(&P->d_reslog, nlog * sizeof(float)), "residuals");
    if (!st) st = check_cuda(cudaMemset(P->d_reslog, 0, nlog * sizeof(float)), "residuals");
    if (!st) st = check_cuda(cudaMemset(P->d_stop, 0, np * sizeof(int)), "residuals");
    P->snaps.assign(np, nullptr);
    for (int i = 0; i < np && !st; ++i)
      st = check_cuda(cudaMalloc(&P->snaps[i], 3 * (size_t)P->h_descs[i].n * sizeof(float)), "residuals");
    if (!st) st = check_cuda(cudaMalloc(&P->d_snaps, np * sizeof(float*)), "residuals");
    if (!st) st = check_cuda(cudaMemcpy(P->d_snaps, P->snaps.data(), np * sizeof(float*), cudaMemcpyHostToDevice), "residuals");
    if (st) return st;
  }
  // the flag pointer in every descriptor (null when off: the kernels test it)
  for (int l = 0; l < P->levels; ++l)
    for (int i = 0; i < np; ++i) P->h_descs[(size_t)l * np + i].stop = on ? P->d_stop + i : nullptr;
  svs_status st = check_cuda(cudaMemcpy(P->d_descs, P->h_descs.data(), P->h_descs.size() * sizeof(Desc),
                                        cudaMemcpyHostToDevice), "residuals");
  if (st) return st;
  P->res_on = on;
  P->res_tol = stop_tol;
  ++P->tile_epoch;  // the captured graph changes
  return SVS_OK;
}

svs_status svs_tvl1_plan_get_residuals(svs_plan* P, float* out, size_t count) {
  SVS_REQUIRE(P && out, "svs_tvl1_plan_get_residuals: null pointer");
  SVS_REQUIRE(P->d_reslog, "svs_tvl1_plan_get_residuals: residuals are not recorded (svs_tvl1_plan_set_residuals)");
  const size_t nlog = (size_t)P->num_pairs * P->levels * std::max(1, P->prm.max_warps);
  SVS_REQUIRE(count == nlog, "svs_tvl1_plan_get_residuals: count must be pairs x levels x max_warps");
  return check_cuda(cudaMemcpy(out, P->d_reslog, nlog * sizeof(float), cudaMemcpyDeviceToHost), "residuals");
}

svs_status svs_tvl1_solve_batch(svs_plan* P, const svs_pair_desc* pairs, int num_pairs,
                                svs_stream_t stream) {
  SVS_REQUIRE(P && pairs, "svs_tvl1_solve_batch: null pointer");
  SVS_REQUIRE(num_pairs == P->num_pairs, "svs_tvl1_solve_batch: pair count differs from the plan");
  bool want_p = false, warm = false;
  for (int i = 0; i < num_pairs; ++i) {
    const svs_pair_desc& q = pairs[i];
    SVS_REQUIRE(q.I0 && q.I1 && q.u_out, "svs_tvl1_solve_batch: null frame or output pointer");
    SVS_REQUIRE(q.nz == P->dims[3 * i] && q.ny == P->dims[3 * i + 1] && q.nx == P->dims[3 * i + 2],
                "svs_tvl1_solve_batch: pair sizes differ from the plan");
    want_p |= q.p_out != nullptr;
    warm |= (q.u_init != nullptr || q.p_init != nullptr);
  }
  warm = warm && P->levels == 1;
  cudaStream_t s = stream;
  svs_status st = SVS_OK;
  for (int i = 0; i < num_pairs && !st; ++i) {
    const size_t b = (size_t)P->h_descs[i].n * sizeof(float);
    st = check_cuda(cudaMemcpyAsync(P->raw[2 * i], pairs[i].I0, b, cudaMemcpyDeviceToDevice, s), "solve: input copy");
    if (!st) st = check_cuda(cudaMemcpyAsync(P->raw[2 * i + 1], pairs[i].I1, b, cudaMemcpyDeviceToDevice, s), "solve: input copy");
  }
  if (st) return st;
  if (warm) {
    for (int i = 0; i < num_pairs; ++i) { P->uinit[i] = pairs[i].u_init; P->pinit[i] = pairs[i].p_init; }
    st = check_cuda(cudaMemcpyAsync(P->d_uinit, P->uinit.data(), num_pairs * sizeof(float*), cudaMemcpyHostToDevice, s), "solve");
    if (!st) st = check_cuda(cudaMemcpyAsync(P->d_pinit, P->pinit.data(), num_pairs * sizeof(float*), cudaMemcpyHostToDevice, s), "solve");
    if (!st) st = check_cuda(cudaStreamSynchronize(s), "solve");
    if (st) return st;
  }
  if (want_p != P->want_p) {
    std::vector<float*> po(num_pairs, nullptr);
    if (want_p) po = P->pout;
    st = check_cuda(cudaMemcpy(P->d_pout, po.data(), num_pairs * sizeof(float*), cudaMemcpyHostToDevice), "solve");
    if (st) return st;
    P->want_p = want_p;
  }
  P->warm = warm;
  if (P->tiles_built_for != P->tile_epoch) {
    st = setup_tiles(*P);
    if (st) return st;
    P->tiles_built_for = P->tile_epoch;
  }
  if (!P->exec || P->graph_tile != P->tile_epoch || P->graph_warm != warm || P->graph_want_p != want_p) {
    if (P->exec) { cudaGraphExecDestroy(P->exec); P->exec = nullptr; }
    cudaGraph_t g = nullptr;
    st = check_cuda(cudaStreamBeginCapture(P->cap_stream, cudaStreamCaptureModeThreadLocal), "solve: capture");
    if (st) return st;
    long long nl = enqueue(*P, P->cap_stream);
    cudaError_t ce = cudaStreamEndCapture(P->cap_stream, &g);
    if ((nl < 0 || ce != cudaSuccess) && P->persistent) {
      // the cooperative launch of the persistent loop could not be captured here: per-iteration
      // launches instead (svs_tvl1_plan_level_persistent then reports 0)
      if (g) cudaGraphDestroy(g);
      g = nullptr;
      cudaGetLastError();
      P->persistent = false;
      st = setup_tiles(*P);
      if (st) return st;
      st = check_cuda(cudaStreamBeginCapture(P->cap_stream, cudaStreamCaptureModeThreadLocal), "solve: capture");
      if (st) return st;
      nl = enqueue(*P, P->cap_stream);
      ce = cudaStreamEndCapture(P->cap_stream, &g);
    }
    if (nl < 0) { if (g) cudaGraphDestroy(g); return fail(SVS_ERR_LAUNCH, std::string("solve: launch failed during capture: ") + cudaGetErrorString(cudaGetLastError())); }
    st = check_cuda(ce, "solve: end capture");
    if (st) return st;
    st = check_cuda(cudaGraphInstantiate(&P->exec, g, 0), "solve: graph instantiate");
    cudaGraphDestroy(g);
    if (st) return st;
    P->graph_kernels = (uint64_t)nl;
    P->graph_tile = P->tile_epoch;
    P->graph_warm = warm;
    P->graph_want_p = want_p;
  }
  st = check_cuda(cudaGraphLaunch(P->exec, s), "solve: graph launch");
  if (st) return st;
  count_launches(P->graph_kernels);
  for (int i = 0; i < num_pairs && !st; ++i) {
    const size_t n = (size_t)P->h_descs[i].n;
    st = check_cuda(cudaMemcpyAsync(pairs[i].u_out, P->uout[i], 3 * n * sizeof(float), cudaMemcpyDeviceToDevice, s), "solve: output copy");
    if (!st && pairs[i].p_out)
      st = check_cuda(cudaMemcpyAsync(pairs[i].p_out, P->pout[i], 9 * n * sizeof(float), cudaMemcpyDeviceToDevice, s), "solve: output copy");
  }
  return st;
}

svs_status svs_tvl1_bench_iterations(svs_plan* P, int level, int count, svs_stream_t stream) {
  SVS_REQUIRE(P, "svs_tvl1_bench_iterations: null plan");
  SVS_REQUIRE(level >= 0 && level < P->levels, "svs_tvl1_bench_iterations: bad level");
  SVS_REQUIRE(count >= 0, "svs_tvl1_bench_iterations: bad count");
  if (P->tiles_built_for != P->tile_epoch) {
    const svs_status st = setup_tiles(*P);
    if (st) return st;
    P->tiles_built_for = P->tile_epoch;
  }
  int cur = 0;
  uint64_t launches = 0;
  fork_groups(*P, level, stream);
  for (int i = 0; i < count; ++i) {
    const int it = P->prm.max_outer_iterations > 0 ? i % P->prm.max_outer_iterations : 0;
    const IterArgs a = iter_args(*P, it, cur);
    launches += level_iteration(*P, level, a, stream);
    cur ^= 1;
  }
  join_groups(*P, level, stream);
  return check_launch("svs_tvl1_bench_iterations", launches);
}

uint64_t svs_tvl1_plan_graph_kernels(const svs_plan* P) { return P ? P->graph_kernels : 0; }

int svs_tvl1_plan_level_tile(const svs_plan* P, int level) {
  return (P && level >= 0 && level < (int)P->level_tile.size()) ? P->level_tile[level] : 0;
}

int svs_tvl1_plan_pair_tile_used(const svs_plan* P, int level, int pair) {
  if (!P || level < 0 || level >= (int)P->pair_used.size() || pair < 0 || pair >= (int)P->pair_used[level].size())
    return 0;
  return P->pair_used[level][pair];
}

int svs_tvl1_auto_tiles(int storage, int num_pairs, const int* dims_host, int sms, int* pair_tile_out) {
  if (num_pairs < 1 || !dims_host || !pair_tile_out || storage < SVS_STORAGE_F32 || storage > SVS_STORAGE_F16_FLOW32)
    return 0;
  for (int i = 0; i < 3 * num_pairs; ++i)
    if (dims_host[i] < 1) return 0;
  return auto_choice(storage, num_pairs, dims_host, sms, pair_tile_out);
}

svs_status svs_tvl1_chunk_plan(int64_t columns, int nz, int64_t slots, int* main_chunks, int* tail_chunks,
                               int64_t* tail_columns) {
  SVS_REQUIRE(columns > 0 && nz > 0 && slots > 0, "svs_tvl1_chunk_plan: columns, nz and slots must be positive");
  SVS_REQUIRE(main_chunks && tail_chunks && tail_columns, "svs_tvl1_chunk_plan: null output");
  const ChunkPlan c = chunk_plan(columns, nz, slots);
  *main_chunks = c.main_c;
  *tail_chunks = c.tail_c;
  *tail_columns = c.tail_cols;
  return SVS_OK;
}

int64_t svs_tvl1_plan_level_ctas(const svs_plan* P, int level) {
  if (!P || level < 0 || level >= (int)P->h_tiles.size()) return 0;
  int64_t n = (int64_t)P->h_tiles[level].size();
  if (level < (int)P->extra.size())
    for (const auto& grp : P->extra[level]) n += (int64_t)grp.h.size();
  return n;
}

svs_status svs_tvl1_plan_check(svs_plan* P) {
  SVS_REQUIRE(P, "svs_tvl1_plan_check: null plan");
  int flags = 0;
  svs_status st = check_cuda(cudaMemcpy(&flags, P->d_status, sizeof(int), cudaMemcpyDeviceToHost), "svs_tvl1_plan_check");
  if (st) return st;
  if (flags) {
    st = check_cuda(cudaMemset(P->d_status, 0, sizeof(int)), "svs_tvl1_plan_check");  // reported once
    if (st) return st;
  }
  if (flags & SVS_DEV_TIMEOUT) return fail(SVS_ERR_TIMEOUT, "a pipeline wait in the iterate kernel timed out; results are invalid");
  return SVS_OK;
}

svs_status svs_tvl1_plan_create_reserve(const svs_tvl1_params* prm, int max_pairs, size_t arena_bytes,
                                        svs_plan** out) {
  SVS_REQUIRE(prm && out, "svs_tvl1_plan_create_reserve: null pointer");
  SVS_REQUIRE(max_pairs > 0, "svs_tvl1_plan_create_reserve: max_pairs must be positive");
  SVS_REQUIRE(prm->num_scales >= 1 && prm->num_scales <= 8, "svs_tvl1_plan_create_reserve: num_scales out of range");
  // a placeholder batch: max_pairs of the smallest cube every level of the pyramid accepts
  const int side = 3 << (prm->num_scales - 1);
  std::vector<int> dims((size_t)3 * max_pairs, side);
  svs_plan* P = nullptr;
  svs_status st = svs_tvl1_plan_create(prm, max_pairs, dims.data(), &P);
  if (st) return st;
  if (arena_bytes > P->arena_bytes) {
    void* bigger = nullptr;
    st = check_cuda(cudaMalloc(&bigger, arena_bytes), "svs_tvl1_plan_create_reserve: device state");
    if (!st) st = check_cuda(cudaMemset(bigger, 0, arena_bytes), "svs_tvl1_plan_create_reserve");
    if (st) {
      cudaFree(bigger);
      svs_tvl1_plan_destroy(P);
      return st;
    }
    cudaFree(P->arena);
    P->arena = bigger;
    P->arena_bytes = arena_bytes;
    carve_batch(*P);
    st = check_cuda(cudaMemcpy(P->d_descs, P->h_descs.data(), P->h_descs.size() * sizeof(Desc), cudaMemcpyHostToDevice),
                    "svs_tvl1_plan_create_reserve");
    if (!st) st = check_cuda(cudaMemcpy(P->d_raw, P->raw.data(), P->raw.size() * sizeof(float*), cudaMemcpyHostToDevice),
                             "svs_tvl1_plan_create_reserve");
    if (!st) st = check_cuda(cudaMemcpy(P->d_uout, P->uout.data(), P->uout.size() * sizeof(float*), cudaMemcpyHostToDevice),
                             "svs_tvl1_plan_create_reserve");
    if (!st) st = check_cuda(cudaMemcpy(P->d_umed, P->umed.data(), P->umed.size() * sizeof(float*), cudaMemcpyHostToDevice),
                             "svs_tvl1_plan_create_reserve");
    if (st) {
      svs_tvl1_plan_destroy(P);
      return st;
    }
  }
  *out = P;
  return SVS_OK;
}

svs_status svs_tvl1_plan_retarget(svs_plan* P, int num_pairs, const int* dims, svs_stream_t stream) {
  SVS_REQUIRE(P && dims, "svs_tvl1_plan_retarget: null pointer");
  SVS_REQUIRE(num_pairs > 0 && num_pairs <= P->capacity,
              "svs_tvl1_plan_retarget: num_pairs must be positive and at most the plan's pair count at creation");
  SVS_REQUIRE(!P->res_on, "svs_tvl1_plan_retarget: not with residuals on (their buffers are sized per pair)");
  std::vector<Desc> descs;
  size_t bytes = 0;
  svs_status st = layout_batch(*P, num_pairs, dims, descs, bytes);
  if (st) return st;
  if (bytes > P->arena_bytes)
    return fail(SVS_ERR_OUT_OF_MEMORY, "svs_tvl1_plan_retarget: the batch needs " + std::to_string(bytes) +
                                           " bytes of device state; the plan holds " + std::to_string(P->arena_bytes));
  cudaStream_t s = stream;
  P->num_pairs = num_pairs;
  P->dims.assign(dims, dims + 3 * num_pairs);
  P->h_descs = std::move(descs);
  carve_batch(*P);
  // clear the state the batch uses (as at creation), then the tables (descriptors with the stop
  // flags off, pointer arrays; the caller's output pointers are filled by each solve)
  st = check_cuda(cudaMemsetAsync(P->arena, 0, bytes, s), "svs_tvl1_plan_retarget");
  if (!st) st = check_cuda(cudaMemcpyAsync(P->d_descs, P->h_descs.data(), P->h_descs.size() * sizeof(Desc),
                                           cudaMemcpyHostToDevice, s), "svs_tvl1_plan_retarget");
  if (!st) st = check_cuda(cudaMemcpyAsync(P->d_raw, P->raw.data(), P->raw.size() * sizeof(float*), cudaMemcpyHostToDevice, s),
                           "svs_tvl1_plan_retarget");
  if (!st) st = check_cuda(cudaMemcpyAsync(P->d_uout, P->uout.data(), P->uout.size() * sizeof(float*), cudaMemcpyHostToDevice, s),
                           "svs_tvl1_plan_retarget");
  if (!st) st = check_cuda(cudaMemcpyAsync(P->d_umed, P->umed.data(), P->umed.size() * sizeof(float*), cudaMemcpyHostToDevice, s),
                           "svs_tvl1_plan_retarget");
  std::vector<float*> nop((size_t)num_pairs, nullptr);
  if (!st) st = check_cuda(cudaMemcpyAsync(P->d_pout, nop.data(), nop.size() * sizeof(float*), cudaMemcpyHostToDevice, s),
                           "svs_tvl1_plan_retarget");
  if (!st) st = check_cuda(cudaStreamSynchronize(s), "svs_tvl1_plan_retarget");  // the host tables may change now
  if (st) return st;
  P->want_p = false;
  P->warm = false;
  P->pair_tile_req.clear();  // pair indices of the earlier batch mean nothing now
  ++P->tile_epoch;           // tiles, tensor maps and the graph follow the new sizes
  return SVS_OK;
}

svs_status svs_tvl1_plan_set_persistent(svs_plan* P, int on) {
  SVS_REQUIRE(P, "svs_tvl1_plan_set_persistent: null plan");
  P->persistent = on != 0;
  ++P->tile_epoch;  // rebuild the per-level choice and recapture the graph
  return SVS_OK;
}

int svs_tvl1_plan_level_persistent(const svs_plan* P, int level) {
  return (P && level >= 0 && level < (int)P->level_persist.size() && P->graph_tile == P->tile_epoch)
             ? (int)P->level_persist[level]
             : 0;
}

svs_status svs_tvl1_plan_set_stall_test(svs_plan* P, int level, int cta, int plane, uint32_t wait_us) {
  SVS_REQUIRE(P, "svs_tvl1_plan_set_stall_test: null plan");
  SVS_REQUIRE(level < P->levels, "svs_tvl1_plan_set_stall_test: bad level");
  P->stall_level = (level >= 0 && cta >= 0 && plane >= 0) ? level : -1;
  P->stall_cta = P->stall_level >= 0 ? cta : -1;
  P->stall_plane = P->stall_level >= 0 ? plane : -1;
  P->wait_us = wait_us ? wait_us : 2000000u;
  ++P->tile_epoch;  // the captured graph carries the launch arguments
  return SVS_OK;
}

}  // extern "C"

// =============================================================================================
// Allocation-free single-pair solve.
//
// For callers that cannot call cudaMalloc: code whose device memory is owned by another
// allocator (a framework's caching pool that has reserved the GPU), and latency-critical loops
// in which an allocation or free would synchronize the device. Everything the solve needs
// beyond the caller's inputs and outputs (pyramid, linearisation, dual state, descriptors and
// tile lists) is carved out of one file-scope device array of kNoAllocScratchBytes.
// =============================================================================================
namespace svs {
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;  // 32 MiB, held by every GPU that loads the library
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kMaxDevices] = {};
CUcontext g_noalloc_ctx[kMaxDevices] = {};

// The calling thread's current driver context (null if it cannot be read).
CUcontext current_context() {
  static PFN_cuCtxGetCurrent_v4000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 4000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
  }
  CUcontext c = nullptr;
  if (fn) fn(&c);
  return c;
}

// Device address of the scratch array on the current device: set up once per device (with that
// device current) through cudaGetSymbolAddress, and again if the device's context has been
// replaced since (a reset reloads the module, and the array may move); in host code the array's
// name is only a host-side stand-in and must never be handed to a kernel.
svs_status noalloc_scratch(unsigned char** out) {
  int dev = 0;
  svs_status st = check_cuda(cudaGetDevice(&dev), "svs_tvl1_solve_noalloc: cudaGetDevice");
  if (st) return st;
  if (dev < 0 || dev >= kMaxDevices) return fail(SVS_ERR_UNSUPPORTED, "svs_tvl1_solve_noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  const CUcontext ctx = current_context();
  if (!g_noalloc_ptr[dev] || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    st = check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "svs_tvl1_solve_noalloc: cudaGetSymbolAddress");
    if (st) return st;
    g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    g_noalloc_ctx[dev] = current_context();  // the lookup makes the primary context current
  }
  *out = g_noalloc_ptr[dev];
  return SVS_OK;
}

// The solve's metadata (descriptors, pointer table, tile lists) reaches the scratch as kernel
// parameters: a launch copies its parameters when it is enqueued, so no host buffer has to
// outlive the call and no host-to-device copy is queued.
struct UploadChunk {
  unsigned char bytes[3840];
};
__global__ void upload_kernel(unsigned char* __restrict__ dst, const __grid_constant__ UploadChunk c, unsigned n) {
  for (unsigned i = threadIdx.x; i < n; i += blockDim.x) dst[i] = c.bytes[i];
}
// Returns the number of launches issued (-1 after a launch error).
long long upload(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  const unsigned char* p = static_cast<const unsigned char*>(src);
  long long launches = 0;
  for (size_t off = 0; off < bytes; off += sizeof(UploadChunk::bytes)) {
    UploadChunk c;
    const unsigned n = (unsigned)std::min(sizeof(c.bytes), bytes - off);
    std::memcpy(c.bytes, p + off, n);
    upload_kernel<<<1, 256, 0, s>>>(static_cast<unsigned char*>(dst) + off, c, n);
    ++launches;
  }
  return cudaPeekAtLastError() == cudaSuccess ? launches : -1;
}

}  // namespace
}  // namespace svs

extern "C" svs_status svs_tvl1_solve_noalloc(const svs_tvl1_params* prm, const float* I0, const float* I1,
                                             int nz, int ny, int nx, float* u_out, svs_stream_t stream) {
  using namespace svs;
  SVS_REQUIRE(prm && I0 && I1 && u_out, "svs_tvl1_solve_noalloc: null pointer");
  SVS_REQUIRE(prm->num_scales >= 1 && prm->num_scales <= 8, "svs_tvl1_solve_noalloc: num_scales out of range");
  SVS_REQUIRE(prm->max_warps >= 0 && prm->max_outer_iterations >= 0, "svs_tvl1_solve_noalloc: negative iteration count");
  SVS_REQUIRE(prm->primaldual_algorithm_type == 1 || prm->primaldual_algorithm_type == 2,
              "svs_tvl1_solve_noalloc: primaldual_algorithm_type must be 1 or 2");
  SVS_REQUIRE(prm->boundary >= 0 && prm->boundary <= 2, "svs_tvl1_solve_noalloc: bad boundary type");
  SVS_REQUIRE(prm->interpolation >= 0 && prm->interpolation <= 2, "svs_tvl1_solve_noalloc: bad interpolation type");
  SVS_REQUIRE(prm->storage >= 0 && prm->storage <= 4, "svs_tvl1_solve_noalloc: bad storage type");
  SVS_REQUIRE(prm->weight_tv >= 0.f, "svs_tvl1_solve_noalloc: weight_tv must be >= 0");
  SVS_REQUIRE(prm->median_kernel == 0 || prm->median_kernel == 1 || prm->median_kernel == 3 ||
                  prm->median_kernel == 5 || prm->median_kernel == 7,
              "svs_tvl1_solve_noalloc: median kernel must be 0, 1, 3, 5 or 7");
  SVS_REQUIRE(nz < 65535 && ny < 65535 && nx < 65535, "svs_tvl1_solve_noalloc: volume dimension too large");

  // A host-only plan: the same launch sequence as svs_tvl1_solve_batch, with every device
  // pointer carved from the scratch array and the plain-load iterate kernel at every level.
  svs_plan P;
  P.prm = *prm;
  P.num_pairs = 1;
  P.levels = prm->num_scales;
  P.dims = {nz, ny, nx};
  P.h_descs.resize(P.levels);
  const size_t ub = flow_bytes(prm->storage), sb = field_bytes(prm->storage);
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  size_t bytes = al(P.levels * sizeof(Desc)) + al(7 * sizeof(float*));
  {
    int z = nz, y = ny, x = nx;
    for (int l = 0; l < P.levels; ++l) {
      if (l > 0) { z = (z + 1) / 2; y = (y + 1) / 2; x = (x + 1) / 2; }
      SVS_REQUIRE(z >= 3 && y >= 3 && x >= 3,
                  "svs_tvl1_solve_noalloc: every pyramid level needs at least 3 nodes per axis");
      Desc& d = P.h_descs[l];
      std::memset(&d, 0, sizeof(d));
      d.nz = z; d.ny = y; d.nx = x;
      d.pitch = (x + 7) / 8 * 8;
      d.n = (long long)z * y * x;
      d.cs = (long long)d.pitch * y * z;
      if (prm->length_type == 0) { d.lz = (float)(z - 1); d.ly = (float)(y - 1); d.lx = (float)(x - 1); }
      else { d.lz = prm->length_z; d.ly = prm->length_y; d.lx = prm->length_x; }
      d.hz = d.lz / (float)(z - 1); d.hy = d.ly / (float)(y - 1); d.hx = d.lx / (float)(x - 1);
      const size_t n = (size_t)d.n, cs = (size_t)d.cs;
      bytes += 2 * al(n * 4) + al(4 * n * 4) + al(6 * cs * sb) + al(cs * sb) + al(3 * cs * sb) +
               2 * al(3 * cs * ub) + 2 * al(9 * cs * sb);
      if (l == 0 && prm->median_kernel > 1) bytes += al(3 * n * 4);
    }
  }
  P.level_tile.assign(P.levels, 6);  // plain-load 32x8
  P.h_tiles.assign(P.levels, {});
  for (int l = 0; l < P.levels; ++l) {
    build_tiles(P, l, 6);
    bytes += al(P.h_tiles[l].size() * sizeof(Tile));
  }
  if (bytes > kNoAllocScratchBytes)
    return fail(SVS_ERR_INVALID_ARG, "svs_tvl1_solve_noalloc: a " + std::to_string(nz) + "x" + std::to_string(ny) + "x" +
                                         std::to_string(nx) + " solve needs " + std::to_string(bytes) +
                                         " bytes of scratch; the allocation-free entry point has " +
                                         std::to_string(kNoAllocScratchBytes) + " (use svs_tvl1_solve_batch)");
  unsigned char* base = nullptr;
  svs_status st = noalloc_scratch(&base);
  if (st) return st;
  char* cur = reinterpret_cast<char*>(base);
  P.d_descs = carve<Desc>(cur, P.levels);
  float** ptrs = carve<float*>(cur, 7);  // raw I0, raw I1, u_out, p_out, median temp, u_init, p_init
  P.d_raw = ptrs;
  P.d_uout = ptrs + 2;
  P.d_pout = ptrs + 3;
  P.d_umed = ptrs + 4;
  P.d_uinit = const_cast<const float**>(ptrs + 5);
  P.d_pinit = const_cast<const float**>(ptrs + 6);
  P.d_tiles.assign(P.levels, nullptr);
  for (int l = 0; l < P.levels; ++l) P.d_tiles[l] = carve<Tile>(cur, P.h_tiles[l].size());
  char* state_begin = cur;
  for (int l = 0; l < P.levels; ++l) {
    Desc& d = P.h_descs[l];
    const size_t n = (size_t)d.n, cs = (size_t)d.cs;
    d.I0 = carve<float>(cur, n);
    d.I1 = carve<float>(cur, n);
    d.ig = carve<float>(cur, 4 * n);
    d.D = carve<char>(cur, 6 * cs * sb);
    d.rc = carve<char>(cur, cs * sb);
    d.gw = carve<char>(cur, 3 * cs * sb);
    d.u[0] = carve<char>(cur, 3 * cs * ub);
    d.u[1] = carve<char>(cur, 3 * cs * ub);
    d.p[0] = carve<char>(cur, 9 * cs * sb);
    d.p[1] = carve<char>(cur, 9 * cs * sb);
  }
  float* umed = prm->median_kernel > 1 ? carve<float>(cur, 3 * (size_t)nz * ny * nx) : nullptr;
  // The blur reads the caller's frames and finalize writes the caller's flow directly.
  P.raw = {const_cast<float*>(I0), const_cast<float*>(I1)};
  P.uout = {u_out};
  P.umed = {umed};
  P.pout = {nullptr};
  std::vector<float*> hp = {P.raw[0], P.raw[1], u_out, nullptr, umed, nullptr, nullptr};
  // step-size schedule and blur weights exactly as svs_tvl1_plan_create builds them
  {
    double sg = prm->sigma, ta = prm->tau;
    for (int it = 0; it < prm->max_outer_iterations; ++it) {
      P.sig_sched.push_back((float)sg);
      P.tau_sched.push_back((float)ta);
      if (prm->primaldual_algorithm_type == 2) {
        const double th = 1.0 / std::sqrt(1.0 + 2.0 * prm->gamma * ta);
        ta *= th;
        sg /= th;
      }
    }
  }
  if (prm->use_gaussian_blur) {
    const double sgm = prm->gaussian_blur_sigma;
    int ks = (int)(sgm * 5);
    if (ks % 2 == 0) ks += 1;
    SVS_REQUIRE(ks <= 9 && ks >= 1, "svs_tvl1_solve_noalloc: gaussian_blur_sigma out of range (kernel size <= 9)");
    const int lo = -((ks + 1) / 2), hi = ks / 2 + 1;
    std::vector<float> t(ks), g(ks), k1(ks);
    for (int i = 0; i < ks; ++i) t[i] = (ks == 1) ? (float)lo : (float)(lo + (double)(hi - lo) * i / (ks - 1));
    float gs = 0.f;
    for (int i = 0; i < ks; ++i) {
      const float a = t[i] / (float)sgm;
      g[i] = std::exp(-(a * a) / 2.0f);
      gs += g[i];
    }
    for (int i = 0; i < ks; ++i) k1[i] = g[i] / gs;
    float tot = 0.f;
    std::vector<float> k3((size_t)ks * ks * ks);
    for (int a = 0; a < ks; ++a)
      for (int b = 0; b < ks; ++b)
        for (int c = 0; c < ks; ++c) { k3[(a * ks + b) * ks + c] = k1[a] * k1[b] * k1[c]; tot += k3[(a * ks + b) * ks + c]; }
    for (size_t i = 0; i < k3.size(); ++i) P.blur.w[i] = k3[i] / tot;
    P.blur_r = ks / 2;
  }
  // Metadata into the scratch (as kernel parameters), then clear the state region so no value
  // from an earlier call is ever read.
  cudaStream_t s = stream;
  long long up = upload(P.d_descs, P.h_descs.data(), P.levels * sizeof(Desc), s);
  const long long up_ptrs = up < 0 ? -1 : upload(ptrs, hp.data(), hp.size() * sizeof(float*), s);
  up = up_ptrs < 0 ? -1 : up + up_ptrs;
  for (int l = 0; l < P.levels && up >= 0; ++l) {
    const long long n = upload(P.d_tiles[l], P.h_tiles[l].data(), P.h_tiles[l].size() * sizeof(Tile), s);
    up = n < 0 ? -1 : up + n;
  }
  if (up < 0) return fail(SVS_ERR_LAUNCH, std::string("svs_tvl1_solve_noalloc: launch failed: ") + cudaGetErrorString(cudaGetLastError()));
  st = check_cuda(cudaMemsetAsync(state_begin, 0, (size_t)(cur - state_begin), s), "svs_tvl1_solve_noalloc");
  if (st) return st;
  P.warm = false;
  const long long nl = enqueue(P, s);
  if (nl < 0) return fail(SVS_ERR_LAUNCH, std::string("svs_tvl1_solve_noalloc: launch failed: ") + cudaGetErrorString(cudaGetLastError()));
  count_launches((uint64_t)(nl + up));
  return SVS_OK;
}
