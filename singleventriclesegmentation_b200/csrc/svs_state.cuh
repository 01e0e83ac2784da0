// Device-side state of the fused solver: storage conversions, the per-(pair, level) descriptor
// with its pitched planar layout, tiles and iteration arguments.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "svs_common.cuh"

namespace svs {

// ------------------------------------------------------------------------- storage conversions
template <typename S> struct Store;
template <> struct Store<float> {
  static __device__ __forceinline__ float ld(const float* p) { return __ldg(p); }
  static __device__ __forceinline__ float sh(const float* p) { return *p; }
  static __device__ __forceinline__ void st(float* p, float v) { *p = v; }
};
template <> struct Store<__nv_bfloat16> {
  static __device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }
  static __device__ __forceinline__ float sh(const __nv_bfloat16* p) { return __bfloat162float(*p); }
  static __device__ __forceinline__ void st(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
};
template <> struct Store<__half> {
  static __device__ __forceinline__ float ld(const __half* p) { return __half2float(__ldg(p)); }
  static __device__ __forceinline__ float sh(const __half* p) { return __half2float(*p); }
  static __device__ __forceinline__ void st(__half* p, float v) { *p = __float2half_rn(v); }
};

// Two x-adjacent values (an even element index, so 8- or 4-byte aligned) as one access; the
// roundings are those of Store<S> applied to each value.
template <typename S> struct Pair;
template <> struct Pair<float> {
  static __device__ __forceinline__ float2 sh(const float* p) { return *reinterpret_cast<const float2*>(p); }
  static __device__ __forceinline__ void st(float* p, float a, float b) {
    *reinterpret_cast<float2*>(p) = make_float2(a, b);
  }
};
template <> struct Pair<__nv_bfloat16> {
  static __device__ __forceinline__ float2 sh(const __nv_bfloat16* p) {
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
  }
  static __device__ __forceinline__ void st(__nv_bfloat16* p, float a, float b) {
    *reinterpret_cast<__nv_bfloat162*>(p) = __floats2bfloat162_rn(a, b);
  }
};
template <> struct Pair<__half> {
  static __device__ __forceinline__ float2 sh(const __half* p) {
    return __half22float2(*reinterpret_cast<const __half2*>(p));
  }
  static __device__ __forceinline__ void st(__half* p, float a, float b) {
    *reinterpret_cast<__half2*>(p) = __floats2half2_rn(a, b);
  }
};

// One (pair, level) of the batch.
// Float fields are dense [nz][ny][nx]: I0, I1, and ig = (I1, dI1/dx, dI1/dy, dI1/dz) as one
// float4 per voxel (16-byte aligned). Iteration-state fields of storage
// type S (D, rc, gw, u[2], p[2]) are planar and PITCHED: component c of voxel (z, y, x) is at
// c*cs + (z*ny + y)*pitch + x, with pitch a multiple of 8 elements so that every row starts on a
// 16-byte boundary (the TMA stride rule) for f32, bf16 and f16 alike.
struct Desc {
  int nz, ny, nx, pitch;
  float hz, hy, hx, pad1;
  float lz, ly, lx, pad2;
  long long n;   // voxels
  long long cs;  // component stride of the pitched fields, = pitch * ny * nz
  const float* I0;
  const float* I1;
  float* ig;
  void* D;
  void* rc;
  void* gw;
  void* u[2];
  void* p[2];
  int* stop;  // optional per-pair flag (residual stopping): non-zero = skip the rest of the level
};

__device__ __forceinline__ long long pidx(const Desc& d, int z, int y, int x) {
  return ((long long)z * d.ny + y) * d.pitch + x;
}

// One CTA of the iterate kernels: a column tile [x0, x0+TX) x [y0, y0+TY) x [z0, z1).
struct Tile {
  int desc;
  int x0, y0;
  int z0z1;  // z0 | z1 << 16
};

struct IterArgs {
  float sigma, tau, factor, wtv;
  int src, bdry;
  // bounded pipeline waits give up after wait_us microseconds; the CTA with blockIdx.x ==
  // stall_cta leaves the copies of its staged plane number stall_plane (counted from its first
  // staged plane) unissued (a test of the timeout path; stall_cta < 0: off)
  unsigned wait_us;
  int stall_cta, stall_plane;
};

// The persistent form of the iteration loop: all `iters` primal-dual iterations of one warp at
// one level in a single cooperative launch (svs_iterate.cuh, iterate_persist_kernel).
struct PersistArgs {
  const float* sig;    // [iters] sigma of each iteration (device; the host float64 schedule rounded)
  const float* tau;    // [iters] tau of each iteration
  float wm, wtv;       // weight_matching (factor = tau * wm), weight_tv
  int src0, bdry;      // ping-pong copy read by the first iteration; boundary type
  int iters;
  unsigned wait_us;    // bound of every pipeline and grid-barrier wait
  int stall_cta, stall_plane;  // the timeout-path test of IterArgs (stall_cta counts tiles)
  unsigned* counter;   // grid-barrier arrivals, zero at launch
};

// TMA descriptors of one (pair, level): the two ping-pong copies of u and p, D, rc and gw.
struct alignas(64) TMaps {
  CUtensorMap u[2];
  CUtensorMap p[2];
  CUtensorMap D;
  CUtensorMap rc;
  CUtensorMap gw;
};

// Device status bits (read back by svs_tvl1_plan_check).
enum { SVS_DEV_TIMEOUT = 1 };

}  // namespace svs
