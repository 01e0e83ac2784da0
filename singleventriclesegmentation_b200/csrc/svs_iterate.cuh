// The fused primal-dual iteration (svs/modules/flow/tvl13d.py:213-253) as one kernel per
// iteration, in two forms:
//   iterate_kernel      plain loads, one z-plane of each field per step, state in registers;
//   iterate_tma_kernel  a multi-stage TMA pipeline: one thread issues cp.async.bulk.tensor
//                       loads of whole plane tiles (u, p, D, rc, gw) DIST planes ahead into
//                       shared-memory rings, completion tracked by mbarriers.
// Both march a TX x TY column tile along z. Thread (tx, ty) of the (TX+2) x (TY+2) block owns
// column (x0-1+tx, y0-1+ty) of the "dual region" (tile plus a one-voxel x/y halo). At plane k:
//   dual:   on the dual region minus its 4 corners, p_new(k) = proj(p + sigma D grad u) and
//           q = D p_new; the z-row of q stays in registers, the x- and y-rows are published;
//   primal: on the tile interior, plane j = k-1 is finished: div = adjoint(q) from the
//           published rows of plane j and the registers of planes j-1 and j+1, then
//           u_new(j) = prox_primal(u - tau div).
// Halo duals are recomputed by neighbouring tiles, so the tiles of one launch are independent
// (u and p are ping-pong buffers). The flow u is stored as SU, everything else as SP.
//
// Difference stencils use per-position coefficients (prev, cur, next) instead of boundary
// branches; with h = 1 the result is bitwise the reference's expression:
//   forward  0.5*(next - prev)/h               differentialOps.cu:540-655 (one-sided at faces
//                                              for NEAREST/REFLECT, zero for MIRROR)
//   adjoint  MIRROR  i>1&&i<N-2: 0.5(prev-next); i>1: 0.5 prev; else -0.5 next
//            others  0<i<N-1: 0.5(prev-next); i=N-1: 0.5(prev+cur); i=0: 0.5(-cur-next)
//                                              differentialOps.cu:658-1039 (then /h)
#pragma once

#include <type_traits>

#include "svs_state.cuh"

namespace svs {

// Elementwise FP32 arithmetic on one voxel (float) or on two x-adjacent voxels at once (float2,
// the packed FP32 instructions of sm_100). Every operation rounds like its scalar counterpart and
// products are fused only where an explicit vfma says so, so the scalar and packed forms give
// bitwise the same result per voxel.
__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ float vmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float vadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <typename T> __device__ __forceinline__ T bcast(float s);
template <> __device__ __forceinline__ float bcast<float>(float s) { return s; }
template <> __device__ __forceinline__ float2 bcast<float2>(float s) { return make_float2(s, s); }
__device__ __forceinline__ float first(float v) { return v; }
__device__ __forceinline__ float first(float2 v) { return v.x; }

template <typename T>
struct StencilV {
  T m, c, p;
};
using Stencil3 = StencilV<float>;
__device__ __forceinline__ StencilV<float2> pack(const Stencil3& a, const Stencil3& b) {
  return {make_float2(a.m, b.m), make_float2(a.c, b.c), make_float2(a.p, b.p)};
}
template <typename T> __device__ __forceinline__ StencilV<T> bcast_st(const Stencil3& a) {
  return {bcast<T>(a.m), bcast<T>(a.c), bcast<T>(a.p)};
}

__device__ __forceinline__ Stencil3 fwd_coef(int i, int n, int bdry, float h) {
  const float a = 0.5f / h;
  if (i > 0 && i < n - 1) return {-a, 0.f, a};
  if (bdry == SVS_BOUNDARY_MIRROR) return {0.f, 0.f, 0.f};
  if (i > 0) return {-a, a, 0.f};  // i == n-1
  return {0.f, -a, a};             // i == 0
}

__device__ __forceinline__ Stencil3 adj_coef(int i, int n, int bdry, float ih) {
  const float a = 0.5f * ih;
  if (bdry == SVS_BOUNDARY_MIRROR) {
    if (i > 1) return (i < n - 2) ? Stencil3{a, 0.f, -a} : Stencil3{a, 0.f, 0.f};
    return {0.f, 0.f, -a};
  }
  if (i > 0) return (i < n - 1) ? Stencil3{a, 0.f, -a} : Stencil3{a, a, 0.f};
  return {0.f, -a, -a};
}

// GEN = false: MIRROR boundary, where every stencil has a zero centre coefficient (the centre
// term is dropped; for h = 1 the result is bitwise that of the three-term form).
template <bool GEN, typename T>
__device__ __forceinline__ T apply3(const StencilV<T>& s, T prev, T cur, T next) {
  if (GEN) return vfma(s.p, next, vfma(s.c, cur, vmul(s.m, prev)));
  return vfma(s.p, next, vmul(s.m, prev));
}

// a0 b0 + a1 b1 + a2 b2
template <typename T>
__device__ __forceinline__ T dot3(T a0, T a1, T a2, T b0, T b1, T b2) {
  return vfma(a2, b2, vfma(a1, b1, vmul(a0, b0)));
}

__device__ __forceinline__ float proj_scale(float nsq, float wtv, float wtv2) {
  // weight_tv == 0 gives sc = 0 (or v = 0), i.e. p = 0 as tvl13d.py:223-224 requires
  return (nsq > wtv2) ? __fmul_rn(wtv, rsqrtf(nsq)) : 1.0f;
}
__device__ __forceinline__ float2 proj_scale(float2 nsq, float wtv, float wtv2) {
  return make_float2(proj_scale(nsq.x, wtv, wtv2), proj_scale(nsq.y, wtv, wtv2));
}

// Dual update of one flow component, tvl13d.py:215-222 with opticalFlowOps.cu:179-208:
// v = p + sigma D g; p_new = v / max(1, |v| / weight_tv), written as v * min(1, weight_tv *
// rsqrt(|v|^2)). D is the packed symmetric tensor (d00 d01 d02 d11 d12 d22).
template <typename T>
__device__ __forceinline__ void dual_row(const T D[6], T ex, T ey, T ez, T& p0, T& p1, T& p2, float sigma,
                                         float wtv, float wtv2) {
  const T d0 = dot3(D[0], D[1], D[2], ex, ey, ez);
  const T d1 = dot3(D[1], D[3], D[4], ex, ey, ez);
  const T d2 = dot3(D[2], D[4], D[5], ex, ey, ez);
  const T sg = bcast<T>(sigma);
  const T v0 = vfma(sg, d0, p0), v1 = vfma(sg, d1, p1), v2 = vfma(sg, d2, p2);
  const T sc = proj_scale(dot3(v0, v1, v2, v0, v1, v2), wtv, wtv2);
  p0 = vmul(v0, sc);
  p1 = vmul(v1, sc);
  p2 = vmul(v2, sc);
}

// Step length along g of the L1 shrinkage, the three cases of opticalFlowOps.cu:140-171 (no
// divergence): rho < -th: +factor; rho > th: -factor; |rho| <= th: -rho/|g|^2 (0 where
// |g|^2 <= 1e-10, the reference's (double)g2 > 1e-10 for a float g2). The reference divides
// each component's product, (-rho g_c)/|g|^2, with IEEE division; this step divides once, with
// the fast approximate divide (__fdividef, within 2 ulp for these operands), and the caller
// multiplies by g_c. Measured on the 68-pair 80^3 level-0 launch: 4.4% faster than an IEEE
// divide (__fdiv_rn). A select, not a branch: the branch form took the 32x8 voxel-pair kernel
// from 168 to 202 registers (one CTA per SM instead of two).
__device__ __forceinline__ float shrink_step(float rho, float g2s, float factor) {
  const float th = __fmul_rn(factor, g2s);
  return (rho < -th) ? factor : (rho > th) ? -factor : (g2s >= 1e-10f ? __fdividef(-rho, g2s) : 0.f);
}
__device__ __forceinline__ float2 shrink_step(float2 rho, float2 g2s, float factor) {
  return make_float2(shrink_step(rho.x, g2s.x, factor), shrink_step(rho.y, g2s.y, factor));
}

// Primal update, tvl13d.py:229-235 with opticalFlowOps.cu:123-175: rho = rc + u.g (u before
// the update), u_new = (u - tau div) + shrinkage step along g.
// The step t needs no divergence; primal_step / primal_apply are the two halves, so a kernel can
// compute t before the dual that the divergence waits for (the same operations either way).
template <typename T>
__device__ __forceinline__ T primal_step(const T u[3], float factor, T rc, const T g[3]) {
  const T rho = vadd(rc, dot3(u[0], u[1], u[2], g[0], g[1], g[2]));
  const T g2s = dot3(g[0], g[1], g[2], g[0], g[1], g[2]);
  return shrink_step(rho, g2s, factor);
}
template <typename T>
__device__ __forceinline__ void primal_apply(const T u[3], const T div[3], float tau, T t, const T g[3], T un[3]) {
  const T mt = bcast<T>(-tau);
#pragma unroll
  for (int c = 0; c < 3; ++c) un[c] = vfma(mt, div[c], u[c]);
#pragma unroll
  for (int c = 0; c < 3; ++c) un[c] = vfma(t, g[c], un[c]);
}
template <typename T>
__device__ __forceinline__ void primal_voxel(const T u[3], const T div[3], float tau, float factor, T rc,
                                             const T g[3], T un[3]) {
  primal_apply(u, div, tau, primal_step(u, factor, rc, g), g, un);
}

// div = (dx + dy) + dz
template <typename T> __device__ __forceinline__ T sum3(T dx, T dy, T dz) { return vadd(vadd(dx, dy), dz); }

// ------------------------------------------------------------------------ plain-load form
template <typename SU, typename SP, int TX, int TY, bool GEN>
__global__ void __launch_bounds__((TX + 2) * (TY + 2))
iterate_kernel(const Tile* __restrict__ tiles, const Desc* __restrict__ descs, IterArgs a) {
  constexpr int PX = TX + 2, PY = TY + 2, UX = TX + 4, UY = TY + 4;
  constexpr int NRING = 2 * (TX + TY);
  __shared__ float su[2][3][UY][UX];
  __shared__ float sq[2][6][PY][PX];

  const Tile T = tiles[blockIdx.x];
  const Desc& Dg = descs[T.desc];
  if (Dg.stop && *Dg.stop) return;  // pair converged for this level
  const int nz = Dg.nz, ny = Dg.ny, nx = Dg.nx;
  const int cs = (int)Dg.cs;
  const int plane = Dg.pitch * ny;
  const int z0 = T.z0z1 & 0xffff, z1 = T.z0z1 >> 16;
  const SU* __restrict__ u_src = reinterpret_cast<const SU*>(Dg.u[a.src]);
  const SP* __restrict__ p_src = reinterpret_cast<const SP*>(Dg.p[a.src]);
  SU* __restrict__ u_dst = reinterpret_cast<SU*>(Dg.u[a.src ^ 1]);
  SP* __restrict__ p_dst = reinterpret_cast<SP*>(Dg.p[a.src ^ 1]);
  const SP* __restrict__ Dm = reinterpret_cast<const SP*>(Dg.D);
  const SP* __restrict__ rcm = reinterpret_cast<const SP*>(Dg.rc);
  const SP* __restrict__ gwm = reinterpret_cast<const SP*>(Dg.gw);

  const int tid = threadIdx.x;
  const int tx = tid % PX, ty = tid / PX;
  const int gx = T.x0 - 1 + tx, gy = T.y0 - 1 + ty;
  const bool in_dom = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
  const bool corner = (tx == 0 || tx == PX - 1) && (ty == 0 || ty == PY - 1);
  const bool dual_on = in_dom && !corner;
  const bool interior = in_dom && tx >= 1 && tx <= TX && ty >= 1 && ty <= TY;
  const int col = gy * Dg.pitch + gx;
  const int bdry = a.bdry;
  const Stencil3 fx = fwd_coef(gx, nx, bdry, Dg.hx), fy = fwd_coef(gy, ny, bdry, Dg.hy);
  const Stencil3 ax = adj_coef(gx, nx, bdry, 1.0f / Dg.hx), ay = adj_coef(gy, ny, bdry, 1.0f / Dg.hy);
  const float ihz = 1.0f / Dg.hz;

  int rx = -1, ry = -1;
  if (tid < NRING) {
    int r = tid;
    if (r < TY) { rx = 0; ry = 2 + r; }
    else if ((r -= TY) < TY) { rx = UX - 1; ry = 2 + r; }
    else if ((r -= TY) < TX) { rx = 2 + r; ry = 0; }
    else { r -= TX; rx = 2 + r; ry = UY - 1; }
  }
  const int rgx = T.x0 - 2 + rx, rgy = T.y0 - 2 + ry;
  const bool ring_on = tid < NRING && rgx >= 0 && rgx < nx && rgy >= 0 && rgy < ny;
  const int rcol = rgy * Dg.pitch + rgx;

  // Cells of out-of-domain columns are never written but are multiplied by zero stencil
  // coefficients at the domain faces: they must hold zeros, not stale bits (0 * NaN = NaN).
  for (int i = tid; i < 2 * 3 * UY * UX; i += blockDim.x) (&su[0][0][0][0])[i] = 0.f;
  for (int i = tid; i < 2 * 6 * PY * PX; i += blockDim.x) (&sq[0][0][0][0])[i] = 0.f;
  __syncthreads();
  const int kb = max(z0 - 1, 0), ke = min(z1, nz - 1);
  float um[3] = {0.f, 0.f, 0.f}, uc[3] = {0.f, 0.f, 0.f}, up[3] = {0.f, 0.f, 0.f};
  if (in_dom) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (kb >= 1) um[c] = Store<SU>::ld(u_src + c * cs + (kb - 1) * plane + col);
      uc[c] = Store<SU>::ld(u_src + c * cs + kb * plane + col);
      if (kb + 1 < nz) up[c] = Store<SU>::ld(u_src + c * cs + (kb + 1) * plane + col);
    }
  }
  float qzmm[3] = {0.f, 0.f, 0.f}, qzm[3] = {0.f, 0.f, 0.f}, qzc[3] = {0.f, 0.f, 0.f};
  const float wtv2 = a.wtv * a.wtv;

  for (int k = kb; k <= ke; ++k) {
    const int slot = k & 1;
    float pk[9], Dk[6];
    if (dual_on) {
      const int o = k * plane + col;
#pragma unroll
      for (int c = 0; c < 9; ++c) pk[c] = Store<SP>::ld(p_src + c * cs + o);
#pragma unroll
      for (int c = 0; c < 6; ++c) Dk[c] = Store<SP>::ld(Dm + c * cs + o);
    }
    const int j = k - 1;
    const bool primal_on = interior && j >= z0 && j < z1;
    float rcj = 0.f, gj[3] = {0.f, 0.f, 0.f};
    if (primal_on) {
      const int o = j * plane + col;
      rcj = Store<SP>::ld(rcm + o);
#pragma unroll
      for (int c = 0; c < 3; ++c) gj[c] = Store<SP>::ld(gwm + c * cs + o);
    }
    if (in_dom) {
#pragma unroll
      for (int c = 0; c < 3; ++c) su[slot][c][ty + 1][tx + 1] = uc[c];
    }
    if (ring_on) {
#pragma unroll
      for (int c = 0; c < 3; ++c) su[slot][c][ry][rx] = Store<SU>::ld(u_src + c * cs + k * plane + rcol);
    }
    __syncthreads();
    if (dual_on) {
      const Stencil3 fz = fwd_coef(k, nz, bdry, Dg.hz);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float ex = apply3<GEN>(fx, su[slot][c][ty + 1][tx], uc[c], su[slot][c][ty + 1][tx + 2]);
        const float ey = apply3<GEN>(fy, su[slot][c][ty][tx + 1], uc[c], su[slot][c][ty + 2][tx + 1]);
        const float ez = apply3<GEN>(fz, um[c], uc[c], up[c]);
        dual_row(Dk, ex, ey, ez, pk[3 * c], pk[3 * c + 1], pk[3 * c + 2], a.sigma, a.wtv, wtv2);
      }
      if (interior && k >= z0 && k < z1) {
        const int o = k * plane + col;
#pragma unroll
        for (int c = 0; c < 9; ++c) Store<SP>::st(p_dst + c * cs + o, pk[c]);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        sq[slot][c][ty][tx] = dot3(Dk[0], Dk[1], Dk[2], pk[3 * c], pk[3 * c + 1], pk[3 * c + 2]);
        sq[slot][3 + c][ty][tx] = dot3(Dk[1], Dk[3], Dk[4], pk[3 * c], pk[3 * c + 1], pk[3 * c + 2]);
        qzc[c] = dot3(Dk[2], Dk[4], Dk[5], pk[3 * c], pk[3 * c + 1], pk[3 * c + 2]);
      }
    }
    if (primal_on) {
      const int ps = slot ^ 1;
      const Stencil3 az = adj_coef(j, nz, bdry, ihz);
      float div[3], un[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float dx = apply3<GEN>(ax, sq[ps][c][ty][tx - 1], sq[ps][c][ty][tx], sq[ps][c][ty][tx + 1]);
        const float dy = apply3<GEN>(ay, sq[ps][3 + c][ty - 1][tx], sq[ps][3 + c][ty][tx], sq[ps][3 + c][ty + 1][tx]);
        div[c] = sum3(dx, dy, apply3<GEN>(az, qzmm[c], qzm[c], qzc[c]));
      }
      primal_voxel(um, div, a.tau, a.factor, rcj, gj, un);
      const int o = j * plane + col;
#pragma unroll
      for (int c = 0; c < 3; ++c) Store<SU>::st(u_dst + c * cs + o, un[c]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      qzmm[c] = qzm[c];
      qzm[c] = qzc[c];
      um[c] = uc[c];
      uc[c] = up[c];
      up[c] = 0.f;
    }
    if (in_dom && k + 2 < nz) {
#pragma unroll
      for (int c = 0; c < 3; ++c) up[c] = Store<SU>::ld(u_src + c * cs + (k + 2) * plane + col);
    }
  }
  if (z1 >= nz) {
    __syncthreads();
    const int j = nz - 1;
    if (interior && j >= z0) {
      const int ps = j & 1;
      const int o = j * plane + col;
      const Stencil3 az = adj_coef(j, nz, bdry, ihz);
      float gj[3], div[3], un[3];
      const float rcj = Store<SP>::ld(rcm + o);
#pragma unroll
      for (int c = 0; c < 3; ++c) gj[c] = Store<SP>::ld(gwm + c * cs + o);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float dx = apply3<GEN>(ax, sq[ps][c][ty][tx - 1], sq[ps][c][ty][tx], sq[ps][c][ty][tx + 1]);
        const float dy = apply3<GEN>(ay, sq[ps][3 + c][ty - 1][tx], sq[ps][3 + c][ty][tx], sq[ps][3 + c][ty + 1][tx]);
        div[c] = sum3(dx, dy, apply3<GEN>(az, qzmm[c], qzm[c], 0.f));
      }
      primal_voxel(um, div, a.tau, a.factor, rcj, gj, un);
#pragma unroll
      for (int c = 0; c < 3; ++c) Store<SU>::st(u_dst + c * cs + o, un[c]);
    }
  }
}

// ------------------------------------------------------------------------------- TMA form
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait: gives up after limit_ns of wall time (IterArgs::wait_us, 2 s by default; a
// tile's loads complete in microseconds).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}
// Plain arrival (release, CTA scope) of this thread on an mbarrier.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// Bounded wait that also gives up as soon as another thread of the CTA has raised `abort`; a
// thread that times out raises it.
__device__ __forceinline__ bool mbar_wait_abort(uint64_t* bar, uint32_t parity, volatile int* abort,
                                                uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (*abort) return false;
    if (global_ns() - t0 > limit_ns) {
      *abort = 1;
      return false;
    }
  }
  return true;
}
// 4D tiled TMA load (no multicast) of one box into shared memory, completion on `bar`.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int x,
                                            int y, int z, int c) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(c), "r"(smem_addr(bar))
      : "memory");
}

__host__ __device__ constexpr int round_up_c(int v, int m) { return (v + m - 1) / m * m; }

__device__ __forceinline__ int gx_of(const Tile& T, int tid, int px) { return T.x0 - 1 + tid % px; }
__device__ __forceinline__ int gy_of(const Tile& T, int tid, int px) { return T.y0 - 1 + tid / px; }

// Shared-memory geometry of the TMA form: flow stored as SU, the rest as SP, tile TX x TY,
// prefetch distance DIST planes.
//   u ring    DIST+2 slots: planes k-1, k, k+1 are read at step k;
//   p/D ring  DIST slots:   plane k is read only by the dual of step k;
//   rc/gw     DIST+2 slots: plane j = k-1 is read after the barrier of step k;
//   mbarrier  one per plane, DIST+2 slots.
// Plane k+DIST is issued after the barrier of step k, into the u/rc-gw slot of plane k-2 and the
// p/D slot of plane k, all of which every thread has finished reading by then. The first plane
// (k = kb-1, the z-neighbour of the first dual plane) carries u only.
template <typename SU, typename SP, int TX, int TY, int DIST, int UPAD = 0>
struct TmaGeom {
  static constexpr int ESU = (int)sizeof(SU), ESP = (int)sizeof(SP);
  static constexpr int AU = 16 / ESU, AP = 16 / ESP;      // 16-byte alignment in elements
  static constexpr int PX = TX + 2, PY = TY + 2;
  // u box: x in [x0-AU, x0-AU+UXB); UPAD extra columns (a multiple of AU) only widen the row
  // pitch in shared memory (a bank-conflict choice), the copy reads them as well
  static constexpr int UXB = round_up_c(TX + AU + 2, AU) + UPAD;
  static constexpr int PXB = round_up_c(TX + AP + 1, AP);  // p/D box: x in [x0-AP, x0-AP+PXB)
  static constexpr int UYB = TY + 4, PYB = TY + 2;         // u rows from y0-2, p/D from y0-1
  static constexpr int U_TX = 3 * UYB * UXB * ESU;
  static constexpr int P_TX = 9 * PYB * PXB * ESP;
  static constexpr int D_TX = 6 * PYB * PXB * ESP;
  static constexpr int RC_TX = TY * TX * ESP;
  static constexpr int GW_TX = 3 * TY * TX * ESP;
  static constexpr int NU = DIST + 2, NPD = DIST, NR = DIST + 2, NB = DIST + 2;
  static constexpr int U_SLOT = round_up_c(U_TX, 128);
  static constexpr int P_SLOT = round_up_c(P_TX, 128);
  static constexpr int D_SLOT = round_up_c(D_TX, 128);
  static constexpr int RC_SLOT = round_up_c(RC_TX, 128);
  static constexpr int GW_SLOT = round_up_c(GW_TX, 128);
  static constexpr int U_OFF = 0;
  static constexpr int PD_OFF = U_OFF + NU * U_SLOT;
  static constexpr int PD_SLOT = P_SLOT + D_SLOT;
  static constexpr int R_OFF = PD_OFF + NPD * PD_SLOT;
  static constexpr int R_SLOT = RC_SLOT + GW_SLOT;
  static constexpr int SQ_OFF = R_OFF + NR * R_SLOT;
  static constexpr int SQ_BYTES = 3 * 6 * PY * PX * 4;
  static constexpr int BAR_OFF = round_up_c(SQ_OFF + SQ_BYTES, 8);
  static constexpr int SMEM = BAR_OFF + NB * 8;
  static constexpr int FULL_TX = U_TX + P_TX + D_TX + RC_TX + GW_TX;
};

template <typename SU, typename SP, int TX, int TY, int DIST, bool GEN>
__global__ void __launch_bounds__((TX + 2) * (TY + 2))
iterate_tma_kernel(const Tile* __restrict__ tiles, const Desc* __restrict__ descs,
                   const TMaps* __restrict__ maps, IterArgs a, int* __restrict__ status) {
  using G = TmaGeom<SU, SP, TX, TY, DIST>;
  constexpr int PX = G::PX, PY = G::PY, AU = G::AU, AP = G::AP, UXB = G::UXB, UYB = G::UYB,
                PXB = G::PXB, PYB = G::PYB;
  static_assert(DIST >= 2, "step k waits for plane k+1, issued at step k+1-DIST");
  extern __shared__ __align__(128) unsigned char smem[];
  float(*sq)[6][PY][PX] = reinterpret_cast<float(*)[6][PY][PX]>(smem + G::SQ_OFF);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + G::BAR_OFF);

  const Tile T = tiles[blockIdx.x];
  const Desc& Dg = descs[T.desc];
  if (Dg.stop && *Dg.stop) return;  // pair converged for this level
  const TMaps* M = maps + T.desc;
  const int nz = Dg.nz, ny = Dg.ny, nx = Dg.nx;
  const int cs = (int)Dg.cs;
  const int plane = Dg.pitch * ny;
  const int z0 = T.z0z1 & 0xffff, z1 = T.z0z1 >> 16;
  const int col0 = gy_of(T, threadIdx.x, G::PX) * Dg.pitch + gx_of(T, threadIdx.x, G::PX);
  SU* __restrict__ u_dst = reinterpret_cast<SU*>(Dg.u[a.src ^ 1]) + col0;  // this thread's column
  SP* __restrict__ p_dst = reinterpret_cast<SP*>(Dg.p[a.src ^ 1]) + col0;
  const CUtensorMap* mu = &M->u[a.src];
  const CUtensorMap* mp = &M->p[a.src];

  const int tid = threadIdx.x;
  const int tx = tid % PX, ty = tid / PX;
  const int gx = T.x0 - 1 + tx, gy = T.y0 - 1 + ty;
  const bool in_dom = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
  const bool corner = (tx == 0 || tx == PX - 1) && (ty == 0 || ty == PY - 1);
  const bool dual_on = in_dom && !corner;
  const bool interior = in_dom && tx >= 1 && tx <= TX && ty >= 1 && ty <= TY;
  const int uo = (ty + 1) * UXB + (tx + AU - 1);  // own column in a u box component
  const int po = ty * PXB + (tx + AP - 1);        // own column in a p/D box component
  const int ro = (ty - 1) * TX + (tx - 1);        // own column in an rc/gw box (interior)
  const int bdry = a.bdry;
  const Stencil3 fx = fwd_coef(gx, nx, bdry, Dg.hx), fy = fwd_coef(gy, ny, bdry, Dg.hy);
  const Stencil3 ax = adj_coef(gx, nx, bdry, 1.0f / Dg.hx), ay = adj_coef(gy, ny, bdry, 1.0f / Dg.hy);
  const float ihz = 1.0f / Dg.hz, hz = Dg.hz;

  const int kb = max(z0 - 1, 0), ke = min(z1, nz - 1);
  const int pl = max(kb - 1, 0), ph = min(ke + 1, nz - 1);  // planes staged by this tile
  const uint64_t wait_ns = (uint64_t)a.wait_us * 1000ull;
  const int stall_r = (int)blockIdx.x == a.stall_cta ? a.stall_plane : -1;
  auto issue = [&](int q) {
    const int r = q - pl;
    if (r == stall_r) return;  // timeout-path test: this plane's copies are never issued
    uint64_t* bar = bars + r % G::NB;
    unsigned char* U = smem + G::U_OFF + (r % G::NU) * G::U_SLOT;
    if (q < kb) {
      mbar_arrive_expect_tx(bar, (uint32_t)G::U_TX);
      tma_load_4d(U, mu, bar, T.x0 - AU, T.y0 - 2, q, 0);
      return;
    }
    unsigned char* PD = smem + G::PD_OFF + ((q - kb) % G::NPD) * G::PD_SLOT;
    unsigned char* R = smem + G::R_OFF + ((q - kb) % G::NR) * G::R_SLOT;
    mbar_arrive_expect_tx(bar, (uint32_t)G::FULL_TX);
    tma_load_4d(U, mu, bar, T.x0 - AU, T.y0 - 2, q, 0);
    tma_load_4d(PD, mp, bar, T.x0 - AP, T.y0 - 1, q, 0);
    tma_load_4d(PD + G::P_SLOT, &M->D, bar, T.x0 - AP, T.y0 - 1, q, 0);
    tma_load_4d(R, &M->rc, bar, T.x0, T.y0, q, 0);
    tma_load_4d(R + G::RC_SLOT, &M->gw, bar, T.x0, T.y0, q, 0);
  };
  auto ubox = [&](int q) {
    return reinterpret_cast<const SU*>(smem + G::U_OFF + ((q - pl) % G::NU) * G::U_SLOT);
  };

  // Published rows of out-of-domain columns are never written but are multiplied by zero
  // stencil coefficients at the domain faces: they must hold zeros (0 * NaN = NaN).
  for (int i = tid; i < 3 * 6 * PY * PX; i += blockDim.x) (&sq[0][0][0][0])[i] = 0.f;
  if (tid == 0) {
    for (int s = 0; s < G::NB; ++s) mbar_init(bars + s, 1);
    mbar_fence_init();
  }
  __syncthreads();
  int issued = pl - 1;  // last plane issued (meaningful in thread 0)
  if (tid == 0) {
    const int last = min(kb + DIST - 1, ph);
    for (int q = pl; q <= last; ++q) issue(q);
    issued = last;
  }
  int waited = pl - 1;  // planes <= waited are complete (per thread)
  bool bad = false;

  float qzmm[3] = {0.f, 0.f, 0.f}, qzm[3] = {0.f, 0.f, 0.f}, qzc[3] = {0.f, 0.f, 0.f};
  float uown_m[3] = {0.f, 0.f, 0.f}, uown_c[3] = {0.f, 0.f, 0.f}, uown_p[3] = {0.f, 0.f, 0.f};
  const float wtv2 = a.wtv * a.wtv;

  for (int k = kb; k <= ke; ++k) {
    const int need = min(k + 1, ph);
    while (waited < need && !bad) {
      ++waited;
      const int r = waited - pl;
      if (!mbar_wait(bars + r % G::NB, (uint32_t)((r / G::NB) & 1), wait_ns)) bad = true;
    }
    const int qs = k % 3;
    // own column of u: planes k-1 and k from the previous step, k+1 read once here
    if (k == kb) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        uown_m[c] = (k - 1 >= pl) ? Store<SU>::sh(ubox(k - 1) + uo + c * UYB * UXB) : 0.f;
        uown_c[c] = Store<SU>::sh(ubox(k) + uo + c * UYB * UXB);
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) uown_p[c] = (k + 1 <= ph) ? Store<SU>::sh(ubox(k + 1) + uo + c * UYB * UXB) : 0.f;
    if (dual_on && !bad) {
      const SU* Uk = ubox(k) + uo;
      const unsigned char* PD = smem + G::PD_OFF + ((k - kb) % G::NPD) * G::PD_SLOT;
      const SP* P = reinterpret_cast<const SP*>(PD) + po;
      const SP* Dm = reinterpret_cast<const SP*>(PD + G::P_SLOT) + po;
      const Stencil3 fz = fwd_coef(k, nz, bdry, hz);
      float pk[9], Dk[6];
#pragma unroll
      for (int c = 0; c < 9; ++c) pk[c] = Store<SP>::sh(P + c * PYB * PXB);
#pragma unroll
      for (int c = 0; c < 6; ++c) Dk[c] = Store<SP>::sh(Dm + c * PYB * PXB);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const SU* u = Uk + c * UYB * UXB;
        const float uc = uown_c[c];
        const float ex = apply3<GEN>(fx, Store<SU>::sh(u - 1), uc, Store<SU>::sh(u + 1));
        const float ey = apply3<GEN>(fy, Store<SU>::sh(u - UXB), uc, Store<SU>::sh(u + UXB));
        const float ez = apply3<GEN>(fz, uown_m[c], uc, uown_p[c]);
        dual_row(Dk, ex, ey, ez, pk[3 * c], pk[3 * c + 1], pk[3 * c + 2], a.sigma, a.wtv, wtv2);
      }
      if (interior && k >= z0 && k < z1) {
        SP* dst = p_dst + k * plane;
#pragma unroll
        for (int c = 0; c < 9; ++c) Store<SP>::st(dst + c * cs, pk[c]);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        sq[qs][c][ty][tx] = dot3(Dk[0], Dk[1], Dk[2], pk[3 * c], pk[3 * c + 1], pk[3 * c + 2]);
        sq[qs][3 + c][ty][tx] = dot3(Dk[1], Dk[3], Dk[4], pk[3 * c], pk[3 * c + 1], pk[3 * c + 2]);
        qzc[c] = dot3(Dk[2], Dk[4], Dk[5], pk[3 * c], pk[3 * c + 1], pk[3 * c + 2]);
      }
    }
    // every thread is done with planes < k-1 (u, rc/gw) and with the p/D of plane k
    if (__syncthreads_or(bad)) {
      bad = true;
      break;
    }
    if (tid == 0 && k + DIST <= ph && k + DIST > issued) {
      issue(k + DIST);
      issued = k + DIST;
    }
    const int j = k - 1;
    if (interior && j >= z0 && j < z1) {
      const int ps = (qs + 2) % 3;  // slot of plane j
      const unsigned char* R = smem + G::R_OFF + ((j - kb) % G::NR) * G::R_SLOT;
      const SP* RC = reinterpret_cast<const SP*>(R) + ro;
      const SP* GW = reinterpret_cast<const SP*>(R + G::RC_SLOT) + ro;
      const Stencil3 az = adj_coef(j, nz, bdry, ihz);
      const float rcj = Store<SP>::sh(RC);
      float gj[3], div[3], un[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        gj[c] = Store<SP>::sh(GW + c * TY * TX);
        const float dx = apply3<GEN>(ax, sq[ps][c][ty][tx - 1], GEN ? sq[ps][c][ty][tx] : 0.f, sq[ps][c][ty][tx + 1]);
        const float dy = apply3<GEN>(ay, sq[ps][3 + c][ty - 1][tx], GEN ? sq[ps][3 + c][ty][tx] : 0.f, sq[ps][3 + c][ty + 1][tx]);
        div[c] = sum3(dx, dy, apply3<GEN>(az, qzmm[c], qzm[c], qzc[c]));
      }
      primal_voxel(uown_m, div, a.tau, a.factor, rcj, gj, un);
      SU* dst = u_dst + j * plane;
#pragma unroll
      for (int c = 0; c < 3; ++c) Store<SU>::st(dst + c * cs, un[c]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      qzmm[c] = qzm[c];
      qzm[c] = qzc[c];
      uown_m[c] = uown_c[c];
      uown_c[c] = uown_p[c];
    }
  }
  if (bad) {
    if (tid == 0) {
      atomicOr(status, SVS_DEV_TIMEOUT);
      // wait (bounded) for the copies this CTA still has in flight before it exits
      for (int q = max(waited + 1, pl); q <= issued; ++q) {
        const int r = q - pl;
        mbar_wait(bars + r % G::NB, (uint32_t)((r / G::NB) & 1), wait_ns);
      }
    }
    return;
  }
  if (z1 >= nz) {
    const int j = nz - 1;
    if (interior && j >= z0) {
      const int ps = j % 3;
      const unsigned char* R = smem + G::R_OFF + ((j - kb) % G::NR) * G::R_SLOT;
      const SP* RC = reinterpret_cast<const SP*>(R) + ro;
      const SP* GW = reinterpret_cast<const SP*>(R + G::RC_SLOT) + ro;
      const Stencil3 az = adj_coef(j, nz, bdry, ihz);
      const float rcj = Store<SP>::sh(RC);
      float gj[3], div[3], un[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        gj[c] = Store<SP>::sh(GW + c * TY * TX);
        const float dx = apply3<GEN>(ax, sq[ps][c][ty][tx - 1], GEN ? sq[ps][c][ty][tx] : 0.f, sq[ps][c][ty][tx + 1]);
        const float dy = apply3<GEN>(ay, sq[ps][3 + c][ty - 1][tx], GEN ? sq[ps][3 + c][ty][tx] : 0.f, sq[ps][3 + c][ty + 1][tx]);
        div[c] = sum3(dx, dy, apply3<GEN>(az, qzmm[c], qzm[c], 0.f));
      }
      primal_voxel(uown_m, div, a.tau, a.factor, rcj, gj, un);
      SU* dst = u_dst + j * plane;
#pragma unroll
      for (int c = 0; c < 3; ++c) Store<SU>::st(dst + c * cs, un[c]);
    }
  }
}

// ------------------------------------------------------------------- split-role TMA form
// The TMA pipeline and tensor maps of iterate_tma_kernel (same boxes), with a different division
// of work: a lane owns V (1 or 2) x-adjacent voxels (for V = 2 read and written as one 8-byte
// f32 or 4-byte 16-bit access), and the lanes are split by role:
//   role 0  interior         TY rows x TX/V lanes (whole warps): dual, p store, q rows, primal,
//                            u store;
//   role 1  halo rows        rows y0-1 and y0+TY, TX/V lanes each: dual and the y-row of q;
//   role 2  halo columns     x0-1 and x0+TX, TY voxels each, one per lane: dual and the x-row
//                            of q.
// One __syncthreads per plane, at the END of step k: step k computes the dual of plane k and the
// primal of plane k-1 (whose x/y rows of q were published before the barrier of step k-1 and
// whose z-neighbour q(k) is in the lane's registers), so the two are independent within the
// step; u of planes k-1, k, k+1 is read from the ring. After the barrier, plane k+DIST is issued
// into the slots of planes k-1 (u, rc/gw) and k (p/D), which nobody reads any more; q rows need
// two slots (plane k written, plane k-1 read).
// The arithmetic of every voxel is the expression sequence of iterate_tma_kernel, so the two
// kernels give bitwise the same result. q rows live in qx [TY][TX+4] (x from x0-2, so V-voxel
// groups start on even indices) and qy [TY+2][TX] (rows from y0-1).
// Value type of a lane: one voxel (float) or two x-adjacent voxels (float2, packed FP32 math).
template <int V> using LaneT = typename std::conditional<V == 2, float2, float>::type;
// Load / store the lane's V voxels of storage type S (for V = 2: one 8-byte f32 or 4-byte 16-bit
// access; the roundings are those of Store<S> per value).
template <int V, typename S> struct Lane;
template <typename S> struct Lane<1, S> {
  static __device__ __forceinline__ float ld(const S* p) { return Store<S>::sh(p); }
  static __device__ __forceinline__ void st(S* p, float v) { Store<S>::st(p, v); }
};
template <typename S> struct Lane<2, S> {
  static __device__ __forceinline__ float2 ld(const S* p) { return Pair<S>::sh(p); }
  static __device__ __forceinline__ void st(S* p, float2 v) { Pair<S>::st(p, v.x, v.y); }
};
template <> struct Lane<1, float> {
  static __device__ __forceinline__ float ld(const float* p) { return *p; }
  static __device__ __forceinline__ void st(float* p, float v) { *p = v; }
};
template <> struct Lane<2, float> {
  static __device__ __forceinline__ float2 ld(const float* p) { return *reinterpret_cast<const float2*>(p); }
  static __device__ __forceinline__ void st(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
};
// x-neighbours of the lane's voxels: L is the value left of the first voxel, R right of the last
__device__ __forceinline__ float prev_x(float L, float) { return L; }
__device__ __forceinline__ float next_x(float, float R) { return R; }
__device__ __forceinline__ float2 prev_x(float L, float2 o) { return make_float2(L, o.x); }
__device__ __forceinline__ float2 next_x(float2 o, float R) { return make_float2(o.y, R); }
// x-direction stencil of the lane's voxels, as packed operations on the shifted pairs (prev_x,
// next_x) or, with SCALAR, as one scalar stencil per voxel written straight into the result's two
// halves (no shifted pair has to be assembled); bitwise the same per voxel.
template <bool GEN, bool SCALAR>
__device__ __forceinline__ float x_stencil(const StencilV<float>& s, float L, float o, float R) {
  return apply3<GEN>(s, L, o, R);
}
template <bool GEN, bool SCALAR>
__device__ __forceinline__ float2 x_stencil(const StencilV<float2>& s, float L, float2 o, float R) {
  if constexpr (SCALAR) {
    return make_float2(apply3<GEN>(Stencil3{s.m.x, s.c.x, s.p.x}, L, o.x, o.y),
                       apply3<GEN>(Stencil3{s.m.y, s.c.y, s.p.y}, o.x, o.y, R));
  } else {
    return apply3<GEN>(s, prev_x(L, o), o, next_x(o, R));
  }
}

template <typename SU, typename SP, int TX, int TY, int DIST, int V, bool AS = false, int UPAD = 0>
struct SplitGeom {
  using B = TmaGeom<SU, SP, TX, TY, DIST, UPAD>;  // box shapes (shared with the tensor maps)
  static_assert(UPAD % B::AU == 0, "padding keeps the 16-byte row alignment");
  static_assert(V == 1 || V == 2, "one or two voxels per lane");
  static_assert(TX % V == 0, "whole lanes per row");
  static constexpr int PW = TX / V;          // lanes per row
  static constexpr int NI = PW * TY;         // role 0 lanes
  static constexpr int NH = 2 * PW;          // role 1 lanes
  static constexpr int NC = 2 * TY;          // role 2 lanes
  static constexpr int NT = NI + NH + NC;
  static_assert(NI % 32 == 0, "role 0 fills whole warps");
  static constexpr int NU = DIST + 1, NPD = DIST, NR = DIST + 1, NB = DIST + 1;
  static constexpr int U_OFF = 0;
  static constexpr int PD_OFF = U_OFF + NU * B::U_SLOT;
  static constexpr int R_OFF = PD_OFF + NPD * B::PD_SLOT;
  static constexpr int SXW = TX + 4;
  static constexpr int SQX_OFF = R_OFF + NR * B::R_SLOT;
  static constexpr int SQX_BYTES = 2 * 3 * TY * SXW * 4;
  static constexpr int SQY_OFF = SQX_OFF + SQX_BYTES;
  static constexpr int SQY_BYTES = 2 * 3 * (TY + 2) * TX * 4;
  static constexpr int BAR_OFF = round_up_c(SQY_OFF + SQY_BYTES, 8);
  // decoupled form (AS): "q rows of plane k published" (2, one per q slot) and "step k done"
  // (DIST+1) barriers, an abort flag, and one producer warp beyond the NT compute lanes
  static constexpr int NQP = AS ? 2 : 0, NFR = AS ? DIST + 1 : 0;
  static constexpr int ABORT_OFF = BAR_OFF + (NB + NQP + NFR) * 8;
  static constexpr int SMEM = ABORT_OFF + (AS ? 8 : 0);
  static constexpr int NT_LAUNCH = NT + (AS ? 32 : 0);
};

// OPT (schedule options of the interior lanes, the same arithmetic either way):
//   kLatePrimal  load the primal inputs of plane k-1 (q rows, u, rc, gw) and compute the
//                shrinkage step AFTER the dual of plane k instead of before it (fewer values live
//                across the dual, a longer dependent chain per plane);
//   kJitDual     load the dual field of one flow component at a time and finish that component
//                (dual, q, p store) before loading the next (fewer values live at once);
//   kRowPairs    place the interior lanes so that a warp holds 16 voxel pairs of each of two rows
//                D apart (RowPairs) instead of consecutive lanes along the rows: every 8-byte
//                shared access of a half-warp is then one row, and the two rows' 4-byte accesses
//                to 16-bit fields fall in disjoint banks;
//   kScalarX     x-direction stencils of a voxel pair as two scalar stencils (x_stencil);
//   kNoSel       q rows stored without zeroing lanes outside the volume (their q is zero);
//   kPeel        planes whose z stencils are the interior ones run a step with those
//                coefficients fixed and both z-neighbour slots present;
//   OPT >> 8     extra columns of the u box in shared memory (row pitch, TmaGeom::UPAD).
enum { kLatePrimal = 1, kJitDual = 2, kRowPairs = 4, kScalarX = 8, kNoSel = 16, kPeel = 32 };
template <typename SP, int PXB, int PW, int TY, int V>
struct RowPairs {
  static constexpr int ROWB = PXB * (int)sizeof(SP);  // bytes per p/D row in shared memory
  static constexpr int pick16() {
    for (int d = 1; d <= 8; d *= 2)
      if (TY % (2 * d) == 0 && (d * ROWB) % 128 == 64) return d;
    return 0;
  }
  // 8-byte accesses (4-byte fields): any row distance is conflict-free
  static constexpr int D = sizeof(SP) == 4 ? 1 : pick16();
  static constexpr bool ok = V == 2 && PW >= 16 && D > 0 && TY % (2 * (D > 0 ? D : 1)) == 0 &&
                             ((PW - 16) * TY) % 32 == 0;
  static constexpr int NPAIRED = 16 * TY;  // lanes placed in row pairs; the rest row by row
};
// What split_body did with its tile: skipped it (the pair had stopped; shared memory untouched),
// finished it, or gave up at a timed-out pipeline wait (the same in every thread of the CTA).
enum { kItemSkipped = 0, kItemDone = 1, kItemTimeout = 2 };
template <typename SU, typename SP, int TX, int TY, int DIST, int V, bool GEN, bool AS, int OPT = 0>
__device__ __forceinline__ int split_body(const Tile* __restrict__ tiles, const int item,
                                           const Desc* __restrict__ descs, const TMaps* __restrict__ maps,
                                           const IterArgs a, int* __restrict__ status) {
  using G = SplitGeom<SU, SP, TX, TY, DIST, V, AS, (OPT >> 8)>;
  using B = typename G::B;
  using T = LaneT<V>;
  constexpr int AU = B::AU, AP = B::AP, UXB = B::UXB, PXB = B::PXB;
  constexpr int UC = B::UYB * UXB, PC = B::PYB * PXB, RCS = TY * TX, SXW = G::SXW;
  static_assert(DIST >= 2, "step k waits for plane k+1, issued at the end of step k+1-DIST");
  extern __shared__ __align__(128) unsigned char smem[];
  float(*sqx)[3][TY][SXW] = reinterpret_cast<float(*)[3][TY][SXW]>(smem + G::SQX_OFF);
  float(*sqy)[3][TY + 2][TX] = reinterpret_cast<float(*)[3][TY + 2][TX]>(smem + G::SQY_OFF);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + G::BAR_OFF);

  const Tile Tl = tiles[item];
  const Desc& Dg = descs[Tl.desc];
  if (Dg.stop && *Dg.stop) return kItemSkipped;  // pair converged for this level
  const TMaps* M = maps + Tl.desc;
  const int nz = Dg.nz, ny = Dg.ny, nx = Dg.nx;
  const int cs = (int)Dg.cs;
  const int plane = Dg.pitch * ny;
  const int z0 = Tl.z0z1 & 0xffff, z1 = Tl.z0z1 >> 16;
  const CUtensorMap* mu = &M->u[a.src];
  const CUtensorMap* mp = &M->p[a.src];

  const int tid = threadIdx.x;
  int role, lx, ly;  // position relative to (x0, y0)
  if (tid < G::NI) {
    role = 0;
    if constexpr ((OPT & kRowPairs) && RowPairs<SP, PXB, G::PW, TY, V>::ok) {
      using RP = RowPairs<SP, PXB, G::PW, TY, V>;
      if (tid < RP::NPAIRED) {
        const int w = tid >> 5, l = tid & 31, b = w / RP::D;  // warp w: rows r and r + D
        const int r = b * 2 * RP::D + (w % RP::D) + ((l >> 4) ? RP::D : 0);
        lx = V * (l & 15);
        ly = r;
      } else {  // pairs 16.. of every row, row by row
        const int i = tid - RP::NPAIRED;
        lx = V * (16 + i % (G::PW - 16));
        ly = i / (G::PW - 16);
      }
    } else {
      lx = V * (tid % G::PW);
      ly = tid / G::PW;
    }
  } else if (tid < G::NI + G::NH) {
    const int h = tid - G::NI;
    role = 1;
    lx = V * (h % G::PW);
    ly = (h < G::PW) ? -1 : TY;
  } else {
    const int h = tid - G::NI - G::NH;
    role = 2;
    lx = (h < TY) ? -1 : TX;
    ly = h % TY;
  }
  const int gx = Tl.x0 + lx, gy = Tl.y0 + ly;
  const bool active = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
  const bool full = gx + V - 1 < nx;          // roles 0/1: every voxel of the lane is inside
  const int uo = (ly + 2) * UXB + (lx + AU);  // own (first) voxel in a u box component
  const int po = (ly + 1) * PXB + (lx + AP);  // own (first) voxel in a p/D box component
  const int ro = ly * TX + lx;                // own voxels in an rc/gw box (role 0)
  const long long col0 = (long long)gy * Dg.pitch + gx;
  SU* __restrict__ u_dst = reinterpret_cast<SU*>(Dg.u[a.src ^ 1]) + col0;
  SP* __restrict__ p_dst = reinterpret_cast<SP*>(Dg.p[a.src ^ 1]) + col0;
  const int bdry = GEN ? a.bdry : (int)SVS_BOUNDARY_MIRROR;  // GEN = false is launched for MIRROR only
  const Stencil3 fx0 = fwd_coef(gx, nx, bdry, Dg.hx), ax0 = adj_coef(gx, nx, bdry, 1.0f / Dg.hx);
  StencilV<T> fx, ax;
  if constexpr (V == 2) {
    fx = pack(fx0, fwd_coef(gx + 1, nx, bdry, Dg.hx));
    ax = pack(ax0, adj_coef(gx + 1, nx, bdry, 1.0f / Dg.hx));
  } else {
    fx = fx0;
    ax = ax0;
  }
  const Stencil3 fy1 = fwd_coef(gy, ny, bdry, Dg.hy);
  const StencilV<T> fy = bcast_st<T>(fy1), ay = bcast_st<T>(adj_coef(gy, ny, bdry, 1.0f / Dg.hy));
  const float ihz = 1.0f / Dg.hz, hz = Dg.hz;

  const int kb = max(z0 - 1, 0), ke = min(z1, nz - 1);
  const int pl = max(kb - 1, 0), ph = min(ke + 1, nz - 1);
  const uint64_t wait_ns = (uint64_t)a.wait_us * 1000ull;
  const int stall_r = item == a.stall_cta ? a.stall_plane : -1;
  auto issue = [&](int q) {
    const int r = q - pl;
    if (r == stall_r) return;  // timeout-path test: this plane's copies are never issued
    uint64_t* bar = bars + r % G::NB;
    unsigned char* U = smem + G::U_OFF + (r % G::NU) * B::U_SLOT;
    if (q < kb) {
      mbar_arrive_expect_tx(bar, (uint32_t)B::U_TX);
      tma_load_4d(U, mu, bar, Tl.x0 - AU, Tl.y0 - 2, q, 0);
      return;
    }
    unsigned char* PD = smem + G::PD_OFF + ((q - kb) % G::NPD) * B::PD_SLOT;
    unsigned char* R = smem + G::R_OFF + ((q - kb) % G::NR) * B::R_SLOT;
    mbar_arrive_expect_tx(bar, (uint32_t)B::FULL_TX);
    tma_load_4d(U, mu, bar, Tl.x0 - AU, Tl.y0 - 2, q, 0);
    tma_load_4d(PD, mp, bar, Tl.x0 - AP, Tl.y0 - 1, q, 0);
    tma_load_4d(PD + B::P_SLOT, &M->D, bar, Tl.x0 - AP, Tl.y0 - 1, q, 0);
    tma_load_4d(R, &M->rc, bar, Tl.x0, Tl.y0, q, 0);
    tma_load_4d(R + B::RC_SLOT, &M->gw, bar, Tl.x0, Tl.y0, q, 0);
  };
  auto ubox = [&](int q) {
    return reinterpret_cast<const SU*>(smem + G::U_OFF + ((q - pl) % G::NU) * B::U_SLOT);
  };
  auto rbox = [&](int q) { return smem + G::R_OFF + ((q - kb) % G::NR) * B::R_SLOT; };

  // q cells that no lane writes (outside the volume, the unused qx column x0+TX+1) are read
  // with zero stencil coefficients: they must hold zeros (0 * NaN = NaN)
  for (int i = tid; i < (G::SQX_BYTES + G::SQY_BYTES) / 4; i += blockDim.x)
    reinterpret_cast<float*>(smem + G::SQX_OFF)[i] = 0.f;
  uint64_t* qpub = bars + G::NB;             // AS: q rows of plane k published, slot (k-kb) & 1
  uint64_t* freed = qpub + G::NQP;           // AS: step k done by every lane, slot (k-kb) % NFR
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + G::ABORT_OFF);
  if (tid == 0) {
    for (int s = 0; s < G::NB; ++s) mbar_init(bars + s, 1);
    if constexpr (AS) {
      for (int s = 0; s < G::NQP; ++s) mbar_init(qpub + s, G::NT);
      for (int s = 0; s < G::NFR; ++s) mbar_init(freed + s, G::NT);
      *abort_flag = 0;
    }
    mbar_fence_init();
  }
  __syncthreads();
  int issued = pl - 1;
  if constexpr (AS) {
    // producer warp: issues every plane once the step that frees its slots is done
    if (tid >= G::NT) {
      if (tid == G::NT) {
        const int last = min(kb + DIST - 1, ph);
        for (int q = pl; q <= last; ++q) issue(q);
        issued = last;
        for (int q = kb + DIST; q <= ph; ++q) {
          const int st = q - DIST - kb;
          if (!mbar_wait_abort(freed + st % G::NFR, (uint32_t)((st / G::NFR) & 1), abort_flag, wait_ns)) break;
          issue(q);
          issued = q;
        }
        if (*abort_flag) {
          atomicOr(status, SVS_DEV_TIMEOUT);
          // wait (bounded) for the copies still in flight before the CTA may exit
          for (int q = max(issued - G::NB + 1, pl); q <= issued; ++q) {
            const int r = q - pl;
            mbar_wait(bars + r % G::NB, (uint32_t)((r / G::NB) & 1), wait_ns);
          }
        }
      }
      return kItemDone;
    }
  } else {
    if (tid == 0) {
      const int last = min(kb + DIST - 1, ph);
      for (int q = pl; q <= last; ++q) issue(q);
      issued = last;
    }
  }
  int waited = pl - 1;
  bool bad = false;

  // q_z of the own voxels (role 0) at planes k-2, k-1, k
  T qmm[3], qm[3], qc[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) qmm[c] = qm[c] = qc[c] = bcast<T>(0.f);
  const float wtv2 = a.wtv * a.wtv;

  // x/y part of the divergence at plane j (q rows of slot j & 1)
  auto load_dxy = [&](int j, T (&dxy)[3]) {
    const int ps = j & 1;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float* qx = &sqx[ps][c][ly][lx + 2];
      const T o = Lane<V, float>::ld(qx);
      const T dx = x_stencil<GEN, (OPT & kScalarX) != 0>(ax, qx[-1], o, qx[V]);
      const T dn = Lane<V, float>::ld(&sqy[ps][c][ly][lx]);
      const T up = Lane<V, float>::ld(&sqy[ps][c][ly + 2][lx]);
      const T oy = GEN ? Lane<V, float>::ld(&sqy[ps][c][ly + 1][lx]) : bcast<T>(0.f);
      dxy[c] = vadd(dx, apply3<GEN>(ay, dn, oy, up));
    }
  };
  // primal of plane j, the part that needs no new dual (run before the dual of plane j+1):
  // own u, the data-term gradient g and the shrinkage step t
  auto primal_pre = [&](int j, T (&uj)[3], T (&g)[3], T& t) {
    const unsigned char* R = rbox(j);
    const SP* RC = reinterpret_cast<const SP*>(R) + ro;
    const SP* GW = reinterpret_cast<const SP*>(R + B::RC_SLOT) + ro;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      uj[c] = Lane<V, SU>::ld(ubox(j) + uo + c * UC);
      g[c] = Lane<V, SP>::ld(GW + c * RCS);
    }
    t = primal_step(uj, a.factor, Lane<V, SP>::ld(RC), g);
  };
  // rest of the primal of plane j: qn = q_z(j+1)
  auto finish_primal = [&](int j, const Stencil3& azs, const T (&dxy)[3], const T (&qn)[3], const T (&uj)[3],
                           const T (&g)[3], T t) {
    const StencilV<T> az = bcast_st<T>(azs);  // adj_coef(j, ...)
    T d[3], n[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) d[c] = vadd(dxy[c], apply3<GEN>(az, qmm[c], qm[c], qn[c]));
    primal_apply(uj, d, a.tau, t, g, n);
    SU* dst = u_dst + (long long)j * plane;
    if (full) {
#pragma unroll
      for (int c = 0; c < 3; ++c) Lane<V, SU>::st(dst + c * cs, n[c]);
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) Store<SU>::st(dst + c * cs, first(n[c]));
    }
  };
  // AS: waits on "q rows of plane j published" and "step j done by every lane"
  auto wait_q = [&](int j) {
    const int r = j - kb;
    return mbar_wait_abort(qpub + (r & 1), (uint32_t)((r >> 1) & 1), abort_flag, wait_ns);
  };
  auto wait_free = [&](int j) {
    if constexpr (AS) {
      const int r = j - kb;
      return mbar_wait_abort(freed + r % G::NFR, (uint32_t)((r / G::NFR) & 1), abort_flag, wait_ns);
    } else {
      return true;  // only the decoupled form waits here
    }
  };

  // One plane step; WITH_PRIMAL: role 0 also finishes plane k-1.
  // kPeel: the z stencils of interior planes (the same values fwd_coef / adj_coef give there)
  const Stencil3 fz_int = fwd_coef(1, 3, bdry, hz), az_int = adj_coef(2, 5, bdry, ihz);
  auto step = [&](const int k, auto with_primal, auto interior) {
    constexpr bool WP = decltype(with_primal)::value;
    constexpr bool INT = decltype(interior)::value;  // both z stencils interior, k-1 and k+1 staged
    const int need = min(k + 1, ph);
    while (waited < need && !bad) {
      ++waited;
      const int r = waited - pl;
      const bool ok = AS ? mbar_wait_abort(bars + r % G::NB, (uint32_t)((r / G::NB) & 1), abort_flag, wait_ns)
                         : mbar_wait(bars + r % G::NB, (uint32_t)((r / G::NB) & 1), wait_ns);
      if (!ok) bad = true;
    }
    if (AS && bad) return;
    const int qs = k & 1;
    const SU* Uk = ubox(k) + uo;
    const unsigned char* PD = smem + G::PD_OFF + ((k - kb) % G::NPD) * B::PD_SLOT;
    const Stencil3 fz1 = INT ? fz_int : fwd_coef(k, nz, bdry, hz);
    // planes k-1 and k+1 are missing only at k = 0 and k = nz-1, where the z stencil's
    // coefficient for them is zero (every boundary type): plane k stands in for them
    const SU* Um = ubox(INT || k - 1 >= pl ? k - 1 : k) + uo;
    const SU* Up = ubox(INT || k + 1 <= ph ? k + 1 : k) + uo;
    if (role == 0) {
      // interior lanes, one block with few branches so that the compiler can interleave the
      // primal of plane k-1 with the dual of plane k; lanes outside the volume compute on the
      // zero fill of the boxes (finite values) and store nothing to global memory
      T dxy[3], uo1[3], gp[3], tp;
      constexpr bool kEarly = !(OPT & kLatePrimal);
      if constexpr (WP && kEarly) {
        if (AS && !wait_q(k - 1)) {
          bad = true;
          return;
        }
        load_dxy(k - 1, dxy);
        primal_pre(k - 1, uo1, gp, tp);
      }
      const StencilV<T> fz = bcast_st<T>(fz1);
      const SP* P = reinterpret_cast<const SP*>(PD) + po;
      const SP* Dm = reinterpret_cast<const SP*>(PD + B::P_SLOT) + po;
      T Dk[6], qxo[3], qyo[3];
#pragma unroll
      for (int c = 0; c < 6; ++c) Dk[c] = Lane<V, SP>::ld(Dm + c * PC);
      const bool p_out = active && !bad && k >= z0 && k < z1;
      SP* pdst = p_dst + (long long)k * plane;
      // the dual of flow component c: p_new, its q = D p_new, and the p store
      auto dual_comp = [&](int c, T& p0, T& p1, T& p2) {
        const SU* u = Uk + c * UC;
        const T o = Lane<V, SU>::ld(u);
        const T ex = x_stencil<GEN, (OPT & kScalarX) != 0>(fx, Store<SU>::sh(u - 1), o, Store<SU>::sh(u + V));
        const T ey = apply3<GEN>(fy, Lane<V, SU>::ld(u - UXB), o, Lane<V, SU>::ld(u + UXB));
        const T ez = apply3<GEN>(fz, Lane<V, SU>::ld(Um + c * UC), o, Lane<V, SU>::ld(Up + c * UC));
        dual_row(Dk, ex, ey, ez, p0, p1, p2, a.sigma, a.wtv, wtv2);
      };
      auto q_comp = [&](int c, const T& p0, const T& p1, const T& p2) {
        qyo[c] = dot3(Dk[1], Dk[3], Dk[4], p0, p1, p2);
        qxo[c] = dot3(Dk[0], Dk[1], Dk[2], p0, p1, p2);
        qc[c] = dot3(Dk[2], Dk[4], Dk[5], p0, p1, p2);
      };
      auto store_p = [&](int c, const T& p) {
        if (full) Lane<V, SP>::st(pdst + c * cs, p);
        else Store<SP>::st(pdst + c * cs, first(p));
      };
      if constexpr (OPT & kJitDual) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          T p0 = Lane<V, SP>::ld(P + (3 * c) * PC), p1 = Lane<V, SP>::ld(P + (3 * c + 1) * PC),
            p2 = Lane<V, SP>::ld(P + (3 * c + 2) * PC);
          dual_comp(c, p0, p1, p2);
          q_comp(c, p0, p1, p2);
          if (p_out) {
            store_p(3 * c, p0);
            store_p(3 * c + 1, p1);
            store_p(3 * c + 2, p2);
          }
        }
      } else {
        T pk[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) pk[c] = Lane<V, SP>::ld(P + c * PC);
#pragma unroll
        for (int c = 0; c < 3; ++c) dual_comp(c, pk[3 * c], pk[3 * c + 1], pk[3 * c + 2]);
#pragma unroll
        for (int c = 0; c < 3; ++c) q_comp(c, pk[3 * c], pk[3 * c + 1], pk[3 * c + 2]);
        if (p_out) {
#pragma unroll
          for (int c = 0; c < 9; ++c) store_p(c, pk[c]);
        }
      }
      // AS: the q slot of plane k was last read by the primal of plane k-2 (step k-1)
      if (AS && k > kb && !wait_free(k - 1)) {
        bad = true;
        return;
      }
      // cells outside the volume keep their zeros (kNoSel: a lane outside the volume computed on
      // the zero fill of the boxes, D = 0, so its q is already exactly zero)
      const T zero = bcast<T>(0.f);
      const bool keep = (OPT & kNoSel) ? true : active;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Lane<V, float>::st(&sqy[qs][c][ly + 1][lx], keep ? qyo[c] : zero);
        Lane<V, float>::st(&sqx[qs][c][ly][lx + 2], keep ? qxo[c] : zero);
      }
      if constexpr (AS) mbar_arrive(qpub + ((k - kb) & 1));
      if constexpr (WP) {
        if constexpr (!kEarly) {
          if (AS && !wait_q(k - 1)) {
            bad = true;
            return;
          }
          load_dxy(k - 1, dxy);
          primal_pre(k - 1, uo1, gp, tp);
        }
        if (active && !bad) finish_primal(k - 1, INT ? az_int : adj_coef(k - 1, nz, bdry, ihz), dxy, qc, uo1, gp, tp);
      }
    } else {
      T qyo[3];
      float qxs[3];
      if (role == 1) {
        if (active && !bad) {
          const StencilV<T> fz = bcast_st<T>(fz1);
          const SP* P = reinterpret_cast<const SP*>(PD) + po;
          const SP* Dm = reinterpret_cast<const SP*>(PD + B::P_SLOT) + po;
          T pk[9], Dk[6];
#pragma unroll
          for (int c = 0; c < 9; ++c) pk[c] = Lane<V, SP>::ld(P + c * PC);
#pragma unroll
          for (int c = 0; c < 6; ++c) Dk[c] = Lane<V, SP>::ld(Dm + c * PC);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const SU* u = Uk + c * UC;
            const T o = Lane<V, SU>::ld(u);
            const T ex = apply3<GEN>(fx, prev_x(Store<SU>::sh(u - 1), o), o, next_x(o, Store<SU>::sh(u + V)));
            const T ey = apply3<GEN>(fy, Lane<V, SU>::ld(u - UXB), o, Lane<V, SU>::ld(u + UXB));
            const T ez = apply3<GEN>(fz, Lane<V, SU>::ld(Um + c * UC), o, Lane<V, SU>::ld(Up + c * UC));
            dual_row(Dk, ex, ey, ez, pk[3 * c], pk[3 * c + 1], pk[3 * c + 2], a.sigma, a.wtv, wtv2);
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) qyo[c] = dot3(Dk[1], Dk[3], Dk[4], pk[3 * c], pk[3 * c + 1], pk[3 * c + 2]);
        }
      } else if (active && !bad) {
        // halo column: one voxel, scalar arithmetic
        const SP* P = reinterpret_cast<const SP*>(PD) + po;
        const SP* Dm = reinterpret_cast<const SP*>(PD + B::P_SLOT) + po;
        float pk[9], Dk[6];
#pragma unroll
        for (int c = 0; c < 9; ++c) pk[c] = Store<SP>::sh(P + c * PC);
#pragma unroll
        for (int c = 0; c < 6; ++c) Dk[c] = Store<SP>::sh(Dm + c * PC);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const SU* u = Uk + c * UC;
          const float o = Store<SU>::sh(u);
          const float ex = apply3<GEN>(fx0, Store<SU>::sh(u - 1), o, Store<SU>::sh(u + 1));
          const float ey = apply3<GEN>(fy1, Store<SU>::sh(u - UXB), o, Store<SU>::sh(u + UXB));
          const float ez = apply3<GEN>(fz1, Store<SU>::sh(Um + c * UC), o, Store<SU>::sh(Up + c * UC));
          dual_row(Dk, ex, ey, ez, pk[3 * c], pk[3 * c + 1], pk[3 * c + 2], a.sigma, a.wtv, wtv2);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) qxs[c] = dot3(Dk[0], Dk[1], Dk[2], pk[3 * c], pk[3 * c + 1], pk[3 * c + 2]);
      }
      // AS: the q slot of plane k was last read by the primal of plane k-2 (step k-1)
      if (AS && k > kb && !wait_free(k - 1)) {
        bad = true;
        return;
      }
      if (active && !bad) {
        if (role == 2) {
#pragma unroll
          for (int c = 0; c < 3; ++c) sqx[qs][c][ly][lx + 2] = qxs[c];
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c) Lane<V, float>::st(&sqy[qs][c][ly + 1][lx], qyo[c]);
        }
      }
      if constexpr (AS) mbar_arrive(qpub + ((k - kb) & 1));
    }
    if constexpr (AS) {
      mbar_arrive(freed + (k - kb) % G::NFR);
    } else {
      // everyone is done with plane k's p/D, plane k-1's u and rc/gw, and q rows of plane k-1
      if (__syncthreads_or(bad)) {
        bad = true;
        return;
      }
      if (tid == 0 && k + DIST <= ph && k + DIST > issued) {
        issue(k + DIST);
        issued = k + DIST;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      qmm[c] = qm[c];
      qm[c] = qc[c];
    }
  };

  // the first one or two steps have no finished plane (j = k-1 < z0)
  const int kp = min(z0 + 1, ke + 1);
  int k = kb;
  for (; k < kp && !bad; ++k) step(k, std::false_type{}, std::false_type{});
  if constexpr ((OPT & kPeel) != 0) {
    // interior steps: 1 <= k <= nz-2 (forward stencil) and j = k-1 interior for the adjoint
    // (MIRROR: 2 <= j <= nz-3; the other boundaries: 1 <= j <= nz-2)
    const int ilo = max(kp, GEN ? 2 : 3), ihi = min(ke, nz - 2);
    for (; k < ilo && k <= ke && !bad; ++k) step(k, std::true_type{}, std::false_type{});
    for (; k <= ihi && !bad; ++k) step(k, std::true_type{}, std::true_type{});
  }
  for (; k <= ke && !bad; ++k) step(k, std::true_type{}, std::false_type{});
  if (bad) {
    if constexpr (AS) {
      *abort_flag = 1;
      atomicOr(status, SVS_DEV_TIMEOUT);
    } else if (tid == 0) {
      atomicOr(status, SVS_DEV_TIMEOUT);
      // wait (bounded) for the copies this CTA still has in flight before it exits
      for (int q = max(waited + 1, pl); q <= issued; ++q) {
        const int r = q - pl;
        mbar_wait(bars + r % G::NB, (uint32_t)((r / G::NB) & 1), wait_ns);
      }
    }
    return kItemTimeout;
  }
  if (z1 >= nz) {
    const int j = nz - 1;
    if (AS && role == 0 && !wait_q(j)) {
      atomicOr(status, SVS_DEV_TIMEOUT);
      return kItemTimeout;
    }
    if (role == 0 && active && j >= z0) {
      T dxy[3], uj[3], g[3], t;
      const T zero[3] = {bcast<T>(0.f), bcast<T>(0.f), bcast<T>(0.f)};
      load_dxy(j, dxy);
      primal_pre(j, uj, g, t);
      finish_primal(j, adj_coef(j, nz, bdry, ihz), dxy, zero, uj, g, t);
    }
  }
  return kItemDone;
}

// The split-role kernel with a register budget for MINB resident CTAs per SM (launch bounds)...
template <typename SU, typename SP, int TX, int TY, int DIST, int V, int MINB, bool GEN, bool AS = false, int OPT = 0>
__global__ void __launch_bounds__(SplitGeom<SU, SP, TX, TY, DIST, V, AS>::NT_LAUNCH, MINB)
iterate_split_kernel(const Tile* __restrict__ tiles, const Desc* __restrict__ descs,
                     const TMaps* __restrict__ maps, IterArgs a, int* __restrict__ status) {
  split_body<SU, SP, TX, TY, DIST, V, GEN, AS, OPT>(tiles, blockIdx.x, descs, maps, a, status);
}
// ...or with an explicit per-thread register cap: the launch-bounds arithmetic rounds a block of
// 5.5 warps up further than the register file requires, so three 176-thread CTAs per SM (6
// warps x 112 registers x 32 lanes each, 64,512 of the 65,536 registers) need the cap spelled out.
template <typename SU, typename SP, int TX, int TY, int DIST, int V, int REGS, bool GEN, bool AS = false, int OPT = 0>
__global__ void __launch_bounds__(SplitGeom<SU, SP, TX, TY, DIST, V, AS>::NT_LAUNCH) __maxnreg__(REGS)
iterate_split_kernel_r(const Tile* __restrict__ tiles, const Desc* __restrict__ descs,
                       const TMaps* __restrict__ maps, IterArgs a, int* __restrict__ status) {
  split_body<SU, SP, TX, TY, DIST, V, GEN, AS, OPT>(tiles, blockIdx.x, descs, maps, a, status);
}

// ------------------------------------------------------------- persistent iteration loop
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// Generic-proxy stores of this thread are ordered before later async-proxy (TMA) accesses.
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// Barrier over every CTA of a co-resident (cooperative) grid. The arrival counter starts at zero
// and grows by gridDim.x per use, so use number g waits for g * gridDim.x arrivals. Bounded:
// thread 0 gives up after limit_ns and the call returns false in every thread of the CTA.
__device__ __forceinline__ bool grid_barrier(unsigned* counter, unsigned target, uint64_t limit_ns) {
  int ok = 1;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(counter, 1u);
    const uint64_t t0 = global_ns();
    while (ld_acquire_gpu(counter) < target) {
      if (global_ns() - t0 > limit_ns) {
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    fence_proxy_async_global();  // this thread issues the next copies, after the acquire
  }
  return __syncthreads_and(ok) != 0;
}

// All iterations of one warp at one level in one launch: the resident CTAs (a cooperative grid)
// take the level's column tiles in turn (tile blockIdx.x, blockIdx.x + gridDim.x, ...), run each
// exactly as iterate_split_kernel does, and meet at a grid barrier after every iteration, the
// tiles of iteration it+1 reading the ping-pong copies iteration it wrote. The schedule of sigma
// and tau per iteration is the host's (tvl13d.py:240-249); the arithmetic per voxel is that of
// the per-iteration launches, so the result is bitwise the same.
template <typename SU, typename SP, int TX, int TY, int DIST, int V, int MINB, bool GEN, int OPT = 0>
__global__ void __launch_bounds__(SplitGeom<SU, SP, TX, TY, DIST, V, false>::NT_LAUNCH, MINB)
iterate_persist_kernel(const Tile* __restrict__ tiles, int ntiles, const Desc* __restrict__ descs,
                       const TMaps* __restrict__ maps, PersistArgs pa, int* __restrict__ status) {
  using G = SplitGeom<SU, SP, TX, TY, DIST, V, false, (OPT >> 8)>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + G::BAR_OFF);
  const uint64_t limit = (uint64_t)pa.wait_us * 1000ull;
  for (int it = 0; it < pa.iters; ++it) {
    IterArgs a;
    a.sigma = pa.sig[it];
    a.tau = pa.tau[it];
    a.factor = __fmul_rn(a.tau, pa.wm);  // opticalFlowOps.cu:440, as the host computes it
    a.wtv = pa.wtv;
    a.src = (pa.src0 + it) & 1;
    a.bdry = pa.bdry;
    a.wait_us = pa.wait_us;
    a.stall_cta = pa.stall_cta;
    a.stall_plane = pa.stall_plane;
    for (int item = blockIdx.x; item < ntiles; item += gridDim.x) {
      const int r = split_body<SU, SP, TX, TY, DIST, V, GEN, false, OPT>(tiles, item, descs, maps, a, status);
      // the item's shared memory (rings, q rows, mbarriers) is free again; after a timed-out
      // pipeline wait this CTA stops, and the others then time out at the grid barrier
      __syncthreads();
      if (r == kItemTimeout) return;
      if (r == kItemDone && threadIdx.x == 0)
        for (int b = 0; b < G::NB; ++b) mbar_inval(bars + b);
    }
    // this iteration's stores (generic proxy) come before any CTA's copies of the next one
    fence_proxy_async_global();
    if (!grid_barrier(pa.counter, (unsigned)(it + 1) * gridDim.x, limit)) {
      if (threadIdx.x == 0) atomicOr(status, SVS_DEV_TIMEOUT);
      return;
    }
  }
}

// Compiled shapes of the split-role form (tile, prefetch distance, voxels per lane, CTAs per SM
// the register budget is sized for, or an explicit register cap, schedule options); instantiated
// in svs_split.cu for the storage modes in `smask` (bit s = SVS_STORAGE s).
struct SplitShape {
  int tx, ty, dist, v, minb;
  bool as;    // decoupled synchronisation (mbarriers and a producer warp instead of __syncthreads)
  int regs;   // > 0: registers per thread (iterate_split_kernel_r), instead of minb
  int opt;    // kLatePrimal | kJitDual
  int smask;  // storage modes compiled
};
constexpr int kAllStorages = 31, kF32AndF16Flow32 = (1 << SVS_STORAGE_F32) | (1 << SVS_STORAGE_F16_FLOW32);
constexpr SplitShape kSplitShapes[] = {
    {32, 8, 3, 2, 2, false, 0, 0, kAllStorages},  {32, 8, 4, 2, 2, false, 0, 0, kAllStorages},
    {16, 16, 3, 2, 2, false, 0, 0, kAllStorages}, {40, 8, 3, 2, 2, false, 0, 0, kAllStorages},
    {32, 16, 3, 2, 1, false, 0, 0, kAllStorages}, {40, 16, 3, 2, 1, false, 0, 0, kAllStorages},
    {32, 8, 3, 1, 2, false, 0, 0, kAllStorages},  {32, 8, 4, 1, 2, false, 0, 0, kAllStorages},
    {16, 16, 3, 1, 2, false, 0, 0, kAllStorages}, {32, 16, 2, 1, 1, false, 0, 0, kAllStorages},
    {32, 16, 3, 1, 1, false, 0, 0, kAllStorages}, {40, 8, 3, 1, 2, false, 0, 0, kAllStorages},
    {40, 8, 3, 2, 2, true, 0, 0, kAllStorages},   {32, 8, 3, 2, 2, true, 0, 0, kAllStorages},
    {16, 16, 3, 1, 2, true, 0, 0, kAllStorages},  {32, 16, 3, 2, 1, true, 0, 0, kAllStorages},
    // placement and schedule options of the 40x8 pair-lane shape (and of the FP32 32x16 and the
    // 16x16 shapes), FP32 and f16-flow32 storage
    {40, 8, 3, 2, 2, false, 0, kRowPairs, kF32AndF16Flow32},
    {40, 8, 3, 2, 2, false, 0, kRowPairs | (8 << 8), kF32AndF16Flow32},
    {40, 8, 3, 2, 2, false, 0, kRowPairs | kScalarX, kF32AndF16Flow32},
    {40, 8, 3, 2, 2, false, 0, kRowPairs | kNoSel, kAllStorages},  // the 16-bit default at widths of 40
    {40, 8, 3, 2, 2, false, 0, kRowPairs | kPeel, kF32AndF16Flow32},
    {40, 8, 3, 2, 2, false, 0, kRowPairs | kScalarX | kNoSel | kPeel, kF32AndF16Flow32},
    {40, 8, 3, 2, 2, false, 0, kRowPairs | kScalarX | kNoSel | kPeel | kJitDual | kLatePrimal, kF32AndF16Flow32},
    {32, 16, 3, 2, 1, false, 0, kScalarX | kNoSel | kPeel, kF32AndF16Flow32},
    {16, 16, 3, 2, 2, false, 0, kScalarX | kNoSel | kPeel, kF32AndF16Flow32}};
constexpr int kNumSplitShapes = sizeof(kSplitShapes) / sizeof(kSplitShapes[0]);

// Split-role variant `idx` for a storage mode. op 0: set the kernels' shared-memory attribute
// and return the TMA box shapes {u x, u y, p x, p y} in `box` (false if the variant does not
// fit); op 1: launch one iteration over `ntiles` tiles on stream s; op 2: resident CTAs per SM
// in box[0] (after op 0).
bool split_variant(int storage, int idx, int op, bool gen, unsigned ntiles, const Tile* tiles, const Desc* descs,
                   const TMaps* maps, const IterArgs* a, int* status, cudaStream_t s, int* box);

template <typename SU, typename SP> constexpr int storage_id() {
  if constexpr (std::is_same<SU, float>::value && std::is_same<SP, float>::value) return SVS_STORAGE_F32;
  else if constexpr (std::is_same<SU, float>::value && std::is_same<SP, __half>::value) return SVS_STORAGE_F16_FLOW32;
  else if constexpr (std::is_same<SU, float>::value) return SVS_STORAGE_BF16_FLOW32;
  else if constexpr (std::is_same<SP, __half>::value) return SVS_STORAGE_F16;
  else return SVS_STORAGE_BF16;
}

// The shapes that also have the persistent form (iterate_persist_kernel): those the automatic
// per-level choice uses (32x16 pairs, 40x8 pairs in row pairs, 32x8 and 16x16 single voxels) and
// the 32x8 pair shape, at prefetch distance 3, block barrier per plane, every storage mode.
constexpr bool has_persist(const SplitShape& S) {
  if (S.as || S.regs != 0 || S.dist != 3 || S.smask != kAllStorages) return false;
  if (S.opt == (kRowPairs | kNoSel)) return S.tx == 40 && S.ty == 8 && S.v == 2;
  if (S.opt != 0) return false;
  return (S.tx == 32 && S.ty == 16 && S.v == 2) || (S.tx == 32 && S.ty == 8 && S.v == 2 && S.minb == 2) ||
         (S.tx == 32 && S.ty == 8 && S.v == 1) || (S.tx == 16 && S.ty == 16 && S.v == 1);
}

// Persistent launch of split-role variant `idx`: all `pa->iters` iterations of one warp at one
// level over `ntiles` tiles, one cooperative grid of the resident CTAs. op 0: set the kernels'
// shared-memory attribute; op 1: launch on stream s. False if the variant has no persistent form
// (has_persist) or the launch failed.
bool split_persist(int storage, int idx, int op, bool gen, unsigned ntiles, const Tile* tiles, const Desc* descs,
                   const TMaps* maps, const PersistArgs* pa, int* status, cudaStream_t s);

}  // namespace svs
