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

struct Stencil3 {
  float m, c, p;
};

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
template <bool GEN>
__device__ __forceinline__ float apply3(const Stencil3& s, float prev, float cur, float next) {
  if (GEN) return fmaf(s.p, next, fmaf(s.c, cur, s.m * prev));
  return fmaf(s.p, next, s.m * prev);
}

// Dual update of one flow component at one voxel, tvl13d.py:215-222 with
// opticalFlowOps.cu:179-208: v = p + sigma D g; p_new = v / max(1, |v| / weight_tv), written as
// v * min(1, weight_tv * rsqrt(|v|^2)).
__device__ __forceinline__ void dual_row(const float D[6], float ex, float ey, float ez, float& p0,
                                         float& p1, float& p2, float sigma, float wtv, float wtv2) {
  const float d0 = D[0] * ex + D[1] * ey + D[2] * ez;
  const float d1 = D[1] * ex + D[3] * ey + D[4] * ez;
  const float d2 = D[2] * ex + D[4] * ey + D[5] * ez;
  const float v0 = p0 + sigma * d0, v1 = p1 + sigma * d1, v2 = p2 + sigma * d2;
  const float nsq = v0 * v0 + v1 * v1 + v2 * v2;
  // weight_tv == 0 gives sc = 0 (or v = 0), i.e. p = 0 as tvl13d.py:223-224 requires
  const float sc = (nsq > wtv2) ? wtv * rsqrtf(nsq) : 1.0f;
  p0 = v0 * sc;
  p1 = v1 * sc;
  p2 = v2 * sc;
}

// Primal update at one voxel, tvl13d.py:229-235 with opticalFlowOps.cu:123-175:
// rho = rc + u.g (u before the update), u_new = (u - tau div) + shrinkage step.
__device__ __forceinline__ void primal_voxel(const float u[3], const float div[3], float tau,
                                             float factor, float rc, const float g[3], float un[3]) {
  const float rho = rc + (u[0] * g[0] + u[1] * g[1] + u[2] * g[2]);
  const float g2s = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
#pragma unroll
  for (int c = 0; c < 3; ++c) un[c] = u[c] - tau * div[c];
  // the three cases of opticalFlowOps.cu:140-171 as one step length along g (no divergence):
  // rho < -th: +factor; rho > th: -factor; |rho| <= th: -rho/|g|^2 (0 where |g|^2 <= 1e-10,
  // the reference's (double)g2 > 1e-10 for a float g2)
  const float th = factor * g2s;
  const float t = (rho < -th) ? factor : (rho > th) ? -factor : (g2s >= 1e-10f ? __fdividef(-rho, g2s) : 0.f);
#pragma unroll
  for (int c = 0; c < 3; ++c) un[c] = fmaf(t, g[c], un[c]);
}

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
        sq[slot][c][ty][tx] = Dk[0] * pk[3 * c] + Dk[1] * pk[3 * c + 1] + Dk[2] * pk[3 * c + 2];
        sq[slot][3 + c][ty][tx] = Dk[1] * pk[3 * c] + Dk[3] * pk[3 * c + 1] + Dk[4] * pk[3 * c + 2];
        qzc[c] = Dk[2] * pk[3 * c] + Dk[4] * pk[3 * c + 1] + Dk[5] * pk[3 * c + 2];
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
        div[c] = (dx + dy) + apply3<GEN>(az, qzmm[c], qzm[c], qzc[c]);
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
        div[c] = (dx + dy) + apply3<GEN>(az, qzmm[c], qzm[c], 0.f);
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
// Bounded wait: gives up after kMbarWaitNs of wall time (a tile's loads complete in microseconds).
constexpr uint64_t kMbarWaitNs = 2000000000ull;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > kMbarWaitNs) return false;
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
template <typename SU, typename SP, int TX, int TY, int DIST>
struct TmaGeom {
  static constexpr int ESU = (int)sizeof(SU), ESP = (int)sizeof(SP);
  static constexpr int AU = 16 / ESU, AP = 16 / ESP;      // 16-byte alignment in elements
  static constexpr int PX = TX + 2, PY = TY + 2;
  static constexpr int UXB = round_up_c(TX + AU + 2, AU);  // u box: x in [x0-AU, x0-AU+UXB)
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
  auto issue = [&](int q) {
    const int r = q - pl;
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
      if (!mbar_wait(bars + r % G::NB, (uint32_t)((r / G::NB) & 1))) bad = true;
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
        sq[qs][c][ty][tx] = Dk[0] * pk[3 * c] + Dk[1] * pk[3 * c + 1] + Dk[2] * pk[3 * c + 2];
        sq[qs][3 + c][ty][tx] = Dk[1] * pk[3 * c] + Dk[3] * pk[3 * c + 1] + Dk[4] * pk[3 * c + 2];
        qzc[c] = Dk[2] * pk[3 * c] + Dk[4] * pk[3 * c + 1] + Dk[5] * pk[3 * c + 2];
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
        div[c] = (dx + dy) + apply3<GEN>(az, qzmm[c], qzm[c], qzc[c]);
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
        mbar_wait(bars + r % G::NB, (uint32_t)((r / G::NB) & 1));
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
        div[c] = (dx + dy) + apply3<GEN>(az, qzmm[c], qzm[c], 0.f);
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
template <int V, typename S> struct Lane;
template <typename S> struct Lane<1, S> {
  static __device__ __forceinline__ void sh(const S* p, float (&o)[1]) { o[0] = Store<S>::sh(p); }
  static __device__ __forceinline__ void st(S* p, const float (&v)[1]) { Store<S>::st(p, v[0]); }
};
template <typename S> struct Lane<2, S> {
  static __device__ __forceinline__ void sh(const S* p, float (&o)[2]) {
    const float2 t = Pair<S>::sh(p);
    o[0] = t.x;
    o[1] = t.y;
  }
  static __device__ __forceinline__ void st(S* p, const float (&v)[2]) { Pair<S>::st(p, v[0], v[1]); }
};
template <> struct Lane<1, float> {
  static __device__ __forceinline__ void sh(const float* p, float (&o)[1]) { o[0] = *p; }
  static __device__ __forceinline__ void st(float* p, const float (&v)[1]) { *p = v[0]; }
};
template <> struct Lane<2, float> {
  static __device__ __forceinline__ void sh(const float* p, float (&o)[2]) {
    const float2 t = *reinterpret_cast<const float2*>(p);
    o[0] = t.x;
    o[1] = t.y;
  }
  static __device__ __forceinline__ void st(float* p, const float (&v)[2]) {
    *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
  }
};

template <typename SU, typename SP, int TX, int TY, int DIST, int V>
struct SplitGeom {
  using B = TmaGeom<SU, SP, TX, TY, DIST>;  // box shapes (shared with the tensor maps)
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
  static constexpr int SMEM = BAR_OFF + NB * 8;
};

template <typename SU, typename SP, int TX, int TY, int DIST, int V, int MINB, bool GEN>
__global__ void __launch_bounds__(SplitGeom<SU, SP, TX, TY, DIST, V>::NT, MINB)
iterate_split_kernel(const Tile* __restrict__ tiles, const Desc* __restrict__ descs,
                     const TMaps* __restrict__ maps, IterArgs a, int* __restrict__ status) {
  using G = SplitGeom<SU, SP, TX, TY, DIST, V>;
  using B = typename G::B;
  constexpr int AU = B::AU, AP = B::AP, UXB = B::UXB, PXB = B::PXB;
  constexpr int UC = B::UYB * UXB, PC = B::PYB * PXB, RCS = TY * TX, SXW = G::SXW;
  static_assert(DIST >= 2, "step k waits for plane k+1, issued at the end of step k+1-DIST");
  extern __shared__ __align__(128) unsigned char smem[];
  float(*sqx)[3][TY][SXW] = reinterpret_cast<float(*)[3][TY][SXW]>(smem + G::SQX_OFF);
  float(*sqy)[3][TY + 2][TX] = reinterpret_cast<float(*)[3][TY + 2][TX]>(smem + G::SQY_OFF);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + G::BAR_OFF);

  const Tile T = tiles[blockIdx.x];
  const Desc& Dg = descs[T.desc];
  const TMaps* M = maps + T.desc;
  const int nz = Dg.nz, ny = Dg.ny, nx = Dg.nx;
  const int cs = (int)Dg.cs;
  const int plane = Dg.pitch * ny;
  const int z0 = T.z0z1 & 0xffff, z1 = T.z0z1 >> 16;
  const CUtensorMap* mu = &M->u[a.src];
  const CUtensorMap* mp = &M->p[a.src];

  const int tid = threadIdx.x;
  int role, lx, ly;  // position relative to (x0, y0)
  if (tid < G::NI) {
    role = 0;
    lx = V * (tid % G::PW);
    ly = tid / G::PW;
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
  const int gx = T.x0 + lx, gy = T.y0 + ly;
  const bool active = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
  const bool full = gx + V - 1 < nx;          // roles 0/1: every voxel of the lane is inside
  const int uo = (ly + 2) * UXB + (lx + AU);  // own (first) voxel in a u box component
  const int po = (ly + 1) * PXB + (lx + AP);  // own (first) voxel in a p/D box component
  const int ro = ly * TX + lx;                // own voxels in an rc/gw box (role 0)
  const long long col0 = (long long)gy * Dg.pitch + gx;
  SU* __restrict__ u_dst = reinterpret_cast<SU*>(Dg.u[a.src ^ 1]) + col0;
  SP* __restrict__ p_dst = reinterpret_cast<SP*>(Dg.p[a.src ^ 1]) + col0;
  const int bdry = GEN ? a.bdry : (int)SVS_BOUNDARY_MIRROR;  // GEN = false is launched for MIRROR only
  Stencil3 fx[V], ax[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    fx[v] = fwd_coef(gx + v, nx, bdry, Dg.hx);
    ax[v] = adj_coef(gx + v, nx, bdry, 1.0f / Dg.hx);
  }
  const Stencil3 fy = fwd_coef(gy, ny, bdry, Dg.hy);
  const Stencil3 ay = adj_coef(gy, ny, bdry, 1.0f / Dg.hy);
  const float ihz = 1.0f / Dg.hz, hz = Dg.hz;

  const int kb = max(z0 - 1, 0), ke = min(z1, nz - 1);
  const int pl = max(kb - 1, 0), ph = min(ke + 1, nz - 1);
  auto issue = [&](int q) {
    const int r = q - pl;
    uint64_t* bar = bars + r % G::NB;
    unsigned char* U = smem + G::U_OFF + (r % G::NU) * B::U_SLOT;
    if (q < kb) {
      mbar_arrive_expect_tx(bar, (uint32_t)B::U_TX);
      tma_load_4d(U, mu, bar, T.x0 - AU, T.y0 - 2, q, 0);
      return;
    }
    unsigned char* PD = smem + G::PD_OFF + ((q - kb) % G::NPD) * B::PD_SLOT;
    unsigned char* R = smem + G::R_OFF + ((q - kb) % G::NR) * B::R_SLOT;
    mbar_arrive_expect_tx(bar, (uint32_t)B::FULL_TX);
    tma_load_4d(U, mu, bar, T.x0 - AU, T.y0 - 2, q, 0);
    tma_load_4d(PD, mp, bar, T.x0 - AP, T.y0 - 1, q, 0);
    tma_load_4d(PD + B::P_SLOT, &M->D, bar, T.x0 - AP, T.y0 - 1, q, 0);
    tma_load_4d(R, &M->rc, bar, T.x0, T.y0, q, 0);
    tma_load_4d(R + B::RC_SLOT, &M->gw, bar, T.x0, T.y0, q, 0);
  };
  auto ubox = [&](int q) {
    return reinterpret_cast<const SU*>(smem + G::U_OFF + ((q - pl) % G::NU) * B::U_SLOT);
  };
  auto rbox = [&](int q) { return smem + G::R_OFF + ((q - kb) % G::NR) * B::R_SLOT; };

  // q cells that no lane writes (outside the volume, the unused qx column x0+TX+1) are read
  // with zero stencil coefficients: they must hold zeros (0 * NaN = NaN)
  for (int i = tid; i < (G::SQX_BYTES + G::SQY_BYTES) / 4; i += blockDim.x)
    reinterpret_cast<float*>(smem + G::SQX_OFF)[i] = 0.f;
  if (tid == 0) {
    for (int s = 0; s < G::NB; ++s) mbar_init(bars + s, 1);
    mbar_fence_init();
  }
  __syncthreads();
  int issued = pl - 1;
  if (tid == 0) {
    const int last = min(kb + DIST - 1, ph);
    for (int q = pl; q <= last; ++q) issue(q);
    issued = last;
  }
  int waited = pl - 1;
  bool bad = false;

  // q_z of the own voxels (role 0) at planes k-2, k-1, k
  float qmm[V][3] = {}, qm[V][3] = {}, qc[V][3] = {};
  const float wtv2 = a.wtv * a.wtv;

  // x/y part of the divergence at plane j (q rows of slot j & 1), loaded before the dual
  auto load_dxy = [&](int j, float (&dxy)[V][3]) {
    const int ps = j & 1;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float* qx = &sqx[ps][c][ly][lx + 2];
      float o[V], dn[V], up[V], oy[V];
      Lane<V, float>::sh(qx, o);
      const float L = qx[-1], R = qx[V];
      Lane<V, float>::sh(&sqy[ps][c][ly][lx], dn);
      Lane<V, float>::sh(&sqy[ps][c][ly + 2][lx], up);
      if (GEN) Lane<V, float>::sh(&sqy[ps][c][ly + 1][lx], oy);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const float prev = v == 0 ? L : o[v - 1], next = v == V - 1 ? R : o[v + 1];
        const float dx = apply3<GEN>(ax[v], prev, GEN ? o[v] : 0.f, next);
        dxy[v][c] = dx + apply3<GEN>(ay, dn[v], GEN ? oy[v] : 0.f, up[v]);
      }
    }
  };
  // primal of plane j: qn = q_z(j+1), uj = own u at plane j
  auto finish_primal = [&](int j, const float (&dxy)[V][3], const float (&qn)[V][3], const float (&uj)[V][3]) {
    const unsigned char* R = rbox(j);
    const SP* RC = reinterpret_cast<const SP*>(R) + ro;
    const SP* GW = reinterpret_cast<const SP*>(R + B::RC_SLOT) + ro;
    const Stencil3 az = adj_coef(j, nz, bdry, ihz);
    float rc[V], g[3][V], n[3][V];
    Lane<V, SP>::sh(RC, rc);
#pragma unroll
    for (int c = 0; c < 3; ++c) Lane<V, SP>::sh(GW + c * RCS, g[c]);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      float d[3], gv[3], nv[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        d[c] = dxy[v][c] + apply3<GEN>(az, qmm[v][c], qm[v][c], qn[v][c]);
        gv[c] = g[c][v];
      }
      primal_voxel(uj[v], d, a.tau, a.factor, rc[v], gv, nv);
#pragma unroll
      for (int c = 0; c < 3; ++c) n[c][v] = nv[c];
    }
    SU* dst = u_dst + (long long)j * plane;
    if (full) {
#pragma unroll
      for (int c = 0; c < 3; ++c) Lane<V, SU>::st(dst + c * cs, n[c]);
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) Store<SU>::st(dst + c * cs, n[c][0]);
    }
  };

  // One plane step; WITH_PRIMAL: role 0 also finishes plane k-1.
  auto step = [&](const int k, auto with_primal) {
    constexpr bool WP = decltype(with_primal)::value;
    const int need = min(k + 1, ph);
    while (waited < need && !bad) {
      ++waited;
      const int r = waited - pl;
      if (!mbar_wait(bars + r % G::NB, (uint32_t)((r / G::NB) & 1))) bad = true;
    }
    const int qs = k & 1;
    const SU* Uk = ubox(k) + uo;
    const unsigned char* PD = smem + G::PD_OFF + ((k - kb) % G::NPD) * B::PD_SLOT;
    const Stencil3 fz = fwd_coef(k, nz, bdry, hz);
    // planes k-1 and k+1 are missing only at k = 0 and k = nz-1, where the z stencil's
    // coefficient for them is zero (every boundary type): plane k stands in for them
    const SU* Um = ubox(k - 1 >= pl ? k - 1 : k) + uo;
    const SU* Up = ubox(k + 1 <= ph ? k + 1 : k) + uo;
    if (role != 2) {
      if (active && !bad) {
        float dxy[V][3];
        if (WP && role == 0) load_dxy(k - 1, dxy);
        // own voxels at planes k-1, k, k+1
        float um[V][3], uc[V][3], up[V][3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float m[V], o[V], n[V];
          Lane<V, SU>::sh(Um + c * UC, m);
          Lane<V, SU>::sh(Uk + c * UC, o);
          Lane<V, SU>::sh(Up + c * UC, n);
#pragma unroll
          for (int v = 0; v < V; ++v) {
            um[v][c] = m[v];
            uc[v][c] = o[v];
            up[v][c] = n[v];
          }
        }
        const SP* P = reinterpret_cast<const SP*>(PD) + po;
        const SP* Dm = reinterpret_cast<const SP*>(PD + B::P_SLOT) + po;
        float pv[9][V], Dv[6][V];
#pragma unroll
        for (int c = 0; c < 9; ++c) Lane<V, SP>::sh(P + c * PC, pv[c]);
#pragma unroll
        for (int c = 0; c < 6; ++c) Lane<V, SP>::sh(Dm + c * PC, Dv[c]);
        float pk[V][9], Dk[V][6];
#pragma unroll
        for (int v = 0; v < V; ++v) {
#pragma unroll
          for (int c = 0; c < 9; ++c) pk[v][c] = pv[c][v];
#pragma unroll
          for (int c = 0; c < 6; ++c) Dk[v][c] = Dv[c][v];
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const SU* u = Uk + c * UC;
          const float L = Store<SU>::sh(u - 1), R = Store<SU>::sh(u + V);
          float dn[V], upy[V];
          Lane<V, SU>::sh(u - UXB, dn);
          Lane<V, SU>::sh(u + UXB, upy);
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const float prev = v == 0 ? L : uc[v - 1][c], next = v == V - 1 ? R : uc[v + 1][c];
            const float ex = apply3<GEN>(fx[v], prev, uc[v][c], next);
            const float ey = apply3<GEN>(fy, dn[v], uc[v][c], upy[v]);
            const float ez = apply3<GEN>(fz, um[v][c], uc[v][c], up[v][c]);
            dual_row(Dk[v], ex, ey, ez, pk[v][3 * c], pk[v][3 * c + 1], pk[v][3 * c + 2], a.sigma, a.wtv, wtv2);
          }
        }
        if (role == 0) {
          if (k >= z0 && k < z1) {
            SP* dst = p_dst + (long long)k * plane;
            if (full) {
#pragma unroll
              for (int c = 0; c < 9; ++c) {
                float t[V];
#pragma unroll
                for (int v = 0; v < V; ++v) t[v] = pk[v][c];
                Lane<V, SP>::st(dst + c * cs, t);
              }
            } else {
#pragma unroll
              for (int c = 0; c < 9; ++c) Store<SP>::st(dst + c * cs, pk[0][c]);
            }
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            float qx[V], qy[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
              const float* D = Dk[v];
              const float* p = &pk[v][3 * c];
              qx[v] = D[0] * p[0] + D[1] * p[1] + D[2] * p[2];
              qy[v] = D[1] * p[0] + D[3] * p[1] + D[4] * p[2];
              qc[v][c] = D[2] * p[0] + D[4] * p[1] + D[5] * p[2];
            }
            Lane<V, float>::st(&sqx[qs][c][ly][lx + 2], qx);
            Lane<V, float>::st(&sqy[qs][c][ly + 1][lx], qy);
          }
          if (WP) finish_primal(k - 1, dxy, qc, um);
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            float qy[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
              const float* D = Dk[v];
              const float* p = &pk[v][3 * c];
              qy[v] = D[1] * p[0] + D[3] * p[1] + D[4] * p[2];
            }
            Lane<V, float>::st(&sqy[qs][c][ly + 1][lx], qy);
          }
        }
      }
    } else if (active && !bad) {
      // halo column: one voxel
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
        const float m = Store<SU>::sh(Um + c * UC);
        const float n = Store<SU>::sh(Up + c * UC);
        const float ex = apply3<GEN>(fx[0], Store<SU>::sh(u - 1), o, Store<SU>::sh(u + 1));
        const float ey = apply3<GEN>(fy, Store<SU>::sh(u - UXB), o, Store<SU>::sh(u + UXB));
        const float ez = apply3<GEN>(fz, m, o, n);
        dual_row(Dk, ex, ey, ez, pk[3 * c], pk[3 * c + 1], pk[3 * c + 2], a.sigma, a.wtv, wtv2);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c)
        sqx[qs][c][ly][lx + 2] = Dk[0] * pk[3 * c] + Dk[1] * pk[3 * c + 1] + Dk[2] * pk[3 * c + 2];
    }
    // everyone is done with plane k's p/D, plane k-1's u and rc/gw, and q rows of plane k-1
    if (__syncthreads_or(bad)) {
      bad = true;
      return;
    }
    if (tid == 0 && k + DIST <= ph && k + DIST > issued) {
      issue(k + DIST);
      issued = k + DIST;
    }
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        qmm[v][c] = qm[v][c];
        qm[v][c] = qc[v][c];
      }
  };

  // the first one or two steps have no finished plane (j = k-1 < z0)
  const int kp = min(z0 + 1, ke + 1);
  int k = kb;
  for (; k < kp && !bad; ++k) step(k, std::false_type{});
  for (; k <= ke && !bad; ++k) step(k, std::true_type{});
  if (bad) {
    if (tid == 0) {
      atomicOr(status, SVS_DEV_TIMEOUT);
      // wait (bounded) for the copies this CTA still has in flight before it exits
      for (int q = max(waited + 1, pl); q <= issued; ++q) {
        const int r = q - pl;
        mbar_wait(bars + r % G::NB, (uint32_t)((r / G::NB) & 1));
      }
    }
    return;
  }
  if (z1 >= nz) {
    const int j = nz - 1;
    if (role == 0 && active && j >= z0) {
      float dxy[V][3], uj[V][3];
      const float zero[V][3] = {};
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float o[V];
        Lane<V, SU>::sh(ubox(j) + uo + c * UC, o);
#pragma unroll
        for (int v = 0; v < V; ++v) uj[v][c] = o[v];
      }
      load_dxy(j, dxy);
      finish_primal(j, dxy, zero, uj);
    }
  }
}

// Compiled shapes of the split-role form (tile, prefetch distance, voxels per lane, CTAs per SM
// the register budget is sized for); instantiated in svs_split.cu.
struct SplitShape {
  int tx, ty, dist, v, minb;
};
constexpr SplitShape kSplitShapes[] = {
    {32, 8, 3, 2, 1},  {32, 8, 4, 2, 1}, {16, 16, 3, 2, 1}, {40, 8, 3, 2, 2}, {32, 16, 3, 2, 1},
    {40, 16, 3, 2, 1}, {32, 8, 3, 1, 2}, {32, 8, 4, 1, 2},  {16, 16, 3, 1, 2}, {32, 16, 2, 1, 1},
    {32, 16, 3, 1, 1}, {40, 8, 3, 1, 2}};
constexpr int kNumSplitShapes = sizeof(kSplitShapes) / sizeof(kSplitShapes[0]);

// Split-role variant `idx` for a storage mode. op 0: set the kernels' shared-memory attribute
// and return the TMA box shapes {u x, u y, p x, p y} in `box` (false if the variant does not
// fit); op 1: launch one iteration over `ntiles` tiles on stream s; op 2: resident CTAs per SM
// in box[0] (after op 0).
bool split_variant(int storage, int idx, int op, bool gen, unsigned ntiles, const Tile* tiles, const Desc* descs,
                   const TMaps* maps, const IterArgs* a, int* status, cudaStream_t s, int* box);

}  // namespace svs
