// The fused primal-dual iteration (svs/modules/flow/tvl13d.py:213-253) as one kernel per
// iteration, in two forms:
//   iterate_kernel      plain loads, one z-plane of each field per step, state in registers;
//   iterate_tma_kernel  a multi-stage TMA pipeline: one thread issues cp.async.bulk.tensor
//                       loads of whole plane tiles (u, p, D, rc, gw) several planes ahead into a
//                       shared-memory ring, completion tracked by mbarriers.
// Both march a TX x TY column tile along z. Thread (tx, ty) of the (TX+2) x (TY+2) block owns
// column (x0-1+tx, y0-1+ty) of the "dual region" (tile plus a one-voxel x/y halo). At plane k:
//   dual:   on the dual region minus its 4 corners, p_new(k) = proj(p + sigma D grad u) and
//           q = D p_new; the z-row of q stays in registers, the x- and y-rows are published;
//   primal: on the tile interior, plane j = k-1 is finished: div = adjoint(q) from the
//           published rows of plane j and the registers of planes j-1 and j+1, then
//           u_new(j) = prox_primal(u - tau div).
// Halo duals are recomputed by neighbouring tiles, so the tiles of one launch are independent
// (u and p are ping-pong buffers). The arithmetic of both forms is identical.
#pragma once

#include "svs_state.cuh"

namespace svs {

// Dual update of one flow component at one voxel, tvl13d.py:215-222 with
// opticalFlowOps.cu:179-208: v = p + sigma D g; p_new = v / max(1, |v| / weight_tv), written as
// v * min(1, weight_tv * rsqrt(|v|^2)). weight_tv == 0 zeroes p (tvl13d.py:223-224).
__device__ __forceinline__ void dual_row(const float D[6], float ex, float ey, float ez, float& p0,
                                         float& p1, float& p2, float sigma, float wtv, float wtv2) {
  const float d0 = D[0] * ex + D[1] * ey + D[2] * ez;
  const float d1 = D[1] * ex + D[3] * ey + D[4] * ez;
  const float d2 = D[2] * ex + D[4] * ey + D[5] * ez;
  const float v0 = p0 + sigma * d0, v1 = p1 + sigma * d1, v2 = p2 + sigma * d2;
  const float nsq = v0 * v0 + v1 * v1 + v2 * v2;
  const float sc = (nsq > wtv2) ? wtv * rsqrtf(nsq) : 1.0f;
  if (wtv > 0.f) {
    p0 = v0 * sc;
    p1 = v1 * sc;
    p2 = v2 * sc;
  } else {
    p0 = p1 = p2 = 0.f;
  }
}

// Primal update at one voxel, tvl13d.py:229-235 with opticalFlowOps.cu:123-175:
// rho = rc + u.g (u before the update), u_new = (u - tau div) + shrinkage step.
__device__ __forceinline__ void primal_voxel(const float u[3], const float div[3], float tau,
                                             float factor, float rc, const float g[3], float un[3]) {
  const float rho = rc + (u[0] * g[0] + u[1] * g[1] + u[2] * g[2]);
  const float g2s = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
#pragma unroll
  for (int c = 0; c < 3; ++c) un[c] = u[c] - tau * div[c];
  const float th = factor * g2s;
  if (rho < -th) {
#pragma unroll
    for (int c = 0; c < 3; ++c) un[c] += factor * g[c];
  } else if (rho > th) {
#pragma unroll
    for (int c = 0; c < 3; ++c) un[c] -= factor * g[c];
  } else if (g2s >= 1e-10f) {  // the reference's (double)g2 > 1e-10 for a float g2
    const float t = __fdividef(-rho, g2s);
#pragma unroll
    for (int c = 0; c < 3; ++c) un[c] += t * g[c];
  }
}

// ------------------------------------------------------------------------ plain-load form
template <typename S, int TX, int TY>
__global__ void __launch_bounds__((TX + 2) * (TY + 2))
iterate_kernel(const Tile* __restrict__ tiles, const Desc* __restrict__ descs, IterArgs a) {
  constexpr int PX = TX + 2, PY = TY + 2, UX = TX + 4, UY = TY + 4;
  constexpr int NRING = 2 * (TX + TY);
  __shared__ float su[2][3][UY][UX];
  __shared__ float sq[2][6][PY][PX];

  const Tile T = tiles[blockIdx.x];
  const Desc& Dg = descs[T.desc];
  const int nz = Dg.nz, ny = Dg.ny, nx = Dg.nx;
  const float ihz = 1.0f / Dg.hz, ihy = 1.0f / Dg.hy, ihx = 1.0f / Dg.hx;
  const float hz = Dg.hz, hy = Dg.hy, hx = Dg.hx;
  const long long cs = Dg.cs;
  const long long plane = (long long)Dg.pitch * ny;
  const int z0 = T.z0z1 & 0xffff, z1 = T.z0z1 >> 16;
  const S* __restrict__ u_src = reinterpret_cast<const S*>(Dg.u[a.src]);
  const S* __restrict__ p_src = reinterpret_cast<const S*>(Dg.p[a.src]);
  S* __restrict__ u_dst = reinterpret_cast<S*>(Dg.u[a.src ^ 1]);
  S* __restrict__ p_dst = reinterpret_cast<S*>(Dg.p[a.src ^ 1]);
  const S* __restrict__ Dm = reinterpret_cast<const S*>(Dg.D);
  const S* __restrict__ rcm = reinterpret_cast<const S*>(Dg.rc);
  const S* __restrict__ gwm = reinterpret_cast<const S*>(Dg.gw);

  const int tid = threadIdx.x;
  const int tx = tid % PX, ty = tid / PX;
  const int gx = T.x0 - 1 + tx, gy = T.y0 - 1 + ty;
  const bool in_dom = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
  const bool corner = (tx == 0 || tx == PX - 1) && (ty == 0 || ty == PY - 1);
  const bool dual_on = in_dom && !corner;
  const bool interior = in_dom && tx >= 1 && tx <= TX && ty >= 1 && ty <= TY;
  const long long col = (long long)gy * Dg.pitch + gx;

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
  const long long rcol = (long long)rgy * Dg.pitch + rgx;

  const int kb = max(z0 - 1, 0), ke = min(z1, nz - 1);
  float um[3] = {0.f, 0.f, 0.f}, uc[3] = {0.f, 0.f, 0.f}, up[3] = {0.f, 0.f, 0.f};
  if (in_dom) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (kb >= 1) um[c] = Store<S>::ld(u_src + c * cs + (kb - 1) * plane + col);
      uc[c] = Store<S>::ld(u_src + c * cs + kb * plane + col);
      if (kb + 1 < nz) up[c] = Store<S>::ld(u_src + c * cs + (kb + 1) * plane + col);
    }
  }
  float qzmm[3] = {0.f, 0.f, 0.f}, qzm[3] = {0.f, 0.f, 0.f}, qzc[3] = {0.f, 0.f, 0.f};
  const float wtv2 = a.wtv * a.wtv;
  const int bdry = a.bdry;

  for (int k = kb; k <= ke; ++k) {
    const int slot = k & 1;
    float pk[9], Dk[6];
    if (dual_on) {
      const long long o = k * plane + col;
#pragma unroll
      for (int c = 0; c < 9; ++c) pk[c] = Store<S>::ld(p_src + c * cs + o);
#pragma unroll
      for (int c = 0; c < 6; ++c) Dk[c] = Store<S>::ld(Dm + c * cs + o);
    }
    const int j = k - 1;
    const bool primal_on = interior && j >= z0 && j < z1;
    float rcj = 0.f, gj[3] = {0.f, 0.f, 0.f};
    if (primal_on) {
      const long long o = j * plane + col;
      rcj = Store<S>::ld(rcm + o);
#pragma unroll
      for (int c = 0; c < 3; ++c) gj[c] = Store<S>::ld(gwm + c * cs + o);
    }
    if (in_dom) {
#pragma unroll
      for (int c = 0; c < 3; ++c) su[slot][c][ty + 1][tx + 1] = uc[c];
    }
    if (ring_on) {
#pragma unroll
      for (int c = 0; c < 3; ++c) su[slot][c][ry][rx] = Store<S>::ld(u_src + c * cs + k * plane + rcol);
    }
    __syncthreads();
    if (dual_on) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float ex = fwd_axis(su[slot][c][ty + 1][tx], uc[c], su[slot][c][ty + 1][tx + 2], gx, nx, bdry, hx);
        const float ey = fwd_axis(su[slot][c][ty][tx + 1], uc[c], su[slot][c][ty + 2][tx + 1], gy, ny, bdry, hy);
        const float ez = fwd_axis(um[c], uc[c], up[c], k, nz, bdry, hz);
        dual_row(Dk, ex, ey, ez, pk[3 * c], pk[3 * c + 1], pk[3 * c + 2], a.sigma, a.wtv, wtv2);
      }
      if (interior && k >= z0 && k < z1) {
        const long long o = k * plane + col;
#pragma unroll
        for (int c = 0; c < 9; ++c) Store<S>::st(p_dst + c * cs + o, pk[c]);
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
      float div[3], un[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float ax = adj_axis(sq[ps][c][ty][tx - 1], sq[ps][c][ty][tx], sq[ps][c][ty][tx + 1], gx, nx, bdry);
        const float ay = adj_axis(sq[ps][3 + c][ty - 1][tx], sq[ps][3 + c][ty][tx], sq[ps][3 + c][ty + 1][tx], gy, ny, bdry);
        const float az = adj_axis(qzmm[c], qzm[c], qzc[c], j, nz, bdry);
        div[c] = (ax * ihx + ay * ihy) + az * ihz;
      }
      primal_voxel(um, div, a.tau, a.factor, rcj, gj, un);
      const long long o = j * plane + col;
#pragma unroll
      for (int c = 0; c < 3; ++c) Store<S>::st(u_dst + c * cs + o, un[c]);
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
      for (int c = 0; c < 3; ++c) up[c] = Store<S>::ld(u_src + c * cs + (k + 2) * plane + col);
    }
  }
  if (z1 >= nz) {
    __syncthreads();
    const int j = nz - 1;
    if (interior && j >= z0) {
      const int ps = j & 1;
      const long long o = j * plane + col;
      float gj[3], div[3], un[3];
      const float rcj = Store<S>::ld(rcm + o);
#pragma unroll
      for (int c = 0; c < 3; ++c) gj[c] = Store<S>::ld(gwm + c * cs + o);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float ax = adj_axis(sq[ps][c][ty][tx - 1], sq[ps][c][ty][tx], sq[ps][c][ty][tx + 1], gx, nx, bdry);
        const float ay = adj_axis(sq[ps][3 + c][ty - 1][tx], sq[ps][3 + c][ty][tx], sq[ps][3 + c][ty + 1][tx], gy, ny, bdry);
        const float az = adj_axis(qzmm[c], qzm[c], 0.f, j, nz, bdry);
        div[c] = (ax * ihx + ay * ihy) + az * ihz;
      }
      primal_voxel(um, div, a.tau, a.factor, rcj, gj, un);
#pragma unroll
      for (int c = 0; c < 3; ++c) Store<S>::st(u_dst + c * cs + o, un[c]);
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

// Shared-memory geometry of the TMA form for storage S and tile TX x TY with NSTG stages.
template <typename S, int TX, int TY, int NSTG>
struct TmaGeom {
  static constexpr int ES = (int)sizeof(S);
  static constexpr int A = 16 / ES;                       // 16-byte alignment in elements
  static constexpr int PX = TX + 2, PY = TY + 2;
  static constexpr int UXB = round_up_c(TX + A + 2, A);   // u box: x in [x0-A, x0-A+UXB)
  static constexpr int PXB = round_up_c(TX + A + 1, A);   // p/D box: x in [x0-A, x0-A+PXB)
  static constexpr int UYB = TY + 4, PYB = TY + 2;        // u box rows from y0-2, p/D from y0-1
  static constexpr int U_TX = 3 * UYB * UXB * ES;
  static constexpr int P_TX = 9 * PYB * PXB * ES;
  static constexpr int D_TX = 6 * PYB * PXB * ES;
  static constexpr int RC_TX = TY * TX * ES;
  static constexpr int GW_TX = 3 * TY * TX * ES;
  static constexpr int U_OFF = 0;
  static constexpr int P_OFF = round_up_c(U_OFF + U_TX, 128);
  static constexpr int D_OFF = round_up_c(P_OFF + P_TX, 128);
  static constexpr int RC_OFF = round_up_c(D_OFF + D_TX, 128);
  static constexpr int GW_OFF = round_up_c(RC_OFF + RC_TX, 128);
  static constexpr int STAGE = round_up_c(GW_OFF + GW_TX, 128);
  static constexpr int STAGE_TX = U_TX + P_TX + D_TX + RC_TX + GW_TX;
  static constexpr int SQ_OFF = NSTG * STAGE;
  static constexpr int SQ_BYTES = 3 * 6 * PY * PX * 4;
  static constexpr int BAR_OFF = round_up_c(SQ_OFF + SQ_BYTES, 8);
  static constexpr int SMEM = BAR_OFF + NSTG * 8;
};

template <typename S, int TX, int TY, int NSTG>
__global__ void __launch_bounds__((TX + 2) * (TY + 2))
iterate_tma_kernel(const Tile* __restrict__ tiles, const Desc* __restrict__ descs,
                   const TMaps* __restrict__ maps, IterArgs a, int* __restrict__ status) {
  using G = TmaGeom<S, TX, TY, NSTG>;
  constexpr int PX = G::PX, PY = G::PY, A = G::A, UXB = G::UXB, UYB = G::UYB, PXB = G::PXB,
                PYB = G::PYB;
  // Planes k-1, k, k+1 are read at step k; plane k+DIST is issued after the step's barrier into
  // the slot of plane k-2. Step k waits for plane k+1, issued at step k+1-DIST: DIST >= 2.
  static_assert(NSTG >= 4, "the TMA pipeline needs at least 4 stages");
  constexpr int DIST = NSTG - 2;  // prefetch distance in planes
  extern __shared__ __align__(128) unsigned char smem[];
  float(*sq)[6][PY][PX] = reinterpret_cast<float(*)[6][PY][PX]>(smem + G::SQ_OFF);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + G::BAR_OFF);

  const Tile T = tiles[blockIdx.x];
  const Desc& Dg = descs[T.desc];
  const TMaps* M = maps + T.desc;
  const int nz = Dg.nz, ny = Dg.ny, nx = Dg.nx;
  const float ihz = 1.0f / Dg.hz, ihy = 1.0f / Dg.hy, ihx = 1.0f / Dg.hx;
  const float hz = Dg.hz, hy = Dg.hy, hx = Dg.hx;
  const long long cs = Dg.cs;
  const long long plane = (long long)Dg.pitch * ny;
  const int z0 = T.z0z1 & 0xffff, z1 = T.z0z1 >> 16;
  S* __restrict__ u_dst = reinterpret_cast<S*>(Dg.u[a.src ^ 1]);
  S* __restrict__ p_dst = reinterpret_cast<S*>(Dg.p[a.src ^ 1]);
  const CUtensorMap* mu = &M->u[a.src];
  const CUtensorMap* mp = &M->p[a.src];

  const int tid = threadIdx.x;
  const int tx = tid % PX, ty = tid / PX;
  const int gx = T.x0 - 1 + tx, gy = T.y0 - 1 + ty;
  const bool in_dom = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
  const bool corner = (tx == 0 || tx == PX - 1) && (ty == 0 || ty == PY - 1);
  const bool dual_on = in_dom && !corner;
  const bool interior = in_dom && tx >= 1 && tx <= TX && ty >= 1 && ty <= TY;
  const long long col = (long long)gy * Dg.pitch + gx;
  const int ux = tx + A - 1, uy = ty + 1;  // own column in the u box
  const int px = tx + A - 1, py = ty;      // own column in the p/D boxes

  const int kb = max(z0 - 1, 0), ke = min(z1, nz - 1);
  const int pl = max(kb - 1, 0), ph = min(ke + 1, nz - 1);  // planes staged by this tile

  auto stage = [&](int q) -> unsigned char* { return smem + ((q - pl) % NSTG) * G::STAGE; };
  auto issue = [&](int q) {
    unsigned char* st = stage(q);
    uint64_t* bar = bars + (q - pl) % NSTG;
    mbar_arrive_expect_tx(bar, (uint32_t)G::STAGE_TX);
    tma_load_4d(st + G::U_OFF, mu, bar, T.x0 - A, T.y0 - 2, q, 0);
    tma_load_4d(st + G::P_OFF, mp, bar, T.x0 - A, T.y0 - 1, q, 0);
    tma_load_4d(st + G::D_OFF, &M->D, bar, T.x0 - A, T.y0 - 1, q, 0);
    tma_load_4d(st + G::RC_OFF, &M->rc, bar, T.x0, T.y0, q, 0);
    tma_load_4d(st + G::GW_OFF, &M->gw, bar, T.x0, T.y0, q, 0);
  };

  if (tid == 0) {
    for (int s = 0; s < NSTG; ++s) mbar_init(bars + s, 1);
    mbar_fence_init();
  }
  __syncthreads();
  int issued = pl - 1;  // last plane issued (meaningful in thread 0)
  if (tid == 0) {
    const int last = min(kb + DIST - 1, ph);
    for (int q = pl; q <= last; ++q) issue(q);
    issued = last;
  }
  int waited = pl - 1;  // every thread: planes <= waited are complete
  bool bad = false;

  auto uval = [&](int q, int c, int yy, int xx) -> float {
    const S* U = reinterpret_cast<const S*>(stage(q) + G::U_OFF);
    return Store<S>::sh(U + (c * UYB + yy) * UXB + xx);
  };

  float qzmm[3] = {0.f, 0.f, 0.f}, qzm[3] = {0.f, 0.f, 0.f}, qzc[3] = {0.f, 0.f, 0.f};
  const float wtv2 = a.wtv * a.wtv;
  const int bdry = a.bdry;

  for (int k = kb; k <= ke; ++k) {
    const int need = min(k + 1, ph);
    while (waited < need && !bad) {
      ++waited;
      if (!mbar_wait(bars + (waited - pl) % NSTG, (uint32_t)(((waited - pl) / NSTG) & 1))) bad = true;
    }
    if (dual_on && !bad) {
      const S* P = reinterpret_cast<const S*>(stage(k) + G::P_OFF);
      const S* Dm = reinterpret_cast<const S*>(stage(k) + G::D_OFF);
      float pk[9], Dk[6];
#pragma unroll
      for (int c = 0; c < 9; ++c) pk[c] = Store<S>::sh(P + (c * PYB + py) * PXB + px);
#pragma unroll
      for (int c = 0; c < 6; ++c) Dk[c] = Store<S>::sh(Dm + (c * PYB + py) * PXB + px);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float uc = uval(k, c, uy, ux);
        const float ex = fwd_axis(uval(k, c, uy, ux - 1), uc, uval(k, c, uy, ux + 1), gx, nx, bdry, hx);
        const float ey = fwd_axis(uval(k, c, uy - 1, ux), uc, uval(k, c, uy + 1, ux), gy, ny, bdry, hy);
        const float zm = (k - 1 >= pl) ? uval(k - 1, c, uy, ux) : 0.f;
        const float zp = (k + 1 <= ph) ? uval(k + 1, c, uy, ux) : 0.f;
        const float ez = fwd_axis(zm, uc, zp, k, nz, bdry, hz);
        dual_row(Dk, ex, ey, ez, pk[3 * c], pk[3 * c + 1], pk[3 * c + 2], a.sigma, a.wtv, wtv2);
      }
      if (interior && k >= z0 && k < z1) {
        const long long o = k * plane + col;
#pragma unroll
        for (int c = 0; c < 9; ++c) Store<S>::st(p_dst + c * cs + o, pk[c]);
      }
      const int qs = k % 3;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        sq[qs][c][ty][tx] = Dk[0] * pk[3 * c] + Dk[1] * pk[3 * c + 1] + Dk[2] * pk[3 * c + 2];
        sq[qs][3 + c][ty][tx] = Dk[1] * pk[3 * c] + Dk[3] * pk[3 * c + 1] + Dk[4] * pk[3 * c + 2];
        qzc[c] = Dk[2] * pk[3 * c] + Dk[4] * pk[3 * c + 1] + Dk[5] * pk[3 * c + 2];
      }
    }
    // every thread has finished reading planes < k: stage slots of planes <= k-2 are free
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
      const int ps = j % 3;
      const S* RC = reinterpret_cast<const S*>(stage(j) + G::RC_OFF);
      const S* GW = reinterpret_cast<const S*>(stage(j) + G::GW_OFF);
      const int ri = (ty - 1) * TX + (tx - 1);
      const float rcj = Store<S>::sh(RC + ri);
      float gj[3], uj[3], div[3], un[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        gj[c] = Store<S>::sh(GW + c * TY * TX + ri);
        uj[c] = uval(j, c, uy, ux);
        const float ax = adj_axis(sq[ps][c][ty][tx - 1], sq[ps][c][ty][tx], sq[ps][c][ty][tx + 1], gx, nx, bdry);
        const float ay = adj_axis(sq[ps][3 + c][ty - 1][tx], sq[ps][3 + c][ty][tx], sq[ps][3 + c][ty + 1][tx], gy, ny, bdry);
        const float az = adj_axis(qzmm[c], qzm[c], qzc[c], j, nz, bdry);
        div[c] = (ax * ihx + ay * ihy) + az * ihz;
      }
      primal_voxel(uj, div, a.tau, a.factor, rcj, gj, un);
      const long long o = j * plane + col;
#pragma unroll
      for (int c = 0; c < 3; ++c) Store<S>::st(u_dst + c * cs + o, un[c]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      qzmm[c] = qzm[c];
      qzm[c] = qzc[c];
    }
  }
  if (bad) {
    if (tid == 0) {
      atomicOr(status, SVS_DEV_TIMEOUT);
      // wait (bounded) for the copies this CTA still has in flight before it exits
      for (int q = pl; q <= issued; ++q) mbar_wait(bars + (q - pl) % NSTG, (uint32_t)(((q - pl) / NSTG) & 1));
    }
    return;
  }
  if (z1 >= nz) {
    const int j = nz - 1;
    if (interior && j >= z0) {
      const int ps = j % 3;
      const S* RC = reinterpret_cast<const S*>(stage(j) + G::RC_OFF);
      const S* GW = reinterpret_cast<const S*>(stage(j) + G::GW_OFF);
      const int ri = (ty - 1) * TX + (tx - 1);
      const float rcj = Store<S>::sh(RC + ri);
      float gj[3], uj[3], div[3], un[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        gj[c] = Store<S>::sh(GW + c * TY * TX + ri);
        uj[c] = uval(j, c, uy, ux);
        const float ax = adj_axis(sq[ps][c][ty][tx - 1], sq[ps][c][ty][tx], sq[ps][c][ty][tx + 1], gx, nx, bdry);
        const float ay = adj_axis(sq[ps][3 + c][ty - 1][tx], sq[ps][3 + c][ty][tx], sq[ps][3 + c][ty + 1][tx], gy, ny, bdry);
        const float az = adj_axis(qzmm[c], qzm[c], 0.f, j, nz, bdry);
        div[c] = (ax * ihx + ay * ihy) + az * ihz;
      }
      primal_voxel(uj, div, a.tau, a.factor, rcj, gj, un);
      const long long o = j * plane + col;
#pragma unroll
      for (int c = 0; c < 3; ++c) Store<S>::st(u_dst + c * cs + o, un[c]);
    }
  }
}

}  // namespace svs
