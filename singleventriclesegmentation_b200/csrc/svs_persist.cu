// Persistent launches of the split-role iterate kernel (iterate_persist_kernel, svs_iterate.cuh):
// one cooperative grid runs every iteration of one warp at one level. A translation unit of its
// own, so that it compiles in parallel with the per-iteration instantiations.
#include <algorithm>

#include "svs_iterate.cuh"

namespace svs {
namespace {

template <typename SU, typename SP, int I>
bool run_persist(int op, bool gen, unsigned nt, const Tile* tiles, const Desc* descs, const TMaps* maps,
                 const PersistArgs* pa, int* status, cudaStream_t s) {
  constexpr SplitShape S = kSplitShapes[I];
  if constexpr (!has_persist(S) || !(S.smask & (1 << storage_id<SU, SP>()))) {
    return false;
  } else {
    using G = SplitGeom<SU, SP, S.tx, S.ty, S.dist, S.v, false, (S.opt >> 8)>;
    using KFn = void (*)(const Tile*, int, const Desc*, const TMaps*, PersistArgs, int*);
    const KFn kf = iterate_persist_kernel<SU, SP, S.tx, S.ty, S.dist, S.v, S.minb, false, S.opt>;
    const KFn kt = iterate_persist_kernel<SU, SP, S.tx, S.ty, S.dist, S.v, S.minb, true, S.opt>;
    if (G::SMEM > 227 * 1024) return false;
    if (op == 0) {
      if (cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM) != cudaSuccess ||
          cudaFuncSetAttribute(kt, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
      return true;
    }
    const KFn k = gen ? kt : kf;
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, G::NT_LAUNCH, G::SMEM) != cudaSuccess || per_sm < 1) {
      cudaGetLastError();
      return false;
    }
    // every CTA of the grid must be resident at once (the grid barrier waits for all of them):
    // at most SMs x resident CTAs per SM, and the cooperative attribute makes the launch fail
    // rather than start a grid that cannot be
    const unsigned grid = std::max(1u, std::min(nt, (unsigned)(sms * per_sm)));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(G::NT_LAUNCH);
    cfg.dynamicSmemBytes = G::SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeCooperative;
    attr.val.cooperative = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, tiles, (int)nt, descs, maps, *pa, status) == cudaSuccess;
  }
}

template <typename SU, typename SP>
bool dispatch_persist(int idx, int op, bool gen, unsigned nt, const Tile* tiles, const Desc* descs,
                      const TMaps* maps, const PersistArgs* pa, int* status, cudaStream_t s) {
#define SVS_PERSIST(I) \
  case I: return run_persist<SU, SP, I>(op, gen, nt, tiles, descs, maps, pa, status, s);
  static_assert(kNumSplitShapes == 25, "one case per compiled shape");
  switch (idx) {
    SVS_PERSIST(0) SVS_PERSIST(1) SVS_PERSIST(2) SVS_PERSIST(3) SVS_PERSIST(4) SVS_PERSIST(5)
    SVS_PERSIST(6) SVS_PERSIST(7) SVS_PERSIST(8) SVS_PERSIST(9) SVS_PERSIST(10) SVS_PERSIST(11)
    SVS_PERSIST(12) SVS_PERSIST(13) SVS_PERSIST(14) SVS_PERSIST(15) SVS_PERSIST(16) SVS_PERSIST(17)
    SVS_PERSIST(18) SVS_PERSIST(19) SVS_PERSIST(20) SVS_PERSIST(21) SVS_PERSIST(22) SVS_PERSIST(23)
    SVS_PERSIST(24)
    default: return false;
  }
#undef SVS_PERSIST
}

}  // namespace

bool split_persist(int storage, int idx, int op, bool gen, unsigned ntiles, const Tile* tiles, const Desc* descs,
                   const TMaps* maps, const PersistArgs* pa, int* status, cudaStream_t s) {
  switch (storage) {
    case SVS_STORAGE_BF16:
      return dispatch_persist<__nv_bfloat16, __nv_bfloat16>(idx, op, gen, ntiles, tiles, descs, maps, pa, status, s);
    case SVS_STORAGE_F16: return dispatch_persist<__half, __half>(idx, op, gen, ntiles, tiles, descs, maps, pa, status, s);
    case SVS_STORAGE_BF16_FLOW32:
      return dispatch_persist<float, __nv_bfloat16>(idx, op, gen, ntiles, tiles, descs, maps, pa, status, s);
    case SVS_STORAGE_F16_FLOW32:
      return dispatch_persist<float, __half>(idx, op, gen, ntiles, tiles, descs, maps, pa, status, s);
    default: return dispatch_persist<float, float>(idx, op, gen, ntiles, tiles, descs, maps, pa, status, s);
  }
}

}  // namespace svs
