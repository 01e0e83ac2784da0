// Instantiations and launch of the split-role iterate kernel (svs_iterate.cuh) for every storage
// mode and compiled shape, in a translation unit of their own so that they compile in parallel
// with the rest of the library.
#include "svs_iterate.cuh"

namespace svs {
namespace {

template <typename SU, typename SP, int I>
bool run(int op, bool gen, unsigned nt, const Tile* tiles, const Desc* descs, const TMaps* maps,
         const IterArgs* a, int* status, cudaStream_t s, int* box) {
  constexpr SplitShape S = kSplitShapes[I];
  if constexpr (!(S.smask & (1 << storage_id<SU, SP>()))) {
    return false;  // not compiled for this storage mode
  } else {
  using G = SplitGeom<SU, SP, S.tx, S.ty, S.dist, S.v, S.as, (S.opt >> 8)>;
  using KFn = void (*)(const Tile*, const Desc*, const TMaps*, IterArgs, int*);
  KFn kf, kt;
  if constexpr (S.regs > 0) {
    kf = iterate_split_kernel_r<SU, SP, S.tx, S.ty, S.dist, S.v, S.regs, false, S.as, S.opt>;
    kt = iterate_split_kernel_r<SU, SP, S.tx, S.ty, S.dist, S.v, S.regs, true, S.as, S.opt>;
  } else {
    kf = iterate_split_kernel<SU, SP, S.tx, S.ty, S.dist, S.v, S.minb, false, S.as, S.opt>;
    kt = iterate_split_kernel<SU, SP, S.tx, S.ty, S.dist, S.v, S.minb, true, S.as, S.opt>;
  }
  if (op == 2) {  // resident CTAs per SM (after op 0 set the shared-memory attribute)
    if (G::SMEM > 227 * 1024) return false;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, gen ? kt : kf, G::NT_LAUNCH, G::SMEM) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    box[0] = n;
    return true;
  }
  if (op == 0) {
    if (G::SMEM > 227 * 1024) return false;
    if (cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM) != cudaSuccess ||
        cudaFuncSetAttribute(kt, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    box[0] = G::B::UXB;
    box[1] = G::B::UYB;
    box[2] = G::B::PXB;
    box[3] = G::B::PYB;
    return true;
  }
  (gen ? kt : kf)<<<nt, G::NT_LAUNCH, G::SMEM, s>>>(tiles, descs, maps, *a, status);
  return true;
  }
}

template <typename SU, typename SP>
bool dispatch(int idx, int op, bool gen, unsigned nt, const Tile* tiles, const Desc* descs, const TMaps* maps,
              const IterArgs* a, int* status, cudaStream_t s, int* box) {
#define SVS_SPLIT(I) \
  case I: return run<SU, SP, I>(op, gen, nt, tiles, descs, maps, a, status, s, box);
  static_assert(kNumSplitShapes == 25, "one case per compiled shape");
  switch (idx) {
    SVS_SPLIT(0) SVS_SPLIT(1) SVS_SPLIT(2) SVS_SPLIT(3) SVS_SPLIT(4) SVS_SPLIT(5)
    SVS_SPLIT(6) SVS_SPLIT(7) SVS_SPLIT(8) SVS_SPLIT(9) SVS_SPLIT(10) SVS_SPLIT(11)
    SVS_SPLIT(12) SVS_SPLIT(13) SVS_SPLIT(14) SVS_SPLIT(15) SVS_SPLIT(16) SVS_SPLIT(17)
    SVS_SPLIT(18) SVS_SPLIT(19) SVS_SPLIT(20) SVS_SPLIT(21) SVS_SPLIT(22) SVS_SPLIT(23)
    SVS_SPLIT(24)
    default: return false;
  }
#undef SVS_SPLIT
}

}  // namespace

bool split_variant(int storage, int idx, int op, bool gen, unsigned nt, const Tile* tiles, const Desc* descs,
                   const TMaps* maps, const IterArgs* a, int* status, cudaStream_t s, int* box) {
  switch (storage) {
    case SVS_STORAGE_BF16:
      return dispatch<__nv_bfloat16, __nv_bfloat16>(idx, op, gen, nt, tiles, descs, maps, a, status, s, box);
    case SVS_STORAGE_F16: return dispatch<__half, __half>(idx, op, gen, nt, tiles, descs, maps, a, status, s, box);
    case SVS_STORAGE_BF16_FLOW32:
      return dispatch<float, __nv_bfloat16>(idx, op, gen, nt, tiles, descs, maps, a, status, s, box);
    case SVS_STORAGE_F16_FLOW32: return dispatch<float, __half>(idx, op, gen, nt, tiles, descs, maps, a, status, s, box);
    default: return dispatch<float, float>(idx, op, gen, nt, tiles, descs, maps, a, status, s, box);
  }
}

}  // namespace svs
