#!/usr/bin/env bash
# Builds the reference CUDA extension (opticalFlow_cuda_ext.opticalFlow) for sm_100a from the
# reference sources, so that the GPU tests can pin the oracle against the reference itself.
# Test infrastructure only: nothing in the product links or imports the result.
#
# The reference sources are read in place and copied to a scratch folder under /tmp, where one
# token is patched (`.type()` -> `.scalar_type()` inside AT_DISPATCH_FLOATING_TYPES, which the
# reference's torch 2.1 accepted and torch 2.11 rejects). No source is copied into this repo.
# Output: oracle/_ref/opticalFlow_cuda_ext/opticalFlow*.so (git-ignored, travels with the repo).
#
# Register cap: the reference launches every kernel with 768-thread blocks (blockSize(16,16,3)).
# Built for sm_100a with nvcc 12.9, its tricubic vector-field, matrix-field, CNN-warp and
# warp-backward kernels need 88-104 registers per thread, so 768 x regs exceeds the 65,536
# registers of an SM and those launches fail; the reference never checks (cudaSafeCall is a
# no-op unless CUDA_ERROR_CHECK is defined, svs/src/cudaDebug.cuh:15-27), so their outputs stay
# zero and the stock solver returns u = 0 everywhere. -maxrregcount=80 (a build flag, the same
# source and arithmetic) lets every kernel launch. Set REF_MAXRREG= (empty) to build stock.
#
# Where the reference lives: REF_SRC (its svs/src folder), else SVS_REFERENCE_ROOT/svs/src, else a
# checkout named `reference` beside this repository (../reference/svs/src from the repo root).
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
REF_ROOT=${SVS_REFERENCE_ROOT:-$(cd "$HERE/../.." && pwd)/reference}
REF_SRC=${REF_SRC:-$REF_ROOT/svs/src}
OUT="$HERE/_ref/opticalFlow_cuda_ext"
if [ ! -d "$REF_SRC" ]; then
  echo "reference sources not found at $REF_SRC; nothing to build" >&2
  exit 0
fi
SCRATCH=$(mktemp -d /tmp/svs_ref_build.XXXXXX)
cp "$REF_SRC"/*.cu "$REF_SRC"/*.cuh "$REF_SRC"/*.h "$REF_SRC"/bindings.cpp "$SCRATCH"/
sed -i 's/\.type()/.scalar_type()/g' "$SCRATCH"/*.cu
mkdir -p "$OUT" "$SCRATCH/build"
export REF_MAXRREG=${REF_MAXRREG-80}
SCRATCH="$SCRATCH" OUT="$OUT" python - <<'PY'
import os, glob, shutil
from torch.utils import cpp_extension
s = os.environ["SCRATCH"]
srcs = [os.path.join(s, "bindings.cpp")] + sorted(glob.glob(os.path.join(s, "*.cu")))
mod = cpp_extension.load(
    name="opticalFlow", sources=srcs, build_directory=os.path.join(s, "build"),
    extra_cflags=["-O3"],
    extra_cuda_cflags=["-O3", "-gencode", "arch=compute_100a,code=sm_100a"]
                      + ([f"-maxrregcount={os.environ['REF_MAXRREG']}"] if os.environ.get("REF_MAXRREG") else []),
    verbose=False)
so = mod.__file__
shutil.copy(so, os.path.join(os.environ["OUT"], os.path.basename(so)))
open(os.path.join(os.environ["OUT"], "__init__.py"), "w").close()
print("built", os.path.join(os.environ["OUT"], os.path.basename(so)))
PY
