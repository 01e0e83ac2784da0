"""ctypes binding of libsvsflow.so (the C ABI declared in include/svsflow.h).

The library is loaded from this package directory. There is no fallback: if the library is
missing, or no CUDA device is present when an operator runs, the call raises.
"""
from __future__ import annotations

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsvsflow.so")

c_int, c_float, c_double, c_void_p, c_int64, c_size_t = (
    ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_void_p, ctypes.c_int64, ctypes.c_size_t)

SVS_OK = 0
SVS_ERR_TIMEOUT = 4
STATUS_NAMES = {0: "SVS_OK", 1: "SVS_ERR_INVALID_ARG", 2: "SVS_ERR_OUT_OF_MEMORY",
                3: "SVS_ERR_LAUNCH", 4: "SVS_ERR_TIMEOUT", 5: "SVS_ERR_UNSUPPORTED",
                6: "SVS_ERR_CUDA"}

STORAGE = {"f32": 0, "float32": 0, "bf16": 1, "bfloat16": 1, "f16": 2, "float16": 2,
           "bf16-flow32": 3, "f16-flow32": 4}


class TVL1Params(ctypes.Structure):
    """svs_tvl1_params (include/svsflow.h)."""
    _fields_ = [
        ("num_scales", c_int), ("max_warps", c_int), ("max_outer_iterations", c_int),
        ("weight_matching", c_float), ("weight_tv", c_float),
        ("primaldual_algorithm_type", c_int),
        ("sigma", c_double), ("tau", c_double), ("theta", c_double), ("gamma", c_double),
        ("use_anisotropic_diff", c_int), ("alpha", c_float), ("beta", c_float),
        ("use_gaussian_blur", c_int), ("gaussian_blur_sigma", c_float),
        ("interpolation", c_int), ("boundary", c_int),
        ("length_type", c_int), ("length_z", c_float), ("length_y", c_float), ("length_x", c_float),
        ("median_kernel", c_int), ("storage", c_int),
    ]


class PairDesc(ctypes.Structure):
    """svs_pair_desc (include/svsflow.h)."""
    _fields_ = [
        ("nz", c_int), ("ny", c_int), ("nx", c_int),
        ("I0", c_void_p), ("I1", c_void_p), ("u_out", c_void_p), ("p_out", c_void_p),
        ("u_init", c_void_p), ("p_init", c_void_p),
    ]


_SIGS = {
    "svs_last_error": (ctypes.c_char_p, []),
    "svs_version": (c_int, []),
    "svs_launch_count": (ctypes.c_uint64, []),
    "svs_nabla3d_forward": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_float, c_float, c_float, c_int, c_void_p, c_void_p]),
    "svs_nabla3d_backward": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_float, c_float, c_float, c_int, c_void_p, c_void_p]),
    "svs_aniso3d_tangents": (c_int, [c_void_p, c_int64, c_float, c_float, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "svs_aniso3d_apply": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "svs_tvl1_prox_primal": (c_int, [c_void_p, c_int64, c_float, c_float, c_void_p, c_void_p, c_void_p, c_void_p]),
    "svs_tvl1_prox_dual": (c_int, [c_void_p, c_int64, c_float, c_float, c_void_p, c_void_p]),
    "svs_warp3d": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_float, c_float, c_float, c_int, c_int, c_void_p, c_void_p]),
    "svs_warp3d_backward": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_float, c_float, c_float, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "svs_warp_cnn3d": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_float, c_float, c_float, c_int, c_int, c_void_p, c_void_p]),
    "svs_prolongate3d": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_float, c_float, c_float, c_int, c_int, c_int, c_float, c_float, c_float, c_int, c_int, c_void_p, c_void_p]),
    "svs_gauss_blur3d": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p]),
    "svs_median3d": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p]),
    "svs_nabla3d_forward_f64": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_double, c_double, c_double, c_int, c_void_p, c_void_p]),
    "svs_nabla3d_backward_f64": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_double, c_double, c_double, c_int, c_void_p, c_void_p]),
    "svs_aniso3d_tangents_f64": (c_int, [c_void_p, c_int64, c_double, c_double, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "svs_aniso3d_apply_f64": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "svs_tvl1_prox_primal_f64": (c_int, [c_void_p, c_int64, c_double, c_double, c_void_p, c_void_p, c_void_p, c_void_p]),
    "svs_tvl1_prox_dual_f64": (c_int, [c_void_p, c_int64, c_double, c_double, c_void_p, c_void_p]),
    "svs_warp3d_f64": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_double, c_double, c_double, c_int, c_int, c_void_p, c_void_p]),
    "svs_warp3d_backward_f64": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_double, c_double, c_double, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "svs_warp_cnn3d_f64": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_double, c_double, c_double, c_int, c_int, c_void_p, c_void_p]),
    "svs_prolongate3d_f64": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_double, c_double, c_double, c_int, c_int, c_int, c_double, c_double, c_double, c_int, c_int, c_void_p, c_void_p]),
    "svs_gauss_blur3d_f64": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p]),
    "svs_median3d_f64": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p]),
    "svs_tvl1_plan_create": (c_int, [ctypes.POINTER(TVL1Params), c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_void_p)]),
    "svs_tvl1_plan_destroy": (c_int, [c_void_p]),
    "svs_tvl1_plan_device_bytes": (c_size_t, [c_void_p]),
    "svs_tvl1_plan_set_tile": (c_int, [c_void_p, c_int]),
    "svs_tvl1_plan_set_level_tile": (c_int, [c_void_p, c_int, c_int]),
    "svs_tvl1_num_tiles": (c_int, []),
    "svs_tvl1_plan_set_pair_tile": (c_int, [c_void_p, c_int, c_int, c_int]),
    "svs_tvl1_plan_set_level_chunks": (c_int, [c_void_p, c_int, c_int]),
    "svs_tvl1_plan_set_residuals": (c_int, [c_void_p, c_int, c_float]),
    "svs_tvl1_plan_get_residuals": (c_int, [c_void_p, c_void_p, c_size_t]),
    "svs_tvl1_tile_info": (c_int, [c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                                   ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
    "svs_tvl1_tile_occupancy": (c_int, [c_int, c_int, c_int, ctypes.POINTER(c_int)]),
    "svs_tvl1_solve_batch": (c_int, [c_void_p, ctypes.POINTER(PairDesc), c_int, c_void_p]),
    "svs_tvl1_bench_iterations": (c_int, [c_void_p, c_int, c_int, c_void_p]),
    "svs_tvl1_plan_graph_kernels": (ctypes.c_uint64, [c_void_p]),
    "svs_tvl1_plan_level_tile": (c_int, [c_void_p, c_int]),
    "svs_tvl1_plan_pair_tile_used": (c_int, [c_void_p, c_int, c_int]),
    "svs_tvl1_auto_tiles": (c_int, [c_int, c_int, ctypes.POINTER(c_int), c_int, ctypes.POINTER(c_int)]),
    "svs_tvl1_plan_level_ctas": (c_int64, [c_void_p, c_int]),
    "svs_tvl1_chunk_plan": (c_int, [c_int64, c_int, c_int64, c_void_p, c_void_p, c_void_p]),
    "svs_tvl1_plan_check": (c_int, [c_void_p]),
    "svs_tvl1_plan_set_stall_test": (c_int, [c_void_p, c_int, c_int, c_int, ctypes.c_uint32]),
    "svs_tvl1_plan_set_persistent": (c_int, [c_void_p, c_int]),
    "svs_tvl1_plan_retarget": (c_int, [c_void_p, c_int, ctypes.POINTER(c_int), c_void_p]),
    "svs_tvl1_plan_create_reserve": (c_int, [ctypes.POINTER(TVL1Params), c_int, c_size_t, ctypes.POINTER(c_void_p)]),
    "svs_tvl1_plan_level_persistent": (c_int, [c_void_p, c_int]),
    "svs_tvl1_solve_noalloc": (c_int, [ctypes.POINTER(TVL1Params), c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_void_p]),
}

_lib = None


def exported_symbols():
    """Names of the C ABI entry points this binding expects."""
    return list(_SIGS)


def lib():
    """Load (once) and return the library handle."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libsvsflow.so not found at {LIB_PATH}; build it with "
                "`python -m singleventriclesegmentation_b200.build`")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


class SVSError(RuntimeError):
    """A non-zero svs_status from the library."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def check(status: int) -> None:
    if status != SVS_OK:
        msg = lib().svs_last_error()
        raise SVSError(status, msg.decode() if msg else "")


def stream_ptr(device=None) -> int:
    """The current torch CUDA stream of `device` as a raw cudaStream_t."""
    return torch.cuda.current_stream(device).cuda_stream


def ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


def launch_count() -> int:
    return int(lib().svs_launch_count())


def tile_info(tile_id: int) -> dict:
    """Shape of an iterate-kernel variant: {"tx", "ty", "dist", "form", "lane_voxels"} with form
    "plain", "tma" or "split"."""
    v = [ctypes.c_int() for _ in range(5)]
    check(lib().svs_tvl1_tile_info(int(tile_id), *[ctypes.byref(x) for x in v]))
    return {"tx": v[0].value, "ty": v[1].value, "dist": v[2].value,
            "form": ("plain", "tma", "split")[v[3].value], "lane_voxels": v[4].value}


def tile_occupancy(storage: int, tile_id: int, general_boundary: bool = False) -> int:
    """CTAs of a split-role variant one SM holds at once for a storage mode (current device)."""
    n = c_int()
    check(lib().svs_tvl1_tile_occupancy(int(storage), int(tile_id), int(bool(general_boundary)), ctypes.byref(n)))
    return n.value


def auto_tiles(storage: int, dims, sms: int):
    """The automatic iterate-kernel choice for one pyramid level (host arithmetic): `dims` are the
    pairs' (nz, ny, nx) at that level. Returns (level variant, [pair variant or 0 per pair])."""
    n = len(dims)
    arr = (c_int * (3 * n))(*[int(v) for d in dims for v in d])
    out = (c_int * max(n, 1))()
    main = int(lib().svs_tvl1_auto_tiles(int(storage), n, arr, int(sms), out))
    if main == 0:
        raise SVSError(1, "svs_tvl1_auto_tiles: invalid arguments")
    return main, [int(out[i]) for i in range(n)]


def chunk_plan(columns: int, nz: int, slots: int) -> dict:
    """z-chunk plan of the split-role kernels for `columns` column tiles of up to `nz` planes on
    `slots` resident CTAs: {"main_chunks", "tail_chunks", "tail_columns"} (host arithmetic)."""
    m, t, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
    check(lib().svs_tvl1_chunk_plan(int(columns), int(nz), int(slots), ctypes.byref(m), ctypes.byref(t),
                                    ctypes.byref(c)))
    return {"main_chunks": m.value, "tail_chunks": t.value, "tail_columns": c.value}
