"""The C ABI library loads without a GPU and exports every entry point include/svsflow.h declares."""
import ctypes
import os
import re

from singleventriclesegmentation_b200 import _lib
from singleventriclesegmentation_b200.build import LIB, build_library

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "svsflow.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(svs_[a-z0-9_]+)\s*\(", text)))


def test_library_builds_and_loads():
    path = build_library()
    assert os.path.exists(path) and path == LIB
    lib = ctypes.CDLL(path)
    assert lib.svs_version() == 1


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(build_library())
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_header():
    assert set(declared_functions()) == set(_lib.exported_symbols())


def test_argument_errors_are_reported_without_a_gpu():
    lib = _lib.lib()
    st = lib.svs_nabla3d_forward(None, 4, 4, 4, 1, 1.0, 1.0, 1.0, 1, None, None)
    assert st == 1
    assert b"null pointer" in lib.svs_last_error()
    st = lib.svs_median3d(ctypes.c_void_p(16), 4, 4, 4, 3, 4, ctypes.c_void_p(16), None)
    assert st == 1 and b"kernel size" in lib.svs_last_error()


def test_plan_rejects_too_small_pyramids():
    p = _lib.TVL1Params()
    p.num_scales, p.max_warps, p.max_outer_iterations = 3, 1, 1
    p.primaldual_algorithm_type, p.interpolation, p.boundary, p.weight_tv = 2, 2, 1, 0.025
    dims = (ctypes.c_int * 3)(8, 8, 8)  # 8 -> 4 -> 2: the coarsest level is too small
    h = ctypes.c_void_p()
    st = _lib.lib().svs_tvl1_plan_create(ctypes.byref(p), 1, dims, ctypes.byref(h))
    assert st == 1 and b"at least 3 nodes" in _lib.lib().svs_last_error()


def test_tile_info_lists_every_variant():
    n = _lib.lib().svs_tvl1_num_tiles()
    infos = [_lib.tile_info(t) for t in range(1, n + 1)]
    assert {i["form"] for i in infos} == {"plain", "tma", "split"}
    for i in infos:
        assert i["tx"] % 8 == 0 and i["ty"] > 0  # tile origins keep TMA boxes 16-byte aligned
        assert (i["dist"] == 0) == (i["form"] == "plain")
        if i["form"] == "split":
            assert i["lane_voxels"] in (1, 2) and i["dist"] >= 2
            assert (i["tx"] // i["lane_voxels"] * i["ty"]) % 32 == 0  # interior lanes fill whole warps
    import pytest
    for bad in (0, n + 1):
        with pytest.raises(_lib.SVSError):
            _lib.tile_info(bad)
