"""The C ABI library loads without a GPU and exports every entry point include/svsflow.h declares."""
import ctypes
import os
import re

import pytest

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


def _plan_cost(columns, nz, slots, p, fill=3):
    """Makespan in plane steps of a chunk plan, the quantity the plan minimises."""
    cdiv = lambda a, b: -(-a // b)
    main = columns - p["tail_columns"]
    t = cdiv(main * p["main_chunks"], slots) * (cdiv(nz, p["main_chunks"]) + fill) if main else 0
    if p["tail_columns"]:
        t += cdiv(p["tail_columns"] * p["tail_chunks"], slots) * (cdiv(nz, p["tail_chunks"]) + fill)
    return t


def test_chunk_plan_of_the_split_kernels():
    """The z-chunk plan (host arithmetic, no GPU): the 68-pair 80^3 bench level (1360 40x8 columns
    on 148 SMs x 2 CTAs) marches 1184 whole columns and cuts the last 176 into 5 chunks; level 1
    (340 columns of 40 planes) cuts 44 tail columns into 6; one pair's level 0 (20 columns, all of
    them tail) splits every column into 14. Every plan is at least as short as the best uniform
    chunk count, and the whole-wave columns fill whole waves up to one column's chunks."""
    cases = {(1360, 80, 296): (1, 5, 176), (340, 40, 296): (1, 6, 44), (20, 80, 296): (1, 14, 20)}
    for (cols, nz, slots), want in cases.items():
        p = _lib.chunk_plan(cols, nz, slots)
        assert (p["main_chunks"], p["tail_chunks"], p["tail_columns"]) == want, (cols, nz, slots, p)
    for cols in (1, 7, 150, 296, 297, 1000, 1360, 5000):
        for nz in (3, 20, 40, 80, 128):
            for slots in (148, 296, 444):
                p = _lib.chunk_plan(cols, nz, slots)
                assert 1 <= p["main_chunks"] <= p["tail_chunks"] <= nz
                assert 0 <= p["tail_columns"] <= cols
                main = cols - p["tail_columns"]
                r = (main * p["main_chunks"]) % slots
                assert r == 0 or r > slots - p["main_chunks"] or p["tail_columns"] == 0
                best_uniform = min(_plan_cost(cols, nz, slots, {"main_chunks": c, "tail_chunks": c,
                                                                 "tail_columns": 0}) for c in range(1, nz + 1))
                assert _plan_cost(cols, nz, slots, p) <= best_uniform
    with pytest.raises(_lib.SVSError):
        _lib.chunk_plan(0, 80, 296)


def test_automatic_variant_choice():
    """The automatic per-level choice (host arithmetic, no GPU). The 68-pair 80^3 bench: 40x8
    voxel pairs at levels 0 and 1 and 32x8 single voxels at level 2 (20^3), one variant per level;
    FP32 fields: 32x16 voxel pairs. A batch whose level fills the GPU with widths that are and are
    not multiples of 40 gives each width its own variant (all pairs of one width alike, the
    multiples of 40 on the 40x8 shape); too small a batch keeps one variant per level."""
    def tid(tx, ty, v):
        for t in range(1, _lib.lib().svs_tvl1_num_tiles() + 1):
            i = _lib.tile_info(t)
            if i["form"] == "split" and (i["tx"], i["ty"], i["lane_voxels"]) == (tx, ty, v):
                return t
    f16_flow32, f32 = 4, 0
    main0, pairs0 = _lib.auto_tiles(f16_flow32, [(80, 80, 80)] * 68, 148)
    main1, pairs1 = _lib.auto_tiles(f16_flow32, [(40, 40, 40)] * 68, 148)
    main2, pairs2 = _lib.auto_tiles(f16_flow32, [(20, 20, 20)] * 68, 148)
    assert main0 == main1 == 28 and _lib.tile_info(28)["tx"] == 40 and _lib.tile_info(28)["lane_voxels"] == 2
    assert main2 == tid(32, 8, 1)
    assert not any(pairs0 + pairs1 + pairs2)
    mf, pf = _lib.auto_tiles(f32, [(80, 80, 80)] * 68, 148)
    assert mf == tid(32, 16, 2) and not any(pf)
    dims = [(n, n, n) for n in (64, 80, 96, 128, 120, 64, 80, 96, 128, 120) * 6]
    main, pairs = _lib.auto_tiles(f16_flow32, dims, 148)
    used = [p or main for p in pairs]
    by_width = {}
    for d, t in zip(dims, used):
        by_width.setdefault(d[2], set()).add(t)
    assert all(len(s) == 1 for s in by_width.values())
    assert by_width[80] == by_width[120] == {28}
    assert by_width[64] != {28} and by_width[128] != {28}
    small_main, small_pairs = _lib.auto_tiles(f16_flow32, [(64, 64, 64), (80, 80, 80)], 148)
    assert small_main == tid(16, 16, 1) and not any(small_pairs)
    with pytest.raises(_lib.SVSError):
        _lib.auto_tiles(f16_flow32, [(0, 80, 80)], 148)
