"""Autotuner for the fused iterate kernel: picks, per pyramid level of a plan, the kernel variant
(TMA pipeline or plain-load form, tile shape, prefetch distance) with the shortest measured time
on the plan's own state, and caches the choice on disk.

The variants are listed in include/svsflow.h (svs_tvl1_plan_set_tile). A level's "size class" is
the multiset of its volume sizes; the cache key is (GPU name, storage, level sizes).
"""
from __future__ import annotations

import json
import os

import numpy as np
from typing import Dict, List, Optional, Sequence, Tuple

import torch

from . import _lib
from .tvl13d import SolverPlan

CACHE = os.environ.get("SVS_AUTOTUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "svsflow", "autotune.json"))


def _level_dims(dims: Sequence[Tuple[int, int, int]], levels: int) -> List[List[Tuple[int, int, int]]]:
    out = []
    cur = [tuple(d) for d in dims]
    for _ in range(levels):
        out.append(sorted(cur))
        cur = [tuple((v + 1) // 2 for v in d) for d in cur]
    return out


def _variants_signature() -> str:
    """The compiled variant table, so that a cache written by another build is not reused."""
    n = int(_lib.lib().svs_tvl1_num_tiles())
    return ",".join("{tx}x{ty}/{dist}{f}{lane_voxels}".format(f=i["form"][0], **i)
                    for i in map(_lib.tile_info, range(1, n + 1)))


def _key(device, storage: str, level_dims) -> str:
    name = torch.cuda.get_device_name(device).replace(" ", "_")
    sig = ";".join("x".join(map(str, d)) for d in level_dims)
    return f"{name}|{_variants_signature()}|{storage}|{sig}"


def _load() -> Dict[str, int]:
    try:
        with open(CACHE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(db: Dict[str, int]) -> None:
    try:
        os.makedirs(os.path.dirname(CACHE), exist_ok=True)
        tmp = CACHE + ".tmp"
        with open(tmp, "w") as f:
            json.dump(db, f, indent=1, sort_keys=True)
        os.replace(tmp, CACHE)
    except OSError:
        pass


def time_variant(plan: SolverPlan, level: int, tile: int, iters: int = 6) -> Optional[float]:
    """Mean milliseconds per launch of `tile` at `level`, or None if the variant does not fit."""
    plan.set_level_tile(level, tile)
    try:
        plan.bench_iterations(level, 2)
    except _lib.SVSError as e:
        if e.status == 5:  # shared memory or descriptor limits
            return None
        raise
    torch.cuda.synchronize(plan.device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    plan.bench_iterations(level, iters)
    e1.record()
    torch.cuda.synchronize(plan.device)
    return e0.elapsed_time(e1) / iters


def time_level(plan: SolverPlan, level: int, iters: int = 6) -> Optional[float]:
    """Mean milliseconds per iteration of `level` with the plan's current variant assignment
    (all groups of pairs), or None if an assigned variant does not fit."""
    try:
        plan.bench_iterations(level, 2)
    except _lib.SVSError as e:
        if e.status == 5:
            return None
        raise
    torch.cuda.synchronize(plan.device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    plan.bench_iterations(level, iters)
    e1.record()
    torch.cuda.synchronize(plan.device)
    return e0.elapsed_time(e1) / iters


def _pair_level_dims(dims, level: int):
    out = []
    for d in dims:
        d = tuple(d)
        for _ in range(level):
            d = tuple((v + 1) // 2 for v in d)
        out.append(d)
    return out


def tune_classes(plan: SolverPlan, level: int, candidates: Sequence[int], iters: int = 6) -> Dict[int, int]:
    """Per size class of a level (pairs of equal width at that level): try `candidates` for the
    class's pairs while the others keep their variant, timing the whole level (the groups run
    concurrently), and keep a class's choice when it is at least 2% faster. Returns
    {width: tile id} for the classes that left the level's variant."""
    ld = _pair_level_dims(plan.dims, level)
    widths = sorted({d[2] for d in ld})
    if len(widths) < 2:
        return {}
    base = time_level(plan, level, iters)
    chosen = {}
    for w in widths:
        members = [i for i, d in enumerate(ld) if d[2] == w]
        best_t, best_tid = base, 0
        for t in candidates:
            for i in members:
                plan.set_pair_tile(level, i, t)
            ms = time_level(plan, level, iters)
            if ms is not None and ms < best_t * 0.98:
                best_t, best_tid = ms, t
        for i in members:
            plan.set_pair_tile(level, i, best_tid)
        base = best_t
        if best_tid:
            chosen[w] = best_tid
    return chosen


def tune(plan: SolverPlan, storage: str, levels: int, candidates: Optional[Sequence[int]] = None,
         use_cache: bool = True, iters: int = 6, per_class: bool = False, class_candidates: int = 3) -> List[int]:
    """Choose and set the fastest variant per level; returns the chosen ids (level 0 first).
    With per_class, then let each size class of a level take one of the level's
    `class_candidates` fastest variants (tune_classes)."""
    candidates = list(candidates or range(1, int(_lib.lib().svs_tvl1_num_tiles()) + 1))
    db = _load() if use_cache else {}
    chosen = []
    lds = _level_dims(plan.dims, levels)
    for level in range(levels):
        key = _key(plan.device, storage, [lds[level]])
        best = db.get(key)
        ranked = None
        if best is None or per_class:
            timings = {t: time_variant(plan, level, t, iters) for t in candidates}
            timings = {t: v for t, v in timings.items() if v is not None}
            ranked = sorted(timings, key=timings.get)
            best = ranked[0] if best is None else best
            db[key] = best
        plan.set_level_tile(level, best)
        chosen.append(best)
        if per_class and ranked:
            cls = tune_classes(plan, level, [t for t in ranked[:class_candidates + 1] if t != best][:class_candidates],
                               iters)
            plan.class_tiles = getattr(plan, "class_tiles", {})
            plan.class_tiles[level] = cls
    if use_cache:
        _store(db)
    return chosen


def _main(argv=None) -> None:
    """Time the iterate-kernel variants on a batch of identical synthetic pairs:

        python -m singleventriclesegmentation_b200.autotune --pairs 16 --size 80 --storage f32 --tiles 1,2

    Each variant: one short solve (1 warp x 10 iterations per level) to fill the state, then the
    mean time of level-0 iterate launches; prints one JSON line per variant."""
    import argparse
    import json as _json

    from . import synthetic
    from .tvl13d import TVL13DOpticalFlow

    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=16)
    ap.add_argument("--size", type=int, default=80)
    ap.add_argument("--storage", default="f32")
    ap.add_argument("--tiles", default="")
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--level", type=int, default=0)
    ap.add_argument("--chunks", default="0", help="z chunks per column to try at the level (0 = automatic)")
    args = ap.parse_args(argv)
    dev = torch.device("cuda", 0)
    shape = (args.size,) * 3
    I0, I1, _ = synthetic.frame_pair(shape, seed=0, device="cuda")
    I0, I1 = torch.from_numpy(I0).to(dev), torch.from_numpy(I1).to(dev)
    tiles = [int(t) for t in args.tiles.split(",") if t] or list(range(1, int(_lib.lib().svs_tvl1_num_tiles()) + 1))
    bpv = {"f32": 136, "bf16": 68, "f16": 68, "bf16-flow32": 80, "f16-flow32": 80}[args.storage]
    for tid in tiles:
        s = TVL13DOpticalFlow(3, 1, 10, 1.0, 0.025, 2, (0.5, 0.5, 0.25, 1.0), True, (5.0, 0.5), True, 1.0,
                              "CUBIC_HERMITESPLINE", "MIRROR", "numDofs", (1, 1, 1), dev, storage=args.storage)
        s.tile_id = tid
        try:
            plan = s.plan_for([shape] * args.pairs)
            outs = [torch.empty(shape + (3,), device=dev) for _ in range(args.pairs)]
            plan.solve([I0] * args.pairs, [I1] * args.pairs, outs)
            torch.cuda.synchronize()
            plan.check()
            vox = args.pairs * int(np.prod([(n + (1 << args.level) - 1) >> args.level for n in shape]))
            for ch in [int(c) for c in args.chunks.split(",")]:
                plan.set_level_chunks(args.level, ch)
                ms = time_variant(plan, args.level, tid, args.iters)
                plan.check()
                line = {"storage": args.storage, "tile": tid, "level": args.level, "ms": round(ms, 4),
                        "GBs": round(vox * bpv / (ms / 1e3) / 1e9, 1)}
                if ch:
                    line["chunks"] = ch
                print(_json.dumps(line), flush=True)
            plan.close()
        except _lib.SVSError as e:
            print(_json.dumps({"storage": args.storage, "tile": tid, "error": str(e)[:160]}), flush=True)


if __name__ == "__main__":
    _main()
