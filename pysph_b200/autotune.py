"""Launch-shape autotuner for the pair kernels.

For a workload it times whole predictor-corrector steps for every candidate
of cell size (stencil R: cell = support / R), lanes per dest particle and
threads per block, with the neighbour lists and (2D FP32C summation
density) with the shared-memory tiles, and returns the fastest.  On that shape it then tries
the force pass's load-ahead depth (FP32C) and the skin of the kept
neighbour lists: a wider skin means longer lists but fewer rebins, which
pays where particles move fast.  Results are cached per (dim, precision,
particle-count bucket, scene-count bucket), in memory and, when
PYSPH_B200_TUNE_CACHE names a file, in that JSON file.
"""
from __future__ import annotations

import json
import math
import os

import torch

from .engine import Engine

LANES = (1, 2, 4, 8)
BLOCKS = (64, 128, 256)
STENCILS = (1, 2)
SKINS = (0.1, 0.15, 0.25)

_cache: dict = {}


def _key(dim, precision, n, scenes):
    return f"{dim}d-{precision}-n{int(math.log2(max(n, 1)))}-s{int(math.log2(max(scenes, 1)))}"


def _load():
    path = os.environ.get("PYSPH_B200_TUNE_CACHE")
    if path and os.path.exists(path):
        try:
            with open(path) as f:
                _cache.update(json.load(f))
        except (OSError, ValueError):
            pass


def _store():
    path = os.environ.get("PYSPH_B200_TUNE_CACHE")
    if path:
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(_cache, f, indent=1)
        os.replace(tmp, path)


def time_steps(eng: Engine, steps: int = 4, warm: int = 2) -> float:
    """Milliseconds per PC step (CUDA events on the current stream)."""
    for _ in range(warm):
        eng.pc_step()
    stream = torch.cuda.current_stream(eng.device)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        eng.pc_step()
    b.record(stream)
    torch.cuda.synchronize(eng.device)
    return a.elapsed_time(b) / steps


def tiled_ok(scheme, dim, precision, variable_h=False) -> bool:
    """Whether the tiled pair passes apply (2D FP32C, summation density, one
    h per pair)."""
    return (dim == 2 and precision == "fp32c" and not scheme.continuity and not scheme.hks
            and not variable_h)


def autotune(scenes, scheme, dim, precision="fp32c", device=None, stencils=STENCILS,
             lanes=LANES, blocks=BLOCKS, steps=4, force=False, tiled=True):
    """Best {"pairs", "stencil", "lanes", "pair_block", "ms_per_step"} plus the
    table of every candidate timed."""
    _load()
    n = sum(len(a["x"]) for arrays, _ in scenes for a in arrays)
    key = _key(dim, precision, n, len(scenes))
    if not force and key in _cache:
        return _cache[key]
    table = []
    for R in stencils:
        eng = Engine(scenes, scheme, dim=dim, precision=precision, stencil=R,
                     device=device)
        for L in lanes:
            for B in blocks:
                if B % L or B // L < 8:
                    continue
                eng.set_launch(L, B)
                ms = time_steps(eng, steps)
                eng.check_status()
                table.append({"pairs": "lists", "stencil": R, "lanes": L, "pair_block": B,
                              "ms_per_step": ms})
        del eng
        if tiled and tiled_ok(scheme, dim, precision):
            eng = Engine(scenes, scheme, dim=dim, precision=precision, stencil=R,
                         device=device, pairs="tiled")
            for B in blocks:
                if B < 128:
                    continue
                eng.set_launch(1, B)
                ms = time_steps(eng, steps)
                eng.check_status()
                table.append({"pairs": "tiled", "stencil": R, "lanes": 1, "pair_block": B,
                              "ms_per_step": ms})
            del eng
    best = min(table, key=lambda r: r["ms_per_step"])
    best = dict(best, list_batch=4)
    if precision == "fp32c" and best["pairs"] == "lists":
        # load-ahead depth of the force pass's list loop, on the best shape
        eng = Engine(scenes, scheme, dim=dim, precision=precision, stencil=best["stencil"],
                     lanes=best["lanes"], pair_block=best["pair_block"], device=device,
                     list_batch=2)
        ms = time_steps(eng, steps)
        eng.check_status()
        table.append({"pairs": "lists", "stencil": best["stencil"], "lanes": best["lanes"],
                      "pair_block": best["pair_block"], "list_batch": 2, "ms_per_step": ms})
        if ms < best["ms_per_step"]:
            best = dict(table[-1])
        del eng
    # the skin, on enough steps for the rebins to show (fresh engines, so
    # every candidate starts from the same state)
    skin_table = []
    for skin in SKINS:
        eng = Engine(scenes, scheme, dim=dim, precision=precision, stencil=best["stencil"],
                     lanes=best["lanes"], pair_block=best["pair_block"], device=device,
                     list_batch=best.get("list_batch", 4), skin_margin=skin,
                     pairs=best["pairs"])
        ms = time_steps(eng, 4 * steps, warm=steps)
        eng.check_status()
        skin_table.append(dict(pairs=best["pairs"], stencil=best["stencil"], lanes=best["lanes"],
                               pair_block=best["pair_block"],
                               list_batch=best.get("list_batch", 4), skin_margin=skin,
                               ms_per_step=ms))
        del eng
    table.extend(skin_table)
    best = dict(min(skin_table, key=lambda r: r["ms_per_step"]))
    res = dict(best, key=key, table=table)
    _cache[key] = res
    _store()
    return res
