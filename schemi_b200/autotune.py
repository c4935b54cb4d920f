"""Autotuner of the fused march kernel's tile shape.

For a case it times every supported shape -- threads per CTA along x (incl. the two halo
columns), along y in 3D, the number of rows a CTA marches, and whether rows are staged through
shared memory by bulk async copies -- on the case's own state with
CUDA events on the library's stream, the L2 flushed before each timed step, and keeps the
fastest.  Results are cached in a JSON file keyed by (dims, cells per axis, species, EOS,
precision, device name); ``SCHEMI_B200_TUNE_CACHE`` overrides the cache path.

    from schemi_b200 import autotune
    shape = autotune.tune(fvcase)        # applies the best shape to the handle and returns it
"""

from __future__ import annotations

import json
import os
from typing import Dict, List, Optional, Tuple

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_CACHE = os.path.join(HERE, "tune_cache.json")

SHAPES_2D = [(bx, 1, rows, st) for bx in (64, 128, 256) for rows in (8, 16, 32, 64) for st in (0, 1)]
SHAPES_3D = [(bx, by, rows, st) for (bx, by) in ((32, 8), (32, 16), (64, 8)) for rows in (8, 16, 32, 64)
             for st in (0, 1)]


def _cache_path() -> str:
    return os.environ.get("SCHEMI_B200_TUNE_CACHE", DEFAULT_CACHE)


def _key(case, device: str) -> str:
    n = "x".join(str(v) for v in case.n[: case.dims])
    # 2D cases run the warp-strip march (FP32 flux or FP64), whose shapes are timed separately
    kind = ("|warp-strip" if case.precision == "f32flux" else "|warp-strip64") if case.dims == 2 else ""
    return f"{case.dims}d|{n}|ns{case.n_species}|{case.eos}|{case.precision}|{device}{kind}"


def load_cache() -> Dict[str, dict]:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_cache(cache: Dict[str, dict]) -> None:
    try:
        with open(_cache_path(), "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    except OSError:
        pass


def apply_shape(g, shape) -> None:
    g.set_march_shape(*shape[:3])
    g.set_staging(bool(shape[3]) if len(shape) > 3 else True)


def time_shape(g, torch, shape, steps: int = 5, flush=None) -> float:
    """Mean device ms of one step kernel + CFL for `shape` (state is advanced)."""
    apply_shape(g, shape)
    stream = torch.cuda.ExternalStream(g.stream_ptr)
    g.begin_steps()
    if flush is None:
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    with torch.cuda.stream(stream):
        g.step_async()  # first launch of a shape configures it
        ev = []
        for _ in range(steps):
            flush.add_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g.step_async()
            e1.record(stream)
            ev.append((e0, e1))
    torch.cuda.synchronize()
    g.check()
    return sum(a.elapsed_time(b) for a, b in ev) / steps


def tune(g, steps: int = 5, use_cache: bool = True, verbose: bool = False) -> Optional[Tuple[int, int, int, int]]:
    """Pick the fastest march shape for the handle `g` (an FVCase) and apply it."""
    import torch

    from .fv import PATH_MARCH

    if g.path != PATH_MARCH:
        return None
    case = g.case
    device = torch.cuda.get_device_name()
    key = _key(case, device)
    cache = load_cache() if use_cache else {}
    if key in cache and len(cache[key]["shape"]) == 4:
        shape = tuple(cache[key]["shape"])
        apply_shape(g, shape)
        return shape
    shapes: List[Tuple[int, int, int]] = SHAPES_2D if case.dims == 2 else SHAPES_3D
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    results = {}
    for s in shapes:
        try:
            results[s] = time_shape(g, torch, s, steps=steps, flush=flush)
        except Exception as e:  # an unsupported shape is skipped
            if verbose:
                print("skip", s, e)
    best = min(results, key=results.get)
    if verbose:
        for s, ms in sorted(results.items(), key=lambda kv: kv[1]):
            print(f"  shape bx={s[0]} by={s[1]} rows={s[2]} staged={s[3]}: {ms * 1e3:.1f} us/step")
    apply_shape(g, best)
    cache[key] = {"shape": list(best), "ms": results[best],
                  "all": {f"{s[0]}x{s[1]}x{s[2]}x{s[3]}": v for s, v in results.items()}}
    if use_cache:
        save_cache(cache)
    return best
