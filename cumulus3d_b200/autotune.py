"""Autotuner for the half-step kernel variant.

All variants of the half-step kernel produce the same bits, so the choice only affects speed:

* lanes per pixel: one thread per pixel, or two lanes that split the window rows;
* window-weight cache: on or off;
* source sampling: loads from the bordered plane, or a texture gather;
* row-pair f32x2 loops, staged source boxes (cp.async or TMA tensor loads), a persistent launch per run.

The tuner times each candidate on a prefix of the caller's own views and returns the fastest tuning word: a
photometric run of two red-black iterations from random init brings the planes near convergence (the state most
half steps of a schedule see, and the one the staged source boxes are built for), then one more iteration continuing
from it is timed (kernel time from the session's CUDA events).  Results are cached in a JSON file
keyed by (GPU name, window radius, window step, math mode, image size class).
"""
from __future__ import annotations

import json
import os
import pathlib
from typing import Dict, Optional, Sequence

from . import _lib
from .patchstereo import KernelInput, PatchMatchBackend, RunParams

CANDIDATES = (0, 2, 3, 4, 6, 7, 8, 10, 16, 18, 42, 90)  # see PS_TUNE_* in include/patchstereo.h
DEFAULT_CACHE = pathlib.Path(os.environ.get("PS_AUTOTUNE_CACHE",
                                            pathlib.Path(__file__).resolve().parent / "_autotune_cache.json"))


def _size_class(mp: float) -> str:
    return "S" if mp < 0.5 else ("M" if mp < 4 else "L")


def _key(gpu: str, inp: KernelInput, math: str) -> str:
    """(GPU, window, step, math, the set of image size classes of the batch's top level, the largest source count):
    a mixed batch keys on all its sizes, and the source count sets the shared memory of the half step."""
    sizes = "".join(sorted({_size_class(v.levels[-1].width * v.levels[-1].height / 1e6) for v in inp.views}))
    nsrc = max((len(v.sources) for v in inp.views), default=0)
    return f"{gpu}|r{inp.pm.window_radius}|s{inp.pm.window_step}|{math}|{sizes}|n{nsrc}"


def _load(path: pathlib.Path) -> Dict[str, dict]:
    try:
        return json.loads(path.read_text())
    except Exception:
        return {}


def tune(inp: KernelInput, device: int = 0, math: str = "parity", views: Optional[Sequence[int]] = None,
         candidates: Sequence[int] = CANDIDATES, cache: Optional[pathlib.Path] = DEFAULT_CACHE,
         max_views: int = 4, force: bool = False) -> dict:
    """Returns {"tuning": t, "ms": {t: half-step ms}, "cached": bool}."""
    probe = PatchMatchBackend(device, math=math)
    gpu = probe.name()
    probe.close()
    key = _key(gpu, inp, math)
    if cache is not None and not force:
        hit = _load(cache).get(key)
        if hit:
            return dict(hit, cached=True)
    vs = list(views if views is not None else range(len(inp.views)))
    # a prefix, but with one view of every size class of the batch in it
    picked, seen = [], set()
    for v in vs:
        lv = inp.views[v].levels[-1]
        c = _size_class(lv.width * lv.height / 1e6)
        if c not in seen:
            seen.add(c)
            picked.append(v)
    vs = (picked + [v for v in vs if v not in picked])[:max(max_views, len(picked))]
    times = {}
    for t in candidates:
        be = PatchMatchBackend(device, math=math, tuning=t)
        with be.begin(inp) as s:
            lvl = inp.num_levels - 1
            s.run_resident(vs, RunParams(lvl, False, True, 2, 1))  # warm-up (module load, textures), converging
            s.synchronize()
            s.set_profiling(True)
            s.reset_stats()
            s.run_resident(vs, RunParams(lvl, False, False, 1, 2))
            times[t] = s.kernel_stats(_lib.PS_KERNEL_HALF)["ms"]
        be.close()
    best = min(times, key=times.get)
    res = {"tuning": best, "ms": {str(k): round(v, 3) for k, v in times.items()}, "key": key}
    if cache is not None:
        data = _load(cache)
        data[key] = res
        try:
            cache.write_text(json.dumps(data, indent=1))
        except OSError:
            pass
    return dict(res, cached=False)
