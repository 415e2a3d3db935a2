"""Launch-shape autotuner for batched PatchMatch runs (no reference counterpart).

Times each candidate tuning (thread-block shape, lanes per pixel, persistent
launch or one launch per stage) on the caller's batch with device events and
keeps the fastest.  Results do not depend on the choice (scores agree to the
float rounding of the NCC sums), only the time does.  Decisions are cached in
``opensfm_b200/_build/autotune.json`` keyed by the workload's shape.
"""
from __future__ import annotations

import json
import os
import statistics
from typing import Dict, List, Sequence, Tuple

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE = os.path.join(HERE, "_build", "autotune.json")

# (bx, by, variant): variant = lanes per pixel (1, 2, 4, 8) + 16 for the
# persistent launch.
CANDIDATES: List[Tuple[int, int, int]] = [
    (32, 4, 4), (32, 4, 20), (32, 4, 8), (64, 2, 4), (32, 2, 4), (32, 4, 2), (32, 4, 18),
    (32, 4, 1),
]


def workload_key(shapes: Sequence[Tuple[int, int]], n_views: Sequence[int], patch: int) -> str:
    """A key from the depthmap sizes and matching-view counts (order-free)."""
    sig = sorted(f"{h}x{w}v{n}" for (h, w), n in zip(shapes, n_views))
    counts: Dict[str, int] = {}
    for s in sig:
        counts[s] = counts.get(s, 0) + 1
    return f"v2:p{patch}:" + ",".join(f"{k}*{v}" for k, v in sorted(counts.items()))


def _load() -> dict:
    try:
        with open(CACHE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(d: dict) -> None:
    os.makedirs(os.path.dirname(CACHE), exist_ok=True)
    with open(CACHE, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)


def tune(batch, key: str, run_kwargs: dict, candidates=CANDIDATES, repeats: int = 2,
         use_cache: bool = True) -> dict:
    """Picks the fastest candidate for `batch` and leaves it set.

    run_kwargs are passed to ``batch.run`` (e.g. prune=True, graph=True).
    Returns {"choice": (bx, by, variant), "ms": {candidate: ms}, "cached": bool}.
    """
    cache = _load() if use_cache else {}
    if key in cache:
        c = tuple(cache[key]["choice"])
        batch.set_tuning(*c)
        return {"choice": c, "ms": cache[key]["ms"], "cached": True}
    times = {}
    for c in candidates:
        try:
            batch.set_tuning(*c)
            batch.run(**run_kwargs)  # warm-up / graph capture
            batch.synchronize()
            ts = []
            for _ in range(repeats):
                batch.timer_record(0)
                batch.run(**run_kwargs)
                batch.timer_record(1)
                batch.synchronize()
                ts.append(batch.timer_elapsed())
            times[c] = statistics.median(ts)
        except (ValueError, RuntimeError) as e:  # a shape the batch cannot use
            times[c] = float("inf")
    best = min(times, key=times.get)
    batch.set_tuning(*best)
    res = {"choice": best, "ms": {f"{c[0]},{c[1]},{c[2]}": t for c, t in times.items()},
           "cached": False}
    if use_cache:
        cache[key] = {"choice": list(best), "ms": res["ms"]}
        _store(cache)
    return res
