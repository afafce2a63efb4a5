"""Launch-shape tuner for batches of find_HII_bubbles snapshots (rg_find_HII_bubbles_batch).

For one workload shape -- GPU, ReionGridDim, grids per snapshot, snapshots, radii -- it times
every candidate (radii per batch, snapshots per call) on the caller's own grids and keeps the
fastest in a JSON cache next to this file (``tuning_cache.json``), so later runs of the same shape
on the same GPU model start from the tuned values.  The reference's counterpart is FFTW's plan
wisdom, imported and exported around its plans (src/core/reionization.c:726-758).

The tuned values change only how the work is launched: every candidate gives each snapshot the
same results (rg_find_HII_bubbles_batch equals one call per snapshot, and the radius batch only
regroups radii).
"""

from __future__ import annotations

import json
import os
import statistics
import time

CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning_cache.json")
RADIUS_BATCHES = (4, 8, 16)


def shape_key(gpu: str, n: int, grids: int, units: int, radii: int) -> str:
    return f"{gpu}|N={n}|grids={grids}|units={units}|radii={radii}"


def load(path: str = CACHE) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def store(entries: dict, path: str = CACHE) -> bool:
    """Merge entries into the cache; False (nothing kept) where the file cannot be written."""
    cur = load(path)
    cur.update(entries)
    tmp = path + ".tmp"
    try:
        with open(tmp, "w") as f:
            json.dump(cur, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        return False
    return True


def candidates(units: int) -> list[tuple[int, int]]:
    """(radii per batch, snapshots per call): every radius batch with all the snapshots in one
    call, half of them, a quarter, and one at a time."""
    per_call = sorted({units, max(1, units // 2), max(1, units // 4), 1}, reverse=True)
    return [(kb, u) for kb in RADIUS_BATCHES for u in per_call]


def tune(run, sync, units: int, reps: int = 3, clock=time.perf_counter) -> tuple[tuple[int, int], dict]:
    """run(kb, per_call) runs the whole workload once with that launch shape; sync() waits for the
    device.  Each candidate runs once untimed, then `reps` times; the fastest median wins."""
    times = {}
    for kb, per_call in candidates(units):
        run(kb, per_call)
        sync()
        ts = []
        for _ in range(reps):
            t0 = clock()
            run(kb, per_call)
            sync()
            ts.append(clock() - t0)
        times[(kb, per_call)] = statistics.median(ts)
    best = min(times, key=times.get)
    return best, {f"kb={k[0]},per_call={k[1]}": v * 1e3 for k, v in times.items()}


def tuned(key: str, run, sync, units: int, path: str = CACHE, clock=time.perf_counter) -> tuple[int, int]:
    """The cached launch shape of this key, tuned and stored first when absent."""
    entry = load(path).get(key)
    if entry is not None:
        return int(entry["radius_batch"]), int(entry["per_call"])
    (kb, per_call), ms = tune(run, sync, units, clock=clock)
    store({key: {"radius_batch": kb, "per_call": per_call, "ms": ms}}, path)
    return kb, per_call
