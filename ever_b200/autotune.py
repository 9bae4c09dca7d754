"""Autotuner for the trace launch configuration.

Tunables: the event buffer gathered per traversal round (kbuf 8/16/32), the block shape
(64/128/256 threads: 2/4/8 warp packets per block), the traversal (warp packets or one
walk per ray) and whether rays are reordered into coherent packets. The traversal stack
is one 64-entry stack per warp in shared memory (256 B), too small to be worth tuning.

Each candidate runs the caller's workload (one forward + backward) under CUDA events;
the fastest one that finishes without a status flag wins. Results are cached in a JSON
file keyed by GPU name, SH coefficients and power-of-two buckets of the ellipsoid and
ray counts.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import asdict, dataclass
from typing import Callable, Iterable

import torch

from .tracer import Tune


@dataclass
class Candidate:
    kbuf: int
    block: int
    traversal: int = 0
    ordered: bool = True

    def tune(self) -> Tune:
        return Tune(kbuf=self.kbuf, block=self.block, traversal=self.traversal)


DEFAULT_CANDIDATES = [Candidate(k, b, 0, True) for k in (8, 16, 32) for b in (64, 128, 256)] + [
    Candidate(16, 128, 0, False), Candidate(16, 128, 1, True)]


def default_cache_path() -> str:
    base = os.environ.get("EVER_B200_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "ever_b200"))
    return os.path.join(base, "autotune.json")


def workload_key(num_prims: int, num_rays: int, sh_coeffs: int, device=None) -> str:
    name = torch.cuda.get_device_name(device) if torch.cuda.is_available() else "cpu"
    b = lambda x: int(math.log2(max(int(x), 1)))
    return f"{name}|K{sh_coeffs}|N2^{b(num_prims)}|R2^{b(num_rays)}"


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(path, data):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def autotune(run: Callable[[Candidate], int], key: str, candidates: Iterable[Candidate] = DEFAULT_CANDIDATES,
             warmup: int = 1, reps: int = 2, cache_path: str | None = None, force: bool = False):
    """run(candidate) enqueues the workload on the current stream and returns the status
    word of the launch (0 = clean). Returns (best Candidate, {candidate: ms})."""
    cache_path = cache_path or default_cache_path()
    cache = _load(cache_path)
    if not force and key in cache:
        c = cache[key]
        return Candidate(c["kbuf"], c["block"], c["traversal"], c["ordered"]), c.get("timings", {})
    timings = {}
    best, best_ms = None, float("inf")
    for cand in candidates:
        name = f"k{cand.kbuf}-b{cand.block}-t{cand.traversal}-{'ord' if cand.ordered else 'idx'}"
        try:
            for _ in range(warmup):
                run(cand)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            status = 0
            for _ in range(reps):
                status |= int(run(cand))
            e1.record()
            torch.cuda.synchronize()
        except RuntimeError as e:  # a configuration the device rejects is skipped
            timings[name] = f"error: {e}"
            continue
        ms = e0.elapsed_time(e1) / reps
        timings[name] = ms if status == 0 else f"status {status}"
        if status == 0 and ms < best_ms:
            best, best_ms = cand, ms
    if best is None:
        best = Candidate(16, 128, 0, True)
    cache[key] = dict(asdict(best), ms=best_ms, timings=timings)
    _store(cache_path, cache)
    return best, timings
