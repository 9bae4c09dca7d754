"""Autotuner for the trace launch configuration.

Tunables: the event buffer (kbuf 8/16/32: gathered per round, and the frustum phase's
per-ray buffer), the block shape (64/128/256 threads: 2/4/8 warp packets per block), the
traversal (warp packets with the frustum phase, one walk per ray, or warp packets with
gather rounds only), the traversal stack depth (entries in use, 8..64) and whether rays are
reordered into coherent packets.

Each candidate runs the caller's workload (one forward + backward) under CUDA events;
the fastest one that finishes without a status flag wins: a stack too shallow for the
tree raises EVER_STATUS_STACK_OVERFLOW and is rejected. Results are cached in a JSON file
keyed by GPU name, SH coefficients and power-of-two buckets of the ellipsoid and ray
counts; trace_rays looks its workload's key up there (cached_tune) and runs the cached pick
when there is one.
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
    stack_depth: int = 64

    def tune(self) -> Tune:
        return Tune(kbuf=self.kbuf, block=self.block, traversal=self.traversal, stack_depth=self.stack_depth)

    def name(self) -> str:
        return (f"k{self.kbuf}-b{self.block}-t{self.traversal}-s{self.stack_depth}-"
                f"{'ord' if self.ordered else 'idx'}")


DEFAULT_CANDIDATES = ([Candidate(k, b, 0, True) for k in (8, 16, 32) for b in (64, 128, 256)] +
                      [Candidate(16, 128, 2, True), Candidate(16, 128, 0, False), Candidate(16, 128, 1, True)] +
                      [Candidate(16, 128, 0, True, d) for d in (16, 24, 32, 48)])


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
        return _from_entry(cache[key]), cache[key].get("timings", {})
    timings = {}
    best, best_ms = None, float("inf")
    for cand in candidates:
        name = cand.name()
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


def _from_entry(c) -> Candidate:
    return Candidate(c["kbuf"], c["block"], c["traversal"], c["ordered"], c.get("stack_depth", 64))


def cached_tune(num_prims: int, num_rays: int, sh_coeffs: int, device=None, cache_path: str | None = None):
    """The cached pick for this workload's key (no timing run), or None."""
    entry = _load(cache_path or default_cache_path()).get(workload_key(num_prims, num_rays, sh_coeffs, device))
    return _from_entry(entry) if entry else None
