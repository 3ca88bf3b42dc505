"""Project autotuner of the batched engine's execution choices.

The batched form (include/bsam_batch.h) has knobs that change how work is
mapped onto the B200 but not a single result bit (bsam_batch_tuning):

  per_pass    sweep fusion: 0 = every 2D level above the bottom smooths with
              the fused shared-memory stage (all 2*nu colour passes of
              LevelRelax in one launch), 1 = one launch per colour pass
  fused_occ   the fused stage's build: 3 or 4 resident CTAs per SM with one
              tile buffer each (85 or 64 registers per thread), or 2 CTAs per
              SM with two buffers each (the next tile's copies land while the
              current one is computed)
  fused_ctas  CTAs of a fused-stage launch (persistent loop over the stage's
              tiles)
  fused_chunk runs of consecutive tiles a fused-stage CTA takes at a time
  grid_ctas   CTAs of every other stage launch
  tile_chunk  runs of consecutive tiles a CTA of those launches takes at a
              time (a run's tiles mostly share one problem's records)

The tuner times candidates on a sample of the caller's workload with CUDA
events on the engine's stream (a few V-cycle ticks of every sampled problem,
after one warm-up tick), walks the knobs one at a time from the default
(coordinate descent: each knob's best value is kept before the next knob is
searched; the fused stage's build comes first, so that sweep fusion is
judged with its best build), and caches the winner per (GPU, precision, workload class) in a
JSON file.  Results are the same under every candidate;
tests/test_gpu_autotune.py checks that on the GPU.
"""
from __future__ import annotations

import dataclasses
import json
import os
import time

from . import batch as BB

# Search order: the fused stage's build before sweep fusion, so that fusion is
# judged with the fused stage's best build.
KNOBS = ("fused_occ", "per_pass", "fused_ctas", "fused_chunk", "grid_ctas", "tile_chunk")


@dataclasses.dataclass(frozen=True)
class Choice:
    per_pass: int = 0
    fused_occ: int = 0
    fused_ctas: int = 0
    grid_ctas: int = 0
    tile_chunk: int = 0
    fused_chunk: int = 0

    def as_dict(self) -> dict:
        return dataclasses.asdict(self)


def candidates(knob: str, nsm: int) -> list:
    """Values searched for one knob (0 = the engine's default)."""
    if knob == "per_pass":
        return [0, 1]
    if knob == "fused_occ":
        return [2, 3, 4]
    if knob == "fused_ctas":
        return [0, 2 * nsm, 3 * nsm, 8 * nsm]
    if knob == "grid_ctas":
        return [0, 4 * nsm, 8 * nsm, 32 * nsm]
    if knob == "tile_chunk":
        return [0, 1, 4]
    if knob == "fused_chunk":
        return [0, 2]

    raise ValueError(knob)


def workload_class(problems) -> str:
    """Key of a workload: its dimensionality and the sorted set of its root
    sides (a served stream or another batch of the same sizes shares it)."""
    nd = problems[0].ndims
    sides = sorted({int(p.mx[0]) for p in problems})
    return f"{nd}d:" + ",".join(str(s) for s in sides)


def stratified(problems, per_side: int) -> list:
    """The first `per_side` problems of each root side, in workload order."""
    out = []
    for side in sorted({int(p.mx[0]) for p in problems}):
        out += [p for p in problems if int(p.mx[0]) == side][:per_side]
    return out


def _pool_for(problems, precision: int) -> int:
    nd = problems[0].ndims
    with BB.Batch(nd, precision=precision, max_slots=1, pool_bytes=1 << 20) as probe:
        need = sum(probe.footprint(p) for p in problems)
    return int(need * 1.25) + (64 << 20)


def time_choice(problems, precision: int, choice: Choice, ticks: int = 3, reps: int = 2,
                device: int = 0) -> float:
    """Milliseconds of `ticks` V-cycle ticks of every problem under `choice`
    (CUDA events on the engine's stream; best of `reps` fresh engines)."""
    import torch
    best = float("inf")
    nd = problems[0].ndims
    pool = _pool_for(problems, precision)
    for _ in range(reps):
        with BB.Batch(nd, precision=precision, max_slots=len(problems), pool_bytes=pool,
                      device=device, qerrortol=problems[0].qerrortol) as b:
            b.set_tuning(**choice.as_dict())
            for p in problems:
                if b.submit_seeded(p) is None:
                    raise RuntimeError("the tuning sample does not fit its pool")
            b.advance(1)  # warm-up tick (also captures the tick graph)
            b.sync()
            stream = torch.cuda.ExternalStream(b.stream(), device=device)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.advance(ticks)
            e1.record(stream)
            b.sync()
            best = min(best, e0.elapsed_time(e1))
    return best


def search(problems, precision: int, timer=None, nsm: int | None = None,
           device: int = 0) -> dict:
    """Coordinate descent over KNOBS from the default choice.  `timer(choice)`
    returns milliseconds (default: time_choice on `problems`).  Returns the
    best choice, its time, the default's time and every timing taken."""
    if nsm is None:
        import torch
        nsm = torch.cuda.get_device_properties(device).multi_processor_count
    if timer is None:
        def timer(c):
            return time_choice(problems, precision, c, device=device)
    seen = {}

    def t(c):
        if c not in seen:
            seen[c] = timer(c)
        return seen[c]

    best = Choice()
    base = t(best)
    for knob in KNOBS:
        for v in candidates(knob, nsm):
            c = dataclasses.replace(best, **{knob: v})
            if t(c) < t(best):
                best = c
    return {"choice": best.as_dict(), "ms": t(best), "default_ms": base,
            "gain": base / t(best),
            "timings": [{"choice": c.as_dict(), "ms": ms} for c, ms in seen.items()]}


def cache_path() -> str:
    return os.environ.get("BSAM_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "bsam_b200",
                                       "tuning.json"))


def _key(gpu: str, precision: int, wclass: str) -> str:
    return f"{gpu}|{'mixed' if precision == BB.PREC_MIXED else 'fp64'}|{wclass}"


def load_cache(path: str | None = None) -> dict:
    try:
        with open(path or cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def store(key: str, entry: dict, path: str | None = None) -> None:
    path = path or cache_path()
    data = load_cache(path)
    data[key] = entry
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tuned_choice(problems, precision: int, device: int = 0, per_side: int = 16,
                 retune: bool = False, path: str | None = None) -> dict:
    """The cached choice for this GPU, precision and workload class, or a new
    search on a stratified sample of `problems` (stored in the cache)."""
    import torch
    gpu = torch.cuda.get_device_name(device)
    key = _key(gpu, precision, workload_class(problems))
    if not retune:
        hit = load_cache(path).get(key)
        if hit is not None:
            return dict(hit, cached=True, key=key)
    sample = stratified(problems, per_side)
    t0 = time.perf_counter()
    res = search(sample, precision, device=device)
    res["tuning_s"] = time.perf_counter() - t0
    res["sample"] = f"{len(sample)} problems ({per_side} per side), 3 ticks per candidate"
    store(key, res, path)
    return dict(res, cached=False, key=key)
