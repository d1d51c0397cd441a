"""Autotuner for the launch shape of a reconstruction.

The per-plane kernels have compile-time tile shapes (chosen from the line length); what varies
with the problem is how many shots one launch covers: all shots in one launch keeps the GPU
full and amortises launches, while smaller batches keep the transformed volumes closer to L2
and need less workspace.  `tune(pb)` times one SENSE normal-operator application for each
candidate `batch` and one Gauss-Newton statistics call for each candidate `lm_batch` on the
actual problem (CUDA events on the current stream), keeps the fastest, and caches the choice
in a JSON file keyed by problem shape and GPU name, so later reconstructions of the same shape
start from it without timing again.

Cache file: $MOTIONEST_AUTOTUNE_CACHE, else ~/.cache/motionest/autotune.json.
"""
import json
import os
from pathlib import Path

import torch

from . import _lib

_CACHE = None


def cache_path():
    p = os.environ.get("MOTIONEST_AUTOTUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "motionest" / "autotune.json"


def _load():
    global _CACHE
    if _CACHE is None:
        try:
            _CACHE = json.loads(cache_path().read_text())
        except (OSError, ValueError):
            _CACHE = {}
    return _CACHE


def _store(cache):
    p = cache_path()
    try:
        p.parent.mkdir(parents=True, exist_ok=True)
        tmp = p.with_suffix(".tmp")
        tmp.write_text(json.dumps(cache, indent=1, sort_keys=True))
        os.replace(tmp, p)
    except OSError:
        pass  # a read-only home only costs re-tuning


def key_of(pb):
    X, Y, Z = pb.shape
    name = torch.cuda.get_device_name(pb.device)
    return f"{name}|{X}x{Y}x{Z}|C{pb.ncoils}|S{pb.nshots}|n{pb.samples.max_per_shot}"


def _candidates(n, top):
    out, b = [], top
    while b >= 1:
        if b not in out:
            out.append(b)
        b //= 2
    return [c for c in out if c <= n] or [1]


def _time(fn, reps=2):
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def tune(pb, force=False, budget_bytes=None):
    """Choose (batch, lm_batch) for the SenseProblem `pb`, set them on it and return them."""
    cache = _load()
    k = key_of(pb)
    if not force and k in cache:
        choice = cache[k]
        pb.set_batches(choice["batch"], choice["lm_batch"])
        return choice["batch"], choice["lm_batch"]
    lib = _lib.load()
    free, _ = torch.cuda.mem_get_info(pb.device)
    budget = budget_bytes if budget_bytes is not None else int(0.6 * free)
    x = torch.randn(pb.empty_image().shape, dtype=torch.complex64, device=pb.device)
    out = pb.empty_image()
    results = {"normal_ms": {}, "lm_ms": {}}
    best_b, best_t = None, None
    for b in _candidates(pb.nshots, pb.nshots):
        need = lib.me_sense_workspace_bytes(pb.ref, b)
        if need < 0 or need > budget + pb.work.numel():
            continue
        pb.set_batches(b, pb.lm_batch)
        t = _time(lambda: pb.normal(x, out))
        results["normal_ms"][b] = t
        if best_t is None or t < best_t:
            best_b, best_t = b, t
    best_l, best_lt = None, None
    for lb in _candidates(pb.nshots, 16):
        need = lib.me_lm_workspace_bytes(pb.ref, lb)
        if need < 0 or need > budget + pb.work.numel():
            continue
        pb.set_batches(best_b, lb)
        t = _time(lambda: pb.lm_stats(x, _lib.ME_JAC_REFERENCE), reps=1)
        results["lm_ms"][lb] = t
        if best_lt is None or t < best_lt:
            best_l, best_lt = lb, t
    best_b = best_b or 1
    best_l = best_l or 1
    pb.set_batches(best_b, best_l)
    cache[k] = {"batch": best_b, "lm_batch": best_l, "timings": results}
    _store(cache)
    return best_b, best_l
