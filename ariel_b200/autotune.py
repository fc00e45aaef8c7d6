"""Autotuner for the pressure solve's launch shape.

Two knobs change how fast the solve runs but not what it computes (every reduction and every
cell update is fixed by the scene alone, so results are bit-identical across settings):

- ``pcg_blocks_per_sm``: blocks per SM of the persistent solve kernels (1 or 2).  More blocks
  hide more memory latency; fewer blocks make every grid barrier cheaper.
- ``sweep_brick``: the brick of the ordered wavefront sweeps (MIC(0), and the reference
  preconditioner's PRef == 1 path).  Bigger bricks mean fewer dependent brick levels but more
  dependent levels inside each brick.

``tune(descs, params)`` times a few steps of the given scene set for every candidate and
returns a copy of ``params`` with the fastest setting, plus a report.  Results are cached in a
JSON file keyed by device, scene signature, precision and preconditioner
(``ARIEL_TUNE_CACHE``, default ``~/.cache/ariel_b200/tune.json``).
"""
import ctypes as C
import hashlib
import json
import os

from . import _abi as A

BLOCKS_PER_SM = (1, 2)
BRICKS = ((12, 12, 12), (8, 16, 16), (16, 16, 8), (8, 8, 32), (16, 8, 16), (6, 12, 24), (10, 10, 10), (8, 8, 16))


def brick_ok(b):
    """The library's limits on a sweep brick (shared-memory boxes of the general solve kernel)."""
    bx, by, bz = b
    return (1 <= bx <= 31 and 1 <= by <= 31 and 1 <= bz <= 63 and bx * by * bz <= 2048
            and (bx + 1) * (by + 1) * (bz + 1) <= 2744 and bx + by + bz - 2 <= 128)


def _copy_params(p):
    q = A.AsimParams()
    C.pointer(q)[0] = p
    return q


def _signature(descs, params):
    h = hashlib.sha1()
    for d in descs:
        h.update(bytes(d))
    for name in ("precision", "precond", "stop_rule", "tol", "resample_every"):
        h.update(repr(getattr(params, name)).encode())
    return h.hexdigest()[:16]


def _device_name():
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(0)
    except Exception:
        pass
    return "unknown"


def _cache_path():
    return os.environ.get("ARIEL_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "ariel_b200",
                                                           "tune.json"))


def _load_cache():
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store_cache(cache):
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    except OSError:
        pass


def candidates(params):
    """Settings worth timing for these parameters."""
    out = []
    for bps in BLOCKS_PER_SM:
        if params.precond == A.PRECOND_MIC0:
            for b in BRICKS:
                if brick_ok(b):
                    out.append((bps, b))
        else:
            out.append((bps, tuple(params.sweep_brick)))
    return out


def time_solve(descs, params, steps=2, warmup=1):
    """Mean device ms of the solve stage over `steps` steps after `warmup` steps from Init."""
    from .flipsim import Batch
    p = _copy_params(params)
    p.timing = 1
    b = Batch(list(descs), p)
    try:
        b.init()
        b.step(warmup)
        b.synchronize()
        b.timing_reset()
        b.step(steps)
        t = b.timing(max_steps=steps)
        return float(t["stage_ms"][A.STAGE_SOLVE]) / max(t["steps"], 1)
    finally:
        b.close()


def tune(descs, params, steps=2, warmup=1, use_cache=True):
    """Returns (tuned params, report).  The report lists every candidate's solve time."""
    descs = list(descs)
    key = "%s|%s" % (_device_name(), _signature(descs, params))
    cache = _load_cache() if use_cache else {}
    best = None
    report = {"key": key, "cached": False, "timings": []}
    if key in cache:
        best = (cache[key]["pcg_blocks_per_sm"], tuple(cache[key]["sweep_brick"]))
        report["cached"] = True
        report["timings"] = cache[key].get("timings", [])
    else:
        best_ms = None
        for bps, brick in candidates(params):
            p = _copy_params(params)
            p.pcg_blocks_per_sm = bps
            p.sweep_brick[:] = brick
            ms = time_solve(descs, p, steps, warmup)
            report["timings"].append({"pcg_blocks_per_sm": bps, "sweep_brick": list(brick), "solve_ms": ms})
            if best_ms is None or ms < best_ms:
                best_ms, best = ms, (bps, brick)
        if use_cache:
            cache[key] = {"pcg_blocks_per_sm": best[0], "sweep_brick": list(best[1]), "timings": report["timings"]}
            _store_cache(cache)
    out = _copy_params(params)
    out.pcg_blocks_per_sm = best[0]
    out.sweep_brick[:] = best[1]
    report["chosen"] = {"pcg_blocks_per_sm": best[0], "sweep_brick": list(best[1])}
    return out, report
