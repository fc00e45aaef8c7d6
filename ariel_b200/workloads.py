"""Synthetic scene sets of the benchmark configurations (seeded; no dataset is involved).

- ``dambreak(n)``: liquid block x in [0,.4], y in [0,.6], z in [0,1], 8 particles per cell
  (lattice density 0.5) jittered inside their sub-cells, gravity -9.8 y, dt 1/240.
- ``sphere_dambreak(n)``: liquid block x in [0,.35], y in [0,.5], z in [0,1] with a static
  solid sphere of centre (.6,.3,.5) and radius .15, dt 1/480; the benchmark steps it with
  resampling and reseeding (6-10 particles per cell) every 5th step.
- ``uneven_batch(k, seed)``: k scenes with grid sizes drawn from {32,48,64,96,128} and one
  liquid block each filling 20-50% of its domain.
- ``arrival_stream(rate, duration, seed)``: Poisson arrivals (exponential gaps of mean
  1/rate s) of scenes with grid sizes uniform in [48,192] and blocks as in ``uneven_batch``.

A liquid block with fill fraction f starts at the origin, spans the full z extent, has a
height hy drawn uniformly in [.4,.8] and a width hx = f/hy (at most .95).
"""
import numpy as np

from . import _abi as A

BATCH_SIZES = (32, 48, 64, 96, 128)


def dambreak(n, seed=1):
    return A.scene_dambreak(n, liquid_hi=(0.4, 0.6, 1.0), seed=seed)


def sphere_dambreak(n, seed=1):
    return A.scene_dambreak(n, liquid_hi=(0.35, 0.5, 1.0), dt=1.0 / 480.0, seed=seed,
                            spheres=[((0.6, 0.3, 0.5), 0.15)])


def _block(rng):
    f = rng.uniform(0.2, 0.5)
    hy = rng.uniform(0.4, 0.8)
    hx = min(0.95, f / hy)
    return (float(hx), float(hy), 1.0)


def uneven_batch(k=64, seed=7):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(k):
        n = int(rng.choice(BATCH_SIZES))
        out.append(A.scene_dambreak(n, liquid_hi=_block(rng), seed=seed * 1000 + i + 1))
    return out


def arrival_stream(rate=20.0, duration_s=120.0, seed=11, n_lo=48, n_hi=192):
    """[(arrival time s, scene)] over `duration_s` seconds."""
    rng = np.random.default_rng(seed)
    t, out, i = 0.0, [], 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration_s:
            return out
        n = int(rng.integers(n_lo, n_hi + 1))
        out.append((t, A.scene_dambreak(n, liquid_hi=_block(rng), seed=seed * 100000 + i + 1)))
        i += 1
