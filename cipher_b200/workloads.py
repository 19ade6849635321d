"""Seeded synthetic workloads with the shapes of the reference's benchmark
configurations (no dataset exists; the reference ships none).

* alloy_2d:     a CALPHAD two-sublattice alloy, 4 components (3 solutes and a
                vacancy-like balance), two matrix grains with 20
                precipitates, cap 15 (the chemistry configuration, on a
                uniform 512^2 grid instead of an adaptive one)
* batch_domains: 256 independent 2D grain-growth domains, side 2^U[5,8]
                 rounded to a multiple of 32, 8-128 grains each (at most one
                 per ~128 cells, so that no junction exceeds the cap of 8),
                 per-domain seeds (the batched configuration)
* serving_trace: Poisson arrivals of a mix of grain-growth jobs and binary
                 two-phase alloy jobs of 64^2-256^2 cells (the serving
                 configuration, over a shortened window)
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .api import Problem


def alloy_2d(res=(512, 512), seed: int = 2024) -> Problem:
    return Problem.alloy(2, list(res), "calphad2sl", 4, 20, 15, seed, 0)


def batch_domains(n: int = 256, seed: int = 7):
    """[(res, grains, seed)] of the batched configuration"""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        side = int(round(2.0 ** rng.uniform(5.0, 8.0) / 32.0)) * 32
        side = max(32, min(256, side))
        grains = int(rng.integers(8, 129))
        grains = min(grains, max(8, side * side // 128))    # grains of >= ~128 cells
        out.append(([side, side], grains, int(seed * 100003 + k)))
    return out


def batch_problem(spec, cap: int = 8) -> Problem:
    res, grains, s = spec
    return Problem.grain_growth(2, res, grains, cap, s)


def serving_trace(rate: float = 50.0, duration: float = 4.0, seed: int = 11):
    """[(arrival_s, kind, args, init, t_end)]: Poisson(rate) arrivals over
    `duration` seconds; 3 in 4 jobs grain growth (64^2-256^2, 16-64 grains
    with at least ~128 cells per grain, cap 8, to t = 5), 1 in 4 binary
    two-phase alloys (calphaddis, 64^2 or 128^2, 4 seeded particles, cap 8,
    to t = 0.02)"""
    rng = np.random.default_rng(seed)
    t, out, k = 0.0, [], 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        if rng.uniform() < 0.75:
            side = int(rng.choice([64, 128, 256], p=[0.5, 0.35, 0.15]))
            args = ([side, side], min(int(rng.integers(16, 65)), side * side // 128), 8, int(seed * 7919 + k))
            out.append((t, "gg", args, "sharp", 5.0))
        else:
            side = int(rng.choice([64, 128]))
            args = ([side, side], "calphaddis", 2, 4, 8, int(seed * 7919 + k), 0)
            out.append((t, "alloy", args, "sharp", 0.02))
        k += 1
    return out


def trace_problem(kind: str, args) -> Problem:
    if kind == "gg":
        res, ng, cap, s = args
        return Problem.grain_growth(2, res, ng, cap, s)
    res, model, ncp, npr, cap, s, feats = args
    return Problem.alloy(2, res, model, ncp, npr, cap, s, feats)


def ts_opts_for(problem: Problem, **kw) -> L.TSOpts:
    from .api import ts_options
    return ts_options(problem, "2a", **kw)
