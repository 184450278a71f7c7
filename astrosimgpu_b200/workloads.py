"""Synthetic workloads of the benchmark shapes (no external data is used).

- ``sweep_configs``: the batched sweep -- 64 instances of the use_case
  architecture with uneven sizes N in {250, 500, 1000, 2000, 4000} (round
  robin), N_A = N/5, 80/20 E/I, the IP3 weight w_n2a swept over 8 values in
  [0.20, 0.31] crossed with 8 seeds; p_primary = 0.2*500/N keeps the
  in-degree of the 500-neuron model; dt 0.1 ms.
- ``request_stream``: the serving stream -- Poisson arrivals (mean rate
  20/s), N drawn log-uniformly in [500, 200000], N_A = N, in-degree 100
  (the counter-based fixed-in-degree generator), duration U(0.2, 2) s,
  dt 0.1 ms; optionally one 1M/1M request.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from .network import CONFIG_DIR


def base_config(name="use_case") -> dict:
    with open(os.path.join(CONFIG_DIR, name + ".json")) as f:
        return json.load(f)


def sweep_configs(n_instances=64, sim_time_ms=5000.0, sizes=(250, 500, 1000, 2000, 4000),
                  weights=None, seeds=None):
    """JSON texts of the batched-sweep instances."""
    weights = list(np.linspace(0.20, 0.31, 8)) if weights is None else list(weights)
    seeds = list(range(1, 9)) if seeds is None else list(seeds)
    out = []
    base = base_config("use_case")
    for i in range(n_instances):
        w = weights[(i // len(seeds)) % len(weights)]
        s = seeds[i % len(seeds)]
        n = sizes[i % len(sizes)]
        c = json.loads(json.dumps(base))
        c["N"] = {"N_A": n // 5, "N_E": n * 4 // 5, "N_I": n - n * 4 // 5}
        c["connectivity"]["p_primary"] = 0.2 * 500.0 / n
        c["synapse"]["w_n2a"] = float(w)
        c["simulation"].update({"seed": s, "pre_sim_time": 0, "sim_time": sim_time_ms,
                                "record_astro": False, "record_spikes": True})
        out.append(json.dumps(c))
    return out


def serving_config(n: int, seed: int, sim_time_ms: float) -> str:
    c = base_config("use_case")
    c["N"] = {"N_A": n, "N_E": n * 4 // 5, "N_I": n - n * 4 // 5}
    c["connectivity"].update({"p_third_if_primary": 0.2, "pool_size": 1, "pool_type": "block"})
    c["simulation"].update({"seed": seed, "pre_sim_time": 0, "sim_time": sim_time_ms,
                            "record_astro": False})
    return json.dumps(c)


def request_stream(n_requests=40, rate_hz=20.0, n_min=500, n_max=200_000, t_min_s=0.2,
                   t_max_s=2.0, seed=7, big=False):
    """[(arrival_s, n_neurons, sim_time_ms, seed)] of the serving stream."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate_hz)
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        n = max(10, n)
        dur = rng.uniform(t_min_s, t_max_s) * 1000.0
        out.append((t, n, dur, 100 + i))
    if big:
        out.append((t + rng.exponential(1.0 / rate_hz), 1_000_000, 200.0, 99))
    return out
