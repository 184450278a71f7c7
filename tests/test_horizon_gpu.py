"""Parity over the whole benchmarked runs, with the horizons measured on a
B200 stated here.

Rasters: the GPU engine's raster is compared spike for spike with the
reference simulator's own raster of the same run (tests/golden/
raster_<config>.npz, made by tests/golden/make_rasters.py from the reference
built from its sources), from step 0, transient included:

  config               steps (dt)              stated raster horizon
  quick                 25,000 (0.1 ms)        identical for the whole run
  use_case             300,000 (0.1 ms)        identical for the whole run
  bursting             300,000 (0.1 ms)        identical for the whole run
  c0_literal           100,000 (0.1 ms)        identical for the whole run
  paper_sparse_dt005    20,000 (0.05 ms)       identical for the whole run
                       (78,568 spikes; the SIC steady state, every
                       astrocyte above threshold, from step ~16,000 on)

State: GPU and reference advance side by side and the full state (V, w,
g_ex, dg_ex, g_in, dg_in, I_sic, Ca, IP3, h; refractory counters exactly) is
compared every `every` steps with |gpu - ref| <= tol * max(|ref|, 1e-3).
The one source of difference is the last bit of CUDA's exp/log/cos against
the host libm on data-dependent arguments (AdEx spike current, STP decay,
SIC factor, Box-Muller).  Those differences do not grow: they appear as
short bursts while a neuron's potential runs up to the spike peak (the
exponential term amplifies a last-bit difference) and vanish at its reset.
Measured on a B200, the first comparison above 1e-12 came at
  quick: never (max 2e-15)           use_case: step ~163,000
  bursting: step ~165,000            c0_literal: step 65,000 (max 5.1e-11)
  paper_sparse_dt005: step 650 (max 1.6e-12, back to 3e-14 by step 20,000)
so each config asserts 1e-12 up to its stated state horizon and 1e-10 over
the rest of the compared span.
"""
import json

import numpy as np
import pytest

from astrosimgpu_b200 import _lib
from astrosimgpu_b200.network import Batch, Model, Network, Server, config_path
from astrosimgpu_b200.workloads import serving_config
from oracle import ref

pytestmark = pytest.mark.gpu

KEYS = ("V", "w", "g_ex", "dg_ex", "g_in", "dg_in", "I_sic", "Ca", "IP3", "h")
TIGHT = 1e-12
BURST = 1e-10

# name: (state horizon at 1e-12 in steps, steps compared side by side, every)
STATE = {
    "quick": (25_000, 25_000, 250),
    "use_case": (160_000, 300_000, 2000),
    "bursting": (160_000, 300_000, 2000),
    "c0_literal": (64_000, 100_000, 1000),
    "paper_sparse_dt005": (600, 2_000, 50),
}


def rec_all():
    return _lib.RecordOpts(0, 10, 1, 0, 0)


def golden(name):
    import os
    return np.load(os.path.join(os.path.dirname(__file__), "golden", f"raster_{name}.npz"))


def model_of(name, gold):
    sim = float(gold["sim_time_ms"])
    return Model(config_path(name), sim_time=sim)


def first_difference(gs, gsrc, rs, rsrc):
    n = min(len(gs), len(rs))
    bad = np.nonzero((gs[:n] != rs[:n]) | (gsrc[:n] != rsrc[:n]))[0]
    if len(bad):
        return int(min(gs[bad[0]], rs[bad[0]]))
    if len(gs) != len(rs):
        return int(gs[n] if len(gs) > n else rs[n])
    return None


def max_rel(a, b):
    worst = 0.0
    for k in KEYS:
        if len(a[k]):
            d = np.abs(a[k] - b[k]) / np.maximum(np.abs(b[k]), 1e-3)
            worst = max(worst, float(d.max()))
    assert np.array_equal(a["refractory"], b["refractory"])
    return worst


@pytest.mark.parametrize("name", list(STATE))
def test_whole_run_raster_identical(name):
    gold = golden(name)
    m = model_of(name, gold)
    total = int(gold["total_steps"])
    assert m.pre_steps + m.sim_steps == total
    g = Network(m, record=rec_all())
    g.step(total)
    gs, gsrc = g.fetch_spikes()
    first = first_difference(gs, gsrc, gold["steps"].astype(np.int64), gold["sources"])
    assert first is None, f"{name}: rasters differ from step {first} of {total}"
    assert len(gs) == len(gold["steps"]) > 0
    # windowed statistics follow (identical rasters make them equal)
    w = int(gold["window"])
    counts = np.bincount(gs // w, minlength=len(gold["win_spikes"]))
    assert np.array_equal(counts, gold["win_spikes"])
    g.close()


@pytest.mark.parametrize("name", list(STATE))
def test_state_side_by_side(name):
    horizon, span, every = STATE[name]
    gold = golden(name)
    m = model_of(name, gold)
    g = Network(m, record=rec_all())
    r = ref.RefNetwork(path=config_path(name), sim_time=float(gold["sim_time_ms"]))
    step = 0
    worst_tight = worst_all = 0.0
    while step < span:
        g.step(every)
        r.run(every)
        step += every
        e = max_rel(g.state(), r.state())
        worst_all = max(worst_all, e)
        if step <= horizon:
            worst_tight = max(worst_tight, e)
    assert worst_tight <= TIGHT, (name, worst_tight)
    assert worst_all <= BURST, (name, worst_all)
    g.close()


def serving_models(sizes=(20000, 20000, 15000, 12000), seconds=1.0):
    texts = [serving_config(n, 100 + i, seconds * 1000.0) for i, n in enumerate(sizes)]
    models = [Model(text=t, pre_time=0.0, fixed_indegree=100, gen_device=0) for t in texts]
    refs = []
    for t, m in zip(texts, models):
        c = json.loads(t)
        c["connectivity"]["p_primary"] = 0.0  # the tables come from the product's generator
        r = ref.RefNetwork(text=json.dumps(c))
        for which in range(4):
            rs, tg = m.table(which)
            r.load_table(which, rs, tg)
        refs.append(r)
    return models, refs


def test_serving_shapes_against_reference_on_the_same_tables():
    """Fixed-in-degree networks (in-degree 100, N_A = N, the serving
    stream's shape) from the product's counter-based generator, loaded into
    the reference simulator as its connection sets.  Four of them in one
    batch of 67,000 neurons run the forms used at serving scale (the
    high-occupancy kernel, the SIC summed in the neuron role); the same four
    go through the serving loop as requests.  Over 3,000 steps (0.3 s) every
    raster is identical to the reference's, in the batch and in the server;
    the batch's state stays within 1e-10 (measured max 8e-13)."""
    steps, every = 3000, 100
    models, refs = serving_models()
    b = Batch(models, record=rec_all())
    rsp = [[] for _ in refs]
    worst = 0.0
    for _ in range(steps // every):
        b.step(every)
        for i, r in enumerate(refs):
            rsp[i].append(r.run(every))
        for i, r in enumerate(refs):
            worst = max(worst, max_rel(b.state(i), r.state()))
    assert worst <= BURST, worst
    rasters = []
    for i in range(len(refs)):
        gs, gsrc = b.fetch_spikes(i)
        rs = np.concatenate([x[0] for x in rsp[i]])
        rsrc = np.concatenate([x[1] for x in rsp[i]])
        assert first_difference(gs, gsrc, rs, rsrc) is None, i
        assert len(rs) > 0
        rasters.append((rs, rsrc))
    b.close()
    srv = Server()
    ids = [srv.submit(m, steps, keep_spikes=True) for m in models]
    for i, rid in enumerate(ids):
        res = srv.wait(rid, 120000.0)
        assert res.status == 0
        st, src = srv.fetch_spikes(rid)
        assert first_difference(st, src, *rasters[i]) is None, i
    srv.close()
