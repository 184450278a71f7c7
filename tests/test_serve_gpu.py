"""Continuous batching on the B200: requests of different sizes and
durations join and leave the running batch at step boundaries; each
result is bitwise the result of the same network run alone."""
import time

import numpy as np
import pytest

from astrosimgpu_b200 import _lib
from astrosimgpu_b200.network import Model, Network, Server, config_path
from astrosimgpu_b200.workloads import serving_config

pytestmark = pytest.mark.gpu


def alone(model, steps):
    n = Network(model, record=_lib.RecordOpts(0, 10, 1, 0, 0), chunk_steps=64)
    n.step(steps)
    sp = n.fetch_spikes()
    n.close()
    return sp


def test_requests_same_alone_and_in_mix():
    specs = [("quick", 1, 9000), ("use_case", 2, 15000), ("quick", 3, 4000),
             ("bursting", 4, 12000), ("use_case", 5, 7000)]
    models = [Model(config_path(n), seed=s, pre_time=0.0) for n, s, _ in specs]
    srv = Server(chunk_steps=64)
    ids = []
    for m, (_, _, steps) in zip(models, specs):
        ids.append(srv.submit(m, steps))
        time.sleep(0.02)  # staggered arrivals: later ones join a running batch
    res = [srv.wait(i, 60000.0) for i in ids]
    assert all(r.status == 0 for r in res)
    for i, (m, (_, _, steps)) in enumerate(zip(models, specs)):
        st, src = srv.fetch_spikes(ids[i])
        a_st, a_src = alone(m, steps)
        assert np.array_equal(st, a_st) and np.array_equal(src, a_src), i
        assert res[i].n_spikes == len(a_st)
        assert st.max(initial=0) < steps
    stats = srv.stats()
    assert stats["peak_resident"] >= 2 and stats["resident"] == 0
    srv.close()


def test_fixed_indegree_requests_and_latency_fields():
    srv = Server(chunk_steps=32)
    models = [Model(text=serving_config(n, 10 + n, 50.0), pre_time=0.0, fixed_indegree=100,
                    gen_device=0) for n in (500, 3000, 20000)]
    ids = [srv.submit(m, m.sim_steps, keep_spikes=False) for m in models]
    res = [srv.wait(i, 120000.0) for i in ids]
    for r, m in zip(res, models):
        assert r.status == 0
        assert r.submit_to_done_ms >= r.submit_to_admit_ms >= 0.0
        assert r.spike_edges >= 0 and r.sic_edges >= 0
    srv.close()


def test_admission_rejects_over_budget_and_cancel():
    small = Model(config_path("quick"), pre_time=0.0)
    big = Model(config_path("paper_sparse_dt005"), pre_time=0.0)
    srv = Server(mem_budget=64 << 20, chunk_steps=16)
    with pytest.raises(_lib.AsgError) as e:
        srv.submit(big, 100)
    assert e.value.status == 2  # ASG_ERR_OOM: alone it exceeds the budget
    rid = srv.submit(small, 10_000_000)  # long request, cancelled while running
    time.sleep(0.2)
    srv.cancel(rid)
    r = srv.wait(rid, 30000.0)
    assert r.status == 9  # ASG_ERR_CANCELLED
    rid2 = srv.submit(small, 200)
    assert srv.wait(rid2, 30000.0).status == 0
    srv.close()


def test_queued_staged_and_running_cancels_with_admission_thread():
    """Admission runs on its own thread: requests are prepared while the
    batch steps, wait for budget in arrival order, and can be cancelled in
    every state (queued, being admitted, staged, running).  Every request
    that finishes is bitwise its run alone."""
    quick = Model(config_path("quick"), pre_time=0.0)
    uc = Model(config_path("use_case"), seed=7, pre_time=0.0)
    srv = Server(chunk_steps=64, max_instances=3)  # the rest wait in the queue
    ids, want = [], []
    for k in range(12):
        m = quick if k % 2 else uc
        steps = 3000 + 500 * k
        ids.append(srv.submit(m, steps))
        want.append((m, steps))
    for k in (1, 6, 11):  # one early (likely running), two later (queued or staged)
        srv.cancel(ids[k])
    for k, rid in enumerate(ids):
        r = srv.wait(rid, 120000.0)
        if k in (1, 6, 11):
            assert r.status in (0, 9)  # it may have finished before the cancel landed
            continue
        assert r.status == 0, k
        st, src = srv.fetch_spikes(rid)
        a_st, a_src = alone(*want[k])
        assert np.array_equal(st, a_st) and np.array_equal(src, a_src), k
    assert srv.stats()["resident"] == 0
    srv.close()
