"""The whole per-timestep path on the B200 against the reference simulator
built from its own sources (oracle/_ref), on the same config and seed.

Parity bar (stated tolerances):
- spike rasters identical over the horizon run here;
- state within 1e-12 relative (|a-b| <= 1e-12 * max(|b|, 1e-3)) over the
  same horizon.  Arithmetic is evaluated in the reference's order without
  contraction; the only source of difference is the last bit of CUDA's
  exp/log/cos against the host libm on data-dependent arguments.
"""
import json

import numpy as np
import pytest

from astrosimgpu_b200 import _lib
from astrosimgpu_b200.network import Batch, Model, Network, config_path
from oracle import ref

pytestmark = pytest.mark.gpu

REL = 1e-12
STATE_KEYS = ("V", "w", "g_ex", "dg_ex", "g_in", "dg_in", "I_sic", "Ca", "IP3", "h")


def rec_all():
    return _lib.RecordOpts(0, 10, 1, 0, 0)


def run_pair(path=None, text=None, steps=1000, chunks=1, **opts):
    m = Model(path=path, text=text, pre_time=0.0)
    g = Network(m, record=rec_all(), **opts)
    r = ref.RefNetwork(path=path, text=text, pre_time=0.0)
    per = steps // chunks
    for _ in range(chunks):
        g.step(per)
    gs, gsrc = g.fetch_spikes()
    rs, rsrc = r.run(per * chunks)
    return g, r, (gs, gsrc), (rs, rsrc)


def assert_state_close(g, r, rel=REL):
    a, b = g.state(), r.state()
    worst = 0.0
    for k in STATE_KEYS:
        d = np.abs(a[k] - b[k]) / np.maximum(np.abs(b[k]), 1e-3)
        worst = max(worst, float(d.max()) if d.size else 0.0)
        assert np.all(d <= rel), (k, float(d.max()))
    assert np.array_equal(a["refractory"], b["refractory"])
    return worst


def assert_same_spikes(gsp, rsp):
    (gs, gsrc), (rs, rsrc) = gsp, rsp
    if not (np.array_equal(gs, rs) and np.array_equal(gsrc, rsrc)):
        n = min(len(gs), len(rs))
        bad = np.nonzero((gs[:n] != rs[:n]) | (gsrc[:n] != rsrc[:n]))[0]
        first = int(bad[0]) if len(bad) else n
        raise AssertionError(f"rasters differ at spike #{first} (gpu {len(gs)} vs ref {len(rs)}) "
                             f"step {gs[first] if first < len(gs) else None}")


@pytest.mark.parametrize("name,steps", [("quick", 4000), ("use_case", 3000), ("bursting", 3000),
                                        ("random_pool", 2000), ("c0_literal", 1500),
                                        ("no_spiking", 1000)])
def test_config_parity(name, steps):
    g, r, gsp, rsp = run_pair(config_path(name), steps=steps, chunks=2)
    assert_same_spikes(gsp, rsp)
    assert len(gsp[0]) > 0 or name == "no_spiking"
    assert_state_close(g, r)
    # STP per source equals every edge of that source
    x, u, t = g.stp()
    tab = r.table(0)
    rs = tab["row_start"]
    for s in range(0, len(rs) - 1, 7):
        if rs[s] < rs[s + 1]:
            e = rs[s]
            assert x[s] == tab["stp_x"][e] and u[s] == tab["stp_u"][e]


def test_paper_sparse_shape_parity():
    """10k neurons, 10k astrocytes, ~10M synapses, dt 0.05 ms, 1.5 ms delays."""
    g, r, gsp, rsp = run_pair(config_path("paper_sparse_dt005"), steps=600, chunks=3)
    assert_same_spikes(gsp, rsp)
    assert len(gsp[0]) > 0
    assert_state_close(g, r)
    assert g.counters()["spike_edges"] > 0


def variants():
    base = json.load(open(config_path("quick")))
    out = []
    v = json.loads(json.dumps(base))
    for k in ("input_exc", "input_inh", "input_astro"):
        v[k]["independent_noise"] = False
    out.append(("shared_noise", v))
    v = json.loads(json.dumps(base))
    v["synapse"]["stp"]["enabled"] = False
    out.append(("stp_off", v))
    v = json.loads(json.dumps(base))
    v["synapse"]["stp"]["tau_fac"] = 50.0
    v["synapse"]["sic_interval"] = 7
    v["connectivity"]["unique_third_out"] = True
    out.append(("fac_interval_unique", v))
    v = json.loads(json.dumps(base))
    v["synapse"]["d_a2n"] = 0.1  # one-step SIC delay: fused SIC path
    v["synapse"]["d_i"] = 0.3
    v["simulation"]["substeps"] = 3
    v["neuron_exc"]["t_ref"] = 2.0
    out.append(("short_delays_substeps_refractory", v))
    v = json.loads(json.dumps(base))
    v["synapse"]["w_e"] = -2.0  # negative excitatory weight routes to the inhibitory input
    v["synapse"]["w_i"] = 3.0
    v["input_exc"]["poiss_rate"] = 400000.0  # lambda > 30: normal approximation
    out.append(("sign_routing_big_lambda", v))
    v = json.loads(json.dumps(base))
    # astrocytes above the SIC threshold from the start, random pools of 5:
    # SIC sums over several astrocytes with multiplicities from step d_a2n on
    v["astrocyte"]["Ca_init"] = 0.35
    v["astrocyte"]["IP3"] = 0.6
    v["connectivity"].update({"pool_type": "random", "pool_size": 5, "p_third_if_primary": 0.6})
    out.append(("active_astrocytes_random_pools", v))
    v = json.loads(json.dumps(base))
    v["synapse"]["d_e"] = 0.1  # one-step spike delay: pushes stay in the spiking block
    v["synapse"]["d_i"] = 0.2
    out.append(("one_step_spike_delay", v))
    return out


@pytest.mark.parametrize("label,cfg", variants(), ids=[v[0] for v in variants()])
def test_variant_parity(label, cfg):
    g, r, gsp, rsp = run_pair(text=json.dumps(cfg), steps=2000, chunks=2)
    assert_same_spikes(gsp, rsp)
    assert_state_close(g, r)
    if label == "active_astrocytes_random_pools":
        assert g.counters()["sic_edges"] > 0


def sic_active_config():
    """paper_sparse_dt005 scaled to 2,500 neurons with ~350 SIC edges per
    target (in-degree ~700) and every astrocyte above the SIC threshold from
    the start; the SIC delay is 20 steps."""
    cfg = json.load(open(config_path("paper_sparse_dt005")))
    cfg["N"].update({"N_E": 2000, "N_I": 500, "N_A": 2500})
    cfg["connectivity"]["p_primary"] = 0.35
    cfg["astrocyte"]["Ca_init"] = 0.35
    cfg["astrocyte"]["IP3"] = 0.6
    return json.dumps(cfg)


def test_sic_active_parity():
    """SIC currents computed by side-stream batches (the default at a 20-step
    delay), against the oracle."""
    text = sic_active_config()
    rs, tg = Model(text=text, pre_time=0.0).table(3)
    assert np.bincount(tg).max() > 320  # the in-kernel form cuts three parts
    g, r, gsp, rsp = run_pair(text=text, steps=400, chunks=2)
    assert_same_spikes(gsp, rsp)
    assert_state_close(g, r)
    assert g.counters()["sic_edges"] > 1_000_000


def test_sic_forms_bitwise():
    """Side-stream batches (graph and plain launches), SIC parts pipelined in
    the step kernel (sic_mode 2), the persistent kernel's single-part role,
    and a persistent run resumed from a checkpoint by a side-batch network
    (which first recomputes the SIC values of the next steps): same bits."""
    m = Model(text=sic_active_config(), pre_time=0.0)
    outs = []
    for opts in (dict(), dict(use_graphs=-1), dict(sic_mode=2), dict(use_graphs=2),
                 dict(chunk_steps=24)):
        n = Network(m, record=rec_all(), **opts)
        n.step(200)
        n.step(200)
        outs.append((n.fetch_spikes(), n.state()))
    p = Network(m, record=rec_all(), use_graphs=2)
    p.step(200)
    blob = p.checkpoint()
    q = Network(m, record=rec_all())
    q.restore(blob)
    q.step(200)
    sp0, st0 = outs[0]
    tail = sp0[0] >= 200
    sq = q.fetch_spikes()
    assert np.array_equal(sq[0], sp0[0][tail]) and np.array_equal(sq[1], sp0[1][tail])
    for k in STATE_KEYS:
        assert np.array_equal(q.state()[k], st0[k]), ("resumed", k)
    for (sp, st) in outs[1:]:
        assert np.array_equal(sp[0], sp0[0]) and np.array_equal(sp[1], sp0[1])
        for k in STATE_KEYS:
            assert np.array_equal(st[k], st0[k]), k


def test_burst_push_paths_bitwise():
    """The initial burst of the paper-sparse network (up to ~400 spikes in a
    step, tens of arrivals per target and slot): the deferred push with every
    block helping, the in-block push, the persistent kernel and the
    high-occupancy form of the step kernel give the same bits, and the
    short-list overflow path is taken."""
    m = Model(config_path("paper_sparse_dt005"), pre_time=0.0)
    outs = []
    for opts in (dict(), dict(push_mode=1), dict(use_graphs=2, block=256), dict(occupancy=2)):
        n = Network(m, record=rec_all(), **opts)
        n.step(800)
        outs.append((n.fetch_spikes(), n.state(), n.counters(), opts, n.current_step,
                     n.last_timing()))
    sp0, st0, c0 = outs[0][:3]
    assert c0["spikes"] > 20000, outs[0][2:]  # the burst happened
    for sp, st, c, opts, cur, tim in outs[1:]:
        assert np.array_equal(sp[0], sp0[0]) and np.array_equal(sp[1], sp0[1]), (
            len(sp[0]), c, opts, cur, tim, float(np.nanmean(st["V"])))
        for k in STATE_KEYS:
            assert np.array_equal(st[k], st0[k]), k


def test_burst_overflow_both_merge_paths_parity():
    """A synchronous burst at high in-degree against the oracle: excitatory
    targets of more than 1024 in-edges (more than 32 bitmap words: merge by
    summary) and inhibitory targets of a few hundred (all words in one batch)
    both receive tens of arrivals in one slot; spikes must be identical and
    the state within the network tolerance."""
    cfg = json.load(open(config_path("paper_sparse_dt005")))
    cfg["N"].update({"N_E": 2400, "N_I": 600, "N_A": 3000})
    cfg["connectivity"]["p_primary"] = 0.5
    text = json.dumps(cfg)
    m = Model(text=text, pre_time=0.0)
    deg_e = np.bincount(m.table(0)[1]).max()
    deg_i = np.bincount(m.table(1)[1]).max()
    assert deg_e > 1024 and deg_i <= 1024, (deg_e, deg_i)
    g, r, gsp, rsp = run_pair(text=text, steps=800, chunks=2)
    assert_same_spikes(gsp, rsp)
    assert_state_close(g, r)
    per_step = np.bincount(gsp[0])
    # ~200 coincident spikes (a fifth of them inhibitory) at p = 0.5: tens of
    # arrivals per target and slot in every ring
    assert per_step.max() > 150, per_step.max()


def test_large_network_sic_forms_bitwise():
    """A network of 2^16+ neurons with short SIC lists (the serving shape,
    astrocytes active from the start): the automatic form (SIC summed in the
    neuron thread, high-occupancy step kernel), the SIC role and the latency
    form of the step kernel give the same bits."""
    from astrosimgpu_b200.workloads import serving_config
    cfg = json.loads(serving_config(70000, 5, 10.0))
    cfg["astrocyte"]["Ca_init"] = 0.35
    cfg["astrocyte"]["IP3"] = 0.6
    m = Model(text=json.dumps(cfg), pre_time=0.0, fixed_indegree=100, gen_device=0)
    outs = []
    for opts in (dict(), dict(sic_mode=2), dict(sic_mode=1, occupancy=1)):
        n = Network(m, record=rec_all(), **opts)
        n.step(60)
        outs.append((n.fetch_spikes(), n.state(), n.counters()))
        del n
    (sp0, st0, c0) = outs[0]
    assert c0["sic_edges"] > 0 and c0["spikes"] > 0, c0
    for sp, st, c in outs[1:]:
        assert np.array_equal(sp[0], sp0[0]) and np.array_equal(sp[1], sp0[1])
        for k in STATE_KEYS:
            assert np.array_equal(st[k], st0[k]), k


def test_sic_modes_and_block_sizes_bitwise():
    """The separate SIC role and the fused form, any block size, per-step
    graph launches, plain launches and the persistent chunk kernel give
    identical bits (the arithmetic per cell does not depend on the launch)."""
    path = config_path("use_case")
    m = Model(path, pre_time=0.0)
    outs = []
    for opts in (dict(sic_mode=1, block=64), dict(sic_mode=2, block=256),
                 dict(sic_mode=0, block=128, chunk_steps=7, use_graphs=-1),
                 dict(block=128, chunk_steps=50, use_graphs=2),
                 dict(block=64, chunk_steps=13, use_graphs=2, pdl=-1),
                 dict(block=96, chunk_steps=32, push_mode=1)):
        n = Network(m, record=rec_all(), **opts)
        n.step(1200)
        outs.append((n.fetch_spikes(), n.state()))
    for (sp, st) in outs[1:]:
        assert np.array_equal(sp[0], outs[0][0][0]) and np.array_equal(sp[1], outs[0][0][1])
        for k in STATE_KEYS:
            assert np.array_equal(st[k], outs[0][1][k]), k


@pytest.mark.parametrize("mode", [1, 2])
def test_batch_equals_single_bitwise(mode):
    """Instances of uneven size packed into one engine give the bits each
    gives alone (graph launches and the persistent chunk kernel)."""
    names = ["quick", "use_case", "quick", "bursting"]
    seeds = [1, 2, 3, 4]
    models = [Model(config_path(n), seed=s, pre_time=0.0) for n, s in zip(names, seeds)]
    b = Batch(models, record=rec_all(), use_graphs=mode)
    b.step(800)
    for i, m in enumerate(models):
        n = Network(m, record=rec_all())
        n.step(800)
        s1, s2 = n.fetch_spikes(), b.fetch_spikes(i)
        assert np.array_equal(s1[0], s2[0]) and np.array_equal(s1[1], s2[1])
        a, c = n.state(), b.state(i)
        for k in STATE_KEYS:
            assert np.array_equal(a[k], c[k]), (i, k)


def test_large_batch_fused_sic_equals_single_bitwise():
    """A batch of 2^16 neurons in all sums SIC in the neuron threads (its
    instances are small, so alone each runs the SIC role): the same bits."""
    cfg = json.load(open(config_path("use_case")))
    cfg["N"].update({"N_E": 6554, "N_I": 1638, "N_A": 1638})
    cfg["connectivity"]["p_primary"] = 0.02
    cfg["astrocyte"]["Ca_init"] = 0.35
    cfg["astrocyte"]["IP3"] = 0.6
    text = json.dumps(cfg)
    models = [Model(text=text, seed=s, pre_time=0.0) for s in range(1, 9)]
    assert sum(m.desc().n_exc + m.desc().n_inh for m in models) >= 1 << 16
    b = Batch(models, record=rec_all())
    b.step(150)
    assert b.counters(0)["sic_edges"] > 0
    for i in (0, 5):
        n = Network(models[i], record=rec_all())
        n.step(150)
        s1, s2 = n.fetch_spikes(), b.fetch_spikes(i)
        assert np.array_equal(s1[0], s2[0]) and np.array_equal(s1[1], s2[1])
        a, c = n.state(), b.state(i)
        for k in STATE_KEYS:
            assert np.array_equal(a[k], c[k]), (i, k)
        n.close()


def test_checkpoint_restore_bitwise():
    """Resume inside a noise interval (step 503; the noise draws change every
    10 steps), in the same network after it ran on and in a new one."""
    m = Model(config_path("use_case"), pre_time=0.0)
    n = Network(m, record=rec_all())
    n.step(503)
    blob = n.checkpoint()
    n.fetch_spikes()
    n.step(700)
    sp1, st1 = n.fetch_spikes(), n.state()
    n.restore(blob)
    n.step(700)
    sp2, st2 = n.fetch_spikes(), n.state()
    fresh = Network(m, record=rec_all())
    fresh.restore(blob)
    fresh.step(700)
    sp3, st3 = fresh.fetch_spikes(), fresh.state()
    for sp, st in ((sp2, st2), (sp3, st3)):
        assert np.array_equal(sp1[0], sp[0]) and np.array_equal(sp1[1], sp[1])
        for k in STATE_KEYS:
            assert np.array_equal(st1[k], st[k]), k


def test_recording_matches_reference_rows():
    """Recorded Ca/IP3 rows of the first cells every record_every steps, as
    Network::run writes them (network.cpp:443-462)."""
    path = config_path("quick")
    m = Model(path, pre_time=0.0)
    n = Network(m, record=_lib.RecordOpts(0, 10, 1, 20, 15))
    r = ref.RefNetwork(path=path, pre_time=0.0)
    n.step(300)
    rec = n.fetch_record()
    assert len(rec["astro_steps"]) == 30 and rec["astro_steps"][-1] == 290
    # replay the reference to step 291 and compare the last row
    r.run(291)
    s = r.state()
    assert np.allclose(rec["Ca"][-1], s["Ca"][:20], rtol=REL, atol=0)
    assert np.allclose(rec["IP3"][-1], s["IP3"][:20], rtol=REL, atol=0)


def test_fixed_indegree_device_equals_host():
    text = json.dumps({"N": {"N_A": 5000, "N_E": 4000, "N_I": 1000},
                       "connectivity": {"p_third_if_primary": 0.7, "pool_size": 3,
                                        "pool_type": "random"}})
    h = Model(text=text, fixed_indegree=50)
    d = Model(text=text, fixed_indegree=50, gen_device=0)
    for which in range(4):
        a, b = h.table(which), d.table(which)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), which


def test_bad_descriptor_is_rejected_cleanly():
    m = Model(config_path("quick"), pre_time=0.0)
    d = m.desc()
    bad = _lib.NetworkDesc.from_buffer_copy(d)
    bad.d_e_steps = 0
    import ctypes as C
    h = C.c_void_p()
    st = _lib.load().asg_create(C.byref(bad), None, None, C.byref(h))
    assert st == 1 and not h
    assert b"delay" in _lib.load().asg_last_error()
