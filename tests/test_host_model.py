"""The product's host side (config loader and network builder in
libasg_b200.so) against the reference built from its sources: the JSON
schema semantics of parameters.cpp:85-205 and Network::build's tables and
per-cell parameters, bit for bit.  CPU only."""
import json

import numpy as np
import pytest

from astrosimgpu_b200 import _lib
from astrosimgpu_b200.network import Model, config_path
from oracle import ref

needs_ref = pytest.mark.skipif(not ref.ref_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("name", ["quick", "use_case", "bursting", "random_pool", "scale_1000",
                                  "c0_literal", "kernel_scaling"])
def test_builder_bitwise(name):
    path = config_path(name)
    m = Model(path)
    r = ref.RefNetwork(path=path)
    for which in range(4):
        t = r.table(which)
        rs, tg = m.table(which)
        assert np.array_equal(t["row_start"], rs), which
        assert np.array_equal(t["target"], tg), which
    cm, cr = m.cells(), r.cells()
    for k in cr:
        assert np.array_equal(cm[k], cr[k]), k
    st = m.stats()
    assert st["ring_slots"] == r.ring_slots
    assert (st["n_primary_exc"], st["n_primary_inh"], st["n_n2a"], st["n_a2n"]) == (
        r.n_primary_exc, r.n_primary_inh, r.n_n2a, r.n_a2n)
    assert (m.dt, m.substeps, m.pre_steps, m.sim_steps) == (r.dt, r.substeps, r.pre_steps,
                                                            r.sim_steps)


@needs_ref
def test_builder_overrides_and_unique():
    path = config_path("quick")
    for seed in (1, 2, 99):
        m = Model(path, seed=seed, n_astro=37)
        r = ref.RefNetwork(path=path, seed=seed, n_astro=37)
        for which in range(4):
            assert np.array_equal(m.table(which)[1], r.table(which)["target"])
    cfg = json.load(open(path))
    cfg["connectivity"]["unique_third_out"] = True
    cfg["connectivity"]["allow_autapses"] = True
    text = json.dumps(cfg)
    m, r = Model(text=text), ref.RefNetwork(text=text)
    for which in range(4):
        assert np.array_equal(m.table(which)[1], r.table(which)["target"])


def test_config_rejects_unknown_keys():
    cfg = json.load(open(config_path("quick")))
    cfg["synapse"]["w_typo"] = 1.0
    with pytest.raises(_lib.AsgError) as e:
        Model(text=json.dumps(cfg), build=False)
    assert e.value.status == 7 and "synapse.w_typo" in str(e.value)


def test_config_errors_and_aliases():
    with pytest.raises(_lib.AsgError):
        Model(text="{ oops }", build=False)
    with pytest.raises(_lib.AsgError):
        Model(text='{"connectivity": {"pool_type": "ring"}}', build=False)
    with pytest.raises(_lib.AsgError):
        Model(text='{"simulation": {"substeps": 0}}', build=False)
    with pytest.raises(_lib.AsgError):
        Model(text='{"synapse": {"sic_interval": 0}}', build=False)
    # '//' comments, aliases and the noise_dt default
    text = """// comment line
    {"simulation": {"dt": 0.05, "seed": 3},   // trailing comment
     "neuron_exc": {"V_m": -55.5}, "astrocyte": {"IP3": 0.3},
     "input_exc": {"gauss_noise_var": 7.0}, "N": {"N_A": 4, "N_E": 8, "N_I": 2}}"""
    m = Model(text=text)
    d = m.desc()
    assert d.V_m_init_exc == -55.5 and d.IP3_init == 0.3
    assert d.input_exc.gauss_noise_std == 7.0
    assert abs(d.input_exc.noise_dt - 0.5) < 1e-15 and d.seed == 3
    assert d.n_exc == 8 and d.n_astro == 4


def test_fixed_indegree_host_properties():
    text = json.dumps({"N": {"N_A": 3000, "N_E": 2400, "N_I": 600},
                       "connectivity": {"p_third_if_primary": 0.5, "pool_size": 1}})
    m = Model(text=text, fixed_indegree=100)
    rs_e, tg_e = m.table(0)
    rs_i, tg_i = m.table(1)
    indeg = np.bincount(np.concatenate([tg_e, tg_i]), minlength=3000)
    assert np.all(indeg == 100)
    src_e = np.repeat(np.arange(2400), np.diff(rs_e))
    assert not np.any(src_e == tg_e)  # no autapses
    frac_exc = len(tg_e) / (len(tg_e) + len(tg_i))
    assert abs(frac_exc - 0.8) < 0.01
    rs_n, tg_n = m.table(2)
    assert abs(len(tg_n) / len(tg_e) - 0.5) < 0.01
    rs_a, tg_a = m.table(3)
    assert len(tg_a) == len(tg_n)
    # block pools of size 1 with N_A == N: each neuron's astrocyte is its own index
    src_a = np.repeat(np.arange(3000), np.diff(rs_a))
    assert np.array_equal(src_a, tg_a)
