"""Pins the C restatement (oracle/asg_oracle.c) to the reference simulator
compiled from its own sources (oracle/_ref): RNG streams, the astrocyte
advance, builder tables, per-cell parameters, spikes and full state over
thousands of steps must agree bit for bit.  Also checks the reference's own
known-answer facts (rng_uniform == CounterRng, tests/test_astrosimgpu.cpp:
113-120; the input jump of astro_advance, :199-202; use_case edge counts)."""
import ctypes as C

import numpy as np
import pytest

from oracle import config as oc
from oracle import ref

CFG = "astrosimgpu_b200/configs/{}.json"

pytestmark = pytest.mark.skipif(not ref.ref_available(), reason="oracle/_ref not built")


def port():
    L = ref.port()
    L.orc_bits.restype = C.c_uint64
    L.orc_bits.argtypes = [C.c_uint64] * 3
    L.orc_uniform.restype = C.c_double
    L.orc_uniform.argtypes = [C.c_uint64] * 3
    L.orc_normal.restype = C.c_double
    L.orc_normal.argtypes = [C.c_uint64] * 2
    return L


def test_rng_streams_bitwise():
    R, P = ref.ref(), port()
    rng = np.random.default_rng(0)
    for _ in range(2000):
        s, st, c = (int(x) for x in rng.integers(0, 2**63, 3))
        assert R.ref_rng_bits(s, st, c) == P.orc_bits(s, st, c)
        assert R.ref_rng_uniform(s, st, c) == P.orc_uniform(s, st, c)
        assert R.ref_rng_normal(s, st) == P.orc_normal(s, st)


def test_counter_rng_methods_bitwise():
    R, P = ref.ref(), port()
    P.orc_rng_init.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64]

    class Rng(C.Structure):
        _fields_ = [("seed", C.c_uint64), ("stream", C.c_uint64), ("counter", C.c_uint64),
                    ("has_spare", C.c_int), ("spare", C.c_double)]
    P.orc_rng_uniform.restype = C.c_double
    P.orc_rng_normal.restype = C.c_double
    P.orc_rng_poisson.restype = C.c_int
    P.orc_rng_poisson.argtypes = [C.c_void_p, C.c_double]
    for kind, lam in ((0, 0.0), (1, 0.0), (2, 0.27), (2, 3.5), (2, 45.0)):
        out = np.zeros(500)
        R.ref_counter_rng(4242, 7, kind, lam, 500, ref._dp(out))
        r = Rng()
        P.orc_rng_init(C.byref(r), 4242, 7)
        fn = {0: lambda: P.orc_rng_uniform(C.byref(r)), 1: lambda: P.orc_rng_normal(C.byref(r)),
              2: lambda: float(P.orc_rng_poisson(C.byref(r), lam))}[kind]
        got = np.array([fn() for _ in range(500)])
        assert np.array_equal(out, got), (kind, lam)


def test_reference_known_answers():
    """The reference's own pinned facts, reproduced through oracle/_ref."""
    R = ref.ref()
    # free rng functions == CounterRng (test_astrosimgpu.cpp:113-120)
    for stream in range(200):
        u = np.zeros(1)
        R.ref_counter_rng(4242, stream, 0, 0.0, 1, ref._dp(u))
        assert u[0] == R.ref_rng_uniform(4242, stream, 0)
        R.ref_counter_rng(4242, stream, 1, 0.0, 1, ref._dp(u))
        assert u[0] == R.ref_rng_normal(4242, stream)
    # use_case edge counts (docs/gpu-port.md:14-15): 39,790 / 9,944 / 8,097
    net = ref.RefNetwork(path=CFG.format("use_case"))
    assert (net.n_primary_exc, net.n_primary_inh, net.n_n2a, net.n_a2n) == (39790, 9944, 8097, 8097)


@pytest.mark.parametrize("name,steps", [("quick", 3000), ("use_case", 2500), ("bursting", 1500),
                                        ("random_pool", 1500), ("no_spiking", 500)])
def test_network_bitwise(name, steps):
    path = CFG.format(name)
    r = ref.RefNetwork(path=path)
    p = oc.PortNetwork(oc.load(path))
    for which in range(4):
        t = r.table(which)
        rs, tg = p.table(which)
        assert np.array_equal(t["row_start"], rs) and np.array_equal(t["target"], tg)
    cr, cp = r.cells(), p.cells()
    for k in cr:
        assert np.array_equal(cr[k], cp[k]), k
    a = r.run(steps)
    b = p.run(steps)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    sa, sb = r.state(), p.state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k


def test_network_variants_bitwise():
    """Options the shipped configs leave at defaults: shared noise, STP off,
    facilitation, sic_interval > 1, unique astrocyte-target pairs."""
    import json
    base = json.load(open(CFG.format("quick")))
    variants = []
    v = json.loads(json.dumps(base))
    v["input_exc"]["independent_noise"] = False
    v["input_inh"]["independent_noise"] = False
    v["input_astro"]["independent_noise"] = False
    variants.append(v)
    v = json.loads(json.dumps(base))
    v["synapse"]["stp"]["enabled"] = False
    variants.append(v)
    v = json.loads(json.dumps(base))
    v["synapse"]["stp"]["tau_fac"] = 50.0
    v["synapse"]["sic_interval"] = 7
    v["connectivity"]["unique_third_out"] = True
    variants.append(v)
    for cfg in variants:
        text = json.dumps(cfg)
        r = ref.RefNetwork(text=text)
        p = oc.PortNetwork(oc.load(text=text))
        a, b = r.run(1500), p.run(1500)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        sa, sb = r.state(), p.state()
        for k in sa:
            assert np.array_equal(sa[k], sb[k]), k
