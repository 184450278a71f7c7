"""Every launch shape of the astrocyte kernel gives the same bits, and the
autotuner leaves the state untouched."""
import numpy as np
import pytest

from astrosimgpu_b200.astro import AstroBackend, ScalingWorkload
from oracle import ref

pytestmark = pytest.mark.gpu


def test_autotune_keeps_state_and_result_bitwise():
    w = ScalingWorkload(10001)
    Ca, IP3, h = w.initial_state()
    g = AstroBackend(Ca, IP3, h)
    shape, us = g.autotune(w, steps=5)
    assert 0 <= shape < 9 and us > 0
    for a, b in zip(g.pull_state(), (Ca, IP3, h)):
        assert np.array_equal(a, b)
    g.run_bernoulli(w, 0, 150)
    r = [a.copy() for a in (Ca, IP3, h)]
    ref.ref_astro_scaling(w, *r, 0, 150, threads=1)
    for a, b in zip(g.pull_state(), r):
        assert np.array_equal(a, b)


def test_every_shape_bitwise():
    """Each launch shape (1, 2 or 4 cells per thread; odd sizes leave 1 to 3
    tail cells) reproduces the oracle bit for bit on the scaling workload
    and on the drop-in path with per-cell parameters."""
    from astrosimgpu_b200 import _lib
    w = ScalingWorkload(10003)  # 10003 = 4 * 2500 + 3
    Ca, IP3, h = w.initial_state()
    r = [a.copy() for a in (Ca, IP3, h)]
    ref.ref_astro_scaling(w, *r, 0, 60, threads=1)
    shape = 0
    while True:
        g = AstroBackend(Ca, IP3, h)
        try:
            g.set_shape(shape)
        except _lib.AsgError:
            break
        g.run_bernoulli(w, 0, 60)
        for a, b in zip(g.pull_state(), r):
            assert np.array_equal(a, b), shape
        g.destroy()
        shape += 1
    assert shape == 9

    # drop-in path: per-cell parameters and an input array
    rng = np.random.default_rng(9)
    n = w.n
    par = [x * (1 + 0.05 * rng.standard_normal(n))
           for x in (w.Ca_tot, w.IP3_0, w.tau_IP3, w.delta_IP3)]
    inputs = [np.where(rng.random(n) < 0.3, rng.random(n), 0.0) for _ in range(3)]
    rCa, rIP3, rh = Ca.copy(), IP3.copy(), h.copy()
    lib = ref.ref()
    for inp in inputs:
        lib.ref_astro_advance(ref._dp(w.consts), n, *[ref._dp(x) for x in par], ref._dp(inp),
                              None, w.h_step, 2, ref._dp(rCa), ref._dp(rIP3), ref._dp(rh))
    for k in range(shape):
        g = AstroBackend(Ca, IP3, h, *par)
        g.set_shape(k)
        for inp in inputs:
            g.push_input(inp)
            g.update(w.consts, w.h_step, 2)
        for a, b in zip(g.destroy(), (rCa, rIP3, rh)):
            assert np.array_equal(a, b), k
