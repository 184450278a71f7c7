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
    assert 0 <= shape < 6 and us > 0
    for a, b in zip(g.pull_state(), (Ca, IP3, h)):
        assert np.array_equal(a, b)
    g.run_bernoulli(w, 0, 150)
    r = [a.copy() for a in (Ca, IP3, h)]
    ref.ref_astro_scaling(w, *r, 0, 150, threads=1)
    for a, b in zip(g.pull_state(), r):
        assert np.array_equal(a, b)
