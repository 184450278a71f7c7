"""Astrocyte update on the B200 against the reference's own astro_advance.

With noise off the astrocyte step has no transcendental function, so the
GPU result must be bitwise equal to the host loop over the reference's
astro_advance (astrocyte_kernel.hpp:71-103) built from its sources.
"""
import numpy as np
import pytest

from astrosimgpu_b200.astro import AstroBackend, ScalingWorkload
from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 2, 7, 1000, 4099])
def test_scaling_workload_bitwise(n):
    w = ScalingWorkload(n)
    Ca, IP3, h = w.initial_state()
    gpu = AstroBackend(Ca, IP3, h)
    gpu.run_bernoulli(w, 0, 300)
    gCa, gIP3, gh = gpu.pull_state()
    rCa, rIP3, rh = Ca.copy(), IP3.copy(), h.copy()
    ref.ref_astro_scaling(w, rCa, rIP3, rh, 0, 300, threads=1)
    assert np.array_equal(gCa, rCa)
    assert np.array_equal(gIP3, rIP3)
    assert np.array_equal(gh, rh)
    # the inputs did move the state (not a trivially idle run)
    assert not np.array_equal(gIP3, IP3)


def test_scaling_resume_matches_single_run():
    w = ScalingWorkload(2048)
    Ca, IP3, h = w.initial_state()
    a = AstroBackend(Ca, IP3, h)
    a.run_bernoulli(w, 0, 130)
    b = AstroBackend(Ca, IP3, h)
    b.run_bernoulli(w, 0, 64)
    b.run_bernoulli(w, 64, 66)
    for x, y in zip(a.pull_state(), b.pull_state()):
        assert np.array_equal(x, y)


def test_drop_in_backend_per_cell_params_and_input():
    """The reference backend's movement points: push input, update, pull Ca."""
    rng = np.random.default_rng(3)
    n = 777
    w = ScalingWorkload(n)
    Ca, IP3, h = w.initial_state()
    Ca_tot = w.Ca_tot * (1 + 0.05 * rng.standard_normal(n))
    IP3_0 = w.IP3_0 * (1 + 0.05 * rng.standard_normal(n))
    tau = w.tau_IP3 * (1 + 0.05 * rng.standard_normal(n))
    delta = w.delta_IP3 * (1 + 0.05 * rng.standard_normal(n))
    gpu = AstroBackend(Ca, IP3, h, Ca_tot, IP3_0, tau, delta)
    rCa, rIP3, rh = Ca.copy(), IP3.copy(), h.copy()
    lib = ref.ref()
    for step in range(50):
        inp = np.where(rng.random(n) < 0.3, rng.random(n), 0.0)
        gpu.push_input(inp)
        gpu.update(w.consts, w.h_step, 2)
        lib.ref_astro_advance(ref._dp(w.consts), n, ref._dp(Ca_tot), ref._dp(IP3_0),
                              ref._dp(tau), ref._dp(delta), ref._dp(inp), None, w.h_step, 2,
                              ref._dp(rCa), ref._dp(rIP3), ref._dp(rh))
        assert np.array_equal(gpu.pull_calcium(), rCa)
    gCa, gIP3, gh = gpu.destroy()
    assert np.array_equal(gIP3, rIP3) and np.array_equal(gh, rh)


def test_drop_in_backend_pipelined_cell_ranges():
    """Large handles copy and update in up to eight cell ranges whose copies
    overlap the updates; the result is the oracle's, bit for bit, including
    at range boundaries, on consecutive steps and when the caller reuses one
    input buffer."""
    rng = np.random.default_rng(5)
    n = 3 * (1 << 18) + 77  # three ranges, the last one ragged
    w = ScalingWorkload(n)
    Ca, IP3, h = w.initial_state()
    Ca_tot = w.Ca_tot * (1 + 0.05 * rng.standard_normal(n))
    IP3_0 = w.IP3_0 * (1 + 0.05 * rng.standard_normal(n))
    tau = w.tau_IP3 * (1 + 0.05 * rng.standard_normal(n))
    delta = w.delta_IP3 * (1 + 0.05 * rng.standard_normal(n))
    gpu = AstroBackend(Ca, IP3, h, Ca_tot, IP3_0, tau, delta)
    rCa, rIP3, rh = Ca.copy(), IP3.copy(), h.copy()
    lib = ref.ref()
    inp = np.empty(n)
    for step in range(4):
        inp[:] = np.where(rng.random(n) < 0.3, rng.random(n), 0.0)
        gpu.push_input(inp)
        gpu.update(w.consts, w.h_step, 2)
        lib.ref_astro_advance(ref._dp(w.consts), n, ref._dp(Ca_tot), ref._dp(IP3_0),
                              ref._dp(tau), ref._dp(delta), ref._dp(inp), None, w.h_step, 2,
                              ref._dp(rCa), ref._dp(rIP3), ref._dp(rh))
        if step % 2:
            assert np.array_equal(gpu.pull_calcium(), rCa), step
    gCa, gIP3, gh = gpu.destroy()
    assert np.array_equal(gCa, rCa) and np.array_equal(gIP3, rIP3) and np.array_equal(gh, rh)


@pytest.mark.parametrize("uniform_params", [False, True])
def test_drop_in_update_without_push_sees_zero_input(uniform_params):
    """The reference kernel zeroes the input after each update, so an update
    with no push before it sees zero input.  The engine reads the input only
    after a push and never writes it; the results must still be the oracle's
    for any mix of pushed and unpushed steps, with per-cell parameters that
    differ or that are all equal (held as scalars)."""
    rng = np.random.default_rng(9)
    n = 1003
    w = ScalingWorkload(n)
    Ca, IP3, h = w.initial_state()
    if uniform_params:
        params = [np.full(n, v) for v in (w.Ca_tot, w.IP3_0, w.tau_IP3, w.delta_IP3)]
    else:
        params = [v * (1 + 0.05 * rng.standard_normal(n))
                  for v in (w.Ca_tot, w.IP3_0, w.tau_IP3, w.delta_IP3)]
    gpu = AstroBackend(Ca, IP3, h, *params)
    rCa, rIP3, rh = Ca.copy(), IP3.copy(), h.copy()
    lib = ref.ref()
    zero = np.zeros(n)
    for step in range(40):
        pushed = step % 3 == 0 or step % 7 == 1
        inp = np.where(rng.random(n) < 0.3, rng.random(n), 0.0) if pushed else zero
        if pushed:
            gpu.push_input(inp)
        gpu.update(w.consts, w.h_step, 1)
        lib.ref_astro_advance(ref._dp(w.consts), n, *[ref._dp(p) for p in params],
                              ref._dp(inp), None, w.h_step, 1, ref._dp(rCa), ref._dp(rIP3),
                              ref._dp(rh))
    gCa, gIP3, gh = gpu.pull_state()
    assert np.array_equal(gCa, rCa) and np.array_equal(gIP3, rIP3) and np.array_equal(gh, rh)
