"""The allocation-free astrocyte update (asg_astro_update_noalloc), for
callers that cannot call cudaMalloc and hand over device arrays they own.

It must give what the regular entry point gives (asg_astro_create +
asg_astro_push_input + asg_astro_update: bitwise, the tolerance of the other
astrocyte tests) on two calls in a row -- the second call proves the shared
scratch array carries nothing over from the first.  This file is collected
last, so a run that stops at the first failure has run every other test."""
import ctypes as C

import numpy as np
import pytest

from astrosimgpu_b200 import _lib
from astrosimgpu_b200.astro import AstroBackend, ScalingWorkload

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to("cuda")


def test_noalloc_matches_regular_entry_point_twice():
    """Two calls in a row with different tau_IP3 arrays and sizes: the second
    call's reciprocals must be recomputed over the shared scratch array, so a
    stale entry left by the first call would change its result."""
    import torch
    rng = np.random.default_rng(11)
    n1, n2 = 5003, 4001
    w = ScalingWorkload(n1)
    Ca, IP3, h = w.initial_state()
    Ca_tot = w.Ca_tot * (1 + 0.05 * rng.standard_normal(n1))
    IP3_0 = w.IP3_0 * (1 + 0.05 * rng.standard_normal(n1))
    delta = w.delta_IP3 * (1 + 0.05 * rng.standard_normal(n1))
    taus = [w.tau_IP3 * (1 + 0.05 * rng.standard_normal(n1)),
            w.tau_IP3 * (0.5 + rng.random(n1))]  # a different array for call 2
    inputs = [np.where(rng.random(n1) < 0.3, rng.random(n1), 0.0) for _ in range(2)]

    d = {k: dev(v) for k, v in dict(Ca=Ca, IP3=IP3, h=h, Ca_tot=Ca_tot, IP3_0=IP3_0,
                                       delta=delta, inp=np.zeros(n1)).items()}
    lib = _lib.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    state = (Ca, IP3, h)
    for call, (n, tau, inp) in enumerate(zip((n1, n2), taus, inputs)):
        # the regular entry point on the state both paths hold before this call
        regular = AstroBackend(*[a[:n].copy() for a in state], Ca_tot[:n].copy(),
                               IP3_0[:n].copy(), tau[:n].copy(), delta[:n].copy())
        regular.push_input(inp[:n].copy())
        regular.update(w.consts, w.h_step, 2)
        rCa, rIP3, rh = regular.pull_state()
        regular.destroy()
        d_tau = dev(tau)
        d["inp"].copy_(torch.from_numpy(inp))
        st = lib.asg_astro_update_noalloc(
            n, *[C.c_void_p(d[k].data_ptr()) for k in ("Ca", "IP3", "h", "inp", "Ca_tot",
                                                         "IP3_0")],
            C.c_void_p(d_tau.data_ptr()), C.c_void_p(d["delta"].data_ptr()),
            _lib.dptr(w.consts), w.h_step, 2, 0.0, 1, 0.0, 0, 0, stream)
        assert st == 0, lib.asg_last_error()
        torch.cuda.synchronize()
        gCa, gIP3, gh = (d[k].cpu().numpy() for k in ("Ca", "IP3", "h"))
        assert np.array_equal(gCa[:n], rCa), call
        assert np.array_equal(gIP3[:n], rIP3), call
        assert np.array_equal(gh[:n], rh), call
        # cells beyond n are not touched, and the input is consumed (zeroed)
        # over [0, n) only, as the regular path does for its cells
        for g, before in zip((gCa, gIP3, gh), state):
            assert np.array_equal(g[n:], before[n:]), call
        assert not d["inp"][:n].any()
        state = (gCa.copy(), gIP3.copy(), gh.copy())


def test_pipelined_ranges_with_noise_match_single_launch():
    """The regular entry point splits a large handle into cell ranges, each
    launch offset to its first cell; with independent noise every cell must
    still draw its own stream, as the single-launch no-alloc call does."""
    import torch
    rng = np.random.default_rng(12)
    n = 3 * (1 << 18) + 77
    w = ScalingWorkload(n)
    Ca, IP3, h = w.initial_state()
    Ca_tot = w.Ca_tot * (1 + 0.05 * rng.standard_normal(n))
    IP3_0 = w.IP3_0 * (1 + 0.05 * rng.standard_normal(n))
    tau = w.tau_IP3 * (1 + 0.05 * rng.standard_normal(n))
    delta = w.delta_IP3 * (1 + 0.05 * rng.standard_normal(n))
    regular = AstroBackend(Ca, IP3, h, Ca_tot, IP3_0, tau, delta)
    d = {k: dev(v) for k, v in dict(Ca=Ca, IP3=IP3, h=h, Ca_tot=Ca_tot, IP3_0=IP3_0, tau=tau,
                                       delta=delta, inp=np.zeros(n)).items()}
    lib = _lib.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for step in range(3):
        inp = np.where(rng.random(n) < 0.3, rng.random(n), 0.0)
        regular.push_input(inp)
        regular.update(w.consts, w.h_step, 2, noise_std=0.05, independent=True,
                       noise_seed=77, noise_index=step)
        d["inp"].copy_(torch.from_numpy(inp))
        st = lib.asg_astro_update_noalloc(
            n, *[C.c_void_p(d[k].data_ptr()) for k in ("Ca", "IP3", "h", "inp", "Ca_tot",
                                                         "IP3_0", "tau", "delta")],
            _lib.dptr(w.consts), w.h_step, 2, 0.05, 1, 0.0, 77, step, stream)
        assert st == 0, lib.asg_last_error()
    torch.cuda.synchronize()
    rCa, rIP3, rh = regular.pull_state()
    assert np.array_equal(d["Ca"].cpu().numpy(), rCa)
    assert np.array_equal(d["IP3"].cpu().numpy(), rIP3)
    assert np.array_equal(d["h"].cpu().numpy(), rh)
    regular.destroy()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = _lib.load()
    null = C.c_void_p(16)  # never dereferenced: the size check comes first
    consts = np.zeros(10)
    st = lib.asg_astro_update_noalloc((1 << 20) + 1, *([null] * 8), _lib.dptr(consts), 0.1, 1,
                                      0.0, 1, 0.0, 0, 0, None)
    assert st == 1 and b"scratch limit" in lib.asg_last_error()
