"""Astrocyte backend on the B200 (Python view of the asg_astro_* C ABI).

``AstroBackend`` has the reference's four movement points
(astrocyte_cuda.hpp:15-27): resident state on create, ``push_input``,
``update``, ``pull_calcium`` and ``destroy`` (state copied back).
``run_bernoulli`` is the astrocyte kernel-scaling workload with its input
generated on the device from the counter RNG.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from . import _lib

CONFIG_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "configs")

# AstroConstants order (astrocyte_kernel.hpp:29-40).
CONST_KEYS = ("Kd_IP3_1", "Kd_IP3_2", "Kd_act", "Kd_inh", "Km_SERCA", "k_IP3R", "rate_IP3R",
              "rate_L", "rate_SERCA", "ratio_ER_cyt")

_MASK = np.uint64(0xFFFFFFFFFFFFFFFF)


def mix64_np(seed, stream, counter):
    """splitmix64 finaliser over seed + stream*phi + counter*c (vectorised, wraps mod 2^64)."""
    seed = np.asarray(seed, dtype=np.uint64)
    stream = np.asarray(stream, dtype=np.uint64)
    counter = np.asarray(counter, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = seed + stream * np.uint64(0x9E3779B97F4A7C15) + counter * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform_np(seed, stream, counter):
    return (mix64_np(seed, stream, counter) >> np.uint64(11)).astype(np.float64) * (
        1.0 / 9007199254740992.0)


def load_astro_block(name: str = "use_case") -> dict:
    with open(os.path.join(CONFIG_DIR, name + ".json")) as f:
        return json.load(f)["astrocyte"]


class ScalingWorkload:
    """The astrocyte kernel-scaling case: N independent Li-Rinzel cells with the
    use_case astrocyte parameters (not randomised), state x0*(1+0.1*(2U-1)),
    U = rng_uniform(seed, cell, k) for k = 0, 1, 2 (Ca, IP3, h); per step an
    IP3 input event of weight 0.2 with probability 0.01; noise off,
    substeps 1, dt 0.1 ms."""

    def __init__(self, n: int, seed: int = 1, p: float = 0.01, weight: float = 0.2,
                 dt: float = 0.1, substeps: int = 1):
        blk = load_astro_block("use_case")
        self.n, self.seed, self.p, self.weight = n, seed, p, weight
        self.dt, self.substeps = dt, substeps
        self.h_step = dt / substeps
        self.consts = np.array([blk[k] for k in CONST_KEYS], dtype=np.float64)
        self.Ca_tot = float(blk["Ca_tot"])
        self.IP3_0 = float(blk["IP3_0"])
        self.tau_IP3 = float(blk["tau_IP3"])
        self.delta_IP3 = float(blk["delta_IP3"])
        self.rest = (float(blk["Ca_init"]), self.IP3_0, float(blk["h_init"]))

    def initial_state(self):
        cells = np.arange(self.n, dtype=np.uint64)
        out = []
        for k, x0 in enumerate(self.rest):
            u = uniform_np(self.seed, cells, k)
            out.append(x0 * (1.0 + 0.1 * (2.0 * u - 1.0)))
        return out  # Ca, IP3, h


class AstroBackend:
    """Resident astrocyte state on the GPU behind the asg_astro_* ABI."""

    def __init__(self, Ca, IP3, h, Ca_tot=None, IP3_0=None, tau_IP3=None, delta_IP3=None):
        lib = _lib.load()
        arrs = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None
                for a in (Ca, IP3, h, Ca_tot, IP3_0, tau_IP3, delta_IP3)]
        self.n = len(arrs[0])
        self._h = C.c_void_p()
        _lib.check(lib.asg_astro_create(self.n, *[_lib.dptr(a) for a in arrs],
                                        C.byref(self._h)), "asg_astro_create")

    def push_input(self, ip3_input):
        a = np.ascontiguousarray(ip3_input, dtype=np.float64)
        _lib.call("asg_astro_push_input", self._h, _lib.dptr(a))

    def update(self, consts, h_step, substeps=1, noise_std=0.0, independent=True,
               shared_noise=0.0, noise_seed=0, noise_index=0):
        c = np.ascontiguousarray(consts, dtype=np.float64)
        _lib.call("asg_astro_update", self._h, _lib.dptr(c), float(h_step), int(substeps),
                  float(noise_std), int(bool(independent)), float(shared_noise),
                  int(noise_seed), int(noise_index))

    def pull_calcium(self):
        out = np.empty(self.n, dtype=np.float64)
        _lib.call("asg_astro_pull_calcium", self._h, _lib.dptr(out))
        return out

    def pull_state(self):
        out = [np.empty(self.n, dtype=np.float64) for _ in range(3)]
        _lib.call("asg_astro_pull_state", self._h, *[_lib.dptr(a) for a in out])
        return out

    def run_bernoulli(self, w: ScalingWorkload, first: int, count: int, uniform=True):
        _lib.call("asg_astro_run_bernoulli", self._h, _lib.dptr(w.consts), w.h_step,
                  w.substeps, w.seed, w.p, w.weight, int(first), int(count), int(uniform),
                  w.Ca_tot, w.IP3_0, w.tau_IP3, w.delta_IP3)
        ms = C.c_double()
        k = C.c_int64()
        _lib.call("asg_astro_last_timing", self._h, C.byref(ms), C.byref(k))
        return ms.value, k.value

    def last_timing(self):
        """(device ms, kernels) of the last run_bernoulli call, or of every
        update since the previous read (waits for them)."""
        ms = C.c_double()
        k = C.c_int64()
        _lib.call("asg_astro_last_timing", self._h, C.byref(ms), C.byref(k))
        return ms.value, k.value

    def run_bernoulli_f32(self, w: ScalingWorkload, first: int, count: int):
        """The same workload in FP32 (the precision study); returns the
        steps' device ms and kernels."""
        _lib.call("asg_astro_run_bernoulli_f32", self._h, _lib.dptr(w.consts), w.h_step,
                  w.substeps, w.seed, w.p, w.weight, int(first), int(count), w.Ca_tot, w.IP3_0,
                  w.tau_IP3, w.delta_IP3)
        return self.last_timing()

    def set_shape(self, shape: int):
        """Use launch shape `shape` (raises AsgError outside the valid range)."""
        _lib.call("asg_astro_set_shape", self._h, int(shape))

    def autotune(self, w: ScalingWorkload, steps=20):
        """Pick the fastest launch shape on a scratch copy (state unchanged)."""
        chosen = C.c_int32()
        us = C.c_double()
        _lib.call("asg_astro_autotune", self._h, _lib.dptr(w.consts), w.h_step, w.substeps,
                  int(steps), C.byref(chosen), C.byref(us))
        return chosen.value, us.value

    def destroy(self):
        if self._h:
            out = [np.empty(self.n, dtype=np.float64) for _ in range(3)]
            _lib.call("asg_astro_destroy", self._h, *[_lib.dptr(a) for a in out])
            self._h = C.c_void_p()
            return out
        return None

    def __del__(self):
        try:
            if self._h:
                _lib.load().asg_astro_destroy(self._h, None, None, None)
        except Exception:
            pass
