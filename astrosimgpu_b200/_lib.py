"""ctypes binding of ``libasg_b200.so`` (the C ABI declared in include/asg_b200.h).

The library is loaded from this package directory.  There is no fallback:
if the shared library is missing or fails to load, every entry point raises,
so nothing can silently run on the CPU instead of the GPU.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libasg_b200.so")

ASG_OK = 0
STATUS_NAMES = {
    0: "ASG_OK", 1: "ASG_ERR_ARG", 2: "ASG_ERR_OOM", 3: "ASG_ERR_CUDA",
    4: "ASG_ERR_UNSUPPORTED", 5: "ASG_ERR_TIMEOUT", 6: "ASG_ERR_OVERFLOW",
    7: "ASG_ERR_CONFIG", 8: "ASG_ERR_STATE", 9: "ASG_ERR_CANCELLED",
    10: "ASG_ERR_NO_DEVICE", 11: "ASG_ERR_NOT_FOUND",
}


class AsgError(RuntimeError):
    """A non-zero status from the C ABI, with asg_last_error()'s text."""

    def __init__(self, status: int, where: str, text: str):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {text}")


_lib = None

c_double_p = C.POINTER(C.c_double)
c_int32_p = C.POINTER(C.c_int32)
c_int64_p = C.POINTER(C.c_int64)
c_uint32_p = C.POINTER(C.c_uint32)
c_uint64_p = C.POINTER(C.c_uint64)


class NeuronParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "C_m", "g_L", "E_L", "V_th", "Delta_T", "a", "tau_w", "V_peak", "t_ref", "E_ex",
        "E_in", "tau_syn_ex", "tau_syn_in", "I_e")]


class AstroParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "Kd_IP3_1", "Kd_IP3_2", "Kd_act", "Kd_inh", "Km_SERCA", "k_IP3R", "rate_IP3R",
        "rate_L", "rate_SERCA", "ratio_ER_cyt", "SIC_scale", "SIC_th")]


class InputParams(C.Structure):
    _fields_ = [("poiss_rate", C.c_double), ("poiss_weight", C.c_double),
                ("gauss_noise_std", C.c_double), ("noise_dt", C.c_double),
                ("independent_noise", C.c_int32)]


class StpParams(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("U", C.c_double), ("tau_rec", C.c_double),
                ("tau_fac", C.c_double)]


class Csr(C.Structure):
    _fields_ = [("n_sources", C.c_uint32), ("row_start", c_uint32_p), ("target", c_uint32_p),
                ("weight", c_double_p), ("delay_steps", c_int32_p), ("stp_x", c_double_p),
                ("stp_u", c_double_p), ("stp_t_last", c_double_p)]


class NetworkDesc(C.Structure):
    _fields_ = [
        ("n_exc", C.c_uint32), ("n_inh", C.c_uint32), ("n_astro", C.c_uint32),
        ("dt", C.c_double), ("substeps", C.c_int32), ("seed", C.c_uint64),
        ("sic_interval", C.c_int32),
        ("d_e_steps", C.c_int32), ("d_i_steps", C.c_int32), ("d_a2n_steps", C.c_int32),
        ("w_e", C.c_double), ("w_i", C.c_double), ("w_n2a", C.c_double), ("w_a2n", C.c_double),
        ("exc", NeuronParams), ("inh", NeuronParams), ("astro", AstroParams),
        ("input_exc", InputParams), ("input_inh", InputParams), ("input_astro", InputParams),
        ("stp", StpParams),
        ("exc_primary", Csr), ("inh_primary", Csr), ("neuron_astro", Csr), ("astro_neuron", Csr),
        ("V_reset", c_double_p), ("b", c_double_p),
        ("Ca_tot", c_double_p), ("IP3_0", c_double_p), ("tau_IP3", c_double_p),
        ("delta_IP3", c_double_p),
        ("Ca_tot_u", C.c_double), ("IP3_0_u", C.c_double), ("tau_IP3_u", C.c_double),
        ("delta_IP3_u", C.c_double),
        ("V_m_init_exc", C.c_double), ("V_m_init_inh", C.c_double), ("Ca_init", C.c_double),
        ("IP3_init", C.c_double), ("h_init", C.c_double),
        ("V", c_double_p), ("w", c_double_p), ("g_ex", c_double_p), ("dg_ex", c_double_p),
        ("g_in", c_double_p), ("dg_in", c_double_p), ("I_sic", c_double_p),
        ("refractory", c_int32_p),
        ("Ca", c_double_p), ("IP3", c_double_p), ("h", c_double_p),
    ]


class RecordOpts(C.Structure):
    _fields_ = [("record_from_step", C.c_int64), ("record_every", C.c_int32),
                ("spikes", C.c_int32), ("astro_max", C.c_uint32), ("neuron_max", C.c_uint32)]


class State(C.Structure):
    _fields_ = [("V", c_double_p), ("w", c_double_p), ("g_ex", c_double_p),
                ("dg_ex", c_double_p), ("g_in", c_double_p), ("dg_in", c_double_p),
                ("I_sic", c_double_p), ("refractory", c_int32_p),
                ("Ca", c_double_p), ("IP3", c_double_p), ("h", c_double_p)]


class EngineOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("chunk_steps", C.c_int32), ("block", C.c_int32),
                ("use_graphs", C.c_int32), ("sic_mode", C.c_int32), ("pdl", C.c_int32),
                ("push_mode", C.c_int32), ("mem_budget", C.c_uint64), ("occupancy", C.c_int32),
                ("astro_precision", C.c_int32)]


class ServeOpts(C.Structure):
    _fields_ = [("engine", EngineOpts), ("mem_budget", C.c_uint64),
                ("max_instances", C.c_int32)]


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("n_spikes", C.c_int64), ("spike_edges", C.c_int64),
                ("sic_edges", C.c_int64), ("submit_to_admit_ms", C.c_double),
                ("submit_to_done_ms", C.c_double), ("mean_rate_hz", C.c_double)]


vp = C.c_void_p
vpp = C.POINTER(C.c_void_p)

# name -> (restype, argtypes); every function returns an int status unless noted.
SIGNATURES = {
    "asg_last_error": (C.c_char_p, []),
    "asg_version": (C.c_char_p, []),
    # single network
    "asg_create": (C.c_int, [C.POINTER(NetworkDesc), C.POINTER(RecordOpts),
                             C.POINTER(EngineOpts), vpp]),
    "asg_step": (C.c_int, [vp, C.c_int64]),
    "asg_current_step": (C.c_int, [vp, c_int64_p]),
    "asg_fetch_spikes": (C.c_int, [vp, c_int64_p, c_uint32_p, C.c_int64, c_int64_p]),
    "asg_fetch_record": (C.c_int, [vp, c_int64_p, c_double_p, c_double_p, C.c_int64, c_int64_p,
                                   c_int64_p, c_double_p, c_double_p, C.c_int64, c_int64_p]),
    "asg_pull_state": (C.c_int, [vp, C.POINTER(State)]),
    "asg_pull_stp": (C.c_int, [vp, c_double_p, c_double_p, c_double_p]),
    "asg_counters": (C.c_int, [vp, c_int64_p, c_int64_p, c_int64_p]),
    "asg_last_timing": (C.c_int, [vp, c_double_p, c_int64_p]),
    "asg_checkpoint_size": (C.c_int, [vp, c_uint64_p]),
    "asg_checkpoint": (C.c_int, [vp, vp, C.c_uint64]),
    "asg_restore": (C.c_int, [vp, vp, C.c_uint64]),
    "asg_destroy": (C.c_int, [vp]),
    "asg_autotune": (C.c_int, [vp, C.c_int32, C.POINTER(EngineOpts)]),
    # batch
    "asg_batch_create": (C.c_int, [C.c_int32, C.POINTER(C.POINTER(NetworkDesc)),
                                   C.POINTER(RecordOpts), C.POINTER(EngineOpts), vpp]),
    "asg_batch_step": (C.c_int, [vp, C.c_int64]),
    "asg_batch_fetch_spikes": (C.c_int, [vp, C.c_int32, c_int64_p, c_uint32_p, C.c_int64,
                                         c_int64_p]),
    "asg_batch_fetch_record": (C.c_int, [vp, C.c_int32, c_int64_p, c_double_p, c_double_p,
                                         C.c_int64, c_int64_p, c_int64_p, c_double_p,
                                         c_double_p, C.c_int64, c_int64_p]),
    "asg_batch_pull_state": (C.c_int, [vp, C.c_int32, C.POINTER(State)]),
    "asg_batch_counters": (C.c_int, [vp, C.c_int32, c_int64_p, c_int64_p, c_int64_p]),
    "asg_batch_last_timing": (C.c_int, [vp, c_double_p, c_int64_p]),
    "asg_batch_autotune": (C.c_int, [vp, C.c_int32, C.POINTER(EngineOpts)]),
    "asg_batch_destroy": (C.c_int, [vp]),
    # serving
    "asg_serve_create": (C.c_int, [C.POINTER(ServeOpts), vpp]),
    "asg_serve_submit": (C.c_int, [vp, C.POINTER(NetworkDesc), C.c_int64, C.c_int32,
                                   c_int64_p]),
    "asg_serve_poll": (C.c_int, [vp, C.c_int64, c_int32_p, C.POINTER(RequestResult)]),
    "asg_serve_wait": (C.c_int, [vp, C.c_int64, C.c_double, C.POINTER(RequestResult)]),
    "asg_serve_fetch_spikes": (C.c_int, [vp, C.c_int64, c_int64_p, c_uint32_p, C.c_int64,
                                         c_int64_p]),
    "asg_serve_cancel": (C.c_int, [vp, C.c_int64]),
    "asg_serve_stats": (C.c_int, [vp, c_int64_p, c_int64_p, c_double_p, c_int32_p, c_int32_p]),
    "asg_serve_destroy": (C.c_int, [vp]),
    # astrocyte backend
    "asg_astro_create": (C.c_int, [C.c_uint32, c_double_p, c_double_p, c_double_p, c_double_p,
                                   c_double_p, c_double_p, c_double_p, vpp]),
    "asg_astro_destroy": (C.c_int, [vp, c_double_p, c_double_p, c_double_p]),
    "asg_astro_set_shape": (C.c_int, [vp, C.c_int32]),
    "asg_astro_push_input": (C.c_int, [vp, c_double_p]),
    "asg_astro_pull_calcium": (C.c_int, [vp, c_double_p]),
    "asg_astro_update": (C.c_int, [vp, c_double_p, C.c_double, C.c_int32, C.c_double, C.c_int32,
                                   C.c_double, C.c_uint64, C.c_uint64]),
    "asg_astro_run_bernoulli": (C.c_int, [vp, c_double_p, C.c_double, C.c_int32, C.c_uint64,
                                          C.c_double, C.c_double, C.c_int64, C.c_int64,
                                          C.c_int32, C.c_double, C.c_double, C.c_double,
                                          C.c_double]),
    "asg_astro_run_bernoulli_f32": (C.c_int, [vp, c_double_p, C.c_double, C.c_int32, C.c_uint64,
                                              C.c_double, C.c_double, C.c_int64, C.c_int64,
                                              C.c_double, C.c_double, C.c_double, C.c_double]),
    "asg_astro_pull_state": (C.c_int, [vp, c_double_p, c_double_p, c_double_p]),
    "asg_astro_last_timing": (C.c_int, [vp, c_double_p, c_int64_p]),
    "asg_astro_autotune": (C.c_int, [vp, c_double_p, C.c_double, C.c_int32, C.c_int32,
                                     c_int32_p, c_double_p]),
    "asg_astro_update_noalloc": (C.c_int, [C.c_uint32] + [vp] * 8 + [c_double_p, C.c_double,
                                           C.c_int32, C.c_double, C.c_int32, C.c_double,
                                           C.c_uint64, C.c_uint64, vp]),
    # host config + builder
    "asg_model_from_json": (C.c_int, [C.c_char_p, C.c_int64, C.c_double, C.c_double, C.c_int64,
                                      vpp]),
    "asg_model_from_file": (C.c_int, [C.c_char_p, C.c_int64, C.c_double, C.c_double, C.c_int64,
                                      vpp]),
    "asg_model_build": (C.c_int, [vp]),
    "asg_model_build_fixed_indegree": (C.c_int, [vp, C.c_uint32, C.c_int32]),
    "asg_model_desc": (C.c_int, [vp, C.POINTER(NetworkDesc)]),
    "asg_model_record_opts": (C.c_int, [vp, C.POINTER(RecordOpts)]),
    "asg_model_scalars": (C.c_int, [vp, c_double_p]),
    "asg_model_stats": (C.c_int, [vp, c_int64_p]),
    "asg_model_free": (C.c_int, [vp]),
    "asg_selftest_barrier_timeout": (C.c_int, [c_int32_p, c_double_p]),
    "asg_calcium_analysis": (C.c_int, [c_double_p, c_double_p, C.c_int32, C.c_int32, C.c_double,
                                       C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double, c_double_p]),
}


def load():
    """Load the library (once) and declare every signature.  Raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; "
            "g.build()'` (no CPU fallback exists)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, where: str) -> None:
    if status != ASG_OK:
        text = load().asg_last_error().decode(errors="replace")
        raise AsgError(status, where, text)


def call(name: str, *args) -> None:
    """Call an int-status entry point and raise AsgError on failure."""
    fn = getattr(load(), name)
    check(fn(*args), name)


def dptr(a):
    """Pointer to a contiguous float64 numpy array (or NULL for None)."""
    if a is None:
        return None
    assert a.dtype.name == "float64" and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(c_double_p)


def i32ptr(a):
    if a is None:
        return None
    assert a.dtype.name == "int32" and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(c_int32_p)


def u32ptr(a):
    if a is None:
        return None
    assert a.dtype.name == "uint32" and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(c_uint32_p)


def i64ptr(a):
    if a is None:
        return None
    assert a.dtype.name == "int64" and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(c_int64_p)
