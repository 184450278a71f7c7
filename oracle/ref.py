"""ctypes view of the checkers (test infrastructure only).

- ``_ref/libastroref.so``: the REFERENCE simulator compiled from its own
  sources (see oracle/Makefile and ref_shim.cpp).
- ``_ref/libastroref_cuda.so``: the reference's native CUDA astrocyte
  backend compiled for sm_100a.
- ``liboracle.so``: the C restatement in asg_oracle.c.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs import this module, and only as the checker or the baseline
being timed; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libastroref.so")
REF_CUDA_LIB = os.path.join(HERE, "_ref", "libastroref_cuda.so")
REF_CLI = os.path.join(HERE, "_ref", "astrosimgpu")
PORT_LIB = os.path.join(HERE, "liboracle.so")

_ref = None
_refcu = None
_port = None

D = C.POINTER(C.c_double)
I32 = C.POINTER(C.c_int32)
U32 = C.POINTER(C.c_uint32)
I64 = C.POINTER(C.c_int64)


def _dp(a):
    return None if a is None else a.ctypes.data_as(D)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref():
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_LIB)
        lib.ref_net_create.restype = C.c_void_p
        lib.ref_net_create.argtypes = [C.c_char_p, C.c_longlong, C.c_double, C.c_double,
                                       C.c_longlong, C.c_char_p, C.c_int]
        lib.ref_net_create_text.restype = C.c_void_p
        lib.ref_net_create_text.argtypes = [C.c_char_p, C.c_longlong, C.c_char_p, C.c_int]
        lib.ref_net_destroy.argtypes = [C.c_void_p]
        lib.ref_net_stats.argtypes = [C.c_void_p, I64]
        lib.ref_net_time.argtypes = [C.c_void_p, D]
        lib.ref_net_table_size.restype = C.c_int64
        lib.ref_net_table_size.argtypes = [C.c_void_p, C.c_int]
        lib.ref_net_table_rows.restype = C.c_int64
        lib.ref_net_table_rows.argtypes = [C.c_void_p, C.c_int]
        lib.ref_net_table.argtypes = [C.c_void_p, C.c_int, U32, U32, D, I32, D, D, D]
        lib.ref_net_cells.argtypes = [C.c_void_p, D, D, D, D, D, D]
        lib.ref_net_state.argtypes = [C.c_void_p, D, I32, D]
        lib.ref_net_ring.argtypes = [C.c_void_p, C.c_int, D]
        lib.ref_net_step.restype = C.c_int
        lib.ref_net_step.argtypes = [C.c_void_p, C.c_int64, U32, C.c_int]
        lib.ref_net_run.restype = C.c_int64
        lib.ref_net_run.argtypes = [C.c_void_p, C.c_int64, C.c_int64, I64, U32, C.c_int64]
        lib.ref_net_sic_factors.argtypes = [C.c_void_p, D]
        lib.ref_net_set_state.argtypes = [C.c_void_p, D, I32, D]
        lib.ref_net_load_table.restype = C.c_int
        lib.ref_net_load_table.argtypes = [C.c_void_p, C.c_int, C.c_int64, U32, U32]
        lib.ref_rng_bits.restype = C.c_uint64
        lib.ref_rng_bits.argtypes = [C.c_uint64] * 3
        lib.ref_rng_uniform.restype = C.c_double
        lib.ref_rng_uniform.argtypes = [C.c_uint64] * 3
        lib.ref_rng_normal.restype = C.c_double
        lib.ref_rng_normal.argtypes = [C.c_uint64] * 2
        lib.ref_counter_rng.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_double, C.c_int, D]
        lib.ref_astro_advance.argtypes = [D, C.c_int64, D, D, D, D, D, D, C.c_double, C.c_int,
                                          D, D, D]
        lib.ref_astro_scaling.restype = C.c_double
        lib.ref_astro_scaling.argtypes = [D, C.c_double, C.c_double, C.c_double, C.c_double,
                                          C.c_double, C.c_int, C.c_uint64, C.c_double,
                                          C.c_double, C.c_int64, C.c_int64, C.c_int64, D, D, D,
                                          C.c_int]
        lib.ref_omp_max_threads.restype = C.c_int
        lib.ref_calcium_analysis.argtypes = [D, D, C.c_int, C.c_int, C.c_double, C.c_double,
                                             C.c_double, C.c_double, C.c_double, C.c_double, D]
        _ref = lib
    return _ref


def refcu():
    global _refcu
    if _refcu is None:
        lib = C.CDLL(REF_CUDA_LIB)
        lib.refcu_create.restype = C.c_void_p
        lib.refcu_create.argtypes = [C.c_uint] + [D] * 7
        lib.refcu_destroy.argtypes = [C.c_void_p, D, D, D]
        lib.refcu_push_input.argtypes = [C.c_void_p, D]
        lib.refcu_pull_calcium.argtypes = [C.c_void_p, D]
        lib.refcu_update.argtypes = [C.c_void_p, D, C.c_double, C.c_int, C.c_double, C.c_int,
                                     C.c_double, C.c_ulonglong, C.c_ulonglong]
        lib.refcu_time_updates.restype = C.c_float
        lib.refcu_time_updates.argtypes = [C.c_void_p, D, C.c_double, C.c_int, C.c_int]
        _refcu = lib
    return _refcu


class RefNetwork:
    """The reference Network built from a config file or JSON text."""

    def __init__(self, path=None, text=None, seed=-1, sim_time=-1.0, pre_time=-1.0,
                 n_astro=-1):
        lib = ref()
        err = C.create_string_buffer(4096)
        if text is not None:
            self.h = lib.ref_net_create_text(text.encode(), seed, err, 4096)
        else:
            self.h = lib.ref_net_create(path.encode(), seed, sim_time, pre_time, n_astro, err,
                                        4096)
        if not self.h:
            raise RuntimeError("reference build failed: " + err.value.decode())
        st = np.zeros(9, dtype=np.int64)
        lib.ref_net_stats(self.h, st.ctypes.data_as(I64))
        (self.n_astro, self.n_exc, self.n_inh, self.n_primary_exc, self.n_primary_inh,
         self.n_n2a, self.n_a2n, self.ring_slots, self.sic_delay) = [int(x) for x in st]
        self.n = self.n_exc + self.n_inh
        t = np.zeros(8)
        lib.ref_net_time(self.h, _dp(t))
        self.dt, self.substeps = float(t[0]), int(t[1])
        self.seed, self.pre_steps, self.sim_steps = int(t[2]), int(t[3]), int(t[4])
        self.step = 0

    def close(self):
        if self.h:
            ref().ref_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def table(self, which: int):
        """CSR of set `which` (0 exc, 1 inh, 2 neuron->astro, 3 astro->neuron)."""
        lib = ref()
        rows = int(lib.ref_net_table_rows(self.h, which))
        m = int(lib.ref_net_table_size(self.h, which))
        rs = np.zeros(rows + 1, np.uint32)
        tg = np.zeros(m, np.uint32)
        w = np.zeros(m)
        d = np.zeros(m, np.int32)
        x = np.full(m, np.nan)
        u = np.full(m, np.nan)
        tl = np.full(m, np.nan)
        lib.ref_net_table(self.h, which, rs.ctypes.data_as(U32), tg.ctypes.data_as(U32), _dp(w),
                          d.ctypes.data_as(I32), _dp(x), _dp(u), _dp(tl))
        return dict(row_start=rs, target=tg, weight=w, delay=d, stp_x=x, stp_u=u, stp_t_last=tl)

    def cells(self):
        n, na = self.n, self.n_astro
        a = [np.zeros(n), np.zeros(n)] + [np.zeros(na) for _ in range(4)]
        ref().ref_net_cells(self.h, *[_dp(x) for x in a])
        return dict(zip(("V_reset", "b", "Ca_tot", "IP3_0", "tau_IP3", "delta_IP3"), a))

    def state(self):
        n, na = self.n, self.n_astro
        n7 = np.zeros(7 * n)
        refr = np.zeros(n, np.int32)
        a3 = np.zeros(3 * na)
        ref().ref_net_state(self.h, _dp(n7), refr.ctypes.data_as(I32), _dp(a3))
        keys = ("V", "w", "g_ex", "dg_ex", "g_in", "dg_in", "I_sic")
        out = {k: n7[i * n:(i + 1) * n].copy() for i, k in enumerate(keys)}
        out["refractory"] = refr
        out["Ca"], out["IP3"], out["h"] = (a3[:na].copy(), a3[na:2 * na].copy(),
                                           a3[2 * na:].copy())
        return out

    def run(self, count: int, cap: int | None = None):
        """Advance `count` steps; returns (steps, sources) of the spikes."""
        cap = cap if cap is not None else self.n * count + 1  # at most one spike per cell-step
        st = np.zeros(cap, np.int64)
        src = np.zeros(cap, np.uint32)
        total = int(ref().ref_net_run(self.h, self.step, count, st.ctypes.data_as(I64),
                                      src.ctypes.data_as(U32), cap))
        if total > cap:
            raise RuntimeError("spike buffer too small")
        self.step += count
        return st[:total], src[:total]

    def set_state(self, st):
        """Overwrite the dynamic state (dict with the keys of state())."""
        keys = ("V", "w", "g_ex", "dg_ex", "g_in", "dg_in", "I_sic")
        n7 = np.ascontiguousarray(np.concatenate([np.asarray(st[k], np.float64) for k in keys]))
        refr = np.ascontiguousarray(st["refractory"], np.int32)
        a3 = np.ascontiguousarray(np.concatenate([np.asarray(st[k], np.float64)
                                                  for k in ("Ca", "IP3", "h")]))
        ref().ref_net_set_state(self.h, _dp(n7), refr.ctypes.data_as(I32), _dp(a3))

    def load_table(self, which: int, row_start, target):
        """Replace connection set `which` by the CSR (row_start, target)."""
        rs = np.ascontiguousarray(row_start, np.uint32)
        tg = np.ascontiguousarray(target, np.uint32)
        if len(tg) == 0:
            tg = np.zeros(1, np.uint32)
        rc = ref().ref_net_load_table(self.h, which, len(rs) - 1, rs.ctypes.data_as(U32),
                                      tg.ctypes.data_as(U32))
        if rc != 0:
            raise ValueError(f"table {which}: {len(rs) - 1} rows do not match the set's sources")

    def sic_factors(self):
        out = np.zeros(self.n_astro)
        ref().ref_net_sic_factors(self.h, _dp(out))
        return out


def ref_astro_scaling(w, Ca, IP3, h, first, count, threads=0):
    """Reference astro_advance over the scaling workload on the host (OpenMP);
    updates Ca/IP3/h in place and returns the loop's wall seconds."""
    return ref().ref_astro_scaling(_dp(w.consts), w.Ca_tot, w.IP3_0, w.tau_IP3, w.delta_IP3,
                                   w.h_step, w.substeps, w.seed, w.p, w.weight, first, count,
                                   len(Ca), _dp(Ca), _dp(IP3), _dp(h), threads)


def port():
    global _port
    if _port is None:
        _port = C.CDLL(PORT_LIB)
    return _port
