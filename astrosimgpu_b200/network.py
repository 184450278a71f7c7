"""Network engine on the B200 (Python view of the asg_model_*, asg_*, asg_batch_*
and asg_serve_* C ABI).

``Model``     the reference's JSON schema and Network::build, on the host.
``Network``   one network on the plain per-step path (asg_create / asg_step).
``Batch``     many instances packed into one engine (asg_batch_*).
``Server``    continuous batching of simulation requests (asg_serve_*).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib

CONFIG_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "configs")


def config_path(name: str) -> str:
    return os.path.join(CONFIG_DIR, name + ".json")


class Model:
    """Configuration + built network tables (host memory, owned by the library)."""

    def __init__(self, path=None, text=None, seed=-1, sim_time=-1.0, pre_time=-1.0,
                 n_astro=-1, build=True, fixed_indegree=None, gen_device=-1):
        self._lib = _lib.load()
        self._h = C.c_void_p()
        if text is not None:
            _lib.call("asg_model_from_json", text.encode(), int(seed), float(sim_time),
                      float(pre_time), int(n_astro), C.byref(self._h))
        else:
            _lib.call("asg_model_from_file", path.encode(), int(seed), float(sim_time),
                      float(pre_time), int(n_astro), C.byref(self._h))
        if build:
            if fixed_indegree is None:
                _lib.call("asg_model_build", self._h)
            else:
                _lib.call("asg_model_build_fixed_indegree", self._h, int(fixed_indegree),
                          int(gen_device))
        s = np.zeros(12)
        _lib.call("asg_model_scalars", self._h, _lib.dptr(s))
        (self.dt, self.substeps, self.seed, self.pre_steps, self.sim_steps, self.record_every,
         self.pre_sim_time, self.sim_time, self.ca_threshold, self.merge_gap, self.hist_window,
         self.hist_shift) = s
        self.substeps = int(self.substeps)
        self.pre_steps, self.sim_steps = int(self.pre_steps), int(self.sim_steps)
        self.record_every = int(self.record_every)

    def desc(self) -> _lib.NetworkDesc:
        d = _lib.NetworkDesc()
        _lib.call("asg_model_desc", self._h, C.byref(d))
        d._owner = self  # keep the model (and its arrays) alive with the view
        return d

    def record_opts(self) -> _lib.RecordOpts:
        r = _lib.RecordOpts()
        _lib.call("asg_model_record_opts", self._h, C.byref(r))
        return r

    def stats(self):
        o = np.zeros(5, np.int64)
        _lib.call("asg_model_stats", self._h, _lib.i64ptr(o))
        return dict(zip(("n_primary_exc", "n_primary_inh", "n_n2a", "n_a2n", "ring_slots"),
                        (int(x) for x in o)))

    def table(self, which: int):
        """CSR (row_start, target) of set `which` (0 exc, 1 inh, 2 n2a, 3 a2n)."""
        d = self.desc()
        c = (d.exc_primary, d.inh_primary, d.neuron_astro, d.astro_neuron)[which]
        n = c.n_sources
        rs = np.ctypeslib.as_array(c.row_start, shape=(n + 1,)).copy() if n else np.zeros(1, np.uint32)
        m = int(rs[-1])
        tg = np.ctypeslib.as_array(c.target, shape=(m,)).copy() if m else np.zeros(0, np.uint32)
        return rs, tg

    def cells(self):
        d = self.desc()
        n, na = d.n_exc + d.n_inh, d.n_astro

        def arr(p, k):
            return np.ctypeslib.as_array(p, shape=(k,)).copy() if k else np.zeros(0)
        return dict(V_reset=arr(d.V_reset, n), b=arr(d.b, n), Ca_tot=arr(d.Ca_tot, na),
                    IP3_0=arr(d.IP3_0, na), tau_IP3=arr(d.tau_IP3, na),
                    delta_IP3=arr(d.delta_IP3, na))

    def close(self):
        if self._h:
            self._lib.asg_model_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def engine_opts(**kw) -> _lib.EngineOpts:
    o = _lib.EngineOpts()
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _alloc_state(n, na):
    st = _lib.State()
    arrs = {k: np.zeros(n) for k in ("V", "w", "g_ex", "dg_ex", "g_in", "dg_in", "I_sic")}
    arrs["refractory"] = np.zeros(n, np.int32)
    for k in ("Ca", "IP3", "h"):
        arrs[k] = np.zeros(na)
    for k, a in arrs.items():
        setattr(st, k, _lib.i32ptr(a) if a.dtype == np.int32 else _lib.dptr(a))
    return st, arrs


class Network:
    """One network on the plain per-step GPU path."""

    def __init__(self, model: Model, record=None, **opts):
        self.model = model
        self.desc = model.desc()
        self.n = self.desc.n_exc + self.desc.n_inh
        self.na = self.desc.n_astro
        rec = record if record is not None else model.record_opts()
        self.rec = rec
        self._h = C.c_void_p()
        _lib.call("asg_create", C.byref(self.desc), C.byref(rec), C.byref(engine_opts(**opts)),
                  C.byref(self._h))

    def step(self, n_steps: int):
        _lib.call("asg_step", self._h, int(n_steps))

    @property
    def current_step(self) -> int:
        s = C.c_int64()
        _lib.call("asg_current_step", self._h, C.byref(s))
        return s.value

    def fetch_spikes(self):
        cnt = C.c_int64()
        _lib.call("asg_fetch_spikes", self._h, None, None, 0, C.byref(cnt))
        n = cnt.value
        st = np.zeros(max(n, 1), np.int64)
        src = np.zeros(max(n, 1), np.uint32)
        _lib.call("asg_fetch_spikes", self._h, _lib.i64ptr(st), _lib.u32ptr(src), n,
                  C.byref(cnt))
        return st[:n], src[:n]

    def fetch_record(self):
        na_rows, nn_rows = C.c_int64(), C.c_int64()
        _lib.call("asg_fetch_record", self._h, None, None, None, 0, C.byref(na_rows), None, None,
                  None, 0, C.byref(nn_rows))
        am, nm = min(self.rec.astro_max, self.na), min(self.rec.neuron_max, self.n)
        a_st = np.zeros(max(na_rows.value, 1), np.int64)
        ca = np.zeros(max(na_rows.value * am, 1))
        ip3 = np.zeros(max(na_rows.value * am, 1))
        n_st = np.zeros(max(nn_rows.value, 1), np.int64)
        v = np.zeros(max(nn_rows.value * nm, 1))
        isic = np.zeros(max(nn_rows.value * nm, 1))
        _lib.call("asg_fetch_record", self._h, _lib.i64ptr(a_st), _lib.dptr(ca), _lib.dptr(ip3),
                  na_rows.value, C.byref(na_rows), _lib.i64ptr(n_st), _lib.dptr(v),
                  _lib.dptr(isic), nn_rows.value, C.byref(nn_rows))
        ra, rn = na_rows.value, nn_rows.value
        return dict(astro_steps=a_st[:ra], Ca=ca[:ra * am].reshape(ra, am),
                    IP3=ip3[:ra * am].reshape(ra, am), neuron_steps=n_st[:rn],
                    V=v[:rn * nm].reshape(rn, nm), I_sic=isic[:rn * nm].reshape(rn, nm))

    def state(self):
        st, arrs = _alloc_state(self.n, self.na)
        _lib.call("asg_pull_state", self._h, C.byref(st))
        return arrs

    def stp(self):
        x, u, t = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        _lib.call("asg_pull_stp", self._h, _lib.dptr(x), _lib.dptr(u), _lib.dptr(t))
        return x, u, t

    def counters(self):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        _lib.call("asg_counters", self._h, C.byref(a), C.byref(b), C.byref(c))
        return dict(spike_edges=a.value, sic_edges=b.value, spikes=c.value)

    def last_timing(self):
        ms, k = C.c_double(), C.c_int64()
        _lib.call("asg_last_timing", self._h, C.byref(ms), C.byref(k))
        return ms.value, k.value

    def autotune(self, steps=64):
        """Pick the fastest launch shape on a snapshot (state unchanged)."""
        o = _lib.EngineOpts()
        _lib.call("asg_autotune", self._h, int(steps), C.byref(o))
        return {f: getattr(o, f) for f, _ in _lib.EngineOpts._fields_}

    def checkpoint(self) -> bytes:
        n = C.c_uint64()
        _lib.call("asg_checkpoint_size", self._h, C.byref(n))
        buf = C.create_string_buffer(n.value)
        _lib.call("asg_checkpoint", self._h, buf, n.value)
        return buf.raw

    def restore(self, blob: bytes):
        buf = C.create_string_buffer(blob, len(blob))
        _lib.call("asg_restore", self._h, buf, len(blob))

    def close(self):
        if self._h:
            _lib.load().asg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many network instances advanced together (asg_batch_*)."""

    def __init__(self, models, record=None, **opts):
        self.models = list(models)
        self.descs = [m.desc() for m in self.models]
        arr = (C.POINTER(_lib.NetworkDesc) * len(self.descs))(
            *[C.pointer(d) for d in self.descs])
        rec = record if record is not None else _lib.RecordOpts(0, 1, 1, 0, 0)
        self.rec = rec
        self._h = C.c_void_p()
        _lib.call("asg_batch_create", len(self.descs), arr, C.byref(rec),
                  C.byref(engine_opts(**opts)), C.byref(self._h))

    def step(self, n_steps: int):
        _lib.call("asg_batch_step", self._h, int(n_steps))

    def fetch_spikes(self, inst: int):
        cnt = C.c_int64()
        _lib.call("asg_batch_fetch_spikes", self._h, inst, None, None, 0, C.byref(cnt))
        n = cnt.value
        st = np.zeros(max(n, 1), np.int64)
        src = np.zeros(max(n, 1), np.uint32)
        _lib.call("asg_batch_fetch_spikes", self._h, inst, _lib.i64ptr(st), _lib.u32ptr(src), n,
                  C.byref(cnt))
        return st[:n], src[:n]

    def fetch_record(self, inst: int):
        """Recorded rows of instance `inst` since its last fetch (see
        Network.fetch_record)."""
        na_rows, nn_rows = C.c_int64(), C.c_int64()
        _lib.call("asg_batch_fetch_record", self._h, inst, None, None, None, 0, C.byref(na_rows),
                  None, None, None, 0, C.byref(nn_rows))
        d = self.descs[inst]
        n, na = d.n_exc + d.n_inh, d.n_astro
        am, nm = min(self.rec.astro_max, na), min(self.rec.neuron_max, n)
        a_st = np.zeros(max(na_rows.value, 1), np.int64)
        ca = np.zeros(max(na_rows.value * am, 1))
        ip3 = np.zeros(max(na_rows.value * am, 1))
        n_st = np.zeros(max(nn_rows.value, 1), np.int64)
        v = np.zeros(max(nn_rows.value * nm, 1))
        isic = np.zeros(max(nn_rows.value * nm, 1))
        _lib.call("asg_batch_fetch_record", self._h, inst, _lib.i64ptr(a_st), _lib.dptr(ca),
                  _lib.dptr(ip3), na_rows.value, C.byref(na_rows), _lib.i64ptr(n_st),
                  _lib.dptr(v), _lib.dptr(isic), nn_rows.value, C.byref(nn_rows))
        ra, rn = na_rows.value, nn_rows.value
        return dict(astro_steps=a_st[:ra], Ca=ca[:ra * am].reshape(ra, am),
                    IP3=ip3[:ra * am].reshape(ra, am), neuron_steps=n_st[:rn],
                    V=v[:rn * nm].reshape(rn, nm), I_sic=isic[:rn * nm].reshape(rn, nm))

    def state(self, inst: int):
        d = self.descs[inst]
        st, arrs = _alloc_state(d.n_exc + d.n_inh, d.n_astro)
        _lib.call("asg_batch_pull_state", self._h, inst, C.byref(st))
        return arrs

    def counters(self, inst: int):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        _lib.call("asg_batch_counters", self._h, inst, C.byref(a), C.byref(b), C.byref(c))
        return dict(spike_edges=a.value, sic_edges=b.value, spikes=c.value)

    def last_timing(self):
        ms, k = C.c_double(), C.c_int64()
        _lib.call("asg_batch_last_timing", self._h, C.byref(ms), C.byref(k))
        return ms.value, k.value

    def autotune(self, steps=64):
        o = _lib.EngineOpts()
        _lib.call("asg_batch_autotune", self._h, int(steps), C.byref(o))
        return {f: getattr(o, f) for f, _ in _lib.EngineOpts._fields_}

    def close(self):
        if self._h:
            _lib.load().asg_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous batching of simulation requests (asg_serve_*)."""

    def __init__(self, mem_budget=0, max_instances=256, **opts):
        o = _lib.ServeOpts()
        o.engine = engine_opts(**opts)
        o.mem_budget = int(mem_budget)
        o.max_instances = int(max_instances)
        self._h = C.c_void_p()
        _lib.call("asg_serve_create", C.byref(o), C.byref(self._h))
        self._keep = {}

    def submit(self, model: Model, n_steps: int, keep_spikes=True) -> int:
        d = model.desc()
        rid = C.c_int64()
        _lib.call("asg_serve_submit", self._h, C.byref(d), int(n_steps), int(keep_spikes),
                  C.byref(rid))
        return rid.value

    def poll(self, rid: int):
        done = C.c_int32()
        res = _lib.RequestResult()
        _lib.call("asg_serve_poll", self._h, int(rid), C.byref(done), C.byref(res))
        return bool(done.value), res

    def wait(self, rid: int, timeout_ms=-1.0):
        res = _lib.RequestResult()
        _lib.call("asg_serve_wait", self._h, int(rid), float(timeout_ms), C.byref(res))
        return res

    def fetch_spikes(self, rid: int):
        cnt = C.c_int64()
        _lib.call("asg_serve_fetch_spikes", self._h, int(rid), None, None, 0, C.byref(cnt))
        n = cnt.value
        st = np.zeros(max(n, 1), np.int64)
        src = np.zeros(max(n, 1), np.uint32)
        _lib.call("asg_serve_fetch_spikes", self._h, int(rid), _lib.i64ptr(st), _lib.u32ptr(src),
                  n, C.byref(cnt))
        return st[:n], src[:n]

    def cancel(self, rid: int):
        _lib.call("asg_serve_cancel", self._h, int(rid))

    def stats(self):
        ch, k, ms, r, pk = C.c_int64(), C.c_int64(), C.c_double(), C.c_int32(), C.c_int32()
        _lib.call("asg_serve_stats", self._h, C.byref(ch), C.byref(k), C.byref(ms), C.byref(r),
                  C.byref(pk))
        return dict(chunks=ch.value, kernels=k.value, device_ms=ms.value, resident=r.value,
                    peak_resident=pk.value)

    def close(self):
        if self._h:
            _lib.load().asg_serve_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def calcium_analysis(times, ca, threshold, merge_gap, win_start, win_end, width, shift):
    """Calcium analysis of traces (asg_calcium_analysis, the semantics of the
    reference's analysis.cpp): `times` and `ca` are cells x samples.  Returns
    active cells, transients, mean duration (ms), pairs correlated and the
    mean pairwise correlation."""
    t = np.ascontiguousarray(times, np.float64)
    c = np.ascontiguousarray(ca, np.float64)
    out = np.zeros(5)
    _lib.call("asg_calcium_analysis", _lib.dptr(t), _lib.dptr(c), int(c.shape[0]),
              int(c.shape[1]), float(threshold), float(merge_gap), float(win_start),
              float(win_end), float(width), float(shift), _lib.dptr(out))
    return dict(active=int(out[0]), transients=int(out[1]), mean_duration_ms=float(out[2]),
                pairs=int(out[3]), correlation=float(out[4]))
