"""Config reader for the C restatement (test infrastructure only).

Restates the reference's load_config (parameters.cpp:85-205) with the
defaults of parameters.hpp:14-198 and packs the resolved values into the
flat ORC_* array that asg_oracle.c's orc_net_build takes.
"""
from __future__ import annotations

import ctypes as C
import json
import re

import numpy as np

ASTRO_DEFAULTS = dict(Ca_tot=2.0, IP3_0=0.16, Kd_IP3_1=0.13, Kd_IP3_2=0.9434, Kd_act=0.08234,
                      Kd_inh=1.049, Km_SERCA=0.1, SIC_scale=1.0, SIC_th=0.19669,
                      delta_IP3=0.0002, k_IP3R=0.0002, rate_IP3R=0.006, rate_L=0.00011,
                      rate_SERCA=0.0009, ratio_ER_cyt=0.185, tau_IP3=7142.0, Ca_init=0.073,
                      h_init=0.793, IP3_init=0.16)
NEURON_KEYS = ("C_m", "g_L", "E_L", "V_th", "Delta_T", "a", "b", "tau_w", "V_reset", "V_peak",
               "t_ref", "E_ex", "E_in", "tau_syn_ex", "tau_syn_in", "I_e", "V_m_init")
NEURON_DEFAULTS = dict(C_m=281.0, g_L=30.0, E_L=-70.6, V_th=-50.4, Delta_T=2.0, a=4.0, b=80.5,
                       tau_w=144.0, V_reset=-60.0, V_peak=0.0, t_ref=0.0, E_ex=0.0, E_in=-85.0,
                       tau_syn_ex=0.2, tau_syn_in=2.0, I_e=0.0, V_m_init=-70.6)


def strip_comments(text: str) -> str:
    out = []
    for line in text.splitlines():
        # '//' outside strings (config strings hold no '//')
        i = line.find("//")
        out.append(line if i < 0 else line[:i])
    return "\n".join(out)


def load(path=None, text=None, seed=None):
    if text is None:
        with open(path) as f:
            text = f.read()
    j = json.loads(strip_comments(text))
    N = j.get("N", {})
    sim = j.get("simulation", {})
    c = {"N_A": N.get("N_A", 100), "N_E": N.get("N_E", 400), "N_I": N.get("N_I", 100),
         "dt": sim.get("dt", 0.1), "substeps": sim.get("substeps", 1),
         "seed": sim.get("seed", 1) if seed is None else seed}
    a = dict(ASTRO_DEFAULTS)
    for k, v in j.get("astrocyte", {}).items():
        a["IP3_init" if k == "IP3" else k] = v
    c["astro"] = a

    def neuron(blk):
        p = dict(NEURON_DEFAULTS)
        for k, v in blk.items():
            p["V_m_init" if k == "V_m" else k] = v
        return p

    c["exc"] = neuron(j.get("neuron_exc", {}))
    c["inh"] = neuron(j.get("neuron_inh", {}))

    def inp(blk):
        d = dict(poiss_rate=0.0, poiss_weight=1.0, std=0.0, noise_dt=0.0, independent=True)
        for k, v in blk.items():
            if k in ("gauss_noise_var", "gauss_noise_std"):
                d["std"] = v
            elif k == "independent_noise":
                d["independent"] = v
            else:
                d[k] = v
        if d["noise_dt"] <= 0.0:
            d["noise_dt"] = 10.0 * c["dt"]
        return d

    c["in_a"], c["in_e"], c["in_i"] = (inp(j.get("input_astro", {})), inp(j.get("input_exc", {})),
                                       inp(j.get("input_inh", {})))

    def rnd(blk):
        if blk is None:
            return dict(enabled=False, lower=1.0, upper=1.0, var=0.0)
        d = dict(enabled=True, lower=1.0, upper=1.0, var=0.0)
        d.update(blk)
        return d

    c["rnd_a"] = rnd(j.get("randomize_astro"))
    c["rnd_n"] = rnd(j.get("randomize_neuron"))
    s = dict(w_e=5.0, w_i=-5.0, w_n2a=0.2, w_a2n=1.0, d_e=1.0, d_i=1.0, d_a2n=1.0,
             sic_interval=1)
    syn = j.get("synapse", {})
    for k, v in syn.items():
        if k != "stp":
            s[k] = v
    stp = dict(enabled=True, U=0.5, tau_rec=800.0, tau_fac=0.0)
    stp.update(syn.get("stp", {}))
    s["stp"] = stp
    c["syn"] = s
    conn = dict(p_primary=0.2, p_third_if_primary=0.2, pool_size=1, pool_type="block",
                allow_autapses=False, unique_third_out=False)
    conn.update(j.get("connectivity", {}))
    c["conn"] = conn
    return c


def to_flat(c) -> np.ndarray:
    a, s, cn = c["astro"], c["syn"], c["conn"]
    v = [c["N_A"], c["N_E"], c["N_I"], c["dt"], c["substeps"], float(c["seed"])]
    v += [a[k] for k in ("Ca_tot", "IP3_0", "Kd_IP3_1", "Kd_IP3_2", "Kd_act", "Kd_inh",
                         "Km_SERCA", "SIC_scale", "SIC_th", "delta_IP3", "k_IP3R", "rate_IP3R",
                         "rate_L", "rate_SERCA", "ratio_ER_cyt", "tau_IP3", "Ca_init", "h_init",
                         "IP3_init")]
    v += [c["exc"][k] for k in NEURON_KEYS]
    v += [c["inh"][k] for k in NEURON_KEYS]
    v += [s["w_e"], s["w_i"], s["w_n2a"], s["w_a2n"], s["d_e"], s["d_i"], s["d_a2n"],
          s["sic_interval"], float(bool(s["stp"]["enabled"])), s["stp"]["U"],
          s["stp"]["tau_rec"], s["stp"]["tau_fac"]]
    v += [cn["p_primary"], cn["p_third_if_primary"], cn["pool_size"],
          float(cn["pool_type"] == "random"), float(bool(cn["allow_autapses"])),
          float(bool(cn["unique_third_out"]))]
    for key in ("in_a", "in_e", "in_i"):
        d = c[key]
        v += [d["poiss_rate"], d["poiss_weight"], d["std"], d["noise_dt"],
              float(bool(d["independent"]))]
    for key in ("rnd_a", "rnd_n"):
        d = c[key]
        v += [float(bool(d["enabled"])), d["lower"], d["upper"], d["var"]]
    return np.array(v, dtype=np.float64)


class PortNetwork:
    """The C restatement's network (asg_oracle.c)."""

    def __init__(self, cfg: dict):
        from . import ref
        self.lib = ref.port()
        L = self.lib
        L.orc_net_build.restype = C.c_void_p
        L.orc_net_build.argtypes = [C.POINTER(C.c_double)]
        L.orc_net_free.argtypes = [C.c_void_p]
        L.orc_net_table_size.restype = C.c_int64
        L.orc_net_table_size.argtypes = [C.c_void_p, C.c_int]
        L.orc_net_table.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint32)]
        L.orc_net_cells.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 6
        L.orc_net_step.restype = C.c_int
        L.orc_net_step.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_uint32), C.c_int]
        L.orc_net_state.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32),
                                    C.POINTER(C.c_double)]
        flat = to_flat(cfg)
        self.h = L.orc_net_build(flat.ctypes.data_as(C.POINTER(C.c_double)))
        self.NA, self.NE, self.NI = int(cfg["N_A"]), int(cfg["N_E"]), int(cfg["N_I"])
        self.N = self.NE + self.NI
        self.step = 0

    def close(self):
        if self.h:
            self.lib.orc_net_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def table(self, which):
        m = int(self.lib.orc_net_table_size(self.h, which))
        rows = {0: self.NE, 1: self.NI, 2: self.NE, 3: self.NA}[which]
        rs = np.zeros(rows + 1, np.uint32)
        tg = np.zeros(max(m, 1), np.uint32)
        self.lib.orc_net_table(self.h, which, rs.ctypes.data_as(C.POINTER(C.c_uint32)),
                               tg.ctypes.data_as(C.POINTER(C.c_uint32)))
        return rs, tg[:m]

    def cells(self):
        a = [np.zeros(self.N), np.zeros(self.N)] + [np.zeros(self.NA) for _ in range(4)]
        self.lib.orc_net_cells(self.h, *[x.ctypes.data_as(C.POINTER(C.c_double)) for x in a])
        return dict(zip(("V_reset", "b", "Ca_tot", "IP3_0", "tau_IP3", "delta_IP3"), a))

    def run(self, count):
        buf = np.zeros(self.N + 1, np.uint32)
        steps, srcs = [], []
        for s in range(self.step, self.step + count):
            k = self.lib.orc_net_step(self.h, s, buf.ctypes.data_as(C.POINTER(C.c_uint32)),
                                      len(buf))
            steps += [s] * k
            srcs += list(buf[:k])
        self.step += count
        return np.array(steps, np.int64), np.array(srcs, np.uint32)

    def state(self):
        n, na = self.N, self.NA
        n7 = np.zeros(7 * max(n, 1))
        refr = np.zeros(max(n, 1), np.int32)
        a3 = np.zeros(3 * max(na, 1))
        self.lib.orc_net_state(self.h, n7.ctypes.data_as(C.POINTER(C.c_double)),
                               refr.ctypes.data_as(C.POINTER(C.c_int32)),
                               a3.ctypes.data_as(C.POINTER(C.c_double)))
        keys = ("V", "w", "g_ex", "dg_ex", "g_in", "dg_in", "I_sic")
        out = {k: n7[i * n:(i + 1) * n].copy() for i, k in enumerate(keys)}
        out["refractory"] = refr[:n]
        out["Ca"], out["IP3"], out["h"] = a3[:na].copy(), a3[na:2 * na].copy(), a3[2 * na:3 * na].copy()
        return out
