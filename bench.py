#!/usr/bin/env python3
"""Benchmark of the B200 per-timestep engine.

Headline workload (one JSON line on rank 0): the astrocyte kernel-scaling
case at N = 1e7 independent Li-Rinzel cells (use_case astrocyte parameters,
IP3 input events Bernoulli(0.01) of weight 0.2 per 0.1 ms step, FP64,
noise off).  One "step" is one timestep of all N cells.

- value: cell-updates/s with the state resident in HBM, input generated on
  the device from the counter RNG; device time from CUDA events on the
  engine's stream, max over ranks.
- e2e: the same metric through the drop-in C ABI of the reference's CUDA
  astrocyte backend (asg_astro_push_input / asg_astro_update /
  asg_astro_pull_calcium), i.e. per step an 8N-byte host->device input copy
  and an 8N-byte device->host calcium copy from pinned host memory, exactly
  the movement pattern of the reference's published GPU numbers.
- roofline: the binding one is the FP64 pipe (FP64 flops counted by ncu per
  cell-step / launch time, against 148 SMs x 64 FP64 lanes x 2 flops x the
  sampled SM clock); the HBM roofline (48 algorithmic bytes per cell-step
  against the measured copy bandwidth) is reported beside it.
- cpu_baseline: the reference's own astro_advance (built from its sources,
  oracle/_ref) over a bounded sample on the host cores with OpenMP.
- reference_cuda_kernel: the reference's astro_update_kernel built for
  sm_100a on the same GPU, and the same-contract A/B against it: the
  drop-in asg_astro_update (per-cell parameter arrays, resident state,
  back-to-back updates, no copies) on the calls the reference kernel is
  timed on.
- network_c0 / network_c2: the plain one-network path over the whole run of
  use_case (20 s transient + 10 s) and paper_sparse at dt 0.05 ms (1 s),
  each beside the reference CLI (OpenMP) timed on a bounded sample of the
  same run on the host cores.
- batched_c3: 64 instances of uneven size, 5 s each, batched vs one network
  per launch.  serving_c4: a Poisson request stream (with one 1M-neuron /
  1M-astrocyte request) through the continuous-batching server.
  network_1m: that 1M network alone on the plain path.

Multi-GPU: the astrocyte cells are independent, so N GPUs each run their
own N-cell instance (weak scaling, no collective); rank 0 reports the sum.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "neuron-updates/s & HBM GB/s vs roofline; batched/served vs plain; p50/p99 lat"
BYTES_PER_CELL_STEP = 48  # Ca, IP3, h: read + write, FP64
# Per cell-step of astro_step_kernel<uniform, bernoulli> (substeps 1), from
# an ncu capture of the headline workload (profiles/astro_step_kernel_N1e7.md):
# FP64 thread instructions executed (DADD + DMUL + DFMA + the rest of the
# FP64 pipe) and FP64 flops (DFMA counted twice).
FP64_INST_PER_CELL_STEP = 313  # 64 DADD + 109 DMUL + 134 DFMA + 6 other
FP64_FLOP_PER_CELL_STEP = 441
FP64_LANES_PER_SM = 64
# dram__bytes_read.sum + dram__bytes_write.sum of one astro_step_kernel launch
# at N = 1e7, from the same capture.
NCU_TRAFFIC_PER_LAUNCH = {10_000_000: 420_352_512}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def headline_config(cells, world):
    """The workload both arms report (identical keys and values)."""
    return {"workload": f"astrocyte kernel scaling, N={cells} cells per GPU, 1 step = 1 "
                        "timestep (0.1 ms) of all cells, Bernoulli(0.01) IP3 input w=0.2, "
                        "use_case astrocyte parameters, noise off, seed 1",
            "cells": cells, "parallelism": f"replicas x{world}",
            "l2": "working set 24 B/cell = 240 MB at N=1e7 > 126 MB L2 (no flush needed)"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled around the timed region.

    The sampler is started and its first sample awaited before the timed
    region begins; samples taken from that point until it stops are kept
    (line-buffered output, 20 ms period)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.error = None

    def __enter__(self):
        import shutil
        cmd = ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
               "--format=csv,noheader,nounits", "-lms", "20"]
        if shutil.which("stdbuf"):
            cmd = ["stdbuf", "-oL"] + cmd
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                         text=True, bufsize=1)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception as e:  # noqa: BLE001
            self.error = str(e)
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.05)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if not self.lines:
                try:
                    self.error = self.proc.stderr.read()[:200]
                except Exception:
                    pass

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                    "error": self.error or (self.lines[:1] or [None])[0]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl" if os.environ.get("ASG_BENCH_GLOO") is None else "gloo",
                                timeout=datetime.timedelta(seconds=120))
        pg = dist
    return rank, world, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def pinned(n):
    """Pinned host float64 buffer as a numpy array (torch allocates it)."""
    import torch
    t = torch.empty(n, dtype=torch.float64, pin_memory=True)
    return t, t.numpy()


def sm_count():
    import torch
    return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count


def bench_astro_scaling(args, rank, world, pg):
    import numpy as np
    import torch

    from astrosimgpu_b200 import _lib
    from astrosimgpu_b200.astro import AstroBackend, ScalingWorkload, uniform_np

    n = args.cells
    w = ScalingWorkload(n, seed=1 + rank)
    Ca, IP3, h = w.initial_state()
    eng = AstroBackend(Ca, IP3, h)
    shape, tuned_us = eng.autotune(w, steps=30)  # 9 shapes x 2 passes x 30 steps, ~0.15 s
    step = 0
    for _ in range(args.warmup):  # untimed
        eng.run_bernoulli(w, step, 1)
        step += 1
    torch.cuda.synchronize()
    barrier(pg)
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clk:
        dev_ms, kernels = eng.run_bernoulli(w, step, args.steps)
        torch.cuda.synchronize()
    barrier(pg)
    step += args.steps
    dev_ms = max_over_ranks(pg, dev_ms)
    per_launch_us = dev_ms * 1e3 / args.steps
    value = n * world * args.steps / (dev_ms * 1e-3)
    clocks = clk.summary()

    # e2e through the drop-in ABI (per-cell parameter arrays, as the
    # reference backend holds them): H2D input + update + D2H Ca per step.
    eng_e2e = AstroBackend(Ca, IP3, h, np.full(n, w.Ca_tot), np.full(n, w.IP3_0),
                           np.full(n, w.tau_IP3), np.full(n, w.delta_IP3))
    # Two pinned input buffers, filled before the timed region (the
    # caller's input of alternate steps), and one pinned Ca buffer.
    ein_bufs = [pinned(n) for _ in range(2)]
    eca_t, eca = pinned(n)
    cells = np.arange(n, dtype=np.uint64)
    for k, (_, buf) in enumerate(ein_bufs):
        u = uniform_np(w.seed, cells, 1000 + 10_000 + k)
        buf[:] = np.where(u < w.p, w.weight, 0.0)
    e2e_steps = max(3, min(args.steps, 20))
    for k in range(2):  # warm-up of the copy path
        eng_e2e.push_input(ein_bufs[k % 2][1])
        eng_e2e.update(w.consts, w.h_step, w.substeps)
        eca[:] = eng_e2e.pull_calcium()
    torch.cuda.synchronize()
    barrier(pg)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L = _lib.load()
    ein_ptrs = [_lib.dptr(buf) for _, buf in ein_bufs]
    for k in range(e2e_steps):
        _lib.check(L.asg_astro_push_input(eng_e2e._h, ein_ptrs[k % 2]), "push")
        _lib.check(L.asg_astro_update(eng_e2e._h, _lib.dptr(w.consts), w.h_step, w.substeps, 0.0,
                                      1, 0.0, 0, 0), "update")
        _lib.check(L.asg_astro_pull_calcium(eng_e2e._h, _lib.dptr(eca)), "pull")
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    barrier(pg)
    wall = max_over_ranks(pg, wall)
    e2e_value = n * world * e2e_steps / wall
    del ein_bufs, eca_t
    eng_e2e.destroy()

    peak, peak_kind = load_peaks()
    achieved = BYTES_PER_CELL_STEP * n / (per_launch_us * 1e-6) / 1e9
    hbm = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "traffic": NCU_TRAFFIC_PER_LAUNCH.get(n),
           "traffic_unit": "bytes per launch (ncu dram read + write)",
           "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
           else peak_kind, "bytes_per_launch": BYTES_PER_CELL_STEP * n}
    roofline = dict(hbm)
    if FP64_FLOP_PER_CELL_STEP is not None and clocks.get("sm_mhz"):
        sms = sm_count()
        peak_tf = sms * FP64_LANES_PER_SM * 2 * clocks["sm_mhz"] * 1e6 / 1e12
        ach_tf = FP64_FLOP_PER_CELL_STEP * n / (per_launch_us * 1e-6) / 1e12
        inst_rate = FP64_INST_PER_CELL_STEP * n / (per_launch_us * 1e-6)
        roofline = {"bound": "fp64", "achieved": ach_tf, "peak": peak_tf, "unit": "TFLOP/s",
                    "frac": ach_tf / peak_tf,
                    "fp64_pipe_inst_frac": inst_rate / (sms * FP64_LANES_PER_SM *
                                                        clocks["sm_mhz"] * 1e6),
                    "flop_per_cell_step": FP64_FLOP_PER_CELL_STEP,
                    "inst_per_cell_step": FP64_INST_PER_CELL_STEP,
                    "peak_source": f"{sms} SMs x {FP64_LANES_PER_SM} FP64 lanes x 2 flops x "
                                   "median sampled SM clock",
                    "traffic": NCU_TRAFFIC_PER_LAUNCH.get(n),
                    "hbm": hbm}
    roofline["kernel"] = "astro_step_kernel<uniform,bernoulli>"
    out = {
        "value": value, "ms_per_step": dev_ms / args.steps, "kernels": kernels,
        "per_launch_us": per_launch_us,
        "e2e": {"value": e2e_value, "unit": "cell-updates/s",
                "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                "steps": e2e_steps, "path": "asg_astro_push_input+update+pull_calcium"},
        "roofline": roofline, "clocks": clocks, "launch_shape": shape,
    }
    return out, (w, Ca, IP3, h)


def network_bytes(n, na, astro_uniform, spike_edges, sic_edges, steps, sic_steps):
    """Algorithmic HBM bytes of `steps` network steps: 144 B per neuron-step,
    56 B (uniform astrocyte parameters) or 88 B per astrocyte-step, 68 B per
    delivered spike edge, 4 B per active SIC edge plus 8 B per astrocyte
    factor and 8 B per neuron SIC value on each SIC step."""
    return (144 * n + (56 if astro_uniform else 88) * na) * steps + 68 * spike_edges + \
        4 * sic_edges + (8 * na + 8 * n) * sic_steps


def run_network(m, uniform, calls, steady_calls=0, **opts):
    """Whole run of model `m` on the plain path in `calls` equal calls;
    device time per call, roofline over the run (and its last calls)."""
    from astrosimgpu_b200 import _lib
    from astrosimgpu_b200.network import Network
    hbm, src = load_peaks()
    net = Network(m, record=_lib.RecordOpts(0, 10, 1, 0, 0), **opts)
    total = m.pre_steps + m.sim_steps
    per = max(1, total // calls)
    rows = []
    prev = net.counters()
    kernels = 0
    wall0 = time.perf_counter()
    for _ in range(calls):
        net.step(per)
        ms, k = net.last_timing()
        c = net.counters()
        rows.append((ms, c["spike_edges"] - prev["spike_edges"], c["sic_edges"] - prev["sic_edges"],
                     c["spikes"] - prev["spikes"]))
        kernels += k
        prev = c
    wall_s = time.perf_counter() - wall0
    n, na = net.n, net.na
    net.close()

    def summary(sel):
        ms = sum(r[0] for r in sel)
        steps = per * len(sel)
        se, sic = sum(r[1] for r in sel), sum(r[2] for r in sel)
        sic_steps = steps if sic > 0 else 0
        gb = network_bytes(n, na, uniform, se, sic, steps, sic_steps) / (ms * 1e-3) / 1e9
        us = ms * 1e3 / steps
        return {"steps": steps, "device_ms": ms, "us_per_step": us,
                "sim_s_per_wall_s": (m.dt * 1e-3) / (us * 1e-6),
                "neuron_updates_per_s": n / (us * 1e-6),
                "synaptic_events_per_s": (se + sic) / (ms * 1e-3),
                "roofline": {"bound": "hbm", "achieved": gb, "peak": hbm, "unit": "GB/s",
                             "frac": gb / hbm, "peak_source": src}}
    out = {"neurons": n, "astrocytes": na, "dt_ms": m.dt, "kernels": kernels,
           "spikes": sum(r[3] for r in rows), "wall_s_including_host": wall_s,
           "per_call_us_per_step": [round(r[0] * 1e3 / per, 2) for r in rows],
           "engine_opts": opts}
    out.update(summary(rows))
    if steady_calls:
        out["steady_state_last_%d_steps" % (per * steady_calls)] = summary(rows[-steady_calls:])
    return out, rows, per


def reference_cli_sample(config_file, sim_ms, pre_ms, seed=1, timeout=600):
    """The reference CLI (oracle/_ref/astrosimgpu, OpenMP on every host core,
    OMP_PROC_BIND=spread) on `sim_ms` of recorded time after `pre_ms` of
    transient; sim-s/wall-s from its own phase timers (run.txt's
    real-time factor, recorded window only)."""
    from oracle import ref
    threads = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="spread")
    with tempfile.TemporaryDirectory() as out:
        t0 = time.perf_counter()
        r = subprocess.run([ref.REF_CLI, "-c", config_file, "-o", out, "-t", str(sim_ms),
                            "-p", str(pre_ms), "-s", str(seed), "--no-analysis"], env=env,
                           capture_output=True, text=True, timeout=timeout)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(r.stderr[-300:])
        text = open(os.path.join(out, "run.txt")).read()
    rtf = float(re.search(r"real-time factor\s+([0-9.eE+-]+)", text).group(1))
    omp = int(re.search(r"OpenMP threads\s+(\d+)", text).group(1))
    phases = {}
    for key, label in (("input_gen", "background input"), ("update_astro", "update astrocytes"),
                       ("update_neuron", "update neurons"), ("spike_cd", "spike delivery"),
                       ("sic_gd", r"SIC gather\+deliver"), ("deliver", "arrival application")):
        mm = re.search(label + r"\s+([0-9.]+)", text)
        if mm:
            phases[key] = float(mm.group(1))
    return {"value": 1.0 / rtf, "unit": "sim-s/wall-s", "cores": omp, "kind": "reference",
            "process_wall_s": wall, "phase_seconds": phases,
            "sample": f"reference CLI (oracle/_ref/astrosimgpu, OpenMP {omp} threads, "
                      f"OMP_PROC_BIND=spread): {sim_ms} ms recorded after {pre_ms} ms of "
                      "transient, sim-s/wall-s from its run.txt real-time factor"}


def bench_network_c0(cpu=True):
    """use_case as shipped, the C0 throughput run: 20 s transient + 10 s."""
    from astrosimgpu_b200.network import Model, config_path
    m = Model(config_path("use_case"), sim_time=10000.0)
    out, rows, per = run_network(m, uniform=False, calls=10)
    out["config"] = "use_case, 20 s transient + 10 s recorded, dt 0.1 ms, seed 1"
    if cpu:
        try:
            c = reference_cli_sample(config_path("use_case"), 2000.0, 0.0)
            out["cpu_baseline"] = c
            out["gpu_over_cpu_sim_s_per_wall_s"] = out["sim_s_per_wall_s"] / c["value"]
        except Exception as e:  # noqa: BLE001
            out["cpu_baseline"] = {"unavailable": str(e)[:200]}
    return out


def bench_network_c2(cpu=True, **opts):
    """paper_sparse at dt 0.05 ms, 1.5 ms delays: the whole 1 s (20,000
    steps) in 20 calls, with the SIC-active steady state (last 5,000)."""
    from astrosimgpu_b200.network import Model, config_path
    name = "paper_sparse_dt005"
    uniform = not json.load(open(config_path(name))).get("randomize_astro", {}).get("enabled",
                                                                                      False)
    t0 = time.perf_counter()
    m = Model(config_path(name), pre_time=0.0)
    build_s = time.perf_counter() - t0
    out, rows, per = run_network(m, uniform=uniform, calls=20, steady_calls=5, **opts)
    out["config"] = name + " (10k neurons, 10k astrocytes, ~10M synapses, dt 0.05 ms, 1 s)"
    out["build_s"] = build_s
    if cpu:
        try:
            sample_ms = 200.0
            c = reference_cli_sample(config_path(name), sample_ms, 0.0)
            c["sample"] += ("; the first 4,000 steps, before the SIC steady state (the "
                            "reference's cheapest window)")
            out["cpu_baseline"] = c
            k = int(round(sample_ms / m.dt / per))
            gpu_ms = sum(r[0] for r in rows[:k])
            gpu_rate = (k * per * m.dt * 1e-3) / (gpu_ms * 1e-3)
            out["gpu_sim_s_per_wall_s_same_window"] = gpu_rate
            out["gpu_over_cpu_same_window"] = gpu_rate / c["value"]
        except Exception as e:  # noqa: BLE001
            out["cpu_baseline"] = {"unavailable": str(e)[:200]}
    return out


def bench_network_1m():
    """The largest serving request alone: 1M neurons, 1M astrocytes, fixed
    in-degree 100 (device generator), 1,000 steps of 0.1 ms."""
    from astrosimgpu_b200.network import Model
    from astrosimgpu_b200.workloads import serving_config
    t0 = time.perf_counter()
    m = Model(text=serving_config(1_000_000, 99, 100.0), pre_time=0.0, fixed_indegree=100,
              gen_device=0)
    build_s = time.perf_counter() - t0
    out, rows, per = run_network(m, uniform=False, calls=4)
    out["config"] = "1M neurons / 1M astrocytes, fixed in-degree 100, use_case parameters, 100 ms"
    out["build_s"] = build_s
    return out


def bench_batched(sim_ms=5000.0, n_inst=64, autotune=True):
    """64-instance sweep: batched engine vs one network per launch."""
    from astrosimgpu_b200 import _lib
    from astrosimgpu_b200.network import Batch, Model, Network
    from astrosimgpu_b200.workloads import sweep_configs
    texts = sweep_configs(n_inst, sim_ms)
    models = [Model(text=t, pre_time=0.0) for t in texts]
    steps = models[0].sim_steps
    dt = models[0].dt
    rec = _lib.RecordOpts(0, 10, 1, 0, 0)
    plain_ms, plain_kernels = 0.0, 0
    for m in models:  # plain path: each instance on its own, one after another
        net = Network(m, record=rec, chunk_steps=64)
        net.step(64)  # warm (graph capture)
        net.step(steps)
        ms, k = net.last_timing()
        plain_ms += ms
        plain_kernels += k
        net.close()
    b = Batch(models, record=rec, chunk_steps=128)
    tuned = b.autotune(1024) if autotune else None  # long enough to rank chunk lengths
    b.step(64)
    b.step(steps)
    bms, bk = b.last_timing()
    sim_s = n_inst * steps * dt * 1e-3
    spikes = sum(b.counters(i)["spikes"] for i in range(n_inst))
    neurons = sum(mm.desc().n_exc + mm.desc().n_inh for mm in models)
    b.close()
    return {"instances": n_inst, "steps": steps, "sim_ms_each": steps * dt,
            "total_neurons": neurons,
            "batched_ms": bms, "plain_ms": plain_ms,
            "batched_sim_s_per_wall_s": sim_s / (bms * 1e-3),
            "plain_sim_s_per_wall_s": sim_s / (plain_ms * 1e-3),
            "speedup": plain_ms / bms, "batched_kernels": bk, "plain_kernels": plain_kernels,
            "batched_us_per_step": bms * 1e3 / steps, "autotuned": tuned,
            "spikes": spikes}


def bench_serving(n_req=100, rate_hz=20.0, big=True, **opts):
    """Poisson request stream through the continuous-batching server."""
    import numpy as np
    from astrosimgpu_b200.network import Model, Server
    from astrosimgpu_b200.workloads import request_stream, serving_config
    stream = request_stream(n_req, rate_hz, big=big)
    t0 = time.perf_counter()
    models = [Model(text=serving_config(n, sd, dur), pre_time=0.0, fixed_indegree=100,
                    gen_device=0) for (_, n, dur, sd) in stream]
    build_s = time.perf_counter() - t0
    srv = Server(**opts)
    ids = []
    start = time.perf_counter()
    for (arr, n, dur, sd), m in zip(stream, models):
        delay = arr - (time.perf_counter() - start)
        if delay > 0:
            time.sleep(delay)
        ids.append(srv.submit(m, m.sim_steps, keep_spikes=False))
    res = [srv.wait(i) for i in ids]
    wall = time.perf_counter() - start
    st = srv.stats()
    srv.close()
    lat = np.array([r.submit_to_done_ms for r in res])
    adm = np.array([r.submit_to_admit_ms for r in res])
    events = sum(r.spike_edges + r.sic_edges for r in res)
    sim_s = sum(dur for (_, _, dur, _) in stream) * 1e-3
    neuron_steps = sum(n * m.sim_steps for (_, n, _, _), m in zip(stream, models))
    return {"requests": len(res), "arrival_rate_hz": rate_hz,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "admit_p50_ms": float(np.percentile(adm, 50)),
            "admit_p99_ms": float(np.percentile(adm, 99)),
            "wall_s": wall, "synaptic_events_per_s": events / wall,
            "sim_s_per_wall_s": sim_s / wall, "neuron_updates_per_s": neuron_steps / wall,
            "gpu_busy_frac": st["device_ms"] * 1e-3 / wall,
            "peak_resident": st["peak_resident"], "kernels": st["kernels"],
            "device_ms": st["device_ms"], "build_s": build_s,
            "largest_request_neurons": max(int(n) for (_, n, _, _) in stream),
            "sizes": [int(n) for (_, n, _, _) in stream],
            "statuses": sorted(set(int(r.status) for r in res))}


def reference_cuda_kernel(w, Ca, IP3, h, steps):
    """The reference's astro_update_kernel (sm_100a build) on the same GPU,
    and the drop-in asg_astro_update on the same contract: per-cell
    parameter arrays given at create, resident state, `steps` back-to-back
    updates with no push in between (the calls refcu_time_updates makes),
    device-timed on each side.  Once with the C1 parameters (equal in every
    cell) and once with per-cell parameters spread +-5 %."""
    import numpy as np

    from astrosimgpu_b200.astro import AstroBackend
    from oracle import ref
    lib = ref.refcu()
    n = len(Ca)
    rng = np.random.default_rng(3)
    sets = {"uniform_values": [np.full(n, v) for v in (w.Ca_tot, w.IP3_0, w.tau_IP3,
                                                       w.delta_IP3)],
            "per_cell_values": [v * (1 + 0.05 * rng.standard_normal(n))
                                for v in (w.Ca_tot, w.IP3_0, w.tau_IP3, w.delta_IP3)]}
    out = {"steps": steps, "note": "reference astro_update_kernel, block 128, built -arch "
                                   "sm_100a, resident state, no copies; ours asg_astro_update"}
    o = [np.empty(n) for _ in range(3)]
    for label, params in sets.items():
        arrs = [np.ascontiguousarray(a) for a in (Ca, IP3, h, *params)]
        s = lib.refcu_create(n, *[ref._dp(a) for a in arrs])
        lib.refcu_time_updates(s, ref._dp(w.consts), w.h_step, w.substeps, 3)
        ref_ms = lib.refcu_time_updates(s, ref._dp(w.consts), w.h_step, w.substeps, steps)
        lib.refcu_destroy(s, *[ref._dp(a) for a in o])
        eng = AstroBackend(Ca, IP3, h, *params)
        eng.autotune(w, steps=20)
        for rep in range(2):  # first pass warms up
            for _ in range(steps):
                eng.update(w.consts, w.h_step, w.substeps)
            ms, _ = eng.last_timing()
        eng.destroy()
        ref_us, us = ref_ms * 1e3 / steps, ms * 1e3 / steps
        out[label] = {"reference_us_per_step": ref_us, "asg_astro_update_us_per_step": us,
                      "speedup": ref_us / us, "cell_updates_per_s": n / (us * 1e-6)}
    out["us_per_step"] = out["uniform_values"]["reference_us_per_step"]
    out["cell_updates_per_s"] = n / (out["us_per_step"] * 1e-6)
    return out


def cpu_baseline(w, budget_s=12.0):
    """Reference astro_advance on the host cores (OpenMP), bounded sample."""
    from oracle import ref
    lib = ref.ref()
    threads = os.cpu_count() or 1
    n = w.n
    Ca, IP3, h = [a.copy() for a in w.initial_state()]
    ref.ref_astro_scaling(w, Ca, IP3, h, 0, 1, threads=threads)  # warm
    steps, secs = 0, 0.0
    while secs < budget_s and steps < 1000:
        secs += ref.ref_astro_scaling(w, Ca, IP3, h, 1 + steps, 1, threads=threads)
        steps += 1
    return {"value": n * steps / secs, "unit": "cell-updates/s", "cores": threads,
            "kind": "reference",
            "sample": f"{steps} steps x {n} cells of the same workload through the reference's "
                      f"astro_advance (OpenMP, {threads} threads, oracle/_ref)",
            "omp_max_threads": int(lib.ref_omp_max_threads())}


def run_reference_arm(args, rank, world, pg):
    """--impl reference: the reference's CPU implementation on the host cores."""
    if rank != 0:
        return 0
    from astrosimgpu_b200.astro import ScalingWorkload

    from oracle import ref
    threads = os.cpu_count() or 1
    w = ScalingWorkload(args.cells)
    Ca, IP3, h = [a.copy() for a in w.initial_state()]
    step = 0
    for _ in range(args.warmup):
        ref.ref_astro_scaling(w, Ca, IP3, h, step, 1, threads=threads)
        step += 1
    secs = ref.ref_astro_scaling(w, Ca, IP3, h, step, args.steps, threads=threads)
    value = args.cells * args.steps / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": secs * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": headline_config(args.cells, world),
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"{args.steps} full steps of {args.cells} cells through the "
                                   "reference's astro_advance (OpenMP), oracle/_ref"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


SUBS = ("network_c0", "network_c2", "batched_c3", "serving_c4", "network_1m")


def main():
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cells", type=int, default=10_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the reference CUDA kernel and sub-benchmarks")
    ap.add_argument("--skip", default="", help="comma list of sub-benchmarks to skip: "
                    + ",".join(SUBS))
    ap.add_argument("--engine-mode", type=int, default=1,
                    help="network engine launches (--only network_c2): 1 graphs of per-step "
                         "kernels, 2 persistent chunk kernel")
    ap.add_argument("--only", default="", choices=("", "astro") + SUBS,
                    help="run one part alone and print its JSON (profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank, world, local, pg = dist_setup(args.gpus)
    if args.impl == "reference":
        rc = run_reference_arm(args, rank, world, pg)
        if pg is not None:
            pg.destroy_process_group()
        return rc

    import torch
    torch.cuda.set_device(local)
    subs = {"network_c0": lambda: bench_network_c0(cpu=not args.no_cpu_baseline),
            "network_c2": lambda: bench_network_c2(cpu=not args.no_cpu_baseline),
            "batched_c3": bench_batched, "serving_c4": bench_serving,
            "network_1m": bench_network_1m}
    if args.only and args.only != "astro":
        fn = subs[args.only]
        if args.only == "network_c2":
            fn = lambda: bench_network_c2(cpu=False, use_graphs=max(args.engine_mode, 1))  # noqa
        print(json.dumps({args.only: fn()}), flush=True)
        return 0
    res, (w, Ca, IP3, h) = bench_astro_scaling(args, rank, world, pg)
    if args.only == "astro":
        print(json.dumps({"astro": {k: res[k] for k in ("value", "per_launch_us", "roofline",
                                                        "e2e", "clocks")}}))
        return 0

    extras = {}
    if rank == 0 and not args.no_extras:
        try:
            extras["reference_cuda_kernel"] = reference_cuda_kernel(w, Ca, IP3, h,
                                                                    min(args.steps, 50))
        except Exception as e:  # noqa: BLE001
            extras["reference_cuda_kernel"] = {"unavailable": str(e)[:200]}
        for key in SUBS:
            if key in args.skip:
                continue
            try:
                extras[key] = subs[key]()
            except Exception as e:  # noqa: BLE001
                extras[key] = {"unavailable": f"{type(e).__name__}: {str(e)[:300]}"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w)

    if rank == 0:
        line = {
            "metric": METRIC, "value": res["value"], "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": res["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": headline_config(args.cells, world),
            "e2e": res["e2e"], "gpu_launches": res["kernels"], "roofline": res["roofline"],
            "clocks": res["clocks"], "per_launch_us": res["per_launch_us"],
            "launch_shape": res["launch_shape"],
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        line.update(extras)
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
