"""Regenerate tests/golden/sweep_stats_5s.json: per-instance statistics of
the 64-instance batched sweep (astrosimgpu_b200/workloads.py sweep_configs:
N in {250, 500, 1000, 2000, 4000} round robin, N_A = N/5, w_n2a swept over
8 values in [0.20, 0.31] crossed with 8 seeds, 5 s each, no transient) as
the reference simulator itself produces them (oracle/_ref/libastroref.so,
built from the reference sources by oracle/Makefile).

    python tests/golden/make_sweep_stats.py [processes]

Per instance: the spike count, mean firing rate and a SHA-256 of the raster
(int64 steps then uint32 sources of each stepping call, in order) over the
5 s, and the
calcium analysis of the reference's analysis.cpp (event detection, sliding-
window rates, mean pairwise correlation; ref_calcium_analysis in
oracle/ref_shim.cpp) over every astrocyte's Ca sampled every 100 steps (the
config's record_every), at the steps Network::run records
((step - pre_steps) % record_every == 0, network.cpp:451).

Each instance is also run a second time with one neuron's initial membrane
potential moved by one unit in the last place.  The difference between the
two runs is the spread chaos alone produces from a last-bit difference, the
scale the GPU tests use for their tolerances after the raster horizon."""
import hashlib
import json
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SIM_MS = 5000.0
EVERY = 100


def analysis_params(text):
    from astrosimgpu_b200.network import Model
    m = Model(text=text, pre_time=0.0, build=False)
    width, shift = m.hist_window, m.hist_shift
    if width >= m.sim_time and m.sim_time > 0:
        width, shift = m.sim_time / 10.0, m.sim_time / 50.0
    return m.ca_threshold, m.merge_gap, width, shift


def run_one(args):
    idx, text, perturb = args
    from oracle import ref
    r = ref.RefNetwork(text=text)
    if perturb:
        st = r.state()
        st["V"][0] = np.nextafter(st["V"][0], np.inf)
        r.set_state(st)
    steps = r.sim_steps
    samples, times = [], []
    raster = hashlib.sha256()
    spikes = 0

    def advance(k):
        nonlocal spikes
        st, src = r.run(k)
        spikes += len(st)
        raster.update(np.ascontiguousarray(st, np.int64).tobytes())
        raster.update(np.ascontiguousarray(src, np.uint32).tobytes())

    advance(1)
    done = 1
    samples.append(r.state()["Ca"].copy())
    times.append(0.0)
    while done + EVERY <= steps:
        advance(EVERY)
        done += EVERY
        samples.append(r.state()["Ca"].copy())
        times.append((done - 1) * r.dt)
    if done < steps:
        advance(steps - done)
    ca = np.ascontiguousarray(np.array(samples).T)  # cells x samples
    t = np.ascontiguousarray(np.tile(np.array(times), (ca.shape[0], 1)))
    thr, gap, width, shift = analysis_params(text)
    out = np.zeros(5)
    ref.ref().ref_calcium_analysis(ref._dp(t), ref._dp(ca), ca.shape[0], ca.shape[1], thr, gap,
                                   0.0, SIM_MS, width, shift, ref._dp(out))
    return idx, perturb, {"spikes": int(spikes), "rate_hz": spikes * 1000.0 / (SIM_MS * r.n),
                          "raster_sha256": raster.hexdigest(),
                          "active": int(out[0]), "transients": int(out[1]),
                          "mean_duration_ms": float(out[2]), "pairs": int(out[3]),
                          "correlation": float(out[4])}


def main():
    from astrosimgpu_b200.workloads import sweep_configs
    procs = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    texts = sweep_configs(64, SIM_MS)
    jobs = [(i, t, p) for i, t in enumerate(texts) for p in (False, True)]
    res = {}
    with mp.get_context("spawn").Pool(procs) as pool:
        for idx, perturb, st in pool.imap_unordered(run_one, jobs):
            res.setdefault(idx, {})["perturbed" if perturb else "reference"] = st
            print(idx, "perturbed" if perturb else "reference", st, flush=True)
    insts = []
    for i, t in enumerate(texts):
        c = json.loads(t)
        insts.append({"index": i, "neurons": c["N"]["N_E"] + c["N"]["N_I"],
                      "astrocytes": c["N"]["N_A"], "w_n2a": c["synapse"]["w_n2a"],
                      "seed": c["simulation"]["seed"], **res[i]})
    with open(os.path.join(HERE, "sweep_stats_5s.json"), "w") as f:
        json.dump({"sim_ms": SIM_MS, "record_every": EVERY, "instances": insts}, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
