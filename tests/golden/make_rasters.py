"""Regenerate tests/golden/raster_<config>.npz: the reference simulator's own
spike raster and windowed statistics over the whole benchmarked run of a
shipped configuration (oracle/_ref/libastroref.so, the reference compiled
from its sources by oracle/Makefile, stepped through oracle/ref_shim.cpp's
ref_net_run: the phases of Network::run, network.cpp:385-431).

    python tests/golden/make_rasters.py [config ...]

Runs (steps from 0, every spike recorded, transient included):
  quick               0.5 s transient + 2 s   = 25,000 steps of 0.1 ms
  use_case, bursting  20 s transient + 10 s   = 300,000 steps of 0.1 ms
  c0_literal          10 s                    = 100,000 steps of 0.1 ms
  paper_sparse_dt005  1 s                     = 20,000 steps of 0.05 ms

Each file holds the raster (step, source) in step order and sources ascending
within a step, and per window of `window` steps: the spike count and, at the
window's last step, the number of astrocytes whose SIC factor is non-zero
(Ca above the SIC threshold), the mean astrocyte Ca and the mean membrane
potential.  The GPU tests compare the engine's run with these: identical
rasters up to the stated horizon, windowed statistics after it."""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# name: (sim_time_ms override or None for the file's, window steps)
RUNS = {
    "quick": (None, 1000),
    "use_case": (10000.0, 10000),
    "bursting": (10000.0, 10000),
    "c0_literal": (None, 5000),
    "paper_sparse_dt005": (None, 1000),
}


def generate(name: str) -> str:
    from astrosimgpu_b200.network import config_path
    from oracle import ref
    sim, window = RUNS[name]
    r = ref.RefNetwork(path=config_path(name), sim_time=-1.0 if sim is None else sim)
    total = r.pre_steps + r.sim_steps
    steps, sources = [], []
    win_spikes, win_active, win_ca, win_v = [], [], [], []
    t0 = time.time()
    done = 0
    while done < total:
        k = min(window, total - done)
        st, src = r.run(k)
        steps.append(st.astype(np.int32))
        sources.append(src.astype(np.uint32))
        win_spikes.append(len(st))
        win_active.append(int(np.count_nonzero(r.sic_factors())))
        s = r.state()
        win_ca.append(float(s["Ca"].mean()) if len(s["Ca"]) else 0.0)
        win_v.append(float(s["V"].mean()))
        done += k
    out = os.path.join(HERE, f"raster_{name}.npz")
    np.savez_compressed(out, steps=np.concatenate(steps), sources=np.concatenate(sources),
                        win_spikes=np.array(win_spikes, np.int64),
                        win_active=np.array(win_active, np.int32),
                        win_mean_ca=np.array(win_ca), win_mean_v=np.array(win_v),
                        total_steps=np.int64(total), window=np.int64(window),
                        sim_time_ms=np.float64(-1.0 if sim is None else sim),
                        n_neurons=np.int64(r.n), n_astro=np.int64(r.n_astro),
                        dt=np.float64(r.dt))
    print(f"{name}: {total} steps, {sum(win_spikes)} spikes, {time.time() - t0:.1f} s -> {out}",
          flush=True)
    return out


def main():
    names = sys.argv[1:] or list(RUNS)
    for n in names:
        generate(n)


if __name__ == "__main__":
    main()
