"""Regenerate tests/golden/indegree_stats.json: statistics of the reference
simulator on the serving stream's network shape with its own connectivity
rule -- pairwise Bernoulli with p_primary = 100 / N, i.e. a mean in-degree of
100 -- at N = 2,000, 5,000 and 10,000 neurons (N_A = N, use_case
parameters, every excitatory synapse recruiting an astrocyte of the
target's block pool with p = 0.2), seeds 1-3, 1 s of 0.1 ms steps.

    python tests/golden/make_indegree_stats.py

The reference has no fixed-in-degree rule; the engine's counter-based
generator (asg_model_build_fixed_indegree) builds exactly 100 inputs per
neuron.  Above ~20k neurons the serving shapes have no oracle but these
statistics: the firing rate and the astrocyte activity of the two
connectivity rules at the sizes the reference can still build.  Per run:
mean firing rate over the second, and at its end the fraction of
astrocytes above the SIC threshold and the mean Ca."""
import json
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SIZES = (2000, 5000, 10000)
SEEDS = (1, 2, 3)
SIM_MS = 1000.0


def config_text(n, seed):
    from astrosimgpu_b200.workloads import serving_config
    c = json.loads(serving_config(n, seed, SIM_MS))
    c["connectivity"]["p_primary"] = 100.0 / n
    return json.dumps(c)


def run_one(args):
    n, seed = args
    from oracle import ref
    r = ref.RefNetwork(text=config_text(n, seed))
    st, _ = r.run(r.sim_steps)
    f = r.sic_factors()
    s = r.state()
    return n, seed, {"spikes": int(len(st)), "rate_hz": len(st) * 1000.0 / (SIM_MS * r.n),
                     "active_frac": float(np.count_nonzero(f)) / max(len(f), 1),
                     "mean_ca": float(s["Ca"].mean()), "edges": int(r.n_primary_exc +
                                                                    r.n_primary_inh)}


def main():
    jobs = [(n, s) for n in SIZES for s in SEEDS]
    out = {}
    with mp.get_context("spawn").Pool(min(len(jobs), os.cpu_count() or 1)) as pool:
        for n, seed, st in pool.imap_unordered(run_one, jobs):
            out[f"{n}/{seed}"] = st
            print(n, seed, st, flush=True)
    with open(os.path.join(HERE, "indegree_stats.json"), "w") as f:
        json.dump({"sim_ms": SIM_MS, "rule": "Bernoulli p_primary = 100/N", "runs": out}, f,
                  indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
