"""Regenerate astrosimgpu_b200/configs/*.json from the reference's config/*.json.

The engine reads the reference's own JSON schema.  The parameter values of
the shipped model configurations are the inputs the parity tests and the
benchmark run on, so they are carried over as plain JSON (comments and prose
dropped, keys and numbers unchanged).  Run in a checkout that has the
reference sources named by the environment variable ASTROSIMGPU_REF.  Two derived files follow the
benchmark shapes: paper_sparse_dt005 (dt 0.05 ms, 1.5 ms delays, config C2)
and c0_literal (use_case with p_primary 0.1, every excitatory synapse
recruiting from a random pool of 100, 1.5 ms delays).
"""
import json
import os
import re
import sys

REF = os.environ.get("ASTROSIMGPU_REF")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..",
                   "astrosimgpu_b200", "configs")


def strip_comments(text: str) -> str:
    return "\n".join(line for line in text.splitlines() if not re.match(r"^\s*//", line))


def main():
    if not REF or not os.path.isdir(os.path.join(REF, "config")):
        sys.exit("set ASTROSIMGPU_REF to the reference checkout (the directory holding config/)")
    os.makedirs(OUT, exist_ok=True)
    names = ["use_case", "bursting", "quick", "paper_sparse", "kernel_scaling", "no_spiking",
             "random_pool", "scale_1000"]
    cfgs = {}
    for n in names:
        with open(os.path.join(REF, "config", n + ".json")) as f:
            cfgs[n] = json.loads(strip_comments(f.read()))
    ps = json.loads(json.dumps(cfgs["paper_sparse"]))
    ps["simulation"]["dt"] = 0.05
    ps["simulation"]["pre_sim_time"] = 0
    ps["simulation"]["sim_time"] = 1000
    ps["synapse"]["d_e"] = 1.5
    ps["synapse"]["d_i"] = 1.5
    cfgs["paper_sparse_dt005"] = ps
    lit = json.loads(json.dumps(cfgs["use_case"]))
    lit["connectivity"].update({"p_primary": 0.1, "p_third_if_primary": 1.0, "pool_size": 100,
                                "pool_type": "random"})
    lit["synapse"]["d_e"] = 1.5
    lit["synapse"]["d_i"] = 1.5
    lit["simulation"]["pre_sim_time"] = 0
    lit["simulation"]["sim_time"] = 10000
    cfgs["c0_literal"] = lit
    for n, c in cfgs.items():
        with open(os.path.join(OUT, n + ".json"), "w") as f:
            json.dump(c, f, indent=2)
            f.write("\n")
    print("wrote", len(cfgs), "configs to", os.path.normpath(OUT))


if __name__ == "__main__":
    sys.exit(main())
