"""Regenerate tests/golden/stats_*.json: long-run statistics of the reference
simulator itself (oracle/_ref/astrosimgpu, built from the reference sources by
oracle/Makefile) on the shipped configurations.

    python tests/golden/make_stats.py [seconds]

For use_case (IP3 weight w_n2a = 0.20) and bursting (0.31), seed 1, the
recorded window of `seconds` (default 60) after the config's 20 s transient,
it runs the reference CLI and keeps the summary lines of its run.txt: spikes,
mean firing rate, astrocytes with transients, mean pairwise correlation.
These are the figures the reference's own docs quote for the synchrony
transition (60 s: correlation 0.0106 vs 0.4177)."""
import json
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CLI = os.path.join(ROOT, "oracle", "_ref", "astrosimgpu")


def parse(run_txt: str) -> dict:
    out = {}
    for key, pat in (("spikes", r"spikes recorded\s+(\d+)"),
                     ("rate_hz", r"mean firing rate\s+([0-9.]+)"),
                     ("active", r"astrocytes with transients\s+(\d+)\s*/\s*(\d+)"),
                     ("transients", r"transients detected\s+(\d+)"),
                     ("correlation", r"mean pairwise correlation\s+(-?[0-9.]+)")):
        m = re.search(pat, run_txt)
        if m:
            out[key] = float(m.group(1))
            if key == "active":
                out["astro_recorded"] = int(m.group(2))
    return out


def main():
    secs = float(sys.argv[1]) if len(sys.argv) > 1 else 60.0
    res = {"seconds": secs, "seed": 1, "transient_ms": 20000.0, "runs": {}}
    for name in ("use_case", "bursting"):
        cfg = os.path.join(ROOT, "astrosimgpu_b200", "configs", name + ".json")
        with tempfile.TemporaryDirectory() as out:
            subprocess.run([CLI, "-c", cfg, "-o", out, "-t", str(secs * 1000.0), "-s", "1"],
                           check=True, capture_output=True)
            with open(os.path.join(out, "run.txt")) as f:
                res["runs"][name] = parse(f.read())
        print(name, res["runs"][name], flush=True)
    with open(os.path.join(HERE, f"stats_{int(secs)}s.json"), "w") as f:
        json.dump(res, f, indent=2)
        f.write("\n")


if __name__ == "__main__":
    main()
