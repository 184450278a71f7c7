"""The reference's precision study (docs/experiments.md, "Single or double
precision"): is FP32 enough for the Li-Rinzel calcium dynamics?  Its method
is `real = float`; here the opt-in FP32 astrocyte form of the engine
(asg_engine_opts.astro_precision = 32, the CLI's --astro-fp32) against the
FP64 product path.

Measured on a B200 (60 s after the 20 s transient, seed 1):

  run                  rate (Hz)   astrocytes active   mean pairwise correlation
  use_case  FP64        0.4808         46 / 100              0.0106
  use_case  FP32        0.4789         39 / 100              0.0092
  bursting  FP64        0.6277        100 / 100              0.4177
  bursting  FP32        0.6292        100 / 100              0.3875

The regime transition survives in FP32, but the statistics move by more than
the FP64 path's tolerance against the reference (active astrocytes 46 -> 39,
bursting correlation -7 %); FP64 stays the product.  Throughput of the
astrocyte-only workload at 10^7 cells: 179 us per step in FP32 against
277 us in FP64 in the same launch shape (232 us in FP64's best shape), not
the doubling the reference hoped for: the update stays bound by its
divisions.  After 1,000 steps the FP32 state is within 2e-5 relative of the
FP64 one (mean 6e-7).

Stated here: the transition is kept (use_case below 0.05, bursting - use_case
above 0.25) and the 1,000-step drift stays below 1e-4 relative."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from astrosimgpu_b200.astro import AstroBackend, ScalingWorkload

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "astrosimgpu_b200", "astrosim_b200")
CFG = os.path.join(ROOT, "astrosimgpu_b200", "configs")

pytestmark = pytest.mark.gpu


def test_fp32_scaling_workload_drift():
    n = 100_003
    w = ScalingWorkload(n)
    Ca, IP3, h = w.initial_state()
    a64 = AstroBackend(Ca, IP3, h)
    a32 = AstroBackend(Ca, IP3, h)
    a64.run_bernoulli(w, 0, 1000)
    a32.run_bernoulli_f32(w, 0, 500)
    a32.run_bernoulli_f32(w, 500, 500)  # resumes from its float state
    for x, y in zip(a32.pull_state(), a64.pull_state()):
        assert np.all(np.isfinite(x))
        rel = np.abs(x - y) / np.maximum(np.abs(y), 1e-12)
        assert rel.max() < 1e-4, rel.max()
        assert rel.max() > 0.0  # it is a different arithmetic, not the FP64 path


def correlation(config, fp32):
    with tempfile.TemporaryDirectory() as out:
        args = [CLI, "-c", os.path.join(CFG, config + ".json"), "-o", out, "-t", "60000", "-s",
                "1"] + (["--astro-fp32"] if fp32 else [])
        r = subprocess.run(args, capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, r.stderr[-1000:]
        text = open(os.path.join(out, "run.txt")).read()
    assert "FP32 astrocytes" in text
    return float(re.search(r"mean pairwise correlation\s+(-?[0-9.]+)", text).group(1))


def test_fp32_astrocytes_keep_the_synchrony_transition():
    low = correlation("use_case", True)
    high = correlation("bursting", True)
    assert low < 0.05 and high - low > 0.25, (low, high)
