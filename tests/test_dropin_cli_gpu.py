"""The drop-in compiled for real: the reference's own command-line simulator
(its main.cpp, parameters, recorder, analysis, builder -- built from the
reference sources by integration/Makefile) bound to the B200 engine two
ways -- Network::run on the engine (integration/network_b200.cpp), and the
reference's own ASTROSIMGPU_CUDA astrocyte branches on the engine's
asg_astro_* calls (integration/astrocyte_b200.cpp) -- against the
unmodified reference CLI (oracle/_ref/astrosimgpu) on the same config and
seed.

Both write spikes.csv, astrocytes.csv and run.txt through the reference's
Recorder and summary code.  With Network::run bound, the files must agree
byte for byte: the spike file, the astrocyte traces (6 significant digits,
the reference's formatting) and the run summary's counts, rate and calcium
analysis.  With the astrocyte backend bound, the spike file and the summary
must agree, and so must the traces' Ca column, to one unit in the sixth
significant digit (the astrocyte noise's Box-Muller log and cos come from
CUDA on the GPU and from the host libm in the reference, which can move a
printed digit).  Their IP3 column is the reference CUDA backend's own: its
movement points pull only Ca back each step (astrocyte.cpp:195-200), so the
host's IP3 -- what the recorder prints -- stays at its initial value, as it
does in the reference's CUDA build."""
import os
import re
import subprocess
import tempfile
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "integration", "_build", "astrosimgpu_b200")
DROPIN_ASTRO = os.path.join(ROOT, "integration", "_build", "astrosimgpu_b200_astro")
REF_CLI = os.path.join(ROOT, "oracle", "_ref", "astrosimgpu")
CFG = os.path.join(ROOT, "astrosimgpu_b200", "configs")

pytestmark = pytest.mark.gpu

SUMMARY_KEYS = ("astrocytes", "excitatory neurons", "inhibitory neurons",
                "exc -> neuron synapses", "inh -> neuron synapses", "neuron -> astrocyte",
                "astrocyte -> neuron", "spikes recorded", "mean firing rate",
                "astrocytes with transients", "transients detected", "mean duration",
                "pairs correlated", "mean pairwise correlation")


def run(cli, config, out, *args):
    t0 = time.time()
    r = subprocess.run([cli, "-c", config, "-o", out, *args], capture_output=True, text=True,
                       timeout=900, env=dict(os.environ, OMP_NUM_THREADS="4"))
    assert r.returncode == 0, (cli, r.stdout[-1000:], r.stderr[-1000:])
    print(f"{os.path.basename(cli)} {config} {args}: {time.time() - t0:.1f} s")
    with open(os.path.join(out, "run.txt")) as f:
        text = f.read()
    lines = {}
    for key in SUMMARY_KEYS:
        m = re.search(r"^" + re.escape(key) + r"\s+(.*)$", text, re.M)
        if m:
            lines[key] = m.group(1).strip()
    return lines


@pytest.mark.parametrize("cli,name,args", [
    (DROPIN, "use_case", ("-t", "1000", "-p", "0", "-s", "1")),
    (DROPIN, "bursting", ("-t", "2000", "-p", "500", "-s", "3")),
    (DROPIN_ASTRO, "use_case", ("-t", "1000", "-p", "0", "-s", "1")),
])
def test_reference_cli_bound_to_b200(cli, name, args):
    assert os.path.exists(cli), f"{cli} not built (integration/Makefile)"
    cfg = os.path.join(CFG, name + ".json")
    whole_step = cli == DROPIN
    with tempfile.TemporaryDirectory() as a, tempfile.TemporaryDirectory() as b:
        got = run(cli, cfg, a, *args)
        want = run(REF_CLI, cfg, b, *args)
        for f in ("spikes.csv", "astrocytes.csv"):
            with open(os.path.join(a, f)) as fa, open(os.path.join(b, f)) as fb:
                ta, tb = fa.read(), fb.read()
            assert ta.count("\n") > 1
            if whole_step or f == "spikes.csv":
                assert ta == tb, f"{name}: {f} differs"
                continue
            ra = [line.split(",") for line in ta.splitlines()[1:]]
            rb = [line.split(",") for line in tb.splitlines()[1:]]
            assert [r[:2] for r in ra] == [r[:2] for r in rb]
            ca_a = np.array([float(r[2]) for r in ra])
            ca_b = np.array([float(r[2]) for r in rb])
            assert np.all(np.abs(ca_a - ca_b) <= 1.01e-5 * np.abs(ca_b) + 1e-12), f"{name}: Ca"
    if whole_step:
        assert got == want
    else:
        for key in ("spikes recorded", "mean firing rate", "astrocytes with transients",
                    "transients detected"):
            assert got.get(key) == want.get(key), key
        if "mean pairwise correlation" in want:
            assert abs(float(got["mean pairwise correlation"]) -
                       float(want["mean pairwise correlation"])) <= 1e-3
    assert int(got["spikes recorded"]) > 0
