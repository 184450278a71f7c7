"""div_by, the engine's division by a run-time constant through the
host-rounded reciprocal (astrosimgpu_b200/csrc/asg_device.cuh), is bitwise
the IEEE quotient the reference computes.

tests/div_by_check.cu runs the engine's own div_by (compiled for the host:
the host fma is IEEE's correctly rounded fused multiply-add, as the GPU's is)
against IEEE division over operand classes: random normal operands (the
domain of Markstein's theorem), the engine's own divisors with numerators of
the magnitudes the model produces, and the cases the theorem excludes -- a
numerator small enough for the remainder to be subnormal, subnormal
quotients, quotients at the overflow threshold, mantissas of all ones and
powers of two, and signed zeros.  Every class must match bit for bit: the
excluded cases take the IEEE division itself.  div_diff_by, the astrocyte
right-hand side's form without the exponent test, is checked the same way on
differences with a parameter operand of magnitude in [2^-906, 2^976] (the
range the engine enforces for Ca_tot and IP3_0) and any other operand."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    exe = str(tmp_path_factory.mktemp("divby") / "div_by_check")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-x", "cu", "-Wno-deprecated-gpu-targets",
                    "-I" + os.path.join(ROOT, "astrosimgpu_b200", "csrc"),
                    "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "div_by_check.cu"), "-o", exe],
                   check=True, capture_output=True)
    return exe


@pytest.mark.parametrize("seed", [1, 2])
def test_div_by_equals_ieee_division(checker, seed):
    out = subprocess.run([checker, "50000000", str(seed)], check=True, capture_output=True,
                         text=True)
    rows = {}
    for line in out.stdout.splitlines():
        name, cases, bad = line.split()
        rows[name] = (int(cases), int(bad))
    assert set(rows) == {"random", "engine", "tiny_a", "sub_q", "huge", "hard", "zero",
                         "neg_zero", "diff"}
    for name, (cases, bad) in rows.items():
        assert cases > 0, name
        assert bad == 0, (name, cases, bad, out.stderr[:500])
    assert rows["random"][0] == 50_000_000
