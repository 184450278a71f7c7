"""The C-ABI library loads on a machine without a GPU and exports every
entry point declared in include/asg_b200.h; entry points that need a device
fail cleanly with a status code instead of aborting."""
import ctypes as C
import os
import re

import pytest

from astrosimgpu_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "asg_b200.h")).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(asg_\w+)\(", text, re.M)))


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_header():
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_version_and_error_text():
    lib = _lib.load()
    assert b"sm_100a" in lib.asg_version()
    assert lib.asg_step(None, 1) == 1  # ASG_ERR_ARG on a NULL handle
    assert b"NULL" in lib.asg_last_error()


def test_no_device_is_a_status_not_an_abort():
    from conftest import have_gpu
    if have_gpu():
        pytest.skip("a GPU is visible")
    h = C.c_void_p()
    opts = _lib.EngineOpts()
    from astrosimgpu_b200.network import Model, config_path
    m = Model(config_path("quick"))
    d = m.desc()
    st = _lib.load().asg_create(C.byref(d), None, C.byref(opts), C.byref(h))
    assert st in (_lib.ASG_OK + 10, 3)  # ASG_ERR_NO_DEVICE (or a CUDA init error)


# ctypes mirrors of the header's structs (astrosimgpu_b200/_lib.py), by C name.
MIRRORS = {
    "asg_neuron_params": "NeuronParams", "asg_astro_params": "AstroParams",
    "asg_input": "InputParams", "asg_stp": "StpParams", "asg_csr": "Csr",
    "asg_network_desc": "NetworkDesc", "asg_record_opts": "RecordOpts",
    "asg_state": "State", "asg_engine_opts": "EngineOpts", "asg_serve_opts": "ServeOpts",
    "asg_request_result": "RequestResult",
}


def test_struct_layouts_match_header(tmp_path):
    """Every ctypes mirror has the size and field offsets the C compiler gives
    the header's struct (a field added on one side only would shift the
    arguments the library reads)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "asg_b200.h"', "int main(void) {"]
    for cname, pyname in MIRRORS.items():
        st = getattr(_lib, pyname)
        lines.append(f'printf("{pyname} size %zu\\n", sizeof({cname}));')
        for fname, _ in st._fields_:
            lines.append(f'printf("{pyname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True,
                               text=True).stdout.splitlines():
        name, field, value = line.split()
        got[(name, field)] = int(value)
    for cname, pyname in MIRRORS.items():
        st = getattr(_lib, pyname)
        assert got[(pyname, "size")] == C.sizeof(st), pyname
        for fname, _ in st._fields_:
            assert got[(pyname, fname)] == getattr(st, fname).offset, (pyname, fname)


def test_astro_create_rejects_a_partial_parameter_set():
    """All four per-cell parameter arrays or none: a partial set is refused on
    the host (before any device work), so no update can read a missing array."""
    import numpy as np
    lib = _lib.load()
    n = 8
    a = [np.ones(n) for _ in range(7)]
    h = C.c_void_p()
    for missing in range(3, 7):
        args = [_lib.dptr(x) if i != missing else None for i, x in enumerate(a)]
        st = lib.asg_astro_create(n, *args, C.byref(h))
        assert st == 1, missing  # ASG_ERR_ARG
        assert b"all four per-cell parameter arrays" in lib.asg_last_error()
        assert not h.value
