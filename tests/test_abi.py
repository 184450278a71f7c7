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
