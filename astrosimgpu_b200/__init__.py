"""B200-native per-timestep engine for the astrosimgpu neuron-astrocyte network.

The compute path is ``libasg_b200.so`` (hand-written sm_100a FP64 kernels
behind the C ABI of ``include/asg_b200.h``); this package is a thin ctypes
view of it for tests, benchmarks and scripting.
"""
from . import _lib  # noqa: F401

__all__ = ["_lib"]
