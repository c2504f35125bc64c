"""nepheline_b200: the physics world step's solver stage on an NVIDIA B200.

The product is the C-ABI shared library lib/libnepheline_b200.so (include/nepheline_b200.h);
this package holds its CUDA sources (csrc/), the record layouts (abi), seeded synthetic
workloads (scenes) and a thin ctypes binding (solver).
"""
from . import abi  # noqa: F401

__version__ = "0.1.0"
