"""sputnipic_b200: B200-native particle mover + particle-to-grid deposition for
sputniPIC, behind the reference's own entry points.

* ``sputnipic_b200.dropin``: the reference interface (setGrid, mover_PC,
  interpP2G, mover_interp, ...) over ctypes mirrors of the reference structs;
* ``sputnipic_b200.device``: the device-pointer plain form over torch tensors;
* ``sputnipic_b200.workload``: seeded synthetic GEM workloads.

All compute runs in libsputnipic_b200.so (CUDA, sm_100a).
"""
from . import workload  # noqa: F401

__all__ = ["workload", "dropin", "device", "load_library"]


def load_library():
    from . import _lib
    return _lib.load()
