"""tigerpm_b200: a B200-native (sm_100a) PME kick behind TigerPM's interface.

The compute lives in libtigerpm_b200.so (CUDA kernels + C ABI, include/tpm.h);
this package holds its ctypes binding (_lib), the host-side mirror of the
reference interface (api) and the seeded synthetic inputs (workloads).
"""
from . import workloads  # noqa: F401

__all__ = ["api", "workloads", "load"]


def load():
    """Load the CUDA library (raises if it has not been built)."""
    from . import _lib
    return _lib.load()


def __getattr__(name):
    if name == "api":
        from . import api
        return api
    raise AttributeError(name)
