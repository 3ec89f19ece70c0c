"""pypsi_b200 -- PSI's phase-space-sheet voxelization on NVIDIA B200 (sm_100a).

``pypsi_b200.PSI`` is the drop-in module: ``Grid``, ``Mesh`` (loaders 'array',
'block', 'gadget2', 'gevolution'), ``voxels`` (modes 'density' and
'annihilation'), ``RStarTree`` and ``VDF`` behave as in PyPSI's ``PSI``
extension (src/PSI.c) and run on the GPU through ``libpsi_b200.so`` (C ABI in
include/psi_b200.h).  ``capi`` binds the C ABI for device-resident arrays,
``autograd`` the adjoint, ``parallel`` several GPUs.

The native library is mapped on first use of ``lib``, ``PSI`` or ``capi``, so
that the pure-Python helpers (``synth``, ``metrics``) import without it.
There is no CPU fallback: that first use raises if the library has not been
built (``python pypsi_b200/build.py``), and every GPU call raises if no CUDA
device is visible.
"""
from __future__ import annotations

import ctypes
import importlib
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpsi_b200.so")

_lib = None


def _load_lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python pypsi_b200/build.py`")
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def __getattr__(name: str):
    if name == "lib":
        return _load_lib()
    if name == "PSI":
        _load_lib()
        return importlib.import_module(".PSI", __name__)  # the CPython extension, linked against libpsi_b200.so
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


__all__ = ["PSI", "lib", "LIB_PATH"]
