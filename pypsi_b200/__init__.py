"""pypsi_b200 -- PSI's phase-space-sheet voxelization on NVIDIA B200 (sm_100a).

``pypsi_b200.PSI`` is the drop-in module: ``Grid``, ``Mesh`` (loaders 'array',
'block', 'gadget2', 'gevolution'), ``voxels`` (modes 'density' and
'annihilation'), ``RStarTree`` and ``VDF`` behave as in PyPSI's ``PSI``
extension (src/PSI.c) and run on the GPU through ``libpsi_b200.so`` (C ABI in
include/psi_b200.h).  ``capi`` binds the C ABI for device-resident arrays,
``autograd`` the adjoint, ``parallel`` several GPUs.

There is no CPU fallback: importing the package raises if the native library
has not been built (``python pypsi_b200/build.py``), and every GPU call raises
if no CUDA device is visible.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpsi_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `python pypsi_b200/build.py`")

lib = ctypes.CDLL(LIB_PATH)

from . import PSI  # noqa: E402  (the CPython extension, linked against libpsi_b200.so)

__all__ = ["PSI", "lib", "LIB_PATH"]
