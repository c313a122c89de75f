"""Write the seventeen assemble_jacobian_kernel_mex inputs as raw float64 files.

The plain-C harness (replay.c) reads them back; the argument meaning and layout
are the reference gateway's (src/mex/assemble_jacobian_kernel_mex.cpp:10-40).
"""
from __future__ import annotations

import os

import numpy as np

NAMES = ("P", "T", "Dofs", "Signs", "Tags", "SolA", "Qw", "CurlRef", "lin", "isNon", "maxB", "brk", "coe",
         "start", "cnt", "coeStart")


def write_inputs(directory, P, T1, Dofs1, Signs, Tags, SolA, Qw, CurlRef, packed):
    """All index arrays 1-based doubles, as Assembler.m passes them."""
    os.makedirs(directory, exist_ok=True)
    arrays = (P, T1, Dofs1, Signs, Tags, SolA, Qw, CurlRef) + tuple(packed.as_tuple())
    for name, a in zip(NAMES, arrays):
        np.ascontiguousarray(a, dtype="<f8").tofile(os.path.join(directory, f"{name}.f64"))


def read_output(directory, name):
    return np.fromfile(os.path.join(directory, f"{name}.f64"), dtype="<f8")
