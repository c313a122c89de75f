"""The binding layers above the C ABI: MEX gateways and the plain-C harness."""
import glob
import os
import subprocess

import numpy as np
import pytest
from conftest import ROOT, bits_equal, load_golden, packed_from_golden

GXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
GCC = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"


@pytest.mark.parametrize("src", sorted(glob.glob(os.path.join(ROOT, "magpackage_b200", "mex", "*.cpp"))))
def test_mex_gateways_compile(src):
    """Each gateway compiles against a mex.h (the oracle's stand-in here; MATLAB's own
    header in a real build) and the C ABI header."""
    out = subprocess.run([GXX, "-std=c++11", "-fsyntax-only", "-Wall", "-Werror",
                          "-I" + os.path.join(ROOT, "oracle", "mex_shim"), "-I" + os.path.join(ROOT, "include"),
                          src], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr


def test_harness_compiles(tmp_path):
    exe = tmp_path / "replay"
    out = subprocess.run([GCC, "-O2", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
                          os.path.join(ROOT, "magpackage_b200", "harness", "replay.c"),
                          "-L" + os.path.join(ROOT, "magpackage_b200"), "-lmagasm", "-o", str(exe)],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stderr


@pytest.mark.gpu
def test_harness_replays_golden(tmp_path):
    from magpackage_b200.harness.write_inputs import read_output, write_inputs

    d = load_golden("cube3")
    inp, outd = tmp_path / "in", tmp_path / "out"
    outd.mkdir()
    write_inputs(str(inp), d["P"], d["T0"] + 1, d["t2e"] + 1, d["sign"], d["tags"], d["sol"], d["qw"],
                 d["curl"], packed_from_golden(d))
    exe = tmp_path / "replay"
    lib = os.path.join(ROOT, "magpackage_b200")
    subprocess.run([GCC, "-O2", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "magpackage_b200", "harness", "replay.c"), "-L" + lib, "-lmagasm",
                    "-Wl,-rpath," + lib, "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(inp), str(outd)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for name, key in (("I", "jac_I"), ("J", "jac_J"), ("V", "jac_V"), ("R_idx", "jac_Ridx"),
                      ("R_val", "jac_Rval")):
        assert bits_equal(read_output(str(outd), name), d[key]), name
