"""The binding layers above the C ABI: MEX gateways and the plain-C harness."""
import glob
import os
import subprocess

import numpy as np
import pytest
from conftest import ROOT, bits_equal, load_golden, packed_from_golden

GXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
GCC = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"


GATEWAYS = sorted(glob.glob(os.path.join(ROOT, "magpackage_b200", "mex", "*.cpp")))


@pytest.mark.parametrize("src", GATEWAYS)
def test_mex_gateways_compile(src):
    """Each gateway compiles against a mex.h (the tests' stand-in here; MATLAB's own
    header in a real build) and the C ABI header."""
    out = subprocess.run([GXX, "-std=c++11", "-fsyntax-only", "-Wall", "-Werror",
                          "-I" + os.path.join(ROOT, "tests", "mex_host"), "-I" + os.path.join(ROOT, "include"),
                          src], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr


@pytest.mark.parametrize("name,nargs,msg", [
    ("assemble_jacobian_kernel_mex", 16, "Expected 17 inputs (18 with the sparse-output flag)."),
    ("assemble_jacobian_kernel_mex", 19, "Expected 17 inputs (18 with the sparse-output flag)."),
    ("assemble_curl_curl_kernel_mex", 6, "Expected 7 inputs (8 with Ndof)."),
    ("assemble_mass_kernel_mex", 9, "Expected 7 inputs (8 with Ndof)."),
    ("assemble_source_kernel_mex", 8, "Expected 7 inputs."),
    ("assemble_winding_kernel_mex", 10, "Expected 11 inputs."),
])
def test_gateway_rejects_argument_count(tmp_path, name, nargs, msg):
    """The gateways link against libmagasm and raise MagPackage:Args, as the reference's
    do, before any device work (runs without a GPU)."""
    from mex_host.gateway import Gateway, GatewayError, build

    gw = Gateway(build(name, tmp_path))
    with pytest.raises(GatewayError, match="MagPackage:Args: " + msg.replace("(", r"\(").replace(")", r"\)")):
        gw(5, *([0.0] * nargs))


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
