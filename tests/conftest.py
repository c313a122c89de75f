import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100a) device")


@pytest.fixture(scope="session")
def oracle_port():
    from oracle.oracle import Port, build

    if not os.path.exists(os.path.join(ROOT, "oracle", "libmagoracle.so")):
        build()
    return Port()


@pytest.fixture(scope="session")
def oracle_ref():
    from oracle.oracle import RefMex, ref_available

    if not ref_available():
        pytest.skip("reference MEX build (oracle/_ref) not present")
    return RefMex()


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def packed_from_golden(d):
    from magpackage_b200.material import PackedMaterials

    return PackedMaterials(d["mat_lin"], d["mat_isnon"], d["mat_maxb"], d["mat_brk"], d["mat_coe"],
                           d["mat_start"], d["mat_cnt"], d["mat_coestart"])


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    if a.shape != b.shape:
        return False
    # +0.0 and -0.0 compare equal by value; everything else must match bit for bit
    return bool(np.all((a.view(np.int64) == b.view(np.int64)) | ((a == 0) & (b == 0))))
