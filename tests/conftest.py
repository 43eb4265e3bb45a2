import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from sp3mm4amg_b200.problems import CSR  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden_cases.npz")
REF_TEST_DIR = "/root/reference/code/test"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (run with -m gpu)")


def _unpack(z, prefix):
    return CSR(z[f"{prefix}_indptr"], z[f"{prefix}_indices"], z[f"{prefix}_data"],
               tuple(int(x) for x in z[f"{prefix}_shape"]))


def golden_cases():
    """{name: {R, A, P, pair, direct, symb_ra, ub_ra}} from the committed fixture."""
    z = np.load(GOLDEN)
    out = {}
    for name in z["cases"]:
        name = str(name)
        d = {k: _unpack(z, f"{name}__{k}") for k in ("R", "A", "P", "pair", "direct")}
        d["symb_ra"] = z[f"{name}__symb_ra"]
        d["ub_ra"] = z[f"{name}__ub_ra"]
        out[name] = d
    return out


@pytest.fixture(scope="session")
def golden():
    return golden_cases()


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle.Oracle()


@pytest.fixture(scope="session")
def reference_fixture():
    """The reference's bundled 14^3 quadruple (R, AC, P, AC_next), read in place."""
    if not os.path.isdir(REF_TEST_DIR):
        pytest.skip("reference tree not present")
    import oracle
    return tuple(oracle.load_mm(os.path.join(REF_TEST_DIR, n)) for n in ("r", "ac", "p", "ac_next"))
