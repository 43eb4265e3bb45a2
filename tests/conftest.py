import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from sp3mm4amg_b200.problems import CSR  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden_cases.npz")
REF_FIXTURE = os.path.join(ROOT, "tests", "golden", "reference_fixture.npz")
from oracle import REF_TEST_DIR  # noqa: E402


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


def reference_fixture_arrays():
    """The reference's bundled quadruple code/test/{r,ac,p,ac_next} (R, AC,
    P, AC_next), as the committed fixture holds it (tests/golden/
    make_golden.py reads the files with the reference's own MatrixMarket
    loader)."""
    z = np.load(REF_FIXTURE)
    return tuple(_unpack(z, n) for n in ("r", "ac", "p", "ac_next"))


@pytest.fixture(scope="session")
def reference_fixture():
    return reference_fixture_arrays()
