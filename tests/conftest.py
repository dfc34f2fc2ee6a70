import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from networkit_b200.graph import InCSR  # noqa: E402

GOLDEN_NAMES = ["wikivote_directed", "wikivote_undirected", "celegans", "looptest1", "looptest2",
                "matlab8"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def load_golden(name):
    """(InCSR, dict of reference results) of a fixture made by make_golden.py."""
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    weighted = bool(d["weighted"])
    ex = d["exists"]
    csr = InCSR(int(d["z"]), int(ex.sum()), d["in_ptr"], d["in_col"],
                d["in_w"] if weighted else None, d["wdeg"], d["outdeg"],
                None if ex.all() else ex, bool(d["directed"]))
    return csr, {k: d[k] for k in d.files}


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    return oracle
