import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def kats():
    with open(os.path.join(GOLDEN, "reference_kats.json")) as f:
        return json.load(f)


def kat_lp(entry, lower_ub_inf=True):
    """A reference KAT as a typed LP dict.  The reference tests pass upper_bound
    = 0 for Lower columns; with lower_ub_inf those bounds become +inf (the value
    an MPS-loaded Lower column carries)."""
    n = entry["n"]
    ub = list(entry["col_ub"])
    if lower_ub_inf:
        ub = [1e300 if entry["col_type"][j] == 4 else ub[j] for j in range(n)]
    return dict(m=entry["m"], n=n, row_ptr=np.array(entry["row_ptr"], np.int32),
                col_idx=np.array(entry["col_idx"], np.int32), val=np.array(entry["val"]),
                c=np.array(entry["c"]), col_type=np.array(entry["col_type"], np.int32),
                col_lb=np.array(entry["col_lb"]), col_ub=np.array(ub),
                row_type=np.array(entry["row_type"], np.int32), row_lb=np.array(entry["row_lb"]),
                row_ub=np.array(entry["row_ub"]))


def highs(lp):
    from scipy.optimize import linprog
    from parallel_ds_b200.lp import to_scipy
    return linprog(lp["c"], A_ub=to_scipy(lp), b_ub=lp["b"], bounds=(0, None), method="highs-ds")


def feasibility(lp, x):
    """max primal violation of A x <= b, x >= 0 (structural x)."""
    from parallel_ds_b200.lp import to_scipy
    A = to_scipy(lp)
    r = A @ x - lp["b"]
    return max(float(np.max(r, initial=0.0)), float(np.max(-x, initial=0.0)))
