"""The oracle's numpy restatement of the LP generator (oracle/lpgen.py, used
by bench.py's reference arm so that arm loads no product library) against the
product's ds_gen_lp: identical arrays, bit for bit."""
import numpy as np
import pytest

from oracle import lpgen as G
from parallel_ds_b200 import _lib
from parallel_ds_b200 import lp as L


@pytest.mark.parametrize("kind,kw", [
    (_lib.GEN_DENSITY, dict(m=60, n=120, density=0.1, seed=3)),
    (_lib.GEN_DENSITY, dict(m=200, n=400, density=0.05, seed=2000)),
    (_lib.GEN_PER_COL, dict(m=300, n=600, per_col=8, seed=1)),
    (_lib.GEN_BLOCK, dict(m=2 * 40 + 5, n=2 * 80, blocks=2, block_m=40, block_n=80, link_rows=5,
                          block_density=0.05, link_density=0.1, seed=9)),
])
def test_restatement_matches_library(kind, kw):
    a = L.generate(kind, **kw)
    b = G.generate(kind, **kw)
    for key in ("row_ptr", "col_idx", "val", "b", "c"):
        np.testing.assert_array_equal(np.asarray(a[key]), np.asarray(b[key]), err_msg=key)


def test_learned_workload_seed():
    a, b = L.learned(2000), G.learned(2000)
    for key in ("row_ptr", "col_idx", "val", "b", "c"):
        np.testing.assert_array_equal(np.asarray(a[key]), np.asarray(b[key]), err_msg=key)


def test_batched_instances():
    for i in (0, 5, 17):
        a = L.batched_instance(7, i, 16, 64, 0.10)
        b = G.batched_instance(7, i, 16, 64, 0.10)
        assert a["m"] == b["m"]
        for key in ("row_ptr", "col_idx", "val", "b", "c"):
            np.testing.assert_array_equal(np.asarray(a[key]), np.asarray(b[key]), err_msg=key)
