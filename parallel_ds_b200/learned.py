"""Learned leaving-row pricing: the network handle, training data and training.

The network (csrc/mlp.cu) is an MLP 12 -> 64 -> 64 -> 1 whose logit estimates
whether the basic variable of a candidate leaving row is nonbasic at the
optimum ("leaves for good").  CHUZR ranks candidate rows by
``w_i * (mix + (1 - mix) * sigmoid(logit_i))`` with ``w_i`` the dual
steepest-edge weight and falls back to the plain DSE row when the network's row
has ``sigmoid(logit) < margin``; optimality is still decided by the primal
feasibility test, so the network only changes the pivot order.

Training data are feature traces of plain (DSE) solves: every ``every``
iterations the features of each candidate row, labelled 1 when the row's basic
variable is not in the final optimal basis.  Forward, backward and Adam run on
the GPU (tcgen05 BF16 MMAs with FP32 accumulation).
"""
import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import DsError, ptr

NUM_FEATURES = _lib.NUM_FEATURES
NPARAMS = _lib.MLP_NPARAMS
HIDDEN = 64
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")
DEFAULT_WEIGHTS = os.path.join(WEIGHTS_DIR, "scorer_m2000_n4000_d1.npz")

# offsets in the flat fp32 parameter vector (ds_api.h order)
OFF_W1 = 0
OFF_B1 = OFF_W1 + HIDDEN * NUM_FEATURES
OFF_W2 = OFF_B1 + HIDDEN
OFF_B2 = OFF_W2 + HIDDEN * HIDDEN
OFF_W3 = OFF_B2 + HIDDEN
OFF_B3 = OFF_W3 + HIDDEN


def init_params(seed=0):
    """He-initialised parameters (flat float32, ds_api.h order)."""
    r = np.random.default_rng(seed)
    p = np.zeros(NPARAMS, np.float32)
    p[OFF_W1:OFF_B1] = r.normal(0, np.sqrt(2.0 / NUM_FEATURES), HIDDEN * NUM_FEATURES)
    p[OFF_W2:OFF_B2] = r.normal(0, np.sqrt(2.0 / HIDDEN), HIDDEN * HIDDEN)
    p[OFF_W3:OFF_B3] = r.normal(0, np.sqrt(1.0 / HIDDEN), HIDDEN)
    return p


class LeavingRowScorer:
    """A network handle (ds_model) on one GPU."""

    def __init__(self, params=None, device=0):
        self.L = _lib.lib()
        self.h = C.c_void_p()
        rc = self.L.ds_model_create(device, C.byref(self.h))
        if rc != 0:
            raise DsError(rc, "ds_model_create")
        self.device = device
        self.meta = {}
        self.set_params(init_params() if params is None else params)

    def __del__(self):
        try:
            if self.h:
                self.L.ds_model_destroy(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            raise DsError(rc, what)

    def set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.shape != (NPARAMS,):
            raise ValueError(f"expected {NPARAMS} parameters, got {p.shape}")
        self._check(self.L.ds_model_set_params(self.h, ptr(p, C.c_float), NPARAMS), "ds_model_set_params")

    def params(self):
        p = np.zeros(NPARAMS, np.float32)
        self._check(self.L.ds_model_get_params(self.h, ptr(p, C.c_float), NPARAMS), "ds_model_get_params")
        return p

    def forward(self, X, hidden=False):
        X = np.ascontiguousarray(X, dtype=np.float32)
        rows = X.shape[0]
        z = np.zeros(rows, np.float32)
        H1 = np.zeros((rows, HIDDEN), np.float32) if hidden else None
        H2 = np.zeros((rows, HIDDEN), np.float32) if hidden else None
        self._check(self.L.ds_model_forward(self.h, ptr(X, C.c_float), rows, ptr(z, C.c_float),
                                            ptr(H1, C.c_float), ptr(H2, C.c_float)), "ds_model_forward")
        return (z, H1, H2) if hidden else z

    def gradients(self, X, y):
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        g = np.zeros(NPARAMS, np.float32)
        loss = C.c_float(0)
        self._check(self.L.ds_model_gradients(self.h, ptr(X, C.c_float), ptr(y, C.c_float), X.shape[0],
                                              ptr(g, C.c_float), C.byref(loss)), "ds_model_gradients")
        return g, float(loss.value)

    def train(self, X, y, epochs=10, batch=4096, lr=1e-3, seed=0):
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        loss = C.c_float(0)
        self._check(self.L.ds_model_train(self.h, ptr(X, C.c_float), ptr(y, C.c_float), X.shape[0], epochs,
                                          batch, lr, seed, C.byref(loss)), "ds_model_train")
        return float(loss.value)

    def attach(self, solver):
        """Use this network for a CudaDualSimplex solver's learned pricing."""
        rc = self.L.ds_set_model(solver.h, self.h)
        if rc != 0:
            raise DsError(rc, "ds_set_model")

    def save(self, path, **meta):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez(path, params=self.params(), **{k: np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, path=DEFAULT_WEIGHTS, device=0):
        with np.load(path) as f:
            m = cls(f["params"], device=device)
            m.meta = {k: f[k] for k in f.files if k != "params"}
        return m


# ------------------------------------------------------------------ training data
def solve_with_trace(lp, every=8, cap=1 << 20, device=0, refactor_interval=100, seed=12345):
    """Plain DSE solve of a generated LP with the feature trace on.

    Returns (result dict, features [k x 12] float32, labels [k] float32, meta [k x 3]).
    A record is labelled 1 when its basic variable is not in the final basis."""
    from .solver import CudaDualSimplex, problem_from_lp
    s = CudaDualSimplex(problem_from_lp(lp), refactor_interval=refactor_interval, seed=seed, device=device)
    s.initDualSimplex()
    s.set_feature_trace(every, cap)
    sol = s.solve()
    F, M, total = s.feature_trace()
    basis = s.basis()
    in_final = np.zeros(lp["n"] + lp["m"], bool)
    in_final[basis] = True
    y = (~in_final[M[:, 2]]).astype(np.float32) if len(M) else np.zeros(0, np.float32)
    res = dict(status=s.status(), objective=sol.Z, iterations=sol.iterations, trace_total=total,
               stats=s.stats())
    return res, F, y, M
