"""ctypes binding of libds_b200.so (the C ABI declared in include/ds_api.h).

The library is built in-tree (``python -m parallel_ds_b200.build``); importing
this module never falls back to anything else: a missing library raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libds_b200.so")

DS_OK = 0
ERRORS = {-1: "DS_ERR_ARG", -2: "DS_ERR_CUDA", -3: "DS_ERR_STATE", -4: "DS_ERR_SHAPE",
          -5: "DS_ERR_NUMERIC", -6: "DS_ERR_DEVICE_WAIT", -7: "DS_ERR_CAPACITY"}
STATUS = {0: "unsolved", 1: "optimal", 2: "primal_infeasible", 3: "dual_infeasible",
          4: "iter_limit", 5: "error"}
PRICING_DSE, PRICING_LEARNED = 0, 1
FACTOR_SPARSE, FACTOR_DENSE = 0, 1
GEN_DENSITY, GEN_PER_COL, GEN_BLOCK = 0, 1, 2
NUM_FEATURES = 12
MLP_NPARAMS = 64 * NUM_FEATURES + 64 + 64 * 64 + 64 + 64 + 1


class DsOptions(C.Structure):
    _fields_ = [("refactor_interval", C.c_int), ("max_iterations", C.c_int), ("pricing", C.c_int),
                ("strict_reference", C.c_int), ("seed", C.c_ulonglong), ("device", C.c_int),
                ("stream", C.c_void_p), ("learned_margin", C.c_double), ("verbose", C.c_int),
                ("learned_mix", C.c_double), ("learned_pdhg_iters", C.c_int), ("dense_max_m", C.c_int),
                ("dense_refactor_interval", C.c_int), ("learned_start_iteration", C.c_int),
                ("pdhg_cluster", C.c_int), ("factor_mode", C.c_int)]


class DsStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("phase1_iterations", C.c_int), ("refactors", C.c_int),
                ("restarts", C.c_int), ("perturbed", C.c_int), ("bfrt_flips", C.c_int),
                ("learned_used", C.c_int), ("learned_fallback", C.c_int), ("bump_size", C.c_int),
                ("kernel_launches", C.c_int), ("solve_ms", C.c_double), ("refactor_ms", C.c_double),
                ("pdhg_ms", C.c_double), ("lu_kernel", C.c_int), ("lu_dense", C.c_int),
                ("lu_levels", C.c_int), ("lu_rounds", C.c_int)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class DsGenSpec(C.Structure):
    _fields_ = [("kind", C.c_int), ("m", C.c_int), ("n", C.c_int), ("density", C.c_double),
                ("per_col", C.c_int), ("blocks", C.c_int), ("block_m", C.c_int), ("block_n", C.c_int),
                ("link_rows", C.c_int), ("block_density", C.c_double), ("link_density", C.c_double),
                ("seed", C.c_ulonglong)]


class DsError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None
IP = C.POINTER(C.c_int)
DP = C.POINTER(C.c_double)
FP = C.POINTER(C.c_float)


def lib():
    """Load libds_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise DsError(-3, f"{LIB_PATH} not built; run python -m parallel_ds_b200.build")
    L = C.CDLL(LIB_PATH)
    sig = {
        "ds_default_options": (None, [C.POINTER(DsOptions)]),
        "ds_version": (C.c_char_p, []),
        "ds_create": (C.c_int, [C.POINTER(DsOptions), C.POINTER(C.c_void_p)]),
        "ds_destroy": (C.c_int, [C.c_void_p]),
        "ds_load_csr": (C.c_int, [C.c_void_p, C.c_int, C.c_int, IP, IP, DP, DP, DP, DP, DP, DP]),
        "ds_load_typed": (C.c_int, [C.c_void_p, C.c_int, C.c_int, IP, IP, DP, DP, IP, DP, DP, IP, DP, DP]),
        "ds_solve": (C.c_int, [C.c_void_p]),
        "ds_get_status": (C.c_int, [C.c_void_p]),
        "ds_get_objective": (C.c_double, [C.c_void_p]),
        "ds_get_primal": (C.c_int, [C.c_void_p, DP, DP]),
        "ds_get_dual": (C.c_int, [C.c_void_p, DP]),
        "ds_get_reduced_costs": (C.c_int, [C.c_void_p, DP]),
        "ds_get_iterations": (C.c_int, [C.c_void_p]),
        "ds_get_stats": (C.c_int, [C.c_void_p, C.POINTER(DsStats)]),
        "ds_get_basis": (C.c_int, [C.c_void_p, IP]),
        "ds_last_error": (C.c_char_p, [C.c_void_p]),
        "ds_set_trace": (C.c_int, [C.c_void_p, C.c_int]),
        "ds_get_trace": (C.c_int, [C.c_void_p, IP, IP, DP, DP, IP]),
        "ds_set_feature_trace": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
        "ds_get_feature_trace": (C.c_int, [C.c_void_p, FP, IP, IP, IP]),
        "ds_set_model": (C.c_int, [C.c_void_p, C.c_void_p]),
        "ds_model_set_wait_limit": (C.c_int, [C.c_void_p, C.c_int]),
        "ds_pdhg_estimate": (C.c_int, [C.c_void_p, C.c_int, DP, DP]),
        "ds_model_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
        "ds_model_destroy": (C.c_int, [C.c_void_p]),
        "ds_model_set_params": (C.c_int, [C.c_void_p, FP, C.c_int]),
        "ds_model_get_params": (C.c_int, [C.c_void_p, FP, C.c_int]),
        "ds_model_forward": (C.c_int, [C.c_void_p, FP, C.c_int, FP, FP, FP]),
        "ds_model_gradients": (C.c_int, [C.c_void_p, FP, FP, C.c_int, FP, FP]),
        "ds_model_train": (C.c_int, [C.c_void_p, FP, FP, C.c_int, C.c_int, C.c_int, C.c_float, C.c_ulonglong, FP]),
        "ds_kernel_dse_pricing": (C.c_int, [C.c_int, C.c_int, IP, DP, DP, DP, IP, DP, IP, IP, DP, IP, IP]),
        "ds_kernel_pivot_row": (C.c_int, [C.c_int, C.c_int, IP, IP, DP, IP, DP, DP]),
        "ds_kernel_ratio_test": (C.c_int, [C.c_int, C.c_int, IP, DP, C.c_double, C.c_int, DP, DP, DP, DP,
                                           IP, IP, IP, DP, DP, IP]),
        "ds_kernel_pfi_apply": (C.c_int, [C.c_int, C.c_int, DP, IP, DP, DP, C.c_int]),
        "ds_kernel_last_time": (C.c_int, [DP]),
        "ds_sparse_triangularise": (C.c_int, [C.c_int, IP, IP, IP, IP, IP, IP]),
        "ds_kernel_ratio_test_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                   IP, IP, DP, DP, IP, C.c_void_p]),
        "ds_kernel_launch_count": (C.c_longlong, []),
        "ds_basis_solve": (C.c_int, [C.c_void_p, IP, DP, DP, C.c_int, C.c_int]),
        "ds_profile_solve": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
        "ds_gen_lp": (C.c_longlong, [C.POINTER(DsGenSpec), IP, IP, DP, DP, DP, C.c_longlong]),
        "ds_gen_batch_m": (C.c_int, [C.c_ulonglong, C.c_int, C.c_int, C.c_int]),
        "ds_mps_read": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_longlong),
                                  IP, IP, DP, DP, DP, DP, DP, DP, DP]),
        "ds_load_mps": (C.c_int, [C.c_void_p, C.c_char_p, DP]),
        "ds_mps_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        if hasattr(L, name):
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
    _lib = L
    return L


def ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None
