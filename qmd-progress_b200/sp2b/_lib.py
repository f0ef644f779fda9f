"""ctypes binding of libsp2b.so (the C ABI declared in include/sp2b.h, include/prg_sp2b.h).

There is no CPU fallback: if the library is missing or a call fails, an exception is
raised.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsp2b.so")

SP2B_OK = 0
SP2B_NOT_CONVERGED = 1
SP2B_BAD_ARG = 2
SP2B_CUDA_ERROR = 3
SP2B_TIMEOUT = 4
SP2B_BAD_INPUT = 5
SP2B_NO_DEVICE = 6

PREC_FP64 = 0
PREC_MIXED_FP16 = 1
PREC_MIXED_BF16 = 2
PREC_EXACT_INT8 = 3
MCW_INT8 = 0
MCW_FP64 = 1

STATUS_NAMES = {0: "SP2B_OK", 1: "SP2B_NOT_CONVERGED", 2: "SP2B_BAD_ARG", 3: "SP2B_CUDA_ERROR",
                4: "SP2B_TIMEOUT", 5: "SP2B_BAD_INPUT", 6: "SP2B_NO_DEVICE"}


class Opts(C.Structure):
    _fields_ = [("precision", C.c_int), ("mcweeny", C.c_int), ("mixed_tol", C.c_double),
                ("device_ptrs", C.c_int), ("stream", C.c_void_p), ("verbose", C.c_int),
                ("mcweeny_products", C.c_int), ("refine_tol", C.c_double),
                ("exact_switch", C.c_int)]


class SP2Error(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_llp = C.POINTER(C.c_longlong)
_vp = C.c_void_p
_i, _d = C.c_int, C.c_double

# name -> (restype, argtypes)
_SIGS = {
    "sp2b_opts_default": (_i, [C.POINTER(Opts)]),
    "sp2b_set_default_opts": (_i, [C.POINTER(Opts)]),
    "sp2b_get_default_opts": (_i, [C.POINTER(Opts)]),
    "sp2b_last_error": (C.c_char_p, []),
    "sp2b_sp2_alg2": (_i, [_vp, _vp, _i, _d, _d, _i, _i, C.c_char_p, _d, _i, C.POINTER(Opts), _ip]),
    "sp2b_sp2_alg2_genseq": (_i, [_vp, _vp, _i, _d, _d, _i, _i, C.c_char_p, _d, _vp, _ip, _vp, _i,
                                  C.POINTER(Opts)]),
    "sp2b_sp2_alg2_seq": (_i, [_vp, _vp, _i, _d, _vp, _i, _vp, _i, C.POINTER(Opts)]),
    "sp2b_sp2_alg2_seq_inplace": (_i, [_vp, _i, _d, _vp, _i, _vp, _d, _d, _i, C.POINTER(Opts)]),
    "sp2b_sp2_alg1": (_i, [_vp, _vp, _i, _d, _d, _i, _i, C.c_char_p, _d, _i, C.POINTER(Opts), _ip]),
    "sp2b_sp2_alg1_genseq": (_i, [_vp, _vp, _i, _d, _d, _i, _i, C.c_char_p, _d, _vp, _ip, _vp,
                                  C.POINTER(Opts)]),
    "sp2b_sp2_alg1_seq": (_i, [_vp, _vp, _i, _d, _vp, _i, _vp, C.POINTER(Opts)]),
    "sp2b_sp2_alg1_seq_inplace": (_i, [_vp, _i, _d, _vp, _i, _vp, _d, _d, C.POINTER(Opts)]),
    "sp2b_sp2_basic": (_i, [_vp, _vp, _i, _d, _d, _i, _i, C.c_char_p, _d, _i, C.POINTER(Opts), _ip]),
    "sp2b_sp2_submatrix_inplace": (_i, [_vp, _i, _d, _vp, _i, _vp, _d, _d, _i, C.POINTER(Opts)]),
    "sp2b_sp2_submatrix": (_i, [_vp, _vp, _i, _d, _vp, _i, _vp, _d, _d, _i, C.POINTER(Opts)]),
    "sp2b_sp2_submatrix_inplace_noalloc": (_i, [_vp, _i, _vp, _i, _vp, _d, _d, _i, _vp]),
    "sp2b_gershgorin": (_i, [_vp, _i, _dp, _dp, C.POINTER(Opts)]),
    "sp2b_normalize": (_i, [_vp, _i, _dp, _dp, C.POINTER(Opts)]),
    "sp2b_check_idempotency": (_i, [_vp, _i, _d, _dp, C.POINTER(Opts)]),
    "sp2b_sp2sequence": (_i, [_ip, _ip, _d, _d, _d, _d, _d, _i]),
    "sp2b_homolumogap": (_i, [_vp, _i, _vp, _d, _d, _dp, _dp, _dp]),
    "sp2b_equal_partition": (_i, [_i, _i, _ip, _vp, _vp]),
    "sp2b_subgraph_halos": (_i, [_i, _vp, _vp, _vp, _vp, _i, _vp, _vp, _i, _vp, _vp, C.c_longlong,
                                 _llp, _vp, _vp]),
    "sp2b_subgraph_sp2_loop": (_i, [_i, _vp, _vp, _vp, _i, _vp, _vp, _vp, _vp, _i, _d, _d, _vp, _vp,
                                    _vp, C.POINTER(Opts)]),
    "sp2b_dev_sym_gemm_f32": (_i, [_vp, _vp, _vp, _i, _vp]),
    "sp2b_dev_panel_gemm_f32": (_i, [_vp, _i, _vp, _i, _vp, _vp]),
    "sp2b_dev_normalize_f32": (_i, [_vp, _vp, _i, _d, _d, _vp]),
    "sp2b_dev_sp2_step_f32": (_i, [_vp, _vp, _i, _i, _vp]),
    "sp2b_dev_adjoint_step_f32": (_i, [_vp, _vp, _vp, _vp, _i, _i, _vp]),
    "sp2b_split_dim": (_i, [_i]),
    "sp2b_dev_normalize_split": (_i, [_vp, _i, _d, _d, _vp, _vp, _vp]),
    "sp2b_dev_f32_to_split": (_i, [_vp, _i, _vp, _vp, _vp]),
    "sp2b_dev_split_to_f32": (_i, [_vp, _vp, _i, _d, _vp, _vp]),
    "sp2b_dev_sp2_step_split": (_i, [_vp, _vp, _vp, _vp, _i, _i, _vp]),
    "sp2b_dev_adjoint_step_split": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp]),
    "sp2b_last_solve_info": (_i, [_ip, _ip, _ip, _ip, _vp, _i]),
    "sp2b_last_subgraph_refined": (_i, [_ip, _vp, _i, _vp, _i]),
    "sp2b_graph_square_threshold": (_i, [_i, _vp, _vp, _vp, _d, _vp, _vp, C.c_longlong, _vp,
                                         C.POINTER(Opts)]),
    "sp2b_sp2_fermi_init": (_i, [_vp, _i, _i, _d, _d, _d, _d, _d, _vp, _dp, _dp, _dp, _dp, _ip,
                                 C.POINTER(Opts)]),
    "sp2b_sp2_fermi": (_i, [_vp, _i, _i, _i, _d, _dp, _d, _d, _d, _ip, _d, _d, _d, _vp,
                            C.POINTER(Opts)]),
    "sp2b_sp2_fermi_init_norecs": (_i, [_vp, _i, _ip, _d, _d, _d, _d, _d, _vp, _dp, _dp, _dp,
                                        _dp, _ip, C.POINTER(Opts)]),
    "sp2b_sp2_entropy_function": (_i, [_d, _d, _d, _i, _ip, _dp, _dp, _i]),
    "sp2b_tune_get": (_i, [C.c_char_p, _ip, C.POINTER(C.c_float), _i, _ip]),
    "sp2b_tune_set": (_i, [C.c_char_p, _i]),
    "sp2b_tune_keys": (_i, [C.c_char_p, _i]),
    "sp2b_tune_clear": (_i, []),
    "sp2b_ellpack_to_csr": (_i, [_i, _i, _vp, _vp, _vp, _vp, _vp, _vp, C.c_longlong,
                                 C.POINTER(C.c_longlong), C.POINTER(Opts)]),
    "sp2b_launch_count": (C.c_longlong, []),
    "sp2b_last_exact_switch": (_i, []),
    "sp2b_place_core_rows": (_i, [C.c_longlong, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "sp2b_last_refinement_info": (_i, [_ip, _dp]),
    "sp2b_compute_response_sp2": (_i, [_vp, _vp, _vp, _vp, _i, C.c_double, C.c_double, _i, _i,
                                       C.c_char_p, C.c_double, C.c_double, _i, _vp, _ip, _vp]),
    "sp2b_refinement_timing": (_i, [_dp, C.POINTER(C.c_longlong)]),
    "sp2b_selftest_wait_timeout": (_i, [_i]),
    "sp2b_set_step_timing": (_i, [_i]),
    "sp2b_step_timing": (_i, [_dp, _llp]),
    # PROGRESS-named exports
    "sp2b_bml_wrap_dense": (_vp, [_vp, _i]),
    "sp2b_bml_zero_dense": (_vp, [_i]),
    "sp2b_bml_data": (_dp, [_vp]),
    "sp2b_bml_n": (_i, [_vp]),
    "sp2b_bml_free": (None, [_vp]),
    "sp2b_prg_last_status": (_i, []),
    "prg_sp2_basic": (None, [_vp, _vp, _d, _d, _i, _i, C.c_char_p, _d, _i]),
    "prg_sp2_alg2": (None, [_vp, _vp, _d, _d, _i, _i, C.c_char_p, _d, _i]),
    "prg_sp2_alg2_genseq": (None, [_vp, _vp, _d, _d, _i, _i, C.c_char_p, _d, _vp, _ip, _vp, _i]),
    "prg_sp2_alg2_seq": (None, [_vp, _vp, _d, _vp, _ip, _vp, _i]),
    "prg_sp2_alg1": (None, [_vp, _vp, _d, _d, _i, _i, C.c_char_p, _d, _i]),
    "prg_sp2_alg1_genseq": (None, [_vp, _vp, _d, _d, _i, _i, C.c_char_p, _d, _vp, _ip, _vp]),
    "prg_sp2_alg1_seq": (None, [_vp, _vp, _d, _vp, _ip, _vp]),
    "prg_prg_sp2_alg2_seq_inplace": (None, [_vp, _d, _i, _vp, _ip, _vp, _d, _d]),
    "prg_prg_sp2_alg1_seq_inplace": (None, [_vp, _d, _i, _vp, _ip, _vp, _d, _d]),
    "prg_sp2_submatrix": (None, [_vp, _vp, _d, _vp, _ip, _vp, _d, _d, _i]),
    "prg_sp2_submatrix_inplace": (None, [_vp, _d, _vp, _ip, _vp, _d, _d, _i]),
    "prg_sp2_fermi_init": (None, [_vp, _i, _d, _d, _d, _d, _d, _vp, _dp, _dp, _dp, _dp, _ip]),
    "prg_sp2_fermi": (None, [_vp, _i, _i, _d, _dp, _dp, _dp, _dp, _ip, _d, _d, _d, _vp]),
    "prg_sp2_fermi_init_norecs": (None, [_vp, _ip, _d, _d, _d, _d, _d, _vp, _dp, _dp, _dp, _dp,
                                          _ip, _i]),
    "prg_sp2_entropy_function": (None, [_d, _d, _d, _i, _ip, _dp, _dp]),
    "prg_normalize": (None, [_vp]),
    "prg_check_idempotency": (None, [_vp, _d, _dp]),
}

_lib = None


def lib():
    """Load libsp2b.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"sp2b CUDA library not built: {LIB_PATH} is missing "
                               "(run __graft_entry__.build())")
        L = C.CDLL(LIB_PATH, mode=C.RTLD_GLOBAL)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS.keys())


def last_error() -> str:
    m = lib().sp2b_last_error()
    return m.decode() if m else ""


def check(status: int, where: str):
    if status != SP2B_OK:
        raise SP2Error(status, where, last_error())


def make_opts(precision=PREC_FP64, mcweeny=1, mixed_tol=1e-3, device_ptrs=False, stream=None,
              mcweeny_products=MCW_INT8, refine_tol=None, exact_switch=None):
    o = Opts()
    lib().sp2b_opts_default(C.byref(o))
    if refine_tol is not None:
        o.refine_tol = refine_tol
    if exact_switch is not None:
        o.exact_switch = exact_switch
    o.precision = precision
    o.mcweeny = mcweeny
    o.mcweeny_products = mcweeny_products
    o.mixed_tol = mixed_tol
    o.device_ptrs = 1 if device_ptrs else 0
    o.stream = stream
    return o
