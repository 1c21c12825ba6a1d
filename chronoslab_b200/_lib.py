"""ctypes declarations of the C ABI in include/chronos_b200.h.

Loads chronoslab_b200/libchronos_b200.so (built in-tree by
chronoslab_b200.build).  There is no fallback: a missing library raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libchronos_b200.so")

CHRONOS_FP64 = 0
CHRONOS_FP32 = 1

STATUS = {0: "OK", -1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "ENOTSPD", -5: "EBREAKDOWN",
          -6: "EIO", -7: "ENOTSUP"}


class ChronosError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"chronos {STATUS.get(code, code)}: {msg}")
        self.code = code


class chronos_params(C.Structure):
    _fields_ = [
        ("nLevMax", C.c_int), ("maxCoarseSZ", C.c_int),
        ("nthread", C.c_int), ("nupre", C.c_int), ("nupost", C.c_int), ("nstep", C.c_int),
        ("step_size", C.c_int), ("epsilon", C.c_double), ("smoother_method", C.c_char * 32),
        ("ntv", C.c_int), ("tspace_itmax", C.c_int), ("tspace_tol", C.c_double),
        ("tspace_method", C.c_char * 32), ("init_approx", C.c_int),
        ("SoC_type", C.c_char * 16), ("soc_tau", C.c_double), ("nl_agg", C.c_int),
        ("proltype", C.c_char * 16), ("prol_emin", C.c_char * 16), ("prol_np", C.c_int),
        ("itmax_vol", C.c_int), ("tol_vol", C.c_double), ("dist_min", C.c_int),
        ("dist_max", C.c_int), ("maxcond", C.c_double), ("maxrownrm", C.c_double),
        ("eps_prol", C.c_double), ("updateCF", C.c_int),
        ("patt_pow", C.c_int), ("patt_tau", C.c_double), ("nnzr_max", C.c_int),
        ("itmax_emin", C.c_int), ("energ_tol", C.c_double), ("condmax_emin", C.c_double),
        ("prec_emin", C.c_int), ("solv_emin", C.c_int),
        ("filt_np", C.c_int), ("filt_wgt", C.c_double), ("filt_tol", C.c_double),
        ("filt_tau", C.c_double), ("min_patt", C.c_int),
        ("ascii_input", C.c_int), ("rhs_build", C.c_char * 16), ("symmetric", C.c_int),
        ("solv_method", C.c_char * 16), ("itmax", C.c_int), ("tol", C.c_double),
        ("restart", C.c_int),
        ("precision", C.c_int), ("use_graph", C.c_int), ("seed", C.c_uint64),
        ("fsai_fabs", C.c_int), ("use_bsr", C.c_int), ("exact_outer", C.c_int),
        ("replace_ratio", C.c_double), ("spmv_format", C.c_int), ("batch_grouped", C.c_int),
    ]


class chronos_level_info(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz_A", C.c_int64), ("nnz_G", C.c_int64),
                ("nnz_P", C.c_int64), ("nc", C.c_int), ("omega", C.c_double),
                ("lambda_", C.c_double), ("threads_per_row", C.c_int),
                ("block_rows", C.c_int), ("sell_mask", C.c_int)]


class chronos_profile(C.Structure):
    _fields_ = [("vcycle_ms", C.c_double), ("vcycle_bytes", C.c_double),
                ("top_apply_ms", C.c_double), ("top_apply_bytes", C.c_double),
                ("outer_spmv_ms", C.c_double), ("outer_spmv_bytes", C.c_double),
                ("iteration_bytes", C.c_double), ("kernels_per_iteration", C.c_int),
                ("kernels_per_solve", C.c_int)]


class chronos_prolongation(C.Structure):
    _fields_ = [("nc", C.c_int), ("iat_P_h", C.POINTER(C.c_int)),
                ("ja_P_h", C.POINTER(C.c_int)), ("val_P_h", C.POINTER(C.c_double))]


# int (*)(void *ctx, int level, int n, const int *iat, const int *ja, const double *val,
#         chronos_prolongation *P)
PROLONG_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int),
                         C.POINTER(C.c_int), C.POINTER(C.c_double),
                         C.POINTER(chronos_prolongation))

_i = C.c_int
_i64 = C.c_int64
_u64 = C.c_uint64
_d = C.c_double
_pi = C.POINTER(C.c_int)
_pi64 = C.POINTER(C.c_int64)
_pd = C.POINTER(C.c_double)
_vp = C.c_void_p
_pp = C.POINTER(C.c_void_p)

# name -> argtypes (every function returns int unless listed in _RESTYPE)
SIGNATURES = {
    "chronos_params_default": [C.POINTER(chronos_params)],
    "chronos_params_read": [C.c_char_p, C.POINTER(chronos_params)],
    "chronos_last_error": [C.c_char_p, _i],
    "chronos_version": [],
    "chronos_csr_info": [_vp, _pi, _pi, _pi64],
    "chronos_csr_fetch": [_vp, _pi, _pi, _pd],
    "chronos_csr_free": [_vp],
    "chronos_read_matrix_bin": [C.c_char_p, _pp],
    "chronos_read_ext_bin": [C.c_char_p, _pp],
    "chronos_write_ext_bin": [C.c_char_p, _i, _i, _pi, _pi, _pd],
    "chronos_read_tv_ext_bin": [C.c_char_p, _pi, _pi, _pd],
    "chronos_write_tv_ext_bin": [C.c_char_p, _i, _i, _pd],
    "chronos_hier_dump_ext_bin": [_vp, _i, C.c_char, C.c_char_p],
    "chronos_fsai_pattern": [_i, _pi, _pi, _pd, _i, _i, _d, _i, _i, _pi, _pp],
    "chronos_coarsen": [C.POINTER(chronos_params), _i, _pi, _pi, _pd, _u64, _pi, _pi, _pp],
    "chronos_coarsen_device": [C.POINTER(chronos_params), _i, _pi, _pi, _pd, _u64, _pi, _pi,
                               _pp],
    "chronos_bamg": [C.POINTER(chronos_params), _i, _pi, _pi, _pi, _i, _pd, _pi, _pp],
    "chronos_bamg_device": [C.POINTER(chronos_params), _i, _pi, _pi, _pi, _i, _pd, _pi, _i, _pp,
                            _pi],
    "chronos_emin_pattern": [_i, _i, _i, _pi, _pi, _pd, _pi, _pi, _pd, _pi, _i, _i, _pp, _pi],
    "chronos_emin": [C.POINTER(chronos_params), _i, _pi, _pi, _pd, _i, _pi, _pi, _pd, _pi, _pi,
                     _pi, _i, _pd, _i, _pp, _pd],
    "chronos_fsai_compute": [_i, _i, _i, _d, _d, _i, _i, _i64, _pi64, _pi, _pd, _pi64, _pi64,
                             _pi, _pd, _pi],
    "chronos_fsai_numeric": [_i, _i, _pi64, _pi, _pd, _pi64, _pi, _i, _vp, _pi, _vp],
    "chronos_fsai_numeric_noalloc": [_i, _vp, _vp, _vp, _vp, _vp, _vp, _pi, _vp],
    "chronos_fsai_numeric_batch": [_i, _pi, _pp, _pp, _pp, _pp, _pp, _pp, _pi, _i, _pi],
    "chronos_galerkin_compute": [_i, _i, _pi, _pi, _pd, _pi, _pi, _pd, _pi64, _pp],
    "chronos_galerkin_fetch": [_vp, _pi, _pi, _pd],
    "chronos_galerkin_free": [_vp],
    "chronos_dense_chol": [_i, _pd, _pd],
    "chronos_spmv": [_i, _i, _pi, _pi, _pd, _pd, _pd, _i, _i, _i],
    "chronos_amg_setup": [C.POINTER(chronos_params), _i, _pi, _pi, _pd, _i, _pd, _pp],
    "chronos_amg_setup_prolong": [C.POINTER(chronos_params), _i, _pi, _pi, _pd, PROLONG_FN, _vp,
                                  _pp],
    "chronos_hier_free": [_vp],
    "chronos_hier_save": [_vp, C.c_char_p],
    "chronos_device_bytes": [_pi64],
    "chronos_hier_load": [C.c_char_p, _pp],
    "chronos_hier_nlevels": [_vp, _pi],
    "chronos_hier_level_info": [_vp, _i, C.POINTER(chronos_level_info)],
    "chronos_hier_export": [_vp, _i, C.c_char, _pi, _pi, _pi64, _pi, _pi, _pd],
    "chronos_hier_setup_times": [_vp, _pd],
    "chronos_hier_setup_phases": [_vp, _pd, _i],
    "chronos_hier_profile": [_vp, _i, C.POINTER(chronos_profile)],
    "chronos_diag_fix": [_i, _pi, _pi, _pd],
    "chronos_vcycle": [_vp, _pd, _pd, _i, _vp],
    "chronos_vcycle_dev": [_vp, _i, _vp, _vp, _i, _vp],
    "chronos_pcg": [_vp, _pi, _pi, _pd, _pd, _pd, _i, _d, _pi, _pd, _pi, _pd, _vp],
    "chronos_pcg_dev": [_vp, _vp, _vp, _i, _d, _pi, _pd, _pi, _pd, _vp],
    "chronos_pcg_block": [_vp, _i, _pd, _pd, _i, _d, _pi, _pi, _pd, _vp],
    "chronos_batch_setup": [C.POINTER(chronos_params), _i, _pi, _pp, _pp, _pp, _pp],
    "chronos_batch_solve": [_vp, _pp, _pp, _i, _d, _pi, _pi, _pd],
    "chronos_batch_info": [_vp, _i, _pi, _pi],
    "chronos_batch_setup_phases": [_vp, _pd, _i],
    "chronos_batch_setup_wall": [_vp, _pd],
    "chronos_batch_free": [_vp],
    "chronos_sqmr":[_vp, _pi, _pi, _pd, _pd, _pd, _i, _d, _pi, _pd, _pi],
    "chronos_gmres": [_vp, _pi, _pi, _pd, _pd, _pd, _i, _d, _i, _pi, _pi, _pd, _pi, _pd, _pi],
    "chronos_adjoint_grad": [_vp, _pd, _pd, _i, _d, _pd, _pd, _pi],
}
_RESTYPE = {"chronos_params_default": None, "chronos_version": C.c_char_p}

_lib = None


def load():
    """Loads the library once and declares every signature."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m chronoslab_b200.build` "
                "(or __graft_entry__.build()); there is no CPU fallback")
        lib = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, C.c_int)
        _lib = lib
    return _lib


def last_error():
    buf = C.create_string_buffer(4096)
    load().chronos_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def check(code):
    if code != 0:
        raise ChronosError(code, last_error())
    return code
