"""ctypes binding of ``libphs.so`` (the C ABI declared in include/phs.h).

The library is built in-tree by ``pyheartsim_b200.build``.  There is no
fallback: if the library is missing every call raises, so a missing CUDA
extension can never be mistaken for a working one.
"""
import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libphs.so")

PHS_OK = 0
PHS_ERR_BAD_ARG = 1
PHS_ERR_BAD_TABLE = 2
PHS_WARN_NO_CONVERGE = 3
PHS_ERR_NONFINITE = 4
PHS_ERR_OOM = 5
PHS_ERR_TIMEOUT = 6
PHS_ERR_CUDA = 7
PHS_ERR_UNSUPPORTED = 8
PHS_ERR_STATE = 9

PREC_F32 = 32
PREC_F64 = 64
EGM_F64 = 0
EGM_BF16X3 = 1

CFG_VARIANT = 1
CFG_CTAS_PER_SM = 2
CFG_PROFILE = 3
CFG_TEST_TEAM_OVERCOUNT = 4
CFG_AUTO_BALANCE = 5
CFG_WAVE_INSTANCES = 6
CFG_GROUP_SUMS = 7
CFG_COMPACT_NB = 9
PROFILE_SLOTS = ("rhs", "rhs_wait", "arnoldi_a", "arnoldi_a_wait", "arnoldi_c", "arnoldi_c_wait", "update",
                 "check", "check_wait", "copy", "rhs_reaction", "steps", "arnoldi_iters", "team_ctas", "leader", "barriers")

VFLAG_S1 = 1
VFLAG_S2 = 2
VFLAG_TBLOCK = 4

c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_uint8_p = ctypes.POINTER(ctypes.c_uint8)
c_uint16_p = ctypes.POINTER(ctypes.c_uint16)
c_int8_p = ctypes.POINTER(ctypes.c_int8)
c_float_p = ctypes.POINTER(ctypes.c_float)


class InstanceDesc(ctypes.Structure):
    """Mirror of ``phs_instance_desc``."""
    _fields_ = [
        ("n_voxel", ctypes.c_int64),
        ("model", ctypes.c_int32),
        ("restart", ctypes.c_int32),
        ("nb6", c_int32_p),
        ("coef6", c_double_p),
        ("vflags", c_uint8_p),
        ("vparams", c_double_p),
        ("params", ctypes.c_double * 5),
        ("dt", ctypes.c_double),
        ("j_stim", ctypes.c_double),
        ("n_steps", ctypes.c_int64),
        ("stim", c_uint8_p),
        ("tblock_steps", ctypes.c_int64),
        ("sample_stride", ctypes.c_int32),
        ("n_samples", ctypes.c_int32),
        ("save_h", ctypes.c_int32),
        ("full_cycles", ctypes.c_int32),
        ("u0", ctypes.c_double),
        ("h0", ctypes.c_double),
        ("tol", ctypes.c_double),
        ("atol", ctypes.c_double),
        ("maxiter", ctypes.c_int32),
        ("guess", ctypes.c_int32),
        ("cw", c_double_p),
        ("mask6", c_uint8_p),
        ("nb_edge", c_int32_p),
        ("coef_edge", c_double_p),
        ("device_tables", ctypes.c_int32),
        ("_pad", ctypes.c_int32),
    ]


class OperatorTablesArgs(ctypes.Structure):
    """Mirror of ``phs_operator_tables_args`` (device pointers as void*)."""
    _fields_ = [
        ("n_voxel", ctypes.c_int64),
        ("Delta", ctypes.c_double),
        ("P", ctypes.c_void_p),
        ("nb18", ctypes.c_void_p),
        ("node_flag", ctypes.c_void_p),
        ("order", ctypes.c_void_p),
        ("inv", ctypes.c_void_p),
        ("nb6", ctypes.c_void_p),
        ("coef6", ctypes.c_void_p),
        ("cw", ctypes.c_void_p),
        ("mask6", ctypes.c_void_p),
        ("vflags", ctypes.c_void_p),
        ("vparams", ctypes.c_void_p),
        ("nb_edge", ctypes.c_void_p),
        ("coef_edge", ctypes.c_void_p),
        ("s1", ctypes.c_void_p),
        ("n_s1", ctypes.c_int64),
        ("s2", ctypes.c_void_p),
        ("n_s2", ctypes.c_int64),
        ("iso_word", ctypes.c_void_p),
        ("face_cross", ctypes.c_int32),
        ("edge", ctypes.c_int32),
        ("iso", ctypes.c_int32),
        ("_pad", ctypes.c_int32),
        ("stream", ctypes.c_void_p),
    ]


class InstanceInfo(ctypes.Structure):
    """Mirror of ``phs_instance_info``."""
    _fields_ = [
        ("n_voxel", ctypes.c_int64),
        ("step", ctypes.c_int64),
        ("n_steps", ctypes.c_int64),
        ("samples", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("arnoldi_steps", ctypes.c_int64),
        ("solves", ctypes.c_int64),
        ("max_arnoldi", ctypes.c_int32),
        ("nonconverged", ctypes.c_int32),
        ("arnoldi_sq", ctypes.c_int64),
    ]


# name -> (restype, argtypes); every symbol of include/phs.h
SIGNATURES = {
    "phs_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "phs_version": (ctypes.c_int, []),
    "phs_device_query": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "phs_last_error": (ctypes.c_char_p, []),
    "phs_engine_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "phs_engine_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "phs_instance_add": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(InstanceDesc), ctypes.POINTER(ctypes.c_int)]),
    "phs_instance_remove": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "phs_instance_info_get": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(InstanceInfo)]),
    "phs_engine_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]),
    "phs_instance_read_history": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.c_void_p, ctypes.c_void_p]),
    "phs_instance_read_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                               c_int32_p]),
    "phs_instance_device_ptrs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                                ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(c_int32_p)]),
    "phs_engine_launch_count": (ctypes.c_int64, [ctypes.c_void_p]),
    "phs_engine_config": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64]),
    "phs_step_variants": (ctypes.c_int, [ctypes.c_int, c_int32_p, c_int32_p, c_int32_p]),
    "phs_step_variant_vpt": (ctypes.c_int, [ctypes.c_int, ctypes.c_int32, c_int32_p]),
    "phs_step_variant_layout": (ctypes.c_int, [ctypes.c_int, ctypes.c_int32, c_int32_p, c_int32_p]),
    "phs_instance_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]),
    "phs_engine_rebalance": (ctypes.c_int, [ctypes.c_void_p]),
    "phs_instance_table_bytes": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_int32_p]),
    "phs_simulate": (ctypes.c_int, [ctypes.POINTER(InstanceDesc), ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                    c_int32_p, c_int32_p, ctypes.POINTER(InstanceInfo)]),
    "phs_egm_leadfield_f64": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]),
    "phs_egm_contract_f64": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
                                            ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "phs_split_bf16": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                      ctypes.c_void_p]),
    "phs_egm_bf16x3_workspace": (ctypes.c_int64, [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64]),
    "phs_egm_contract_bf16x3": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                               ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "phs_egm_bf16x3_status": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "phs_egm_contract_bf16x3_cfg": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                                   ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                   ctypes.c_void_p]),
    "phs_egm_bf16x3_config_count": (ctypes.c_int, []),
    "phs_egm_contract_f64_noalloc": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
                                                    ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_void_p]),
    "phs_egm_noalloc_capacity": (ctypes.c_int64, []),
    "phs_egm_normalize": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_void_p]),
    "phs_electrogram": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, c_double_p, c_double_p,
                                       c_double_p, c_double_p, c_double_p, c_int32_p, c_int32_p, c_int8_p,
                                       ctypes.c_double, ctypes.c_int, c_double_p]),
    "phs_lattice_neighbors": (ctypes.c_int, [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p]),
    "phs_equation_parts": (ctypes.c_int, [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p]),
    "phs_operator_flags": (ctypes.c_int, [ctypes.c_int64, ctypes.c_void_p, c_int32_p, ctypes.c_void_p]),
    "phs_operator_tables": (ctypes.c_int, [ctypes.POINTER(OperatorTablesArgs)]),
    "phs_electrode_lat": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_void_p]),
    "phs_conduction_velocity": (ctypes.c_int, [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "phs_interpolate_lat": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p]),
    "phs_activation_times": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                            ctypes.c_int, ctypes.c_double, ctypes.c_int32, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_void_p]),
}

_lib = None
_lock = threading.Lock()


class PhsError(RuntimeError):
    """A C-ABI call returned an error status."""

    def __init__(self, status, where):
        self.status = status
        msg = status_string(status)
        detail = ""
        try:
            detail = lib().phs_last_error().decode()
        except Exception:
            pass
        super().__init__(f"{where}: {msg} (status {status}){'; ' + detail if detail else ''}")


def lib():
    """Load libphs.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m pyheartsim_b200.build` "
                                   "(the CUDA path has no fallback)")
            h = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                f = getattr(h, name)
                f.restype = res
                f.argtypes = args
            _lib = h
    return _lib


def status_string(status):
    try:
        return lib().phs_status_string(int(status)).decode()
    except Exception:
        return f"status {status}"


def check(status, where, allow_warn=False, allow_nonfinite=False):
    """Raise PhsError unless ``status`` is OK (or the no-convergence warning /
    a per-instance non-finite retirement when allowed)."""
    if status == PHS_OK or (allow_warn and status == PHS_WARN_NO_CONVERGE):
        return status
    if allow_nonfinite and status == PHS_ERR_NONFINITE:
        return status
    raise PhsError(status, where)


def ptr(a, ctype):
    """ctypes pointer to a C-contiguous numpy array (None -> NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def vptr(a):
    if a is None:
        return None
    if isinstance(a, int):
        return ctypes.c_void_p(a)
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    assert a.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(a.ctypes.data)


def np_dtype(precision):
    return np.float64 if precision == PREC_F64 else np.float32
