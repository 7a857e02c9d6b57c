"""ctypes binding of libqfb.so (include/qfb.h).

The library is the only compute path: if it is missing, or no CUDA device
is usable when a state is created, the calls raise -- there is no CPU
fallback.  Status codes map onto the reference's exception types:
QFB_EINVAL -> ValueError (std::invalid_argument), anything else ->
RuntimeError (std::runtime_error).
"""

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libqfb.so")

QFB_OK, QFB_EINVAL, QFB_ENOMEM, QFB_EDEVICE, QFB_ETIMEDOUT, QFB_ENOSYS = 0, 22, 12, 5, 110, 38

GATE_DTYPE = np.dtype([("target", "<i4"), ("control", "<i4"), ("mat", "<c16", (4, 4))])
PAULI_DTYPE = np.dtype([("x", "<u8"), ("z", "<u8")])
assert GATE_DTYPE.itemsize == 264 and PAULI_DTYPE.itemsize == 16

class QfbComplex(ctypes.Structure):
    _fields_ = [("re", ctypes.c_double), ("im", ctypes.c_double)]


def cplx(z):
    z = complex(z)
    return QfbComplex(z.real, z.imag)


c_state = ctypes.c_void_p
c_sum = ctypes.c_void_p
c_prog = ctypes.c_void_p
_vp = ctypes.c_void_p
_i32, _i64, _u64, _dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double

# name -> (restype, argtypes); every entry point of include/qfb.h
SIGNATURES = {
    "qfb_version": (ctypes.c_int, []),
    "qfb_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    "qfb_set_stream": (ctypes.c_int, [_vp]),
    "qfb_sync": (ctypes.c_int, []),
    "qfb_launch_count": (ctypes.c_int, [_vp]),
    "qfb_set_tile_wait_limit": (ctypes.c_int, [_u64]),
    "qfb_gates_dense": (ctypes.c_int, [ctypes.c_int]),
    "qfb_ucc_sets_per_cta": (ctypes.c_int, [_vp, _vp]),
    "qfb_c64_create": (ctypes.c_int, [ctypes.c_int, _vp]),
    "qfb_c64_destroy": (ctypes.c_int, [_vp]),
    "qfb_c64_reset": (ctypes.c_int, [_vp]),
    "qfb_c64_upload": (ctypes.c_int, [_vp, _vp, _u64]),
    "qfb_c64_download": (ctypes.c_int, [_vp, _vp, _u64]),
    "qfb_c64_apply_gates": (ctypes.c_int, [_vp, _vp, _i64]),
    "qfb_c64_norm2": (ctypes.c_int, [_vp, _vp]),
    "qfb_pack_create": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp]),
    "qfb_pack_destroy": (ctypes.c_int, [_vp]),
    "qfb_pack_info": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "qfb_pack_buffers": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "qfb_pack_launch": (ctypes.c_int, [_vp, ctypes.c_int]),
    "qfb_pack_run": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp]),
    "qfb_state_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp]),
    "qfb_state_destroy": (ctypes.c_int, [c_state]),
    "qfb_state_info": (ctypes.c_int, [c_state, _vp, _vp]),
    "qfb_state_device_ptr": (ctypes.c_void_p, [c_state]),
    "qfb_state_copy": (ctypes.c_int, [c_state, c_state]),
    "qfb_state_copy_slot": (ctypes.c_int, [c_state, ctypes.c_int, c_state, ctypes.c_int]),
    "qfb_state_reset": (ctypes.c_int, [c_state]),
    "qfb_state_null": (ctypes.c_int, [c_state]),
    "qfb_state_set_basis": (ctypes.c_int, [c_state, ctypes.c_int, _vp, _vp, _i64]),
    "qfb_state_upload": (ctypes.c_int, [c_state, ctypes.c_int, _vp, _u64]),
    "qfb_state_download": (ctypes.c_int, [c_state, ctypes.c_int, _vp, _u64]),
    "qfb_state_sample": (ctypes.c_int, [c_state, ctypes.c_int, _u64, _i64, _vp]),
    "qfb_state_get_amp": (ctypes.c_int, [c_state, ctypes.c_int, _u64, _vp]),
    "qfb_apply_gates": (ctypes.c_int, [c_state, _vp, _i64]),
    "qfb_gates_config": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "qfb_gates_plan": (ctypes.c_int, [_vp, _i64, ctypes.c_int, _vp, _vp, _vp]),
    "qfb_gates_phases": (ctypes.c_int, [_vp, _i64, ctypes.c_int, _vp, _vp]),
    "qfb_gates_regs": (ctypes.c_int, [ctypes.c_int]),
    "qfb_gates_fused": (ctypes.c_int, [ctypes.c_int]),
    "qfb_gates_fused_plan": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "qfb_scale": (ctypes.c_int, [c_state, QfbComplex]),
    "qfb_vdot": (ctypes.c_int, [c_state, c_state, _vp]),
    "qfb_axpy": (ctypes.c_int, [c_state, QfbComplex, c_state]),
    "qfb_sum_create": (ctypes.c_int, [_vp, _vp, _vp, _i64, _i32, _vp]),
    "qfb_sum_destroy": (ctypes.c_int, [c_sum]),
    "qfb_sum_info": (ctypes.c_int, [c_sum, _vp, _vp, _vp]),
    "qfb_sum_expval": (ctypes.c_int, [c_sum, c_state, c_state, _vp]),
    "qfb_sum_apply": (ctypes.c_int, [c_sum, c_state, c_state]),
    "qfb_sum_expval_noalloc": (ctypes.c_int, [c_sum, c_state, c_state, _vp]),
    "qfb_prog_create": (ctypes.c_int, [_vp, _vp, _vp, _i64, _i32, _vp]),
    "qfb_prog_destroy": (ctypes.c_int, [c_prog]),
    "qfb_prog_info": (ctypes.c_int, [c_prog, _vp, _vp, _vp]),
    "qfb_prog_apply": (ctypes.c_int, [c_prog, c_state, _vp, _i32, _i32]),
    "qfb_ucc_gradient": (ctypes.c_int, [c_prog, c_prog, c_state, c_state, _vp, _i32, _vp]),
    "qfb_ucc_create": (ctypes.c_int, [c_prog, c_prog, c_prog, c_sum, ctypes.c_int, _u64,
                                      ctypes.c_int, _vp]),
    "qfb_ucc_destroy": (ctypes.c_int, [_vp]),
    "qfb_ucc_sector": (ctypes.c_int, [_vp, _vp]),
    "qfb_ucc_memory": (ctypes.c_int, [_vp, _vp]),
    "qfb_ucc_set_pool": (ctypes.c_int, [_vp, c_prog]),
    "qfb_ucc_set_residuals": (ctypes.c_int, [_vp, _vp, _vp, _i32]),
    "qfb_ucc_residual_buffer": (ctypes.c_int, [_vp, _vp]),
    "qfb_ucc_eval_residuals": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "qfb_ucc_pool_buffer": (ctypes.c_int, [_vp, _vp]),
    "qfb_ucc_eval_pool": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "qfb_ucc_path": (ctypes.c_int, [_vp, _vp]),
    "qfb_ucc_real_states": (ctypes.c_int, [_vp, _vp]),
    "qfb_ucc_rows": (ctypes.c_int, [_vp, _vp]),
    "qfb_ucc_config": (ctypes.c_int, [ctypes.c_int]),
    "qfb_ucc_tiles": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "qfb_ucc_buffers": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "qfb_ucc_run": (ctypes.c_int, [_vp, ctypes.c_int]),
    "qfb_ucc_capture": (ctypes.c_int, [_vp, ctypes.c_int]),
    "qfb_ucc_eval": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "qfb_ucc_profile": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp]),
}

_lib = None
_lock = threading.Lock()


def _ensure_built():
    if os.path.exists(LIB_PATH):
        return
    # building is part of installing the product; no other path exists
    from . import build as _build
    _build.build()


def lib():
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            _ensure_built()
            if not os.path.exists(LIB_PATH):
                raise ImportError(f"libqfb.so not found at {LIB_PATH}; run "
                                  "`python -m qforte_b200.build`")
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib


def last_error():
    buf = ctypes.create_string_buffer(1024)
    lib().qfb_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc, what=""):
    if rc == QFB_OK:
        return
    msg = last_error()
    if rc == QFB_EINVAL:
        raise ValueError(msg)
    raise RuntimeError(f"{what}: [qfb status {rc}] {msg}" if what else f"[qfb status {rc}] {msg}")


def ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def launch_count():
    v = ctypes.c_uint64(0)
    check(lib().qfb_launch_count(ctypes.byref(v)))
    return v.value


def loaded_path():
    """Path of the loaded library (evidence of the native path)."""
    lib()
    return LIB_PATH
