"""ctypes binding of libmotionest.so (the C ABI declared in include/motionest.h).

The library is the product's compute path.  If it cannot be loaded the package raises at the
first call: there is no CPU fallback.
"""
import ctypes
import os
from pathlib import Path

import torch

_PKG = Path(__file__).resolve().parent
_LIB_PATH = _PKG / "libmotionest.so"

ME_OK = 0
ME_JAC_REFERENCE = 0
ME_JAC_EXACT = 1
ME_GA_REFERENCE = 0
ME_GA_INTENDED = 1

c_i64 = ctypes.c_longlong
c_ptr = ctypes.c_void_p


class MeLayout(ctypes.Structure):
    _fields_ = [("sx", c_i64), ("sy", c_i64), ("sz", c_i64)]


class MeRigidJob(ctypes.Structure):
    _fields_ = [("in_", c_ptr), ("in_vol_stride", c_i64), ("out", c_ptr),
                ("out_vol_stride", c_i64), ("nvol", ctypes.c_int), ("lay", MeLayout),
                ("grid", c_ptr), ("params", c_ptr), ("pstride", ctypes.c_int)]


class MeGrid(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("k", c_ptr * 3), ("tan_rk", c_ptr * 3), ("sin_rk", c_ptr * 3),
        ("tan_st", (c_i64 * 3) * 3), ("sin_st", (c_i64 * 3) * 3),
        ("tan_r", c_ptr * 3), ("sin_r", c_ptr * 3), ("k_uniform", ctypes.c_int * 3),
    ]


class MeSamples(ctypes.Structure):
    _fields_ = [
        ("nshots", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("max_per_shot", ctypes.c_int),
        ("shot_off", c_ptr), ("kx", c_ptr), ("ky", c_ptr), ("ky_off", c_ptr),
        ("ky_order", c_ptr),
    ]


class MeSense(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("ncoils", ctypes.c_int), ("nshots", ctypes.c_int),
        ("mps", c_ptr), ("samples", MeSamples), ("ydat", c_ptr), ("P", c_ptr), ("M", c_ptr),
        ("grid", c_ptr), ("transforms", c_ptr),
    ]


class MotionEstError(RuntimeError):
    pass


_lib = None

# name -> (restype, argtypes)
_SIGS = {
    "me_last_error": (ctypes.c_char_p, []),
    "me_abi_version": (ctypes.c_int, []),
    "me_launch_count": (c_i64, []),
    "me_fft_axis": (ctypes.c_int, [c_ptr, c_i64, c_ptr, c_i64, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, MeLayout, ctypes.c_int,
                                   ctypes.c_int, c_ptr]),
    "me_rigid_apply": (ctypes.c_int, [c_ptr, c_i64, c_ptr, c_i64, ctypes.c_int, MeLayout,
                                      ctypes.POINTER(MeGrid), c_ptr, ctypes.c_int, ctypes.c_int,
                                      c_ptr]),
    "me_rigid_apply_multi": (ctypes.c_int, [ctypes.POINTER(MeRigidJob), ctypes.c_int, c_ptr]),
    "me_rigid_adjoint": (ctypes.c_int, [c_ptr, c_i64, c_ptr, c_i64, ctypes.c_int, MeLayout,
                                        ctypes.POINTER(MeGrid), c_ptr, ctypes.c_int,
                                        ctypes.c_int, c_ptr]),
    "me_rigid_jacobian_workspace_bytes": (c_i64, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "me_rigid_derivative": (ctypes.c_int, [c_ptr, c_ptr, MeLayout, ctypes.POINTER(MeGrid), c_ptr,
                                           ctypes.c_int, ctypes.c_int, c_ptr, c_ptr]),
    "me_rigid_jacobian": (ctypes.c_int, [c_ptr, c_ptr, c_i64, MeLayout, ctypes.POINTER(MeGrid),
                                         c_ptr, ctypes.c_int, c_ptr, c_ptr]),
    "me_sense_workspace_bytes": (c_i64, [ctypes.POINTER(MeSense), ctypes.c_int]),
    "me_lm_workspace_bytes": (c_i64, [ctypes.POINTER(MeSense), ctypes.c_int]),
    "me_sense_precond": (ctypes.c_int, [c_ptr, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, c_ptr, c_ptr, c_ptr]),
    "me_sense_gather": (ctypes.c_int, [ctypes.POINTER(MeSense), c_ptr, c_ptr, c_ptr]),
    "me_sense_normal": (ctypes.c_int, [ctypes.POINTER(MeSense), c_ptr, c_ptr, ctypes.c_int,
                                       c_ptr, c_ptr]),
    "me_sense_rhs": (ctypes.c_int, [ctypes.POINTER(MeSense), c_ptr, ctypes.c_int, c_ptr, c_ptr]),
    "me_sense_residual": (ctypes.c_int, [ctypes.POINTER(MeSense), c_ptr, c_ptr, c_ptr,
                                         ctypes.c_int, c_ptr, c_ptr]),
    "me_sense_residual_norms": (ctypes.c_int, [ctypes.POINTER(MeSense), c_ptr, c_ptr, c_ptr,
                                               ctypes.c_int, c_ptr, c_ptr]),
    "me_sense_forward": (ctypes.c_int, [ctypes.POINTER(MeSense), c_ptr, c_ptr, c_ptr,
                                        ctypes.c_int, c_ptr, c_ptr]),
    "me_sense_forward_volumes": (ctypes.c_int, [ctypes.POINTER(MeSense), c_ptr, c_i64,
                                                ctypes.c_int, ctypes.c_int, c_ptr, c_ptr]),
    "me_sense_adjoint_volumes": (ctypes.c_int, [ctypes.POINTER(MeSense), c_ptr, ctypes.c_int,
                                                ctypes.c_int, c_ptr, c_i64, c_ptr]),
    "me_sense_scatter": (ctypes.c_int, [ctypes.POINTER(MeSense), c_ptr, c_ptr, c_ptr]),
    "me_lm_normal_equations": (ctypes.c_int, [ctypes.POINTER(MeSense), c_ptr, ctypes.c_int,
                                              c_ptr, ctypes.c_int, c_ptr, c_ptr]),
    "me_lm_gradient_workspace_bytes": (c_i64, [ctypes.POINTER(MeSense), ctypes.c_int]),
    "me_lm_gradient": (ctypes.c_int, [ctypes.POINTER(MeSense), c_ptr, ctypes.c_int, c_ptr,
                                      ctypes.c_int, c_ptr, c_ptr]),
    "me_lm_ga_workspace_bytes": (c_i64, [ctypes.POINTER(MeSense), ctypes.c_int]),
    "me_lm_ga_rhs": (ctypes.c_int, [ctypes.POINTER(MeSense), c_ptr, ctypes.c_int, ctypes.c_int,
                                    c_ptr, c_ptr, ctypes.c_double, c_ptr, ctypes.c_int, c_ptr,
                                    c_ptr]),
    "me_lm_propose": (ctypes.c_int, [c_ptr, c_ptr, c_ptr, c_ptr, ctypes.c_int, c_ptr]),
    "me_lm_accept": (ctypes.c_int, [c_ptr, c_ptr, c_ptr, c_ptr, c_ptr, c_ptr, ctypes.c_double,
                                    c_ptr, ctypes.c_int, c_ptr]),
    "me_cg_workspace_bytes": (c_i64, [c_i64]),
    "me_cg_init": (ctypes.c_int, [c_ptr, c_ptr, c_ptr, c_ptr, c_ptr, c_ptr, c_i64, c_ptr, c_ptr]),
    "me_cg_pap": (ctypes.c_int, [c_ptr, c_ptr, c_ptr, c_i64, c_ptr, c_ptr]),
    "me_cg_update": (ctypes.c_int, [c_ptr, c_ptr, c_ptr, c_ptr, c_ptr, c_ptr, c_i64, c_ptr,
                                    c_ptr]),
    "me_cg_direction": (ctypes.c_int, [c_ptr, c_ptr, c_ptr, c_ptr, c_i64, c_ptr]),
    "me_cg_graph_create": (ctypes.c_int, [ctypes.POINTER(MeSense), c_ptr, c_ptr, c_ptr, c_ptr,
                                          c_ptr, c_ptr, c_ptr, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_int, c_ptr, c_ptr, c_ptr,
                                          ctypes.POINTER(c_ptr)]),
    "me_cg_graph_launch": (ctypes.c_int, [c_ptr, c_ptr]),
    "me_cg_graph_body_launches": (c_i64, [c_ptr]),
    "me_cg_graph_account": (None, [c_ptr, ctypes.c_int]),
    "me_cg_graph_destroy": (ctypes.c_int, [c_ptr]),
    "me_dot_re": (ctypes.c_int, [c_ptr, c_ptr, c_ptr, c_i64, c_ptr, c_ptr]),
    "me_max_abs": (ctypes.c_int, [c_ptr, c_i64, c_ptr, c_ptr, c_ptr]),
    "me_dot_re_noalloc": (ctypes.c_int, [c_ptr, c_ptr, c_ptr, c_i64, c_ptr]),
    "me_dft_rows_split": (ctypes.c_int, [c_ptr, c_ptr, c_i64, ctypes.c_int, ctypes.c_int, c_ptr]),
    "me_wait_status": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint)]),
    "me_wait_selftest": (ctypes.c_int, [c_i64, c_ptr]),
}

# me_wait_status bits
ME_WAIT_SENSE_FWD = 0x1
ME_WAIT_SENSE_ADJ = 0x2
ME_WAIT_LINE_PASS = 0x4
ME_WAIT_SELFTEST = 0x100


def lib_path():
    return _LIB_PATH


def load(path=None):
    """Load the shared library (once) and bind every declared entry point."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else _LIB_PATH
    if not p.exists():
        raise MotionEstError(
            f"{p} is missing: build it with `python -m motionest.build` (nvcc, sm_100a). "
            "motionest has no CPU fallback.")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def declared_symbols():
    return list(_SIGS)


def check(rc):
    if rc != ME_OK:
        msg = load().me_last_error().decode(errors="replace")
        if rc == 1:
            raise ValueError(msg)
        raise MotionEstError(f"motionest error {rc}: {msg}")


def wait_status():
    """Synchronise the device and return (and clear) the bits of the kernels' bounded
    barrier waits that ran out since the last call (0: none)."""
    v = ctypes.c_uint(0)
    check(load().me_wait_status(ctypes.byref(v)))
    return v.value


def check_waits():
    """Raise MotionEstError if any bounded wait ran out since the last check."""
    bits = wait_status()
    if bits:
        raise MotionEstError(
            f"a kernel's wait for its bulk copies ran out (status 0x{bits:x}); "
            "the results of the launches since the last check are not valid")


def call(name, *args):
    check(getattr(load(), name)(*args))


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def layout_of(t):
    """me_layout of a [..., X, Y, Z] complex tensor (strides of the last three dims)."""
    s = t.stride()
    return MeLayout(s[-3], s[-2], s[-1])


def require_cuda():
    if not torch.cuda.is_available():
        raise MotionEstError("motionest needs a CUDA device; no CPU fallback exists")
    load()
