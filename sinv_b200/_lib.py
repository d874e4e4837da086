"""ctypes binding of ``libsinvb.so`` (declarations in ``include/sinvb.h``).

The library is loaded lazily on first use.  There is no fallback: when the
shared object is missing, fails to load, or no sm_100 GPU is present, every
entry point raises :class:`SinvbUnavailable`.
"""

import ctypes
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsinvb.so")

OK = 0
EINVAL = -1
ECUDA = -2
EWORKSPACE = -3
EUNSUPPORTED = -4
STATUS_PIVOT = 1
STATUS_TIMEOUT = 2

SYM = 1
SAVE_OFFDIAG = 2
FORCE_GRID = 4
FORCE_CTA = 8
INPLACE = 16

C128, F64, C64, F32 = 0, 1, 2, 3

# Every symbol include/sinvb.h declares, with (restype, argtypes).
_vp = ctypes.c_void_p
_i = ctypes.c_int
_u = ctypes.c_uint
_sz = ctypes.c_size_t
_RGF_ARGS = [_vp, _vp, _vp, _i, _i, _u, _vp, _vp, _vp, _vp, _sz, _vp]
SIGNATURES = {
    "sinvb_version": (_i, []),
    "sinvb_status_string": (ctypes.c_char_p, [_i]),
    "sinvb_rgf_workspace_size": (_sz, [_i, _i, _i, _u]),
    "sinvb_rgf_z": (_i, _RGF_ARGS),
    "sinvb_rgf_d": (_i, _RGF_ARGS),
    "sinvb_rgf_c": (_i, _RGF_ARGS),
    "sinvb_rgf_s": (_i, _RGF_ARGS),
    "sinvb_workspace_status": (_i, [_vp, _vp, ctypes.POINTER(_i)]),
    "sinvb_rgf_batched_workspace_size": (_sz, [_vp, _i, _i, _u]),
    "sinvb_rgf2s_workspace_size": (_sz, [_i, _i, _i, _u]),
    "sinvb_rgf2s_z": (_i, [_vp, _vp, _vp, _i, _i, _u, _vp, _vp, _vp, _vp, _sz, _vp]),
    "sinvb_rgf2s_d": (_i, [_vp, _vp, _vp, _i, _i, _u, _vp, _vp, _vp, _vp, _sz, _vp]),
    "sinvb_rgf_lesser_workspace_size": (_sz, [_i, _i]),
    "sinvb_rgf_lesser_z": (_i, [_vp, _vp, _vp, _vp, _i, _i, _u, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "sinvb_rgf_lesser_batched_workspace_size": (_sz, [_vp, _i, _u]),
    "sinvb_rgf_lesser_batched_z": (_i, [_vp, _i, _u, _vp, _sz, _vp, _vp]),
    "sinvb_rgf_batched_z": (_i, [_vp, _i, _u, _vp, _sz, _vp, _vp]),
    "sinvb_rgf_batched_d": (_i, [_vp, _i, _u, _vp, _sz, _vp, _vp]),
    "sinvb_rgf_batched_stream_z": (_i, [_vp, _i, _u, _vp, _sz, _vp, _vp, _vp, _u, _vp]),
    "sinvb_rgf_batched_stream_d": (_i, [_vp, _i, _u, _vp, _sz, _vp, _vp, _vp, _u, _vp]),
    "sinvb_rgf_batched_stream_sched_z": (_i, [_vp, _i, _u, _vp, _vp, _sz, _vp, _vp, _vp, _u, _vp]),
    "sinvb_rgf_batched_stream_sched_d": (_i, [_vp, _i, _u, _vp, _vp, _sz, _vp, _vp, _vp, _u, _vp]),
    "sinvb_rgf_batched_rerun_z": (_i, [_vp, _vp]),
    "sinvb_rgf_batched_rerun_d": (_i, [_vp, _vp]),
    "sinvb_rgf_batched_set_wait_limit": (_i, [_vp, ctypes.c_double]),
    "sinvb_rgf_batched_sched_workspace_size": (_sz, [_vp, _i, _i, _u, _vp]),
    "sinvb_rgf_batched_sched_z": (_i, [_vp, _i, _u, _vp, _vp, _sz, _vp, _vp]),
    "sinvb_rgf_batched_sched_d": (_i, [_vp, _i, _u, _vp, _vp, _sz, _vp, _vp]),
    "sinvb_rgf_batched_ckpt_z": (_i, [_vp, _i, _u, _vp, _vp, _sz, _vp, _vp]),
    "sinvb_rgf_batched_ckpt_d": (_i, [_vp, _i, _u, _vp, _vp, _sz, _vp, _vp]),
    "sinvb_rgf_adjoint_batched_workspace_size": (_sz, [_vp, _i, _i, _u]),
    "sinvb_rgf_adjoint_batched_z": (_i, [_vp, _i, _u, _vp, _sz, _vp, _vp]),
    "sinvb_rgf_adjoint_batched_d": (_i, [_vp, _i, _u, _vp, _sz, _vp, _vp]),
    "sinvb_rgf_z_noalloc": (_i, [_vp, _vp, _vp, _i, _i, _u, _vp, _vp, _vp, _vp, _vp]),
    "sinvb_rgf_checkpoints": (_i, [_i, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "sinvb_rgf_forward_ckpt_z": (_i, [_vp, _vp, _vp, _i, _i, _u, _vp, _vp, _vp, _vp, _i, _vp, _sz, _vp]),
    "sinvb_rgf_forward_ckpt_d": (_i, [_vp, _vp, _vp, _i, _i, _u, _vp, _vp, _vp, _vp, _i, _vp, _sz, _vp]),
    "sinvb_rgf_adjoint_workspace_size": (_sz, [_i, _i, _i, _u]),
    "sinvb_rgf_adjoint_z": (_i, [_vp] * 10 + [_i, _i, _i, _u, _vp, _vp, _vp, _vp, _sz, _vp]),
    "sinvb_rgf_adjoint_d": (_i, [_vp] * 10 + [_i, _i, _i, _u, _vp, _vp, _vp, _vp, _sz, _vp]),
    "sinvb_fp64_mma_peak": (_i, [_i, ctypes.POINTER(ctypes.c_double), _vp]),
    "sinvb_zgemm_ozaki_workspace_size": (_sz, [_i, _i, _i, _i]),
    "sinvb_zgemm_ozaki": (_i, [_i, _i, _i, ctypes.c_double, _vp, _i, _vp, _i, ctypes.c_double, _vp, _i, _vp, _i,
                               _i, _vp, _sz, _vp]),
    "sinvb_bcr_workspace_size": (_sz, [_i, _i, _i, _u]),
    "sinvb_bcr_z": (_i, _RGF_ARGS),
    "sinvb_bcr_d": (_i, _RGF_ARGS),
    "sinvb_psr_partitions": (_i, [_i, _i]),
    "sinvb_psr_workspace_size": (_sz, [_i, _i, _i, _i, _u]),
    "sinvb_psr_z": (_i, [_vp, _vp, _vp, _i, _i, _i, _u, _vp, _vp, _vp, _vp, _sz, _vp]),
    "sinvb_psr_d": (_i, [_vp, _vp, _vp, _i, _i, _i, _u, _vp, _vp, _vp, _vp, _sz, _vp]),
    "sinvb_pdiv_workspace_size": (_sz, [_i, _i, _i, _i, _u]),
    "sinvb_pdiv_z": (_i, [_vp, _vp, _vp, _i, _i, _i, _u, _vp, _vp, _vp, _vp, _sz, _vp]),
    "sinvb_pdiv_d": (_i, [_vp, _vp, _vp, _i, _i, _i, _u, _vp, _vp, _vp, _vp, _sz, _vp]),
    "sinvb_psr_part_workspace_size": (_sz, [_i, _i, _i, _i, _i]),
    "sinvb_psr_part_z": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "sinvb_psr_part_d": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "sinvb_bcr_batched_workspace_size": (_sz, [_vp, _i, _i, _u]),
    "sinvb_bcr_batched_z": (_i, [_vp, _i, _u, _vp, _sz, _vp, _vp]),
    "sinvb_bcr_batched_d": (_i, [_vp, _i, _u, _vp, _sz, _vp, _vp]),
    "sinvb_bcr_batched_rerun_z": (_i, [_vp, _i, _vp, _vp]),
    "sinvb_bcr_batched_rerun_d": (_i, [_vp, _i, _vp, _vp]),
}

PREC_FP64 = 0
PREC_MIXED = 1 << 8
PREC_DIGITS_SHIFT = 12  # Ozaki digits of the mixed products in flag bits 12-15 (0: 7)


class BatchDesc(ctypes.Structure):
    """``sinvb_batch_desc`` of include/sinvb.h."""
    _fields_ = [("diag", _vp), ("upper", _vp), ("lower", _vp), ("G_diag", _vp), ("G_upper", _vp),
                ("G_lower", _vp), ("n", _i), ("b", _i)]


class AdjointDesc(ctypes.Structure):
    """``sinvb_adjoint_desc`` of include/sinvb.h."""
    _fields_ = [(name, _vp) for name in ("diag", "upper", "lower", "G_diag", "G_upper", "G_lower", "bG_diag",
                                         "bG_upper", "bG_lower", "checkpoints", "aD", "aU", "aL")] + \
        [("n", _i), ("b", _i)]


class LesserDesc(ctypes.Structure):
    """``sinvb_lesser_desc`` of include/sinvb.h."""
    _fields_ = [(name, _vp) for name in ("diag", "upper", "lower", "sigma_lesser", "G_diag", "G_upper", "G_lower",
                                         "GL_diag", "GL_upper")] + [("n", _i), ("b", _i)]


class BatchSchedule(ctypes.Structure):
    """``sinvb_batch_schedule`` of include/sinvb.h."""
    _fields_ = [("team", _vp), ("priority", _vp), ("mixed_min_b", _i), ("reserved", _i)]


class SinvbUnavailable(RuntimeError):
    """The CUDA library cannot run here (not built, no B200, no CUDA)."""


class SinvbError(RuntimeError):
    """A library entry point returned an error code."""

    def __init__(self, code, where=""):
        self.code = code
        super().__init__("%s: %s (code %d)" % (where or "libsinvb", status_string(code), code))


_lock = threading.Lock()
_lib = None


def load(path=LIB_PATH):
    """Load the shared library and bind every declared symbol (no GPU needed)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise SinvbUnavailable("libsinvb.so not built: run `python -m sinv_b200.build` (%s)" % path)
        try:
            lib = ctypes.CDLL(path)
        except OSError as e:
            raise SinvbUnavailable("cannot load %s: %s" % (path, e)) from e
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def status_string(code):
    try:
        return load().sinvb_status_string(int(code)).decode()
    except SinvbUnavailable:
        return "code %d" % code


def check(code, where=""):
    if code != OK:
        raise SinvbError(code, where)


def dtype_code(dtype):
    """Map a numpy / torch dtype to the library's element-type code."""
    name = str(dtype).replace("torch.", "")
    table = {"complex128": C128, "float64": F64, "complex64": C64, "float32": F32}
    if name not in table:
        raise TypeError("unsupported dtype %s (complex128, float64, complex64, float32)" % name)
    return table[name]


def np_dtype(code):
    return {C128: np.complex128, F64: np.float64, C64: np.complex64, F32: np.float32}[code]
