"""ctypes binding of libsigk.so (the C ABI declared in include/sigk.h).

The shared library is built in-tree by ``python -m sigpde_b200.build`` (or
``__graft_entry__.build()``).  There is no fallback: if the library is
missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsigk.so")

SIGK_OK = 0
SIGK_EINVAL = 1
SIGK_ENOMEM = 2
SIGK_ETIMEDOUT = 3
SIGK_ELAUNCH = 4
SIGK_EUNSUPPORTED = 5
_STATUS_NAMES = {0: "SIGK_OK", 1: "SIGK_EINVAL", 2: "SIGK_ENOMEM", 3: "SIGK_ETIMEDOUT", 4: "SIGK_ELAUNCH",
                 5: "SIGK_EUNSUPPORTED"}

SIGK_F32 = 0
SIGK_F64 = 1
SIGK_PREC_FP64 = 0
SIGK_PREC_FP32 = 1
SIGK_PREC_TC32 = 2
SIGK_PREC_TC64 = 3
SIGK_OP_PAIRWISE = 0
SIGK_OP_GRAM = 1
SIGK_OP_GRAM_SYM = 2
SIGK_OP_NORMALIZE = 3
SIGK_STATIC_LINEAR = 0
SIGK_STATIC_RBF = 1
SIGK_STATIC_L1RBF = 2

# Exported symbol -> (restype, argtypes).  Kept in the order of include/sigk.h.
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int
_dbl = ctypes.c_double
_sz = ctypes.c_size_t

class RaggedTcPlan(ctypes.Structure):
    """sigk_ragged_tc_plan (include/sigk.h)."""
    _fields_ = [("a_row0", ctypes.c_void_p), ("b_row0", ctypes.c_void_p), ("a_rows", ctypes.c_int64),
                ("b_rows", ctypes.c_int64), ("inc_off", ctypes.c_void_p), ("inc_elems", ctypes.c_int64),
                ("tiles", ctypes.c_void_p), ("ntiles", ctypes.c_int64), ("tile_n", ctypes.c_int64)]


_plan_p = ctypes.POINTER(RaggedTcPlan)

SIGNATURES = {
    "sigk_version": (ctypes.c_char_p, []),
    "sigk_last_error_string": (ctypes.c_char_p, []),
    "sigk_launch_count": (ctypes.c_uint64, []),
    "sigk_set_wait_limit": (_i64, [_i64]),
    "sigk_workspace_size": (_sz, [_int, _i64, _i64, _i64, _i64, _i64, _int, _int, _int]),
    "sigk_pairwise": (_int, [_vp, _vp, _i64, _i64, _i64, _i64, _int, _int, _dbl, _vp, _vp, _vp, _int, _vp, _sz,
                             _vp]),
    "sigk_gram": (_int, [_vp, _vp, _i64, _i64, _i64, _i64, _i64, _int, _int, _dbl, _vp, _vp, _vp, _int, _vp, _sz,
                         _vp]),
    "sigk_gram_sym": (_int, [_vp, _i64, _i64, _i64, _int, _int, _dbl, _vp, _vp, _int, _vp, _sz, _vp]),
    "sigk_static_workspace_size": (_sz, [_int, _int, _i64, _i64, _i64, _i64, _i64, _int, _int, _int]),
    "sigk_gram_static": (_int, [_int, _int, _dbl, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _int, _int, _vp, _vp, _vp,
                                _int, _vp, _sz, _vp]),
    "sigk_backward_workspace_size": (_sz, [_int, _i64, _i64, _i64, _i64, _i64, _int, _int]),
    "sigk_backward": (_int, [_int, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _int, _int, _dbl, _vp, _vp, _vp, _vp, _vp,
                             _vp, _sz, _vp]),
    "sigk_backward_inc_workspace_size": (_sz, [_i64, _i64, _i64, _int]),
    "sigk_backward_inc": (_int, [_vp, _i64, _i64, _i64, _i64, _i64, _i64, _int, _int, _vp, _vp, _vp, _vp, _i64, _i64,
                                 _i64, _vp, _sz, _vp]),
    "sigk_self_norms": (_int, [_vp, _i64, _i64, _i64, _int, _int, _dbl, _vp, _vp, _sz, _vp]),
    "sigk_normalize": (_int, [_vp, _i64, _i64, _i64, _int, _int, _dbl, _vp, _vp, _dbl, _int, _vp, _vp, _vp, _sz,
                              _vp]),
    "sigk_pairwise_inc": (_int, [_vp, _i64, _i64, _i64, _i64, _i64, _i64, _int, _int, _vp, _vp, _vp, _int, _vp, _sz,
                                 _vp]),
    "sigk_gram_inc": (_int, [_vp, _i64, _i64, _i64, _i64, _i64, _i64, _i64, _i64, _int, _int, _vp, _vp, _int, _vp,
                             _i64, _int, _vp, _sz, _vp]),
    "sigk_normalize_inc": (_int, [_vp, _i64, _i64, _i64, _i64, _i64, _int, _int, _vp, _vp, _dbl, _int, _vp, _vp, _vp,
                                  _sz, _vp]),
    "sigk_ragged_workspace_size": (_sz, [_i64, _i64, _i64, _i64, _i64, _i64, _int]),
    "sigk_pairwise_ragged": (_int, [_vp, _vp, _vp, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _i64,
                                    _i64, _i64, _int, _dbl, _vp, _vp, _vp, _int, _vp, _sz, _vp]),
    "sigk_ragged_tc_workspace_size": (_sz, [_i64, _i64, _i64, _i64, _int, _plan_p]),
    "sigk_pairwise_ragged_tc": (_int, [_vp, _vp, _vp, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _vp,
                                       _i64, _i64, _i64, _int, _dbl, _vp, _vp, _vp, _int, _plan_p, _vp, _sz, _vp]),
    "sigk_ragged_status": (_int, [_vp, _vp]),
    "sigk_gram_noalloc": (_int, [_vp, _vp, _i64, _i64, _i64, _i64, _i64, _int, _int, _dbl, _vp, _vp, _vp, _int, _vp]),
}

_lib = None
_lock = threading.Lock()


class SigkError(RuntimeError):
    """A libsigk entry point returned a non-zero status."""

    def __init__(self, status: int, func: str, message: str):
        super().__init__(f"{func} failed with {_STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def lib() -> ctypes.CDLL:
    """Load libsigk.so once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"libsigk.so is missing at {LIB_PATH}; build it with `python -m sigpde_b200.build` "
                    "(this package has no CPU fallback)")
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def last_error() -> str:
    return lib().sigk_last_error_string().decode()


def call(name: str, *args) -> None:
    """Call an entry point and raise SigkError on a non-zero status."""
    st = getattr(lib(), name)(*args)
    if st != SIGK_OK:
        raise SigkError(st, name, last_error())


def version() -> str:
    return lib().sigk_version().decode()


def launch_count() -> int:
    """Kernels enqueued by libsigk.so since it was loaded (all threads)."""
    return int(lib().sigk_launch_count())


def set_wait_limit(polls: int) -> int:
    """Polls an uneven-batch band wait makes before it gives up (< 0: the default,
    ~4 s); returns the previous setting.  See sigk_set_wait_limit in sigk.h."""
    return int(lib().sigk_set_wait_limit(int(polls)))
