"""ctypes binding of ``libel_b200.so`` (the C ABI in include/energy_level_b200.h).

The library is the only compute path: when it is missing or CUDA is not
available every entry point raises; there is no CPU fallback.  Status codes
map onto the reference engine's exception conventions
(matrix_free.py:135-175, backends.py:9-18): EL_EINVAL -> ValueError,
EL_ENOMEM -> MemoryError, EL_ECANCEL -> RuntimeError('用户取消'),
EL_ENOTCONV / EL_ECUDA -> RuntimeError.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libel_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "energy_level_b200.h")

EL_OK, EL_EINVAL, EL_ENOMEM, EL_ENOTCONV, EL_ECANCEL, EL_ECUDA = range(6)
EL_F32, EL_F64, EL_C64, EL_C128 = range(4)
EL_BASIS_FULL, EL_BASIS_BLOCKADE, EL_BASIS_CHARGE = range(3)
EL_LAYOUT_FULL, EL_LAYOUT_CHAIN, EL_LAYOUT_RING, EL_LAYOUT_TABLE = range(4)
EL_ADJ_AUTO, EL_ADJ_STREAM, EL_ADJ_COOP = range(3)
EL_KPM_DIRECT, EL_KPM_DOUBLING = range(2)
EL_KPM_GENERIC_KERNEL = 0x100

DTYPES = {"float32": EL_F32, "float64": EL_F64, "complex64": EL_C64, "complex128": EL_C128}

_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_u64 = C.c_uint64
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

# name -> (restype, argtypes); every function declared in the header
PROTOTYPES = {
    "el_version": (C.c_int, []),
    "el_ctx_create": (C.c_int, [C.c_int, _vp, C.POINTER(_vp)]),
    "el_ctx_destroy": (C.c_int, [_vp]),
    "el_ctx_set_stream": (C.c_int, [_vp, _vp]),
    "el_ctx_set_cancel": (C.c_int, [_vp, _vp]),
    "el_last_error": (C.c_char_p, [_vp]),
    "el_ctx_launches": (_i64, [_vp]),
    "el_ctx_bytes": (C.c_int, [_vp, C.POINTER(_i64), C.POINTER(_i64)]),
    "el_basis_build": (C.c_int, [_vp, C.c_int, _vp, C.c_int, C.c_int, C.c_int, _i64, C.POINTER(_vp)]),
    "el_basis_info": (C.c_int, [_vp, C.POINTER(_i64), _ip]),
    "el_basis_codes": (C.c_int, [_vp, _vp, _vp]),
    "el_basis_rank": (C.c_int, [_vp, _vp, _vp, _i64, _vp]),
    "el_basis_destroy": (C.c_int, [_vp]),
    "el_ham_create": (C.c_int, [_vp, _vp, _dp, _dp, _dp, C.c_int, _vp, _vp, _dp, C.POINTER(_vp)]),
    "el_ham_set_drive": (C.c_int, [_vp, _vp, _dp, _dp, _dp]),
    "el_ham_set_loss": (C.c_int, [_vp, _vp, _dp]),
    "el_taylor_step": (C.c_int, [_vp, _vp, C.c_int, _vp, C.c_double, C.c_double, _ip]),
    "el_ham_set_exchange": (C.c_int, [_vp, _vp, C.c_int, _vp, _vp, _dp, _dp, _dp, _dp]),
    "el_ham_diag": (C.c_int, [_vp, _vp, C.c_int, _vp]),
    "el_ham_destroy": (C.c_int, [_vp]),
    "el_hv": (C.c_int, [_vp, _vp, C.c_int, C.c_int, _vp, _vp]),
    "el_hv_host": (C.c_int, [_vp, _vp, C.c_int, C.c_int, _vp, _vp]),
    "el_bounds": (C.c_int, [_vp, _vp, C.c_int, C.c_double, _u64, _dp, _dp]),
    "el_kpm_moments": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _u64, _vp,
                                 C.c_int, C.c_double, C.c_double, _dp]),
    "el_lanczos_ground": (C.c_int, [_vp, _vp, C.c_int, _vp, _u64, C.c_int, C.c_int, C.c_double,
                                    C.c_int, C.c_int, _dp, _dp, _ip, _ip, _vp]),
    "el_batch_create": (C.c_int, [_vp, C.c_int, _vp, _vp, _dp, _dp, _vp, _vp, _vp, _dp, C.c_int, C.c_int,
                                  C.c_double, C.POINTER(_vp)]),
    "el_batch_create_graph": (C.c_int, [_vp, C.c_int, _vp, _vp, _dp, _dp, _vp, _vp, _vp, _dp, _vp, _vp, _vp,
                                        C.c_int, C.c_int, C.c_double, C.POINTER(_vp)]),
    "el_batch_run": (C.c_int, [_vp, _vp, C.c_int, C.c_int, _u64]),
    "el_batch_run_coop": (C.c_int, [_vp, _vp, C.c_int, C.c_int, _u64]),
    "el_batch_set_wait_limit": (C.c_int, [_vp, _vp, C.c_int32]),
    "el_batch_want_occupations": (C.c_int, [_vp, _vp, C.c_int]),
    "el_batch_occupations": (C.c_int, [_vp, _vp, _dp]),
    "el_batch_results": (C.c_int, [_vp, _vp, _dp, _dp, _dp, _vp, _vp]),
    "el_batch_destroy": (C.c_int, [_vp]),
    "el_cheb_step": (C.c_int, [_vp, _vp, C.c_int, _vp, C.c_double, C.c_double, _ip]),
    "el_observables": (C.c_int, [_vp, _vp, C.c_int, _vp, _dp, _dp]),
    "el_lanczos_tridiag": (C.c_int, [_vp, _vp, C.c_int, _vp, C.c_int, C.c_int, _dp, _dp,
                                     C.POINTER(C.c_int), _dp, _dp, C.POINTER(C.c_int)]),
    "el_spin_observables": (C.c_int, [_vp, _vp, C.c_int, _vp, C.c_int, _vp, _vp, _dp, _dp, _dp, _dp, _dp]),
    "el_pauli_expect": (C.c_int, [_vp, _vp, C.c_int, _vp, C.c_int, _vp, _vp, C.c_char_p, _dp]),
    "el_observables_noalloc": (C.c_int, [_vp, _vp, C.c_int, _vp, _dp, _dp]),
    "el_adjoint_set_mode": (C.c_int, [_vp, C.c_int]),
    "el_adjoint_pulse": (C.c_int, [_vp, _vp, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _vp, _vp, _vp,
                                   C.c_double, _dp, _dp, _dp, _vp]),
}

_lib = None
_lock = threading.Lock()


class LibraryMissing(RuntimeError):
    pass


def load(path: str | None = None):
    """Load the shared library once and attach prototypes; raise if absent."""
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise LibraryMissing(
                "libel_b200.so not built (%s); run energy_level_b200.build.build()" % p)
        lib = C.CDLL(p)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if path is None:
            _lib = lib
        return lib


def header_functions(header: str = HEADER) -> list[str]:
    """Names of all functions declared in the public header."""
    import re
    text = open(header, encoding="utf-8").read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return sorted(set(re.findall(r"\b(el_[a-z0-9_]+)\s*\(", text)))


def check(rc: int, ctx_handle=None, what: str = ""):
    """Map a status code to the reference's exception conventions."""
    if rc == EL_OK:
        return
    msg = ""
    if ctx_handle is not None:
        raw = load().el_last_error(ctx_handle)
        msg = raw.decode("utf-8", "replace") if raw else ""
    text = "%s: %s" % (what, msg) if what else msg
    if rc == EL_EINVAL:
        raise ValueError(text or "invalid argument")
    if rc == EL_ENOMEM:
        raise MemoryError(text or "out of device memory or budget")
    if rc == EL_ECANCEL:
        raise RuntimeError("用户取消")
    if rc == EL_ENOTCONV:
        raise RuntimeError(text or "not converged")
    raise RuntimeError(text or ("CUDA error (status %d)" % rc))


def dptr(arr):
    """ctypes double* for a contiguous float64 numpy array (or None)."""
    if arr is None:
        return None
    return arr.ctypes.data_as(_dp)
