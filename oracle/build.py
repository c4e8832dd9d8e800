"""Build recipe of the C oracle ``oracle/liboracle_el.so`` (test infrastructure).

gcc with OpenMP, generic x86-64-v2 code so the library runs on any host CPU
it is carried to.  The reference itself is pure Python (nothing to compile),
so there is no ``oracle/_ref`` build.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "el_oracle.c")
LIB = os.path.join(HERE, "liboracle_el.so")


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared", SRC, "-o", LIB + ".tmp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("oracle build failed:\n%s" % res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def load():
    lib = C.CDLL(build())
    dp = C.POINTER(C.c_double)
    lib.oracle_threads.restype = C.c_int
    lib.oracle_set_threads.argtypes = [C.c_int]
    lib.oracle_diag_full.argtypes = [C.c_int, dp, C.c_int, C.c_void_p, C.c_void_p, dp, dp]
    lib.oracle_apply_full.argtypes = [C.c_int, dp, dp, C.c_int, C.c_double, C.c_double, C.c_double,
                                      dp, dp, dp]
    lib.oracle_kpm_full.argtypes = [C.c_int, dp, dp, C.c_double, C.c_double, C.c_int, C.c_int,
                                    C.c_void_p, dp]
    lib.oracle_kpm_full.restype = C.c_int
    return lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def diag_full(n, delta, pairs):
    import numpy as np
    lib = load()
    delta = np.ascontiguousarray(delta, dtype=np.float64)
    pi = np.ascontiguousarray([p[0] for p in pairs], dtype=np.int32)
    pj = np.ascontiguousarray([p[1] for p in pairs], dtype=np.int32)
    V = np.ascontiguousarray([p[2] for p in pairs], dtype=np.float64)
    d = np.empty(1 << n)
    lib.oracle_diag_full(n, _dp(delta), len(V), C.c_void_p(pi.ctypes.data),
                         C.c_void_p(pj.ctypes.data), _dp(V), _dp(d))
    return d


def kpm_full(n, omega, d, c, r, num, probes):
    """Direct-recurrence KPM moments on the full basis (real H)."""
    import numpy as np
    lib = load()
    om = np.ascontiguousarray(np.asarray(omega).real, dtype=np.float64)
    d = np.ascontiguousarray(d, dtype=np.float64)
    pr = np.ascontiguousarray(probes, dtype=np.int8)
    mu = np.zeros(num + 1)
    rc = lib.oracle_kpm_full(n, _dp(om), _dp(d), c, r, num, pr.shape[0], C.c_void_p(pr.ctypes.data), _dp(mu))
    if rc:
        raise RuntimeError("oracle_kpm_full failed (%d)" % rc)
    return mu
