"""ctypes access to the CPU oracle (test infrastructure only).

The oracle is the checker: tests, smoke() and bench.py's CPU baseline call
it; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from olam_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
_LIB = None


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(ORACLE_DIR, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        for name, t in (("oracle_scalar_transport_rk_f32", C.c_float),
                        ("oracle_scalar_transport_rk_f64", C.c_double)):
            f = getattr(_LIB, name)
            f.restype = C.c_int
            f.argtypes = [C.POINTER(abi.Grid), C.POINTER(abi.Opts), C.c_int,
                          C.POINTER(C.POINTER(t)), C.POINTER(C.POINTER(t)),
                          abi.c_int_p, abi.c_int_p, abi.c_float_p, abi.c_float_p,
                          abi.c_double_p, abi.c_float_p, abi.c_float_p,
                          abi.c_float_p, abi.c_int_p, abi.c_float_p, C.POINTER(abi.CflDiag)]
    return _LIB


def scalar_transport(fg, opts, tracers, sct, st, fp64=False, pdef=None, sgsmix=None,
                     akhodx=None, khtopv=None, want_ff=False):
    """Run the oracle's scalar_transport_rk in place on copies; return results.

    tracers, sct: (ntr, mwa, mza) float32 arrays (not modified).
    """
    dt = np.float64 if fp64 else np.float32
    ct = C.c_double if fp64 else C.c_float
    scp = [np.ascontiguousarray(t, dtype=dt).copy() for t in tracers]
    sc = [np.ascontiguousarray(t, dtype=dt).copy() for t in sct]
    ntr = len(scp)
    pd = np.ascontiguousarray(pdef if pdef is not None else np.ones(ntr), dtype=np.int32)
    sg = np.ascontiguousarray(sgsmix if sgsmix is not None else np.zeros(ntr), dtype=np.int32)
    nrk = opts.nrk_scal
    ff = np.zeros((fg.g.mwa, nrk), dtype=np.float32)
    diag = abi.CflDiag()
    f = lib().oracle_scalar_transport_rk_f64 if fp64 else lib().oracle_scalar_transport_rk_f32
    rc = f(C.byref(fg.struct), C.byref(opts), ntr, abi.ptr_array(scp, ct), abi.ptr_array(sc, ct),
           abi.ptr(pd, C.c_int), abi.ptr(sg, C.c_int),
           abi.ptr(np.ascontiguousarray(st.vmasc, np.float32), C.c_float),
           abi.ptr(np.ascontiguousarray(st.wmasc, np.float32), C.c_float),
           abi.ptr(np.ascontiguousarray(st.rho, np.float64), C.c_double),
           abi.ptr(np.ascontiguousarray(st.rho_old, np.float32), C.c_float),
           abi.ptr(np.ascontiguousarray(st.wc, np.float32), C.c_float),
           abi.ptr(None if akhodx is None else np.ascontiguousarray(akhodx, np.float32), C.c_float),
           abi.ptr(None if khtopv is None else np.ascontiguousarray(khtopv, np.int32), C.c_int),
           abi.ptr(ff, C.c_float), C.byref(diag))
    assert rc == 0, f"oracle returned {rc}"
    out = np.stack(scp)
    if want_ff:
        return out, ff, diag
    return out
