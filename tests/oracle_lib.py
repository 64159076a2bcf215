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


def use_native():
    """Switch to the -march=native build of the oracle (same bits, faster),
    built on this machine; keeps the portable build if that fails.  Call it
    before the first oracle call.  Returns the library file in use."""
    global _NAME
    if _LIB is not None:
        return _NAME
    # named for this host's CPU features: a build from another machine is not reused
    import hashlib
    flags = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("flags", "model name")):
                    flags += line
    except OSError:
        pass
    name = "liboracle_native_%s.so" % hashlib.sha1(flags.encode()).hexdigest()[:12]
    r = subprocess.run(["make", "-s", "-C", ORACLE_DIR, "native", "NATIVE_SO=" + name], capture_output=True)
    if r.returncode == 0 and os.path.exists(os.path.join(ORACLE_DIR, name)):
        _NAME = name
    return _NAME


_NAME = "liboracle.so"


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(ORACLE_DIR, _NAME)
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


class State64(C.Structure):
    _fields_ = [(n, abi.c_double_p) for n in (
        "rho", "press", "thil", "wc", "wmc", "vxe", "vye", "vze", "vmc", "vc", "vmasc", "wmasc",
        "alpha_press", "pwfac", "pvfac", "thilt", "vmxet", "vmyet", "vmzet", "vmt")]


DYN_FIELDS = ("rho", "press", "thil", "wc", "wmc", "vxe", "vye", "vze", "vmc", "vc", "vmasc",
              "wmasc", "alpha_press", "pwfac", "pvfac", "thilt", "vmxet", "vmyet", "vmzet", "vmt")


def _dyn_lib():
    L = lib()
    if not hasattr(L, "_dyn_ready"):
        for sfx in ("f32", "f64"):
            getattr(L, f"oracle_dyn_new_{sfx}").restype = C.c_void_p
            getattr(L, f"oracle_dyn_new_{sfx}").argtypes = [C.POINTER(abi.Grid), C.POINTER(abi.Opts)]
            getattr(L, f"oracle_dyn_free_{sfx}").argtypes = [C.c_void_p]
        L.oracle_prog_wrtv_rk_f32.argtypes = [C.c_void_p, C.POINTER(abi.State), C.c_int]
        L.oracle_prog_wrtv_rk_f64.argtypes = [C.c_void_p, C.POINTER(State64), C.c_int]
        L.oracle_tend0_f32.argtypes = [C.c_void_p, C.POINTER(abi.State), abi.c_float_p]
        L.oracle_tend0_f64.argtypes = [C.c_void_p, C.POINTER(State64), abi.c_double_p]
        L.oracle_timeavg_momsc_f32.argtypes = [C.c_void_p, C.POINTER(abi.State)]
        L.oracle_timeavg_momsc_f64.argtypes = [C.c_void_p, C.POINTER(State64)]
        L.oracle_dyn_set_eddy_f32.argtypes = [C.c_void_p, C.POINTER(abi.Eddy)]
        L.oracle_dyn_set_eddy_f64.argtypes = [C.c_void_p, C.POINTER(abi.Eddy)]
        L.oracle_comp_horiz_k_f32.argtypes = [C.c_void_p, C.POINTER(abi.State), abi.c_float_p,
                                              abi.c_float_p, abi.c_int_p, abi.c_int_p]
        L.oracle_comp_horiz_k_f64.argtypes = [C.c_void_p, C.POINTER(State64), abi.c_double_p,
                                              abi.c_double_p, abi.c_int_p, abi.c_int_p]
        L._dyn_ready = True
    return L


class DynOracle:
    """The oracle's prog_wrtv_rk with its saved damping state, on copies of
    the given arrays (dict name -> array in OLAM layout)."""

    def __init__(self, fg, opts, arrays, fp64=False):
        self.L = _dyn_lib()
        self.fp64 = fp64
        self.fg, self.opts = fg, opts
        sfx = "f64" if fp64 else "f32"
        self.h = getattr(self.L, f"oracle_dyn_new_{sfx}")(C.byref(fg.struct), C.byref(opts))
        self.a = {}
        for n in DYN_FIELDS:
            dt = np.float64 if (fp64 or n in ("rho", "press")) else np.float32
            self.a[n] = np.ascontiguousarray(arrays[n], dtype=dt).copy()
        if fp64:
            s = State64()
            for n in DYN_FIELDS:
                setattr(s, n, abi.ptr(self.a[n], C.c_double))
        else:
            s = abi.State()
            for n in DYN_FIELDS:
                setattr(s, n, abi.ptr(self.a[n], C.c_double if n in ("rho", "press") else C.c_float))
        self.s = s

    def prog_wrtv_rk(self, istp=1):
        f = self.L.oracle_prog_wrtv_rk_f64 if self.fp64 else self.L.oracle_prog_wrtv_rk_f32
        rc = f(self.h, C.byref(self.s), istp)
        assert rc == 0, rc

    def tend0(self):
        ro = np.zeros_like(self.a["thil"])
        if self.fp64:
            self.L.oracle_tend0_f64(self.h, C.byref(self.s), abi.ptr(ro, C.c_double))
        else:
            self.L.oracle_tend0_f32(self.h, C.byref(self.s), abi.ptr(ro, C.c_float))
        return ro

    def timeavg_momsc(self):
        f = self.L.oracle_timeavg_momsc_f64 if self.fp64 else self.L.oracle_timeavg_momsc_f32
        f(self.h, C.byref(self.s))

    def set_eddy(self, eddy):
        """Eddy diffusion from an ``abi.Eddy`` (kept alive here; None: off)."""
        self.eddy = eddy
        f = self.L.oracle_dyn_set_eddy_f64 if self.fp64 else self.L.oracle_dyn_set_eddy_f32
        f(self.h, C.byref(eddy) if eddy is not None else None)

    def comp_horiz_k(self):
        """comp_horiz_k into the oracle's own arrays, which its later steps
        use; returns copies (akmodx, akhodx, kmtopv, khtopv)."""
        mza, mva = self.a["thil"].shape[1], self.a["vmc"].shape[0]
        dt = np.float64 if self.fp64 else np.float32
        ct = C.c_double if self.fp64 else C.c_float
        am, ah = np.zeros((mva, mza), dt), np.zeros((mva, mza), dt)
        km, kh = np.zeros(mva, np.int32), np.zeros(mva, np.int32)
        f = self.L.oracle_comp_horiz_k_f64 if self.fp64 else self.L.oracle_comp_horiz_k_f32
        rc = f(self.h, C.byref(self.s), abi.ptr(am, ct), abi.ptr(ah, ct), abi.ptr(km, C.c_int),
               abi.ptr(kh, C.c_int))
        assert rc == 0, rc
        return am, ah, km, kh

    def __del__(self):
        try:
            sfx = "f64" if self.fp64 else "f32"
            getattr(self.L, f"oracle_dyn_free_{sfx}")(self.h)
        except Exception:
            pass


def dyn_arrays(g, ds):
    """OLAM module arrays for prog_wrtv_rk from a synth dynamics state."""
    z = lambda n: np.zeros((n, g.mza), dtype=np.float32)  # noqa: E731
    return dict(rho=ds.rho, press=ds.press, thil=ds.thil, wc=ds.wc, wmc=ds.wmc, vxe=ds.vxe,
                vye=ds.vye, vze=ds.vze, vmc=ds.vmc, vc=ds.vc, vmasc=z(g.mva), wmasc=z(g.mwa),
                alpha_press=ds.alpha_press, pwfac=ds.pwfac, pvfac=ds.pvfac, thilt=z(g.mwa),
                vmxet=z(g.mwa), vmyet=z(g.mwa), vmzet=z(g.mwa), vmt=z(g.mva))


def _adj_lib():
    L = lib()
    if not hasattr(L, "_adj_ready"):
        for name, t in (("oracle_scalar_transport_rk_adjoint_f32", C.c_float),
                        ("oracle_scalar_transport_rk_adjoint_f64", C.c_double)):
            f = getattr(L, name)
            f.restype = C.c_int
            f.argtypes = [C.POINTER(abi.Grid), C.POINTER(abi.Opts), C.c_int,
                          C.POINTER(C.POINTER(t)), C.POINTER(C.POINTER(t)),
                          abi.c_float_p, abi.c_float_p, abi.c_double_p, abi.c_float_p, abi.c_float_p]
        L._adj_ready = True
    return L


def scalar_transport_adjoint(fg, opts, lam, st, fp64=False):
    """The oracle's adjoint of one unlimited scalar_transport_rk step.

    lam: (ntr, mwa, mza) adjoint of the new tracers.  Returns (adjoint of the
    old tracers, adjoint of the tendencies sct), same shape."""
    dt = np.float64 if fp64 else np.float32
    ct = C.c_double if fp64 else C.c_float
    la = [np.ascontiguousarray(x, dtype=dt).copy() for x in lam]
    ls = [np.zeros_like(x) for x in la]
    L = _adj_lib()
    f = L.oracle_scalar_transport_rk_adjoint_f64 if fp64 else L.oracle_scalar_transport_rk_adjoint_f32
    rc = f(C.byref(fg.struct), C.byref(opts), len(la), abi.ptr_array(la, ct), abi.ptr_array(ls, ct),
           abi.ptr(np.ascontiguousarray(st.vmasc, np.float32), C.c_float),
           abi.ptr(np.ascontiguousarray(st.wmasc, np.float32), C.c_float),
           abi.ptr(np.ascontiguousarray(st.rho, np.float64), C.c_double),
           abi.ptr(np.ascontiguousarray(st.rho_old, np.float32), C.c_float),
           abi.ptr(np.ascontiguousarray(st.wc, np.float32), C.c_float))
    assert rc == 0, f"oracle adjoint returned {rc}"
    return np.stack(la), np.stack(ls)


def _winds(st):
    return (abi.ptr(np.ascontiguousarray(st.vmasc, np.float32), C.c_float),
            abi.ptr(np.ascontiguousarray(st.wmasc, np.float32), C.c_float),
            abi.ptr(np.ascontiguousarray(st.rho, np.float64), C.c_double),
            abi.ptr(np.ascontiguousarray(st.rho_old, np.float32), C.c_float),
            abi.ptr(np.ascontiguousarray(st.wc, np.float32), C.c_float))


def scalar_transport_tl(fg, opts, tracers, sct, dtracers, dsct, st, pdef=None):
    """The oracle's step in FP64 and its exact tangent-linear: returns
    (new tracers, the directional derivative of the new tracers along
    (dtracers, dsct)), each (ntr, mwa, mza) float64."""
    L = lib()
    f = L.oracle_scalar_transport_rk_tl_f64
    f.restype = C.c_int
    dp = C.POINTER(C.c_double)
    f.argtypes = [C.POINTER(abi.Grid), C.POINTER(abi.Opts), C.c_int, C.POINTER(dp), C.POINTER(dp),
                  C.POINTER(dp), C.POINTER(dp), abi.c_int_p] + [abi.c_float_p, abi.c_float_p, abi.c_double_p,
                                                                  abi.c_float_p, abi.c_float_p]
    cp = lambda xs: [np.ascontiguousarray(x, np.float64).copy() for x in xs]  # noqa: E731
    s, ds, t, dt = cp(tracers), cp(dtracers), cp(sct), cp(dsct)
    pd = np.ascontiguousarray(pdef if pdef is not None else np.ones(len(s)), dtype=np.int32)
    rc = f(C.byref(fg.struct), C.byref(opts), len(s), abi.ptr_array(s, C.c_double), abi.ptr_array(ds, C.c_double),
           abi.ptr_array(t, C.c_double), abi.ptr_array(dt, C.c_double), abi.ptr(pd, C.c_int), *_winds(st))
    assert rc == 0, f"oracle tangent-linear returned {rc}"
    return np.stack(s), np.stack(ds)


def scalar_transport_adjoint_pd(fg, opts, lam, st, tracers, sct, pdef=None, fp64=False):
    """The oracle's adjoint of one step with the positive-definite limiter
    (iscal_monot = 2) on the forward step from (tracers, sct).  Returns
    (adjoint of the old tracers, adjoint of sct)."""
    dt = np.float64 if fp64 else np.float32
    ct = C.c_double if fp64 else C.c_float
    L = lib()
    f = L.oracle_scalar_transport_rk_adjoint_pd_f64 if fp64 else L.oracle_scalar_transport_rk_adjoint_pd_f32
    f.restype = C.c_int
    tp = C.POINTER(ct)
    f.argtypes = [C.POINTER(abi.Grid), C.POINTER(abi.Opts), C.c_int, C.POINTER(tp), C.POINTER(tp), abi.c_int_p,
                  C.POINTER(tp), C.POINTER(tp)] + [abi.c_float_p, abi.c_float_p, abi.c_double_p, abi.c_float_p,
                                                   abi.c_float_p]
    cp = lambda xs: [np.ascontiguousarray(x, dt).copy() for x in xs]  # noqa: E731
    sf, tf, la = cp(tracers), cp(sct), cp(lam)
    ls = [np.zeros_like(x) for x in la]
    pd = np.ascontiguousarray(pdef if pdef is not None else np.ones(len(la)), dtype=np.int32)
    rc = f(C.byref(fg.struct), C.byref(opts), len(la), abi.ptr_array(sf, ct), abi.ptr_array(tf, ct),
           abi.ptr(pd, C.c_int), abi.ptr_array(la, ct), abi.ptr_array(ls, ct), *_winds(st))
    assert rc == 0, f"oracle adjoint returned {rc}"
    return np.stack(la), np.stack(ls)
