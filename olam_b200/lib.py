"""Loader of libolamgpu.so and thin Python mirror of OLAM's hot-path interface.

The product is the C-ABI library; this module is the host-side mirror of the
reference interface (``init_wrtv_rk``, ``prog_wrtv_rk``,
``scalar_transport_rk(rho_old)``) used by tests and benchmarks.  It loads the
in-tree library and raises if it is missing or fails: there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
# OLAMGPU_LIBRARY selects another build of the library (e.g. a diagnostic one)
LIB_PATH = os.environ.get("OLAMGPU_LIBRARY") or os.path.join(HERE, "libolamgpu.so")
_LIB = None

# every entry point declared in include/olamgpu.h
EXPORTS = [
    "olamgpu_init", "olamgpu_register_scalars", "olamgpu_set_turb", "olamgpu_finalize",
    "olamgpu_strerror", "olamgpu_set_coherence", "olamgpu_sync_to_device", "olamgpu_sync_to_host",
    "olamgpu_set_transport_form", "olamgpu_scalar_transport_rk", "olamgpu_prog_wrtv_rk",
    "olamgpu_tend0", "olamgpu_timeavg_momsc", "olamgpu_stream", "olamgpu_launch_count",
    "olamgpu_profile", "olamgpu_profile_read", "olamgpu_update_scalar_noalloc",
    "olamgpu_scalar_transport_rk_adjoint", "olamgpu_set_eddy", "olamgpu_comp_horiz_k",
    "olamgpu_set_scalars_bottom", "olamgpu_diagvel_t3d", "olamgpu_tracer_maxmin", "olamgpu_mass_sums",
    "olamgpu_timestep", "olamgpu_timestep_diag", "olamgpu_set_halo",
    "olamgpu_set_surface_emission", "olamgpu_window_forward", "olamgpu_window_adjoint",
    "olamgpu_window_memory", "olamgpu_window_rewind", "olamgpu_set_tile_shape", "olamgpu_tile_shape",
]


class OlamGpuError(RuntimeError):
    def __init__(self, rc, msg):
        super().__init__(f"olamgpu status {rc}: {msg}")
        self.rc = rc


def load():
    """Load the in-tree library (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise OlamGpuError(-1, f"{LIB_PATH} not built; run __graft_entry__.build()")
    lib = C.CDLL(LIB_PATH)
    lib.olamgpu_init.argtypes = [C.POINTER(abi.Grid), C.POINTER(abi.Opts), C.POINTER(abi.State)]
    lib.olamgpu_register_scalars.argtypes = [C.c_int, C.POINTER(abi.c_float_p),
                                             C.POINTER(abi.c_float_p), abi.c_int_p, abi.c_int_p]
    lib.olamgpu_set_turb.argtypes = [abi.c_float_p, abi.c_int_p]
    lib.olamgpu_finalize.argtypes = []
    lib.olamgpu_strerror.argtypes = [C.c_int]
    lib.olamgpu_strerror.restype = C.c_char_p
    lib.olamgpu_set_coherence.argtypes = [C.c_int]
    lib.olamgpu_sync_to_device.argtypes = [C.c_uint]
    lib.olamgpu_sync_to_host.argtypes = [C.c_uint]
    lib.olamgpu_set_transport_form.argtypes = [C.c_int]
    lib.olamgpu_scalar_transport_rk.argtypes = [abi.c_float_p, C.POINTER(abi.CflDiag)]
    lib.olamgpu_prog_wrtv_rk.argtypes = [C.c_int]
    lib.olamgpu_tend0.argtypes = [abi.c_float_p]
    lib.olamgpu_timeavg_momsc.argtypes = []
    lib.olamgpu_stream.restype = C.c_void_p
    lib.olamgpu_launch_count.argtypes = [C.c_int]
    lib.olamgpu_launch_count.restype = C.c_ulonglong
    lib.olamgpu_profile.argtypes = [C.c_int, C.c_int]
    lib.olamgpu_profile_read.argtypes = [C.c_int, C.c_char_p, C.POINTER(C.c_double),
                                         C.POINTER(C.c_ulonglong)]
    lib.olamgpu_update_scalar_noalloc.argtypes = [C.c_void_p] * 6 + [C.c_float, C.c_void_p, C.c_void_p]
    lib.olamgpu_scalar_transport_rk_adjoint.argtypes = [abi.c_float_p, C.POINTER(abi.c_float_p),
                                                        C.POINTER(abi.c_float_p)]
    lib.olamgpu_set_eddy.argtypes = [C.POINTER(abi.Eddy)]
    lib.olamgpu_comp_horiz_k.argtypes = []
    lib.olamgpu_set_halo.argtypes = [C.POINTER(abi.Halo)]
    lib.olamgpu_set_scalars_bottom.argtypes = []
    lib.olamgpu_diagvel_t3d.argtypes = []
    lib.olamgpu_tracer_maxmin.argtypes = [abi.c_float_p]
    lib.olamgpu_mass_sums.argtypes = [C.c_int, abi.c_int_p, abi.c_double_p]
    lib.olamgpu_timestep.argtypes = [C.c_uint, C.c_int, abi.c_int_p]
    lib.olamgpu_timestep_diag.argtypes = [abi.c_float_p, abi.c_double_p]
    lib.olamgpu_set_surface_emission.argtypes = [C.POINTER(abi.c_float_p)]
    lib.olamgpu_window_forward.argtypes = [C.c_int, C.c_int, C.c_uint]
    lib.olamgpu_window_adjoint.argtypes = [C.POINTER(abi.c_float_p), C.POINTER(abi.c_float_p)]
    lib.olamgpu_window_memory.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
    lib.olamgpu_window_rewind.argtypes = []
    lib.olamgpu_set_tile_shape.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
    lib.olamgpu_tile_shape.argtypes = [abi.c_int_p, C.c_int, abi.c_int_p, abi.c_float_p]
    for name in EXPORTS:
        if name not in ("olamgpu_strerror", "olamgpu_stream", "olamgpu_launch_count"):
            getattr(lib, name).restype = C.c_int
    _LIB = lib
    return lib


def check(rc):
    if rc != 0:
        msg = load().olamgpu_strerror(rc).decode()
        raise OlamGpuError(rc, msg)


class HostState:
    """OLAM module arrays (mem_basic / mem_tend) in Fortran layout."""

    FIELDS32 = ("thil", "wc", "wmc", "vxe", "vye", "vze", "vmc", "vc", "vmasc", "wmasc",
                "alpha_press", "pwfac", "pvfac", "thilt", "vmxet", "vmyet", "vmzet", "vmt")
    FIELDS64 = ("rho", "press")

    def __init__(self, **arrays):
        self.arrays = {}
        for k, v in arrays.items():
            if v is None:
                continue
            dt = np.float64 if k in self.FIELDS64 else np.float32
            self.arrays[k] = np.ascontiguousarray(v, dtype=dt)
        s = abi.State()
        for k in self.FIELDS32:
            setattr(s, k, abi.ptr(self.arrays.get(k), C.c_float))
        for k in self.FIELDS64:
            setattr(s, k, abi.ptr(self.arrays.get(k), C.c_double))
        self.struct = s

    def __getitem__(self, k):
        return self.arrays[k]


class OlamGpu:
    """Process-wide handle on the library context (one per process, as in OLAM)."""

    def __init__(self, fgrid, opts, state: HostState | None = None):
        self.lib = load()
        self.fgrid, self.opts, self.state = fgrid, opts, state
        check(self.lib.olamgpu_init(C.byref(fgrid.struct), C.byref(opts),
                                    C.byref(state.struct) if state is not None else None))
        self._scalars = None

    # -- reference interface ----------------------------------------------------
    def register_scalars(self, var_p, var_t, pdef=None, sgsmix=None):
        """var_p / var_t: lists of (mwa, mza) float32 arrays OLAM owns."""
        n = len(var_p)
        self._scalars = (var_p, var_t)
        pd = np.ascontiguousarray(pdef if pdef is not None else np.ones(n), dtype=np.int32)
        sg = np.ascontiguousarray(sgsmix if sgsmix is not None else np.zeros(n), dtype=np.int32)
        self._flags = (pd, sg)
        check(self.lib.olamgpu_register_scalars(n, abi.ptr_array(var_p, C.c_float),
                                                abi.ptr_array(var_t, C.c_float),
                                                abi.ptr(pd, C.c_int), abi.ptr(sg, C.c_int)))

    def scalar_transport_rk(self, rho_old=None, want_diag=False):
        diag = abi.CflDiag()
        rp = None if rho_old is None else np.ascontiguousarray(rho_old, dtype=np.float32)
        check(self.lib.olamgpu_scalar_transport_rk(abi.ptr(rp, C.c_float), C.byref(diag)
                                                   if want_diag else None))
        return diag if want_diag else None

    def scalar_transport_rk_adjoint(self, lam, rho_old=None):
        """Adjoint of one unlimited step: lam is a list of (mwa, mza)
        float32 arrays of dJ/d(new scp) per registered tracer; returns
        (dJ/d(old scp), dJ/d(sct)) as lists of new arrays of that shape."""
        lam_io = [np.array(x, dtype=np.float32, order="C", copy=True) for x in lam]
        lsct = [np.zeros_like(x) for x in lam_io]
        lp = abi.ptr_array(lam_io, C.c_float)
        sp = abi.ptr_array(lsct, C.c_float)
        rp = None if rho_old is None else np.ascontiguousarray(rho_old, dtype=np.float32)
        check(self.lib.olamgpu_scalar_transport_rk_adjoint(abi.ptr(rp, C.c_float), lp, sp))
        return lam_io, lsct

    def prog_wrtv_rk(self, istp=1):
        check(self.lib.olamgpu_prog_wrtv_rk(int(istp)))

    def tend0(self, rho_old):
        check(self.lib.olamgpu_tend0(abi.ptr(rho_old, C.c_float)))

    def timeavg_momsc(self):
        check(self.lib.olamgpu_timeavg_momsc())

    def set_eddy(self, eddy):
        """Register the eddy-diffusion inputs (an ``abi.Eddy``; None: off).
        The struct and its arrays must stay alive while registered."""
        self._eddy = eddy
        check(self.lib.olamgpu_set_eddy(C.byref(eddy) if eddy is not None else None))

    def comp_horiz_k(self):
        check(self.lib.olamgpu_comp_horiz_k())

    def set_halo(self, halo):
        """Register a halo plan (an ``abi.Halo``; None: one domain).  The
        struct and its hook must stay alive while registered."""
        self._halo = halo
        check(self.lib.olamgpu_set_halo(C.byref(halo) if halo is not None else None))

    # -- long-step glue ------------------------------------------------------------
    def set_scalars_bottom(self):
        check(self.lib.olamgpu_set_scalars_bottom())

    def diagvel_t3d(self):
        check(self.lib.olamgpu_diagvel_t3d())

    def tracer_maxmin(self, ntr):
        """(ntr, 2) array of (max, -min) per registered scalar."""
        out = np.zeros((ntr, 2), np.float32)
        check(self.lib.olamgpu_tracer_maxmin(abi.ptr(out, C.c_float)))
        return out

    def mass_sums(self, ids=()):
        """[sum rho volt, sum rho volt scalar[i - 1] for i in ids]."""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        out = np.zeros(1 + ids.size, np.float64)
        check(self.lib.olamgpu_mass_sums(int(ids.size), abi.ptr(ids, C.c_int) if ids.size else None,
                                         abi.ptr(out, C.c_double)))
        return out

    def timestep(self, flags=0, mass_ids=()):
        ids = np.ascontiguousarray(mass_ids, dtype=np.int32)
        self._mass_ids = ids
        check(self.lib.olamgpu_timestep(int(flags), int(ids.size), abi.ptr(ids, C.c_int) if ids.size else None))

    def set_surface_emission(self, emis):
        """emis: list (one per registered scalar) of (mwa,) float32 arrays or
        None entries, or None to switch the emission off."""
        if emis is None:
            self._emis = None
            check(self.lib.olamgpu_set_surface_emission(None))
            return
        self._emis = [None if e is None else np.ascontiguousarray(e, dtype=np.float32) for e in emis]
        arr = (abi.c_float_p * len(self._emis))(*[abi.ptr(e, C.c_float) for e in self._emis])
        check(self.lib.olamgpu_set_surface_emission(arr))

    def set_tile_shape(self, T=0, G=0, KS=0, ord=0):
        check(self.lib.olamgpu_set_tile_shape(int(T), int(G), int(KS), int(ord)))

    def tile_shape(self, maxn=32):
        """((T, G, KS, ord) in use, [(T, G, KS, ord, chosen, ms) of the last tuning])."""
        shape = np.zeros(4, np.int32)
        cand = np.zeros(5 * maxn, np.int32)
        ms = np.zeros(maxn, np.float32)
        n = self.lib.olamgpu_tile_shape(abi.ptr(shape, C.c_int), maxn, abi.ptr(cand, C.c_int), abi.ptr(ms, C.c_float))
        if n < 0:
            check(-n)
        log = [tuple(int(x) for x in cand[5 * i:5 * i + 5]) + (float(ms[i]),) for i in range(min(n, maxn))]
        return tuple(int(x) for x in shape), log

    def window_forward(self, nsteps, nchk, flags=0):
        check(self.lib.olamgpu_window_forward(int(nsteps), int(nchk), int(flags)))

    def window_adjoint(self, lam, lam_sct=None, in_place=False):
        """lam: list of (mwa, mza) float32 arrays of dJ/d(scalars after the
        window); returns (dJ/d(scalars before it), dJ/d(tendencies)).  With
        in_place the first result is written into lam's own (C-contiguous
        float32) arrays, and lam_sct, when given, receives the second."""
        if in_place:
            for x in lam:
                if x.dtype != np.float32 or not x.flags.c_contiguous:
                    raise ValueError("in_place needs C-contiguous float32 arrays")
            lam_io = list(lam)
        else:
            lam_io = [np.array(x, dtype=np.float32, order="C", copy=True) for x in lam]
        lsct = lam_sct if lam_sct is not None else [np.zeros_like(x) for x in lam_io]
        for x, y in zip(lam_io, lsct):
            if y.shape != x.shape or y.dtype != np.float32 or not y.flags.c_contiguous:
                raise ValueError("lam_sct arrays must match lam (C-contiguous float32)")
        check(self.lib.olamgpu_window_adjoint(abi.ptr_array(lam_io, C.c_float), abi.ptr_array(lsct, C.c_float)))
        return lam_io, lsct

    def window_rewind(self):
        """The state at the start of the last window back on the device (an
        unlimited window's tracers excepted: send the new ones after it)."""
        check(self.lib.olamgpu_window_rewind())

    def window_memory(self, host_checkpoints=False, segment_steps=0, nsteps=0, nchk=0, lean=False):
        """Where the next window keeps its states: page-locked host memory for
        the checkpoints and the final state (reserved now for nsteps / nchk
        when both are given); how many steps' transport inputs the adjoint
        holds at once (0: a whole segment); lean: the adjoint borrows the
        tracer buffers even when the device has room for its own."""
        flags = (abi.WIN_HOST if host_checkpoints else 0) | (abi.WIN_LEAN if lean else 0)
        check(self.lib.olamgpu_window_memory(flags, int(segment_steps), int(nsteps), int(nchk)))

    def timestep_diag(self, ntr, nmass=0):
        smax = np.zeros((ntr, 2), np.float32)
        sums = np.zeros(1 + nmass, np.float64)
        check(self.lib.olamgpu_timestep_diag(abi.ptr(smax, C.c_float), abi.ptr(sums, C.c_double)))
        return smax, sums

    # -- library controls --------------------------------------------------------
    def set_coherence(self, mode):
        check(self.lib.olamgpu_set_coherence(mode))

    def set_transport_form(self, form):
        check(self.lib.olamgpu_set_transport_form(form))

    def sync_to_device(self, mask=abi.F_ALL):
        check(self.lib.olamgpu_sync_to_device(mask))

    def sync_to_host(self, mask=abi.F_ALL):
        check(self.lib.olamgpu_sync_to_host(mask))

    def stream(self):
        return self.lib.olamgpu_stream()

    def launch_count(self, reset=False):
        return int(self.lib.olamgpu_launch_count(1 if reset else 0))

    def profile(self, enable=True, reset=False):
        check(self.lib.olamgpu_profile(1 if enable else 0, 1 if reset else 0))

    def profile_read(self, maxn=64):
        names = C.create_string_buffer(32 * maxn)
        ms = (C.c_double * maxn)()
        cnt = (C.c_ulonglong * maxn)()
        n = self.lib.olamgpu_profile_read(maxn, names, ms, cnt)
        if n < 0:
            check(-n)
        out = {}
        for i in range(min(n, maxn)):
            nm = names.raw[32 * i:32 * (i + 1)].split(b"\0", 1)[0].decode()
            out[nm] = (float(ms[i]), int(cnt[i]))
        return out

    def close(self):
        check(self.lib.olamgpu_finalize())
