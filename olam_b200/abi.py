"""ctypes mirror of include/olamgpu.h and Fortran-layout packing of a grid.

OLAM hands the library its module arrays through ISO_C_BINDING; this module
does the same from Python so tests and benchmarks drive the library exactly
as the Fortran shim would: column-major (mza, n) arrays, OLAM's 1-based
neighbour indices, and packed derived-type members.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

c_int_p = C.POINTER(C.c_int)
c_float_p = C.POINTER(C.c_float)
c_double_p = C.POINTER(C.c_double)

OK = 0
E_ARG, E_STATE, E_UNSUPPORTED, E_CUDA, E_NOMEM, E_NODEVICE, E_NUMERIC = range(1, 8)

SYNC_EACH_CALL, RESIDENT = 0, 1
TRANSPORT_FUSED, TRANSPORT_PLAIN, TRANSPORT_FUSED_COLUMN = 0, 1, 2

F_RHO, F_PRESS, F_THIL, F_WC, F_WMC, F_VXE, F_VMC, F_VC = (1 << i for i in range(8))
F_VMASC, F_WMASC, F_TEND, F_FACS, F_SCALARS, F_SCALAR_TEND, F_EDDY = (1 << i for i in range(8, 15))
F_ALL = 0xFFFF


class Grid(C.Structure):
    _fields_ = [
        ("mza", C.c_int), ("mwa", C.c_int), ("mva", C.c_int), ("mma", C.c_int),
        ("nw_prog", C.c_int), ("jtw_prog", c_int_p),
        ("nw_wadj", C.c_int), ("jtw_wadj", c_int_p),
        ("nv_prog", C.c_int), ("jtv_prog", c_int_p),
        ("nv_wadj", C.c_int), ("jtv_wadj", c_int_p),
        ("nm_prog", C.c_int), ("jtm_prog", c_int_p),
        ("npoly", c_int_p), ("itab_w_iv", c_int_p), ("itab_w_iw", c_int_p),
        ("itab_w_im", c_int_p), ("itab_w_dirv", c_float_p),
        ("ecvec_vx", c_float_p), ("ecvec_vy", c_float_p), ("ecvec_vz", c_float_p),
        ("iwglobe", c_int_p),
        ("itab_v_iw", c_int_p), ("itab_v_im", c_int_p), ("dxps", c_float_p), ("dyps", c_float_p),
        ("itab_m_iv", c_int_p), ("itab_m_iw", c_int_p), ("itab_m_im", c_int_p),
        ("lpw", c_int_p), ("lpv", c_int_p), ("lpm", c_int_p), ("lve2", c_int_p),
        ("zm", c_float_p), ("zt", c_float_p), ("dzm", c_float_p), ("dzt", c_float_p),
        ("dzim", c_float_p), ("dzit", c_float_p), ("dzt_top", c_float_p), ("dzt_bot", c_float_p),
        ("zfacit", c_float_p),
        ("zwgt_top8", c_double_p), ("zwgt_bot8", c_double_p),
        ("gdz_wgtm8", c_double_p), ("gdz_wgtp8", c_double_p),
        ("gdz_wgtm", c_float_p), ("gdz_wgtp", c_float_p),
        ("wnx", c_float_p), ("wny", c_float_p), ("wnz", c_float_p),
        ("wnxo2", c_float_p), ("wnyo2", c_float_p), ("wnzo2", c_float_p),
        ("vnx", c_float_p), ("vny", c_float_p), ("vnz", c_float_p),
        ("dnu", c_float_p), ("dniu", c_float_p), ("dnv", c_float_p), ("dniv", c_float_p),
        ("arw0", c_float_p), ("arm0", c_float_p),
        ("arv", c_float_p), ("arw", c_float_p), ("volt", c_double_p), ("volti", c_float_p),
        ("volwi", c_float_p), ("volvi", c_float_p),
        ("gxps_coef", c_float_p), ("gyps_coef", c_float_p),
        ("a_w", c_float_p), ("a_wu", c_float_p), ("xy_h", c_float_p), ("xy_hu", c_float_p),
        ("xx0_v", c_float_p), ("xy0_v", c_float_p), ("yy0_v", c_float_p),
        ("xx0_vu", c_float_p), ("xy0_vu", c_float_p), ("yy0_vu", c_float_p),
        ("xx_yy", c_float_p), ("xx_yy_m", c_float_p),
    ]


class Opts(C.Structure):
    _fields_ = [
        ("dtlm", C.c_double), ("dtsm", C.c_double), ("nacoust", C.c_int),
        ("nrk_wrtv", C.c_int), ("nrk_scal", C.c_int),
        ("thil_horiz_adv_order", C.c_int), ("wind_horiz_adv_order", C.c_int),
        ("scal_horiz_adv_order", C.c_int),
        ("ithil_monot", C.c_int), ("iwind_monot", C.c_int), ("iscal_monot", C.c_int),
        ("divh_damp_fact", C.c_float), ("divh_damp_level", C.c_int), ("divh_damp_short", C.c_int),
        ("vort_damp_fact", C.c_float), ("vort_damp_level", C.c_int), ("vort_damp_short", C.c_int),
        ("fcoriol", C.c_float), ("mdomain", C.c_int),
        ("krayf_bot", C.c_int), ("rayf_cof", c_float_p), ("dn01d", c_float_p),
        ("th01d", c_float_p), ("vc03d", c_float_p),
        ("krayfw_bot", C.c_int), ("rayf_cofw", c_float_p), ("initial", C.c_int),
    ]


class State(C.Structure):
    _fields_ = [
        ("rho", c_double_p), ("press", c_double_p),
        ("thil", c_float_p), ("wc", c_float_p), ("wmc", c_float_p),
        ("vxe", c_float_p), ("vye", c_float_p), ("vze", c_float_p),
        ("vmc", c_float_p), ("vc", c_float_p), ("vmasc", c_float_p), ("wmasc", c_float_p),
        ("alpha_press", c_float_p), ("pwfac", c_float_p), ("pvfac", c_float_p),
        ("thilt", c_float_p), ("vmxet", c_float_p), ("vmyet", c_float_p), ("vmzet", c_float_p),
        ("vmt", c_float_p),
    ]


# olamgpu_halo's exchange hook
HALO_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.POINTER(C.c_float)),
                      C.POINTER(C.c_size_t), C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.c_size_t), C.c_void_p)


class Halo(C.Structure):
    """olamgpu_halo: the halo plan of a rank and its exchange hook."""
    _fields_ = [("nnb", C.c_int), ("rank", c_int_p), ("nsend", c_int_p), ("send_cols", c_int_p),
                ("nrecv", c_int_p), ("recv_cols", c_int_p), ("host_staged", C.c_int),
                ("exchange", HALO_FN), ("user", C.c_void_p),
                ("nsend_v", c_int_p), ("send_v", c_int_p), ("nrecv_v", c_int_p), ("recv_v", c_int_p),
                ("nsend_m", c_int_p), ("send_m", c_int_p), ("nrecv_m", c_int_p), ("recv_m", c_int_p)]


def make_halo(send, recv, fn, host_staged=True, vm=None):
    """A Halo over a plan {rank: local 0-based column indices} (olam_b200.decomp)
    and a Python hook fn(ranks, sendbufs, recvbufs) -> int on numpy views of
    the buffers (host-staged).  vm: (send_v, recv_v, send_m, recv_m) plans of
    the acoustic step, or None.  The returned struct keeps its arrays."""
    ranks = sorted(set(send) | set(recv) | (set().union(*[set(d) for d in vm]) if vm else set()))
    rk = np.array(ranks, np.int32)
    ns = np.array([len(send.get(r, ())) for r in ranks], np.int32)
    nr = np.array([len(recv.get(r, ())) for r in ranks], np.int32)
    sc = np.concatenate([np.asarray(send.get(r, []), np.int64) for r in ranks] + [np.zeros(0, np.int64)]) + 1
    rc = np.concatenate([np.asarray(recv.get(r, []), np.int64) for r in ranks] + [np.zeros(0, np.int64)]) + 1
    sc = np.ascontiguousarray(sc, np.int32)
    rc = np.ascontiguousarray(rc, np.int32)

    def hook(user, nnb, rank, sbuf, scount, rbuf, rcount, stream):
        try:
            sv = [np.ctypeslib.as_array(sbuf[i], shape=(scount[i],)) for i in range(nnb)]
            rv = [np.ctypeslib.as_array(rbuf[i], shape=(rcount[i],)) for i in range(nnb)]
            return int(fn([rank[i] for i in range(nnb)], sv, rv))
        except Exception:   # an exception must not cross the C frame
            return 1

    return _halo_struct(ranks, rk, ns, nr, sc, rc, hook, host_staged, vm)


def make_halo_device(send, recv, fn, vm=None):
    """A Halo whose hook gets the library's DEVICE buffers and stream:
    fn(ranks, sendbufs, recvbufs, stream) -> int, each buffer a pair
    (device pointer as int, float count), stream a cudaStream_t as int.
    The hook orders its transfers on that stream (CUDA-aware MPI, NCCL
    send/recv); the library unpacks after it returns, on the same stream."""
    ranks = sorted(set(send) | set(recv) | (set().union(*[set(d) for d in vm]) if vm else set()))
    rk = np.array(ranks, np.int32)
    ns = np.array([len(send.get(r, ())) for r in ranks], np.int32)
    nr = np.array([len(recv.get(r, ())) for r in ranks], np.int32)
    sc = np.ascontiguousarray(np.concatenate([np.asarray(send.get(r, []), np.int64) for r in ranks]
                                             + [np.zeros(0, np.int64)]) + 1, np.int32)
    rc = np.ascontiguousarray(np.concatenate([np.asarray(recv.get(r, []), np.int64) for r in ranks]
                                             + [np.zeros(0, np.int64)]) + 1, np.int32)

    def hook(user, nnb, rank, sbuf, scount, rbuf, rcount, stream):
        try:
            sb = [(C.cast(sbuf[i], C.c_void_p).value or 0, int(scount[i])) for i in range(nnb)]
            rb = [(C.cast(rbuf[i], C.c_void_p).value or 0, int(rcount[i])) for i in range(nnb)]
            return int(fn([rank[i] for i in range(nnb)], sb, rb, stream or 0))
        except Exception:   # an exception must not cross the C frame
            return 1

    return _halo_struct(ranks, rk, ns, nr, sc, rc, hook, False, vm)


def _halo_struct(ranks, rk, ns, nr, sc, rc, hook, host_staged, vm):
    h = Halo()
    h.nnb = len(ranks)
    h.rank, h.nsend, h.nrecv = ptr(rk, C.c_int), ptr(ns, C.c_int), ptr(nr, C.c_int)
    h.send_cols, h.recv_cols = ptr(sc, C.c_int), ptr(rc, C.c_int)
    h.host_staged = 1 if host_staged else 0
    h.exchange = HALO_FN(hook)
    h.user = None
    keep = [rk, ns, nr, sc, rc, h.exchange]
    if vm:
        names = (("nsend_v", "send_v"), ("nrecv_v", "recv_v"), ("nsend_m", "send_m"), ("nrecv_m", "recv_m"))
        for plan, (cname, lname) in zip(vm, names):
            cnt = np.array([len(plan.get(r, ())) for r in ranks], np.int32)
            idx = np.ascontiguousarray(np.concatenate([np.asarray(plan.get(r, []), np.int64) for r in ranks]
                                                      + [np.zeros(0, np.int64)]) + 1, np.int32)
            setattr(h, cname, ptr(cnt, C.c_int))
            setattr(h, lname, ptr(idx, C.c_int))
            keep += [cnt, idx]
    h.keep = tuple(keep)
    return h


# olamgpu_timestep flags
TS_GRAPH, TS_HORIZ_K, TS_MAXMIN, TS_MASS = 1, 2, 4, 8
WIN_HOST, WIN_LEAN = 1, 2


class Eddy(C.Structure):
    """olamgpu_eddy: the acoustic step's eddy-diffusion inputs."""
    _fields_ = [
        ("vkm", c_float_p), ("vkh", c_float_p), ("agamma", c_float_p), ("akm_sfc", c_float_p),
        ("sfluxt", c_float_p), ("kmtop", c_int_p), ("khtop", c_int_p), ("kpblh", c_int_p),
        ("theta", c_float_p), ("tair", c_float_p), ("akmodx", c_float_p), ("akhodx", c_float_p),
        ("kmtopv", c_int_p), ("khtopv", c_int_p), ("lsw", c_int_p), ("nsw_max", C.c_int),
        ("mrlw", c_int_p), ("mrlv", c_int_p), ("mrls", C.c_int), ("idiffk", c_int_p),
        ("akmin", c_float_p), ("test_case", C.c_int), ("cp", C.c_float),
        ("krayfmix_bot", C.c_int), ("rayf_cofmix", c_float_p),
    ]


def make_eddy(d):
    """An Eddy struct over the arrays of dict ``d`` (kept referenced by the
    returned struct's ``keep`` attribute)."""
    e = Eddy()
    keep = {}
    for name, ct in (("vkm", C.c_float), ("vkh", C.c_float), ("agamma", C.c_float),
                     ("akm_sfc", C.c_float), ("sfluxt", C.c_float), ("kmtop", C.c_int),
                     ("khtop", C.c_int), ("kpblh", C.c_int), ("theta", C.c_float),
                     ("tair", C.c_float), ("akmodx", C.c_float), ("akhodx", C.c_float),
                     ("kmtopv", C.c_int), ("khtopv", C.c_int), ("lsw", C.c_int), ("mrlw", C.c_int),
                     ("mrlv", C.c_int), ("idiffk", C.c_int), ("akmin", C.c_float),
                     ("rayf_cofmix", C.c_float)):
        a = d.get(name)
        if a is None:
            continue
        dt = np.int32 if ct is C.c_int else np.float32
        a = np.ascontiguousarray(a, dtype=dt)
        d[name] = a
        keep[name] = a
        setattr(e, name, ptr(a, ct))
    e.nsw_max, e.mrls, e.test_case = int(d["nsw_max"]), int(d["mrls"]), int(d["test_case"])
    e.cp, e.krayfmix_bot = float(d["cp"]), int(d["krayfmix_bot"])
    e.keep = keep
    return e


class CflDiag(C.Structure):
    _fields_ = [
        ("cfl_max", C.c_float), ("cfl_k", C.c_int), ("cfl_iwglobe", C.c_int),
        ("cflh_max", C.c_float), ("cflh_k", C.c_int), ("cflh_iwglobe", C.c_int),
        ("w_max", C.c_float), ("w_k", C.c_int), ("w_iwglobe", C.c_int),
    ]


def ptr(a, ctype):
    """Pointer to a contiguous numpy array (None stays NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))


class FortranGrid:
    """Fortran-layout copy of a synth Grid plus the ctypes struct over it.

    Keeps every array alive for as long as the struct is used.
    """

    def __init__(self, g):
        self.g = g
        keep = {}

        def i32(a, plus1=False):
            a = np.ascontiguousarray(a, dtype=np.int32)
            if plus1:
                a = a + 1          # 0-based array index -> OLAM's 1-based index
            keep[id(a)] = a
            return a

        def f32(a):
            a = np.ascontiguousarray(a, dtype=np.float32)
            keep[id(a)] = a
            return a

        def f64(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep[id(a)] = a
            return a

        s = Grid()
        s.mza, s.mwa, s.mva, s.mma = g.mza, g.mwa, g.mva, g.mma
        if hasattr(g, "jtw_prog"):
            # a rank's part of a decomposed grid (olam_b200.decomp): its own
            # loop tables, 1-based
            lists = {n: i32(getattr(g, n)) for n in ("jtw_prog", "jtw_wadj", "jtv_prog", "jtv_wadj",
                                                      "jtm_prog")}
            self.lists = lists
            s.nw_prog, s.jtw_prog = lists["jtw_prog"].size, ptr(lists["jtw_prog"], C.c_int)
            s.nw_wadj, s.jtw_wadj = lists["jtw_wadj"].size, ptr(lists["jtw_wadj"], C.c_int)
            s.nv_prog, s.jtv_prog = lists["jtv_prog"].size, ptr(lists["jtv_prog"], C.c_int)
            s.nv_wadj, s.jtv_wadj = lists["jtv_wadj"].size, ptr(lists["jtv_wadj"], C.c_int)
            s.nm_prog, s.jtm_prog = lists["jtm_prog"].size, ptr(lists["jtm_prog"], C.c_int)
        else:
            # global domain: every real point is prognostic and adjacent
            self.jtw = i32(np.arange(2, g.mwa + 1))
            self.jtv = i32(np.arange(2, g.mva + 1))
            self.jtm = i32(np.arange(2, g.mma + 1))
            s.nw_prog = s.nw_wadj = g.mwa - 1
            s.nv_prog = s.nv_wadj = g.mva - 1
            s.nm_prog = g.mma - 1
            s.jtw_prog = s.jtw_wadj = ptr(self.jtw, C.c_int)
            s.jtv_prog = s.jtv_wadj = ptr(self.jtv, C.c_int)
            s.jtm_prog = ptr(self.jtm, C.c_int)

        def tab(a):
            # tables hold 0-based array indices where 0 = dummy; entries past
            # npoly are 0 -> OLAM's 1 (the dummy point), as Fortran leaves them
            return i32(a, plus1=True)

        s.npoly = ptr(i32(g.npoly), C.c_int)
        s.itab_w_iv = ptr(tab(g.itab_w_iv), C.c_int)
        s.itab_w_iw = ptr(tab(g.itab_w_iw), C.c_int)
        s.itab_w_im = ptr(tab(g.itab_w_im), C.c_int)
        s.itab_w_dirv = ptr(f32(g.dirv), C.c_float)
        s.ecvec_vx = ptr(f32(g.ecvec_vx), C.c_float)
        s.ecvec_vy = ptr(f32(g.ecvec_vy), C.c_float)
        s.ecvec_vz = ptr(f32(g.ecvec_vz), C.c_float)
        s.iwglobe = ptr(i32(g.iwglobe), C.c_int)
        s.itab_v_iw = ptr(tab(g.itab_v_iw), C.c_int)
        s.itab_v_im = ptr(tab(g.itab_v_im), C.c_int)
        s.dxps = ptr(f32(g.dxps), C.c_float)
        s.dyps = ptr(f32(g.dyps), C.c_float)
        s.itab_m_iv = ptr(tab(g.itab_m_iv), C.c_int)
        s.itab_m_iw = ptr(tab(g.itab_m_iw), C.c_int)
        s.itab_m_im = ptr(tab(g.itab_m_im), C.c_int)
        s.lpw = ptr(i32(g.lpw), C.c_int)
        s.lpv = ptr(i32(g.lpv), C.c_int)
        s.lpm = ptr(i32(g.lpm), C.c_int)
        s.lve2 = ptr(i32(g.lve2), C.c_int)
        for name in ("zm", "zt", "dzm", "dzt", "dzim", "dzit", "dzt_top", "dzt_bot", "zfacit",
                     "gdz_wgtm", "gdz_wgtp", "wnx", "wny", "wnz", "wnxo2", "wnyo2", "wnzo2",
                     "vnx", "vny", "vnz", "dnu", "dniu", "dnv", "dniv", "arw0", "arm0",
                     "arv", "arw", "volti", "volwi", "volvi", "gxps_coef", "gyps_coef",
                     "xy_h", "xy_hu", "xx0_v", "xy0_v", "yy0_v", "xx0_vu", "xy0_vu", "yy0_vu",
                     "xx_yy", "xx_yy_m"):
            setattr(s, name, ptr(f32(getattr(g, name)), C.c_float))
        for name in ("zwgt_top8", "zwgt_bot8", "gdz_wgtm8", "gdz_wgtp8", "volt"):
            setattr(s, name, ptr(f64(getattr(g, name)), C.c_double))
        # a_w is Fortran (mza,2,2); the synth array is [i][j][k] -> [j][i][k]
        s.a_w = ptr(f32(np.transpose(g.a_w, (1, 0, 2))), C.c_float)
        s.a_wu = ptr(f32(np.transpose(g.a_wu, (1, 0, 2))), C.c_float)
        self.struct = s
        self._keep = keep


def make_opts(dtlm, nacoust=1, nrk_scal=2, nrk_wrtv=3, scal_order=2, thil_order=2,
              wind_order=2, iscal_monot=0, ithil_monot=0, iwind_monot=0,
              divh_damp_fact=0.1, divh_damp_level=3, divh_damp_short=1,
              vort_damp_fact=0.075, vort_damp_level=3, vort_damp_short=1,
              omega=7.29212e-5):
    o = Opts()
    o.dtlm = float(dtlm)
    o.nacoust = int(nacoust)
    o.dtsm = float(dtlm) / float(np.float32(nacoust))
    o.nrk_wrtv, o.nrk_scal = nrk_wrtv, nrk_scal
    o.thil_horiz_adv_order, o.wind_horiz_adv_order = thil_order, wind_order
    o.scal_horiz_adv_order = scal_order
    o.ithil_monot, o.iwind_monot, o.iscal_monot = ithil_monot, iwind_monot, iscal_monot
    o.divh_damp_fact, o.divh_damp_level, o.divh_damp_short = divh_damp_fact, divh_damp_level, divh_damp_short
    o.vort_damp_fact, o.vort_damp_level, o.vort_damp_short = vort_damp_fact, vort_damp_level, vort_damp_short
    o.fcoriol = np.float32(2.0 * omega)
    o.mdomain = 0
    o.krayf_bot = 10 ** 6
    o.krayfw_bot = 10 ** 6
    o.initial = 1
    return o


def ptr_array(arrays, ctype):
    """C array of pointers to the given numpy arrays."""
    arr_t = C.POINTER(ctype) * len(arrays)
    return arr_t(*[ptr(a, ctype) for a in arrays])
