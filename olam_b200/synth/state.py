"""Seeded synthetic atmospheric states for the benchmark configurations.

Everything here is written from the mathematics; no reference initial
condition code is used.  Arrays follow the layout of ``grid.py``: ``(n, mza)``
C-contiguous (Fortran ``(mza, n)``), slot 0 = OLAM's dummy point.

* Dry atmosphere: ``thil = theta``; pressure from OLAM's equation of state
  ``p = alpha_press * (rho*thil)**(cp/cv)`` with ``alpha_press = pc1*rdry**cpocv``
  (``modules/mem_basic.f90:50,101-109``).
* Transport winds: ``vmasc`` is the long-step mean horizontal mass flux through
  a V face (``vmc*arv``), ``wmasc`` through a W face; the end-of-step density
  is advanced from ``rho_old`` with the same discrete divergence, as OLAM's
  acoustic solver does (``omodel/prog_wrtv_rk.f90:823``), so density and
  tracer mass stay consistent.
"""
from __future__ import annotations

import numpy as np

from .grid import ERAD, F32

CP, CV = 1004.0, 717.0
RDRY = CP - CV
P00 = 1.0e5
GRAV = 9.81
OMEGA = 7.29212e-5
ROCP = RDRY / CP
CPOCV = CP / CV
PC1 = (1.0 / P00) ** (RDRY / CV)
ALPHA_DRY = np.float32(PC1 * RDRY ** CPOCV)


class State:
    pass


def _latlon(g):
    return np.radians(g.glatw.astype(np.float64)), np.radians(g.glonw.astype(np.float64))


def _east_north(lat, lon):
    east = np.stack([-np.sin(lon), np.cos(lon), np.zeros_like(lon)], axis=-1)
    north = np.stack([-np.sin(lat) * np.cos(lon), -np.sin(lat) * np.sin(lon), np.cos(lat)],
                     axis=-1)
    return east, north


def hydrostatic(g, t_sfc=250.0, lapse=0.0, p_sfc=1.0e5, theta_pert=None):
    """Temperature/pressure/density columns at T levels (float64, (mwa, mza))."""
    zt = g.zt.astype(np.float64)
    temp = np.maximum(t_sfc - lapse * zt, 200.0 if lapse > 0 else 1.0)
    # integrate d ln p / dz = -g/(R T) exactly for piecewise-linear T
    z = np.linspace(0.0, zt.max() + 1.0, 4001)
    tz = np.maximum(t_sfc - lapse * z, 200.0 if lapse > 0 else 1.0)
    lnp = np.log(p_sfc) - np.concatenate(
        [[0.0], np.cumsum(0.5 * (GRAV / (RDRY * tz[1:]) + GRAV / (RDRY * tz[:-1]))
                          * np.diff(z))])
    p = np.exp(np.interp(zt, z, lnp))
    theta = temp * (P00 / p) ** ROCP
    th = np.broadcast_to(theta, (g.mwa, g.mza)).copy()
    if theta_pert is not None:
        th += theta_pert
    # density from the equation of state with the (possibly perturbed) theta
    pc = np.broadcast_to(p, (g.mwa, g.mza)).copy()
    rho = (pc / float(ALPHA_DRY)) ** (1.0 / CPOCV) / th
    return th, pc, rho


def zonal_wind(g, kind, amp):
    """Eastward wind u(lat, z) at V points, returned as a 3-D vector field."""
    latv = np.radians(g.glatv.astype(np.float64))
    lonv = np.radians(g.glonv.astype(np.float64))
    east, _ = _east_north(latv, lonv)
    zt = g.zt.astype(np.float64)
    if kind == "solid":
        prof = np.cos(latv)[:, None] * np.ones_like(zt)[None, :]
    else:  # mid-latitude jets centred at +-45 deg, peaking at 10 km
        prof = (np.exp(-((np.abs(latv) - np.radians(45.0)) / np.radians(12.0)) ** 2)[:, None]
                * np.exp(-((zt - 1.0e4) / 6.0e3) ** 2)[None, :])
    u = amp * prof
    return u[..., None] * east[:, None, :]          # (mva, mza, 3)


def vertical_mass_flux(g, rho, amp, seed):
    """A smooth seeded W-face mass flux (kg/s) with both signs, zero at bottom/top."""
    rng = np.random.default_rng(seed)
    lat, lon = _latlon(g)
    a, b, c = rng.uniform(0, 2 * np.pi, 3)
    horiz = np.sin(3 * lon + a) * np.cos(2 * lat + b) + 0.5 * np.sin(5 * lon - c)
    zm = g.zm.astype(np.float64)
    ztop = zm[-1]
    vert = np.sin(np.pi * np.clip(zm / ztop, 0, 1))
    rhow = 0.5 * (rho + np.roll(rho, -1, axis=1))
    w = amp * horiz[:, None] * vert[None, :]                 # m/s
    wm = w * rhow * g.arw.astype(np.float64)
    wm[:, 0] = 0.0
    wm[:, -1] = 0.0
    wm[0] = 0.0
    return wm


def flux_divergence(g, vmasc, wmasc):
    """Sum_j dirv*vmasc + wmasc(k-1) - wmasc(k) for every W column (float64)."""
    iv = g.itab_w_iv
    div = np.einsum("nj,njk->nk", g.dirv.astype(np.float64), vmasc[iv].astype(np.float64))
    w = wmasc.astype(np.float64)
    wm1 = np.concatenate([np.zeros((g.mwa, 1)), w[:, :-1]], axis=1)
    return div + wm1 - w


def transport_state(g, dtlm, ntr, jet_amp=35.0, w_amp=0.05, seed=1234,
                    tracer_kind="lognormal", median=1.0e-8, sigma_ln=1.5,
                    clip=(1.0e-12, 1.0e-6), zero_frac=0.1, zero_above=15000.0,
                    bell=None, solid=False, t_sfc=300.0, lapse=6.5e-3):
    """Inputs of ``scalar_transport_rk``: winds, densities and tracers.

    Returns a State with ``vmasc (mva,mza) f32``, ``wmasc (mwa,mza) f32``,
    ``rho_old (mwa,mza) f32``, ``rho (mwa,mza) f64``, ``wc`` and
    ``tracers (ntr, mwa, mza) f32`` plus zero tendencies ``sct``.
    """
    rng = np.random.default_rng(seed)
    s = State()
    th, p, rho0 = hydrostatic(g, t_sfc=t_sfc, lapse=lapse)
    uvec = zonal_wind(g, "solid" if solid else "jet", jet_amp)
    vn = np.stack([g.vnx, g.vny, g.vnz], axis=1).astype(np.float64)
    vc = np.einsum("vkc,vc->vk", uvec, vn)
    iw1, iw2 = g.itab_v_iw[:, 0], g.itab_v_iw[:, 1]
    rhov = 0.5 * (rho0[iw1] + rho0[iw2])
    vmasc = (rhov * vc * g.arv.astype(np.float64)).astype(F32)
    vmasc[0] = 0.0
    vmasc[:, 0] = 0.0
    wmasc = vertical_mass_flux(g, rho0, w_amp, seed + 1).astype(F32)
    rho_old = rho0.astype(F32)
    rho_old[0] = 0.0
    div = flux_divergence(g, vmasc, wmasc)
    rho = rho_old.astype(np.float64) + dtlm * g.volti.astype(np.float64) * div
    rho[:, 0] = rho[:, 1]
    rho[0] = 0.0
    s.vmasc, s.wmasc, s.rho_old, s.rho = vmasc, wmasc, rho_old, rho
    # wc for check_cfls' max-|W| diagnostic
    s.wc = (wmasc.astype(np.float64) / np.maximum(
        0.5 * (rho0 + np.roll(rho0, -1, axis=1)) * g.arw.astype(np.float64), 1e-30)
    ).astype(F32)
    s.wc[0] = 0.0
    mza = g.mza
    if tracer_kind == "bell":
        lat, lon = _latlon(g)
        lat0, lon0 = bell if bell is not None else (
            rng.uniform(-0.6, 0.6), rng.uniform(-np.pi, np.pi))
        d = np.arccos(np.clip(np.sin(lat) * np.sin(lat0)
                              + np.cos(lat) * np.cos(lat0) * np.cos(lon - lon0), -1, 1))
        r = d * ERAD
        q = np.where(r < 1.5e6, 0.5 * (1.0 + np.cos(np.pi * r / 1.5e6)), 0.0)
        tr = np.broadcast_to(q[:, None], (g.mwa, mza)).astype(F32)[None].copy()
        tr = np.repeat(tr, ntr, axis=0)
    else:
        # lognormal fields: smooth horizontal/vertical structure per tracer
        lat, lon = _latlon(g)
        zt = g.zt.astype(np.float64)
        tr = np.empty((ntr, g.mwa, mza), dtype=F32)
        for n in range(ntr):
            a = rng.uniform(0, 2 * np.pi, 4)
            m1, m2 = rng.integers(1, 6, 2)
            field = (np.sin(m1 * lon + a[0])[:, None] * np.cos(m2 * lat + a[1])[:, None]
                     + 0.5 * np.sin(2 * np.pi * zt / rng.uniform(5e3, 3e4) + a[2])[None, :])
            field += 0.3 * rng.standard_normal((g.mwa, 1))
            x = median * np.exp(sigma_ln * field / 1.2)
            x = np.clip(x, clip[0], clip[1])
            tr[n] = x.astype(F32)
        nz = int(round(zero_frac * ntr))
        if nz > 0:
            sel = rng.choice(ntr, nz, replace=False)
            above = zt > zero_above
            for n in sel:
                tr[n][:, above] = 0.0
    tr[:, 0] = 0.0
    # below-ground level k=1 mirrors k=lpw=2, as OLAM keeps it
    tr[:, :, 0] = tr[:, :, 1]
    s.tracers = tr
    s.sct = np.zeros_like(tr)
    s.ntr = ntr
    return s


def dynamics_state(g, jet_amp=35.0, kind="jet", t_sfc=300.0, lapse=6.5e-3,
                   theta_sigma=0.5, theta_scale=5.0e5, seed=99):
    """Full prognostic state for ``prog_wrtv_rk`` (module mem_basic arrays)."""
    rng = np.random.default_rng(seed)
    lat, lon = _latlon(g)
    pert = None
    if theta_sigma > 0:
        lat0, lon0 = rng.uniform(-0.8, 0.8), rng.uniform(-np.pi, np.pi)
        d = np.arccos(np.clip(np.sin(lat) * np.sin(lat0)
                              + np.cos(lat) * np.cos(lat0) * np.cos(lon - lon0), -1, 1))
        r = d * ERAD
        zt = g.zt.astype(np.float64)
        pert = (theta_sigma * np.exp(-(r / theta_scale) ** 2)[:, None]
                * np.exp(-((zt - 5.0e3) / 3.0e3) ** 2)[None, :])
    th, p, rho = hydrostatic(g, t_sfc=t_sfc, lapse=lapse, theta_pert=pert)
    s = State()
    s.thil = th.astype(F32)
    s.theta = th.astype(F32)
    s.rho = rho.copy()
    s.rho[0] = 0.0
    rt = (rho * th.astype(F32).astype(np.float64))
    s.press = float(ALPHA_DRY) * rt ** CPOCV
    s.press[0] = 0.0
    uvec = zonal_wind(g, kind, jet_amp)
    vn = np.stack([g.vnx, g.vny, g.vnz], axis=1).astype(np.float64)
    vc = np.einsum("vkc,vc->vk", uvec, vn)
    iw1, iw2 = g.itab_v_iw[:, 0], g.itab_v_iw[:, 1]
    rhov = 0.5 * (rho[iw1] + rho[iw2])
    s.vc = vc.astype(F32)
    s.vmc = (rhov * vc).astype(F32)
    s.vc[0] = 0.0
    s.vmc[0] = 0.0
    s.wc = np.zeros((g.mwa, g.mza), dtype=F32)
    s.wmc = np.zeros((g.mwa, g.mza), dtype=F32)
    # earth-cartesian velocity as vel_t3d_hex would diagnose it
    s.vxe = np.einsum("nj,njk->nk", g.ecvec_vx, s.vc[g.itab_w_iv]).astype(F32)
    s.vye = np.einsum("nj,njk->nk", g.ecvec_vy, s.vc[g.itab_w_iv]).astype(F32)
    s.vze = np.einsum("nj,njk->nk", g.ecvec_vz, s.vc[g.itab_w_iv]).astype(F32)
    for a in (s.vxe, s.vye, s.vze):
        a[:, 0] = a[:, 1]
        a[0] = 0.0
    s.alpha_press = np.full((g.mwa, g.mza), ALPHA_DRY, dtype=F32)
    s.pwfac = np.broadcast_to(g.dzim, (g.mwa, g.mza)).astype(F32).copy()
    s.pvfac = (g.zfacit[None, :] * g.dniv[:, None]).astype(F32)
    return s


def fast_lognormal_tracers(g, ntr, seed=2024, median=1.0e-8, sigma_ln=1.5,
                           clip=(1.0e-12, 1.0e-6), zero_frac=0.1, zero_above=15000.0,
                           dtype=np.float32, as_list=False, cols=None):
    """Large-case tracer fields: seeded lognormal mixing ratios, separable in
    horizontal and vertical so that 100+ full-size fields generate quickly.

    q_n(iw, k) = median * exp(sigma * (h_n(iw) + v_n(k))) clipped to ``clip``;
    ``zero_frac`` of the tracers are zero above ``zero_above`` metres.
    Returns (ntr, mwa, mza) in ``dtype``, or with ``as_list`` a list of
    separately allocated (mwa, mza) arrays (one allocation per tracer, as
    OLAM allocates each scalar_tab(n)%var_p).
    """
    rng = np.random.default_rng(seed)
    lat, lon = _latlon(g)
    zt = g.zt.astype(np.float64)
    # cols: only these W points (a rank's part of the grid), in this order;
    # the values are those of the whole-grid fields at those points
    nw = g.mwa if cols is None else len(cols)
    out = ([np.empty((nw, g.mza), dtype=dtype) for _ in range(ntr)] if as_list
           else np.empty((ntr, nw, g.mza), dtype=dtype))
    nz = int(round(zero_frac * ntr))
    zsel = set(rng.choice(ntr, nz, replace=False).tolist()) if nz else set()
    above = zt > zero_above
    for n in range(ntr):
        a = rng.uniform(0, 2 * np.pi, 3)
        m1, m2 = rng.integers(1, 6, 2)
        h = np.sin(m1 * lon + a[0]) * np.cos(m2 * lat + a[1]) + 0.3 * rng.standard_normal(g.mwa)
        v = 0.5 * np.sin(2 * np.pi * zt / rng.uniform(5e3, 3e4) + a[2])
        if cols is not None:
            h = h[cols]
        eh = (median * np.exp(sigma_ln * h / 1.2)).astype(np.float32)
        ev = np.exp(sigma_ln * v / 1.2).astype(np.float32)
        q = out[n]
        np.multiply(eh[:, None], ev[None, :], out=q)
        np.clip(q, clip[0], clip[1], out=q)
        if n in zsel:
            q[:, above] = 0.0
        q[0] = 0.0
        q[:, 0] = q[:, 1]
    return out


def eddy_inputs(g, rho, thil, press, akmin=0.0, idiffk=1, rayf_mix=False, seed=7):
    """Seeded stand-ins for the PBL scheme's outputs that the acoustic step's
    eddy diffusion reads (convect/mem_turb.f90 arrays, OLAM layout): a
    boundary layer 0.8-1.6 km deep with K(z) = Kmax (z/h)(1 - z/h)^2 scaled
    by density, a small non-local heat term, a surface heat flux and a
    surface momentum exchange on the lowest level.  Returns a dict of
    numpy arrays and scalars for ``abi.make_eddy``."""
    rng = np.random.default_rng(seed)
    mwa, mza, mva = g.mwa, g.mza, g.mva
    zm = g.zm.astype(np.float64)                       # W-level heights, Fortran k = index + 1
    h = rng.uniform(800.0, 1600.0, mwa)                 # boundary-layer depth per column
    kmax_m, kmax_h = rng.uniform(20.0, 60.0, mwa), rng.uniform(25.0, 80.0, mwa)
    z = zm[None, :] / h[:, None]
    shape = np.where((z > 0) & (z < 1), z * (1 - z) ** 2 * 6.75, 0.0)   # peak 1 at z = h/3
    rhow = rho.astype(np.float64)
    vkm = (rhow * kmax_m[:, None] * shape).astype(F32)
    vkh = (rhow * kmax_h[:, None] * shape).astype(F32)
    # top W level (1-based) with a nonzero coefficient
    top = np.array([int(np.max(np.nonzero(shape[i] > 0)[0])) + 1 if (shape[i] > 0).any() else 0
                    for i in range(mwa)], np.int32)
    kpblh = np.maximum(top - 1, 1).astype(np.int32)
    agamma = (1.0e-3 * g.arw.astype(np.float64) * np.clip(1 - z, 0, 1) * (z > 0)).astype(F32)
    sfluxt = rng.uniform(50.0, 200.0, mwa).astype(F32)
    theta = thil.astype(F32).copy()
    tair = (theta.astype(np.float64) * (np.maximum(press, 1.0) / P00) ** ROCP).astype(F32)
    nsw_max = 1
    akm_sfc = rng.uniform(0.01, 0.05, (mwa, nsw_max)).astype(F32)
    for a in (vkm, vkh, agamma, theta, tair):
        a[0] = 0
    sfluxt[0] = 0
    akm_sfc[0] = 0
    top[0] = 0
    kpblh[0] = 0
    rayf = None
    krayfmix_bot = mza + 1
    if rayf_mix:
        krayfmix_bot = mza - 2
        rayf = np.zeros(mza, F32)
        rayf[krayfmix_bot - 1:mza - 1] = np.array([0.02, 0.05], F32)   # m/s, like K / dz
    return dict(vkm=vkm, vkh=vkh, agamma=agamma, akm_sfc=akm_sfc, sfluxt=sfluxt, kmtop=top.copy(),
                khtop=top.copy(), kpblh=kpblh, theta=theta, tair=tair,
                akmodx=np.zeros((mva, mza), F32), akhodx=np.zeros((mva, mza), F32),
                kmtopv=np.ones(mva, np.int32), khtopv=np.ones(mva, np.int32),
                lsw=np.ones(mwa, np.int32), nsw_max=nsw_max, mrlw=np.ones(mwa, np.int32),
                mrlv=np.ones(mva, np.int32), mrls=1, idiffk=np.array([idiffk], np.int32),
                akmin=np.array([akmin], F32), test_case=0, cp=CP, krayfmix_bot=krayfmix_bot,
                rayf_cofmix=rayf)
