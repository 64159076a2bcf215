"""Independent numpy restatement of OLAM's plain tracer update (test only).

Written separately from the C++ oracle, array-at-a-time, in float64, to
cross-check the oracle's loop-by-loop restatement:

* grad_t2d / grad_t2d_quadratic   omodel/grad_lib.f90:236-341
* scalar_v_column                 omodel/scalar_transport_rk.F90:474-534
* grad_z_quadratic                omodel/grad_lib.f90:166-229
* scalar_w_column                 omodel/scalar_transport_rk.F90:537-612
* the RK loop of scalar_transport_rk without implicit columns or limiters
  (scalar_transport_rk.F90:95-111, 137-152, 223-381)
* tracer_maxmin                   outils/check_nans.F90:164-203
* compute_mass_sums / mass_sum_from_*   outils/check_nans.F90:207-550

Arrays use the synth grid layout: (n, mza), slot 0 = dummy point.
"""
from __future__ import annotations

import numpy as np


def transport_plain(g, st, tracers, sct, dtlm, nrk=2, order=2):
    mza = g.mza
    vm = st.vmasc.astype(np.float64)
    wm = st.wmasc.astype(np.float64)
    rho_old = st.rho_old.astype(np.float64)
    rho = st.rho.astype(np.float64)
    if nrk == 3:
        rhos = rho            # update_scalar receives rhos(:,:,nrk) = rho
        dtlr = dtlm * np.array([1.0 / 3.0, 0.5, 1.0])
    else:
        rhos = rho
        dtlr = dtlm * np.array([0.5, 1.0])
    del rho_old
    out = []
    for q0, t0 in zip(tracers, sct):
        q0 = q0.astype(np.float64)
        t0 = t0.astype(np.float64)
        s = q0.copy()
        for ist in range(nrk):
            s = plain_stage(g, vm, wm, rhos, s, q0, t0, dtlr[ist], order)
        out.append(s)
    return np.stack(out)


def plain_stage(g, vm, wm, rhos, s, q0, t0, dtr, order=2):
    """One update_scalar call (explicit columns), float64."""
    mza = g.mza
    vm = vm.astype(np.float64)
    wm = wm.astype(np.float64)
    nb = g.itab_w_iw.astype(np.int64)
    ev = g.itab_w_iv.astype(np.int64)
    valid = np.arange(7)[None, :] < g.npoly[:, None]
    dirv = g.dirv.astype(np.float64) * valid
    iw1, iw2 = g.itab_v_iw[:, 0].astype(np.int64), g.itab_v_iw[:, 1].astype(np.int64)
    volti = g.volti.astype(np.float64)
    aw = g.a_w.astype(np.float64)              # [i][j][k]
    d = (s[nb] - s[:, None, :]) * valid[..., None]        # (mwa, 7, mza)
    if order == 2:
        gx = np.einsum("wn,wnk->wk", g.gxps_coef.astype(np.float64), d)
        gy = np.einsum("wn,wnk->wk", g.gyps_coef.astype(np.float64), d)
        planes = [gx, gy]
        coef = [g.dxps, g.dyps]
    else:
        planes = [np.einsum("wn,wnk->wk", g.xy_h[:, :, m].astype(np.float64), d)
                  for m in range(5)]
        coef = [g.dxps, g.dyps, g.xx0_v, g.xy0_v, g.yy0_v]
    s1 = s[iw1].copy()
    s2 = s[iw2].copy()
    for c, p in zip(coef, planes):
        s1 += c[:, 0, None].astype(np.float64) * p[iw1]
        s2 += c[:, 1, None].astype(np.float64) * p[iw2]
    upv = np.where(vm < 0, s2, s1)
    # horizontal flux divergence
    fd = np.einsum("wn,wnk->wk", dirv, vm[ev] * (upv[ev] - q0[:, None, :]))
    # vertical quadratic reconstruction (bounded, zero-gradient BCs);
    # dsk[:, kd] = ds at the top of level kd, dskm1[:, kd] below it
    dsk = np.zeros((g.mwa, mza))
    dskm1 = np.zeros((g.mwa, mza))
    dsk[:, 1:mza - 1] = s[:, 2:] - s[:, 1:-1]
    dskm1[:, 2:] = s[:, 2:] - s[:, 1:-1]
    sb = s + dsk * aw[0, 0][None] + dskm1 * aw[1, 0][None]
    stp = s + dsk * aw[0, 1][None] + dskm1 * aw[1, 1][None]
    upw = np.zeros((g.mwa, mza))
    upw[:, 0] = s[:, 1]                            # scp_upw(kb-1) = scp(kb)
    upw[:, 1:mza - 1] = np.where(wm[:, 1:mza - 1] < 0, sb[:, 2:mza], stp[:, 1:mza - 1])
    upw[:, mza - 1] = s[:, mza - 1]                # scp_upw(mza) = scp(mza)
    wmm1 = np.concatenate([np.zeros((g.mwa, 1)), wm[:, :-1]], axis=1)
    upm1 = np.concatenate([np.zeros((g.mwa, 1)), upw[:, :-1]], axis=1)
    fd = fd + (wmm1 * (upm1 - q0) - wm * (upw - q0))
    new = q0 + dtr * (t0 + volti * fd) / np.where(rhos == 0, 1.0, rhos)
    new[:, 0] = new[:, 1]
    new[0] = 0.0
    return new


def limited_last_stage(g, scp, scp0, rhos, vm, wm, dtr, mode, order=2):
    """One update_scalar_monot (mode 1) or update_scalar_pd (mode 2) call,
    explicit columns only (scalar_transport_rk.F90:619-1081, 1085-1472),
    float64, array-at-a-time.  scp is the stage input, scp0 the (already
    pre-updated) starting value, rhos = rhos(:,:,nrk)."""
    mza = g.mza
    monot = mode == 1
    s = scp.astype(np.float64)
    q0 = scp0.astype(np.float64)
    vm = vm.astype(np.float64)
    wm = wm.astype(np.float64)
    nb = g.itab_w_iw.astype(np.int64)
    ev = g.itab_w_iv.astype(np.int64)
    valid = np.arange(7)[None, :] < g.npoly[:, None]
    dirv = g.dirv.astype(np.float64) * valid
    iw1, iw2 = g.itab_v_iw[:, 0].astype(np.int64), g.itab_v_iw[:, 1].astype(np.int64)
    volti = g.volti.astype(np.float64)
    d = (s[nb] - s[:, None, :]) * valid[..., None]
    if order == 2:
        planes = [np.einsum("wn,wnk->wk", g.gxps_coef.astype(np.float64), d),
                  np.einsum("wn,wnk->wk", g.gyps_coef.astype(np.float64), d)]
        coef = [g.dxps, g.dyps]
    else:
        xy = g.xy_hu if monot else g.xy_h
        planes = [np.einsum("wn,wnk->wk", xy[:, :, m].astype(np.float64), d) for m in range(5)]
        coef = [g.dxps, g.dyps] + ([g.xx0_vu, g.xy0_vu, g.yy0_vu] if monot
                                   else [g.xx0_v, g.xy0_v, g.yy0_v])
    s1 = s[iw1].copy()
    s2 = s[iw2].copy()
    for c, p in zip(coef, planes):
        s1 += c[:, 0, None].astype(np.float64) * p[iw1]
        s2 += c[:, 1, None].astype(np.float64) * p[iw2]
    neg = vm < 0
    lo = np.where(neg, q0[iw2], q0[iw1])
    hiv = np.where(neg, s2, s1) - lo
    sfv = vm * hiv
    # vertical reconstruction: monot = unbounded with constant-gradient BCs
    aw = (g.a_wu if monot else g.a_w).astype(np.float64)
    dsk = np.zeros((g.mwa, mza))
    dskm1 = np.zeros((g.mwa, mza))
    dsk[:, 1:mza - 1] = s[:, 2:] - s[:, 1:-1]
    dskm1[:, 2:] = s[:, 2:] - s[:, 1:-1]
    if monot:
        dskm1[:, 1] = dsk[:, 1]
        dsk[:, mza - 1] = dskm1[:, mza - 1]
    sb = s + dsk * aw[0, 0][None] + dskm1 * aw[1, 0][None]
    stp = s + dsk * aw[0, 1][None] + dskm1 * aw[1, 1][None]
    # low-order face values (face j between levels j and j+1), j = 0..mza-1
    low = np.zeros((g.mwa, mza))
    low[:, 0] = q0[:, 1] if monot else s[:, 1]
    low[:, mza - 1] = q0[:, mza - 1] if monot else s[:, mza - 1]
    low[:, 1:mza - 1] = np.where(wm[:, 1:mza - 1] < 0, q0[:, 2:mza], q0[:, 1:mza - 1])
    hiw = np.zeros((g.mwa, mza))
    hiw[:, 1:mza - 1] = np.where(wm[:, 1:mza - 1] < 0, sb[:, 2:mza], stp[:, 1:mza - 1]) - low[:, 1:mza - 1]
    sfw = wm * hiw
    sfw[:, 0] = 0
    sfw[:, mza - 1] = 0
    sfwm1 = np.concatenate([np.zeros((g.mwa, 1)), sfw[:, :-1]], axis=1)
    wmm1 = np.concatenate([np.zeros((g.mwa, 1)), wm[:, :-1]], axis=1)
    lowm1 = np.concatenate([np.zeros((g.mwa, 1)), low[:, :-1]], axis=1)
    dvm = dirv[..., None] * vm[ev]
    fl = np.einsum("wnk->wk", dvm * (lo[ev] - q0[:, None, :]))
    fl = fl + wmm1 * (lowm1 - q0) - wm * (low - q0)
    fout = np.minimum(dirv[..., None] * sfv[ev], 0).sum(1) + np.minimum(sfwm1, 0) - np.maximum(sfw, 0)
    fin = np.maximum(dirv[..., None] * sfv[ev], 0).sum(1) + np.maximum(sfwm1, 0) - np.minimum(sfw, 0)
    rh = np.where(rhos == 0, 1.0, rhos.astype(np.float64))
    rscp_low = q0 * rh + dtr * volti * fl
    eps0, eps1 = 1e-32, 3e-7
    if monot:
        smax = q0.copy()
        smin = q0.copy()
        up_in = np.zeros((g.mwa, mza), bool)
        up_in[:, 2:] = wm[:, 1:mza - 1] > 0
        q0m1 = np.concatenate([q0[:, :1], q0[:, :-1]], axis=1)
        smax = np.where(up_in, np.maximum(smax, q0m1), smax)
        smin = np.where(up_in, np.minimum(smin, q0m1), smin)
        dn_in = np.zeros((g.mwa, mza), bool)
        dn_in[:, 1:mza - 1] = wm[:, 1:mza - 1] < 0
        q0p1 = np.concatenate([q0[:, 1:], q0[:, -1:]], axis=1)
        smax = np.where(dn_in, np.maximum(smax, q0p1), smax)
        smin = np.where(dn_in, np.minimum(smin, q0p1), smin)
        inflow = dvm > 0
        qn = q0[nb]
        smax = np.maximum(smax, np.where(inflow, qn, -np.inf).max(1))
        smin = np.minimum(smin, np.where(inflow, qn, np.inf).min(1))
        smax = rh * smax
        smin = rh * smin
        dtrp = (1 + eps1) * dtr
        flux_in = np.maximum(dtrp * volti * fin, eps0)
        flux_out = np.minimum(dtrp * volti * fout, -eps0)
        epsr = eps1 * np.abs(rscp_low)
        sc_in = np.maximum(smax - (rscp_low + epsr) - eps0, 0)
        sc_out = np.minimum(smin - (rscp_low - epsr) + eps0, 0)
        s_in = np.minimum(1, sc_in / np.maximum(flux_in, 0.01 * sc_in))
        s_out = np.minimum(1, sc_out / np.minimum(flux_out, 0.01 * sc_out))
        s_in1 = np.concatenate([s_in[:, 1:], s_in[:, -1:]], axis=1)
        s_out1 = np.concatenate([s_out[:, 1:], s_out[:, -1:]], axis=1)
        scw = np.where(sfw < 0, np.minimum(s_in, s_out1), np.minimum(s_in1, s_out))
        scv = np.where(sfv < 0, np.minimum(s_in[iw1], s_out[iw2]), np.minimum(s_in[iw2], s_out[iw1]))
    else:
        mdtrp = -(1 + eps1) * dtr
        flux_out = np.maximum(mdtrp * volti * fout, eps0)
        sc_out = np.maximum((1 - eps1) * rscp_low - eps0, 0)
        so = np.minimum(1, sc_out / np.maximum(flux_out, 0.01 * sc_out))
        so1 = np.concatenate([so[:, 1:], so[:, -1:]], axis=1)
        scw = np.where(sfw < 0, so1, so)
        scv = np.where(sfv < 0, so[iw2], so[iw1])
    upw = low.copy()
    upw[:, 1:mza - 1] = low[:, 1:mza - 1] + hiw[:, 1:mza - 1] * scw[:, 1:mza - 1]
    upv = lo + hiv * scv
    fd = np.einsum("wnk->wk", dvm * (upv[ev] - q0[:, None, :]))
    upwm1 = np.concatenate([np.zeros((g.mwa, 1)), upw[:, :-1]], axis=1)
    fd = fd + wmm1 * (upwm1 - q0) - wm * (upw - q0)
    new = q0 + dtr * volti * fd / rh
    new[:, 0] = s[:, 0]       # level 1 is not written: it keeps the stage input
    new[0] = 0.0
    return new


def tracer_maxmin(scp, lpw):
    """(ntr, 2): max and -min of each scalar over columns 1.. (every W point
    is in jtw_prog on the synth grid), levels lpw..mza; NaNs skipped."""
    ntr, mwa, mza = scp.shape
    out = np.full((ntr, 2), -np.finfo(np.float32).max, np.float32)
    for iw in range(1, mwa):
        kb = int(lpw[iw]) - 1
        col = scp[:, iw, kb:]
        with np.errstate(invalid="ignore"):
            hi = np.nanmax(np.where(np.isnan(col), -np.inf, col), axis=1)
            lo = np.nanmin(np.where(np.isnan(col), np.inf, col), axis=1)
        out[:, 0] = np.maximum(out[:, 0], hi)
        out[:, 1] = np.maximum(out[:, 1], -lo)
    return out


def mass_sums(rho, volt, scalars, lpw):
    """[sum rho volt, sum rho volt s for s in scalars] over columns 1..,
    levels lpw..mza, in float64 (rho * volt first, as the reference)."""
    out = np.zeros(1 + len(scalars))
    mwa = rho.shape[0]
    for iw in range(1, mwa):
        kb = int(lpw[iw]) - 1
        rv = rho[iw, kb:].astype(np.float64) * volt[iw, kb:].astype(np.float64)
        out[0] += rv.sum()
        for i, s in enumerate(scalars):
            out[1 + i] += (rv * s[iw, kb:].astype(np.float64)).sum()
    return out
