"""Independent numpy restatement of OLAM's plain tracer update (test only).

Written separately from the C++ oracle, array-at-a-time, in float64, to
cross-check the oracle's loop-by-loop restatement:

* grad_t2d / grad_t2d_quadratic   omodel/grad_lib.f90:236-341
* scalar_v_column                 omodel/scalar_transport_rk.F90:474-534
* grad_z_quadratic                omodel/grad_lib.f90:166-229
* scalar_w_column                 omodel/scalar_transport_rk.F90:537-612
* the RK loop of scalar_transport_rk without implicit columns or limiters
  (scalar_transport_rk.F90:95-111, 137-152, 223-381)

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
    nb = g.itab_w_iw.astype(np.int64)          # (mwa, 7)
    ev = g.itab_w_iv.astype(np.int64)
    npoly = g.npoly
    valid = np.arange(7)[None, :] < npoly[:, None]
    dirv = g.dirv.astype(np.float64) * valid
    iw1, iw2 = g.itab_v_iw[:, 0].astype(np.int64), g.itab_v_iw[:, 1].astype(np.int64)
    volti = g.volti.astype(np.float64)
    aw = g.a_w.astype(np.float64)              # [i][j][k]
    out = []
    for q0, t0 in zip(tracers, sct):
        q0 = q0.astype(np.float64)
        t0 = t0.astype(np.float64)
        s = q0.copy()
        for ist in range(nrk):
            dtr = dtlr[ist]
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
            # vertical quadratic reconstruction (bounded, zero-gradient BCs)
            ds = np.zeros((g.mwa, mza + 1))
            ds[:, 1:mza - 1] = s[:, 2:] - s[:, 1:-1]       # ds(k) for k = 2..mza-1 (Fortran)
            # Fortran ds(k) at array index k-1 here: ds[:, j] holds ds(j+1)
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
            s = new
        out.append(s)
    return np.stack(out)
