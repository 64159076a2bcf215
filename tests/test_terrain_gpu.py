"""scalar_transport_rk on a grid with terrain through the C-ABI: a mountain
raises the lowest prognosed level lpw of the columns under it (up to 4
levels) and every face takes the higher floor of its two cells (lpv), so
the reconstruction and the flux divergence drop faces and gradient terms
level by level (the reference's loops start at lpv and lpw).  The tiled
and plain forms are checked against the oracle, and against themselves
with NaN below every floor (values the reference never reads); the tiled
adjoint against the oracle's adjoint; prog_wrtv_rk's long step (with the
prognostic shaved-cell method of the columns beside higher ones) against
the oracle and olamgpu_timestep against the single calls."""
import numpy as np
import pytest

import oracle_lib
from conftest import relerr, small_case
from olam_b200 import abi
from olam_b200.lib import HostState, OlamGpu, OlamGpuError
from test_transport_gpu import TOL32, TOL64

pytestmark = pytest.mark.gpu


def terrain_grid(g0, hmax=4):
    from olam_b200.synth.grid import with_terrain
    return with_terrain(g0, hmax)


def terrain_case(nxp=6, nlev=12, ntr=6, hmax=4, **kw):
    g0, st0 = small_case(nxp=nxp, nlev=nlev, ntr=ntr, **kw)
    return terrain_grid(g0, hmax), st0


def run(g, st, opts, form, tracers=None, prof=False):
    hs = HostState(vmasc=st.vmasc, wmasc=st.wmasc, rho=st.rho, wc=st.wc)
    dev = OlamGpu(abi.FortranGrid(g), opts, hs)
    try:
        dev.set_transport_form(form)
        var_p = [np.ascontiguousarray(t.copy()) for t in (tracers if tracers is not None else st.tracers)]
        var_t = [np.ascontiguousarray(t.copy()) for t in st.sct]
        dev.register_scalars(var_p, var_t)
        if prof:
            dev.profile(True, reset=True)
        dev.scalar_transport_rk(st.rho_old)
        p = dev.profile_read() if prof else None
        return np.stack(var_p), p
    finally:
        dev.close()


def test_terrain_case_has_terrain():
    g, _ = terrain_case()
    assert (g.lpw[1:] > 2).sum() > 20 and (g.lpw[1:] == 2).sum() > 20
    assert g.lpw.max() >= 5
    assert (g.lve2 > 0).sum() > 20


@pytest.mark.parametrize("kw", [dict(), dict(nrk_scal=3), dict(scal_order=3),
                                dict(nrk_scal=3, scal_order=3), dict(iscal_monot=1), dict(iscal_monot=2)])
def test_terrain_parity(kw):
    g, st = terrain_case()
    opts = abi.make_opts(1800.0, **kw)
    fg = abi.FortranGrid(g)
    ref32 = oracle_lib.scalar_transport(fg, opts, st.tracers, st.sct, st)
    ref64 = oracle_lib.scalar_transport(fg, opts, st.tracers, st.sct, st, fp64=True)
    tiled, prof = run(g, st, opts, abi.TRANSPORT_FUSED, prof=True)
    assert "tile_stage1" in prof, prof
    plain, _ = run(g, st, opts, abi.TRANSPORT_PLAIN)
    for out in (tiled, plain):
        for n in range(st.ntr):
            assert relerr(out[n], ref64[n]) < TOL64, (kw, n, relerr(out[n], ref64[n]))
            assert relerr(out[n], ref32[n]) < TOL32, (kw, n, relerr(out[n], ref32[n]))


def test_terrain_parity_implicit():
    # vertical CFL > 1: implicit columns, their solves starting at lpw
    g, st = terrain_case(nxp=5, nlev=12, ntr=4, dtlm=3600.0, seed=7, w_amp=3.0)
    for kw in (dict(), dict(nrk_scal=3)):
        opts = abi.make_opts(3600.0, **kw)
        fg = abi.FortranGrid(g)
        ref64, ff, _ = oracle_lib.scalar_transport(fg, opts, st.tracers, st.sct, st, fp64=True, want_ff=True)
        assert (ff > 0).any()
        out, _ = run(g, st, opts, abi.TRANSPORT_FUSED)
        for n in range(st.ntr):
            assert relerr(out[n], ref64[n]) < TOL64, (kw, n, relerr(out[n], ref64[n]))


@pytest.mark.parametrize("form", [abi.TRANSPORT_FUSED, abi.TRANSPORT_PLAIN])
def test_terrain_never_reads_below_the_floor(form):
    g, st = terrain_case()
    opts = abi.make_opts(1800.0, nrk_scal=3, scal_order=3)
    base, _ = run(g, st, opts, form)
    tr = [t.copy() for t in st.tracers]
    below = np.arange(g.mza)[None, :] < (g.lpw[:, None] - 1)
    below[0] = False
    for t in tr:
        t[below] = np.nan
    out, _ = run(g, st, opts, form, tracers=tr)
    assert np.isfinite(out[:, 1:]).all()
    # the levels below a floor take the floor's value, as with finite inputs
    assert np.array_equal(out[:, 1:], base[:, 1:])


def test_terrain_column_form_rejected():
    g, st = terrain_case()
    with pytest.raises(OlamGpuError):
        run(g, st, abi.make_opts(1800.0), abi.TRANSPORT_FUSED_COLUMN)


@pytest.mark.parametrize("kw", [dict(), dict(nrk_scal=3, scal_order=3)])
def test_terrain_adjoint_matches_oracle(kw):
    from test_adjoint_gpu import _adjoint_vs_oracle
    g, st = terrain_case(ntr=3)
    _adjoint_vs_oracle(g, st, abi.make_opts(1800.0, **kw), 3)


def test_terrain_adjoint_implicit_columns():
    from test_adjoint_gpu import _adjoint_vs_oracle
    g, st = terrain_case(nxp=5, nlev=12, ntr=4, dtlm=3600.0, seed=7, w_amp=3.0)
    _adjoint_vs_oracle(g, st, abi.make_opts(3600.0, nrk_scal=3), 4)


DYN_CASES = [dict(), dict(nrk_wrtv=2), dict(thil_order=3, wind_order=3),
             dict(ithil_monot=1, iwind_monot=1), dict(divh_damp_fact=0.0, vort_damp_fact=0.0)]


@pytest.mark.parametrize("kw", DYN_CASES)
def test_terrain_long_step_parity(kw):
    from test_dynamics_gpu import check_fields, dyn_case, gpu_long_steps, oracle_long_steps
    g0, ds = dyn_case()
    g = terrain_grid(g0)
    fg = abi.FortranGrid(g)
    opts = abi.make_opts(600.0, nacoust=4, **kw)
    arrays = oracle_lib.dyn_arrays(g, ds)
    o64, _ = oracle_long_steps(fg, opts, arrays, 1, True)
    o32, _ = oracle_long_steps(fg, opts, arrays, 1, False)
    hs, _ = gpu_long_steps(fg, opts, arrays, 1, abi.SYNC_EACH_CALL)
    check_fields(hs, o32, o64)


def test_terrain_timestep_matches_single_calls():
    from test_timestep_gpu import Dev, _case, _same
    g0, _, arrays, tr = _case()
    g = terrain_grid(g0)
    opts = abi.make_opts(600.0, nacoust=4)
    out = []
    for one_call in (False, True):
        d = Dev(g, arrays, tr, opts)
        try:
            for _ in range(2):
                if one_call:
                    d.dev.timestep(0)
                else:
                    d.dev.tend0(None)
                    for j in range(1, opts.nacoust + 1):
                        d.dev.prog_wrtv_rk(j)
                    d.dev.timeavg_momsc()
                    d.dev.scalar_transport_rk(None)
                    d.dev.set_scalars_bottom()
            out.append(d.host())
        finally:
            d.close()
    _same(out[0], out[1])
    scp = out[1]["scp"]
    assert np.isfinite(scp[:, 1:]).all()
    # the levels below each column's floor took the floor's value
    for iw in range(1, g.mwa):
        kb = g.lpw[iw] - 1
        assert np.array_equal(scp[:, iw, :kb], np.repeat(scp[:, iw, kb:kb + 1], kb, axis=1))
