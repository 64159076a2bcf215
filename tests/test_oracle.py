"""CPU tests of the oracle (the checker) against properties, an independent
numpy restatement and the committed golden fixtures."""
import os

import numpy as np
import pytest

import oracle_lib
from conftest import relerr, small_case
from olam_b200 import abi
from numpy_ref import transport_plain

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _run(g, st, dt, fp64=False, **kw):
    fg = abi.FortranGrid(g)
    o = abi.make_opts(dt, **{k: v for k, v in kw.items() if k in (
        "nrk_scal", "scal_order", "iscal_monot")})
    pdef = kw.get("pdef")
    return oracle_lib.scalar_transport(fg, o, st.tracers, st.sct, st, fp64=fp64, pdef=pdef,
                                       want_ff=True)


def test_constant_tracer_preserved(case_small):
    g, st = case_small
    tr = st.tracers.copy()
    tr[:] = 0.75
    tr[:, 0] = 0.0

    class S:
        pass
    s2 = S()
    s2.__dict__.update(st.__dict__)
    s2.tracers = tr
    for opts in ({}, {"nrk_scal": 3}, {"scal_order": 3}, {"iscal_monot": 1}, {"iscal_monot": 2}):
        out, ff, _ = _run(g, s2, 1800.0, **opts)
        assert np.abs(out[:, 1:, 1:] - 0.75).max() <= 2e-7, opts


@pytest.mark.parametrize("nrk", [2, 3])
def test_mass_conservation(case_small, nrk):
    g, st = case_small
    out, ff, _ = _run(g, st, 1800.0, fp64=True, nrk_scal=nrk)
    volt = g.volt[1:, 1:]
    for n in range(st.ntr):
        m0 = (st.rho_old[1:, 1:].astype(np.float64) * volt * st.tracers[n][1:, 1:]).sum()
        m1 = (st.rho[1:, 1:] * volt * out[n][1:, 1:]).sum()
        if m0 > 0:
            # rho_old is real(4): the budget closes to float32 round-off of rho
            assert abs(m1 - m0) / m0 < 1e-6


@pytest.mark.parametrize("nrk,order", [(2, 2), (3, 2), (2, 3), (3, 3)])
def test_oracle_vs_numpy_restatement(case_small, nrk, order):
    g, st = case_small
    out64, ff, _ = _run(g, st, 1800.0, fp64=True, nrk_scal=nrk, scal_order=order)
    assert ff.max() == 0.0, "case must stay explicit"
    ref = transport_plain(g, st, st.tracers, st.sct, 1800.0, nrk=nrk, order=order)
    for n in range(st.ntr):
        assert relerr(out64[n][1:], ref[n][1:]) < 1e-12, n


def test_fp32_close_to_fp64(case_small):
    g, st = case_small
    out32, _, _ = _run(g, st, 1800.0)
    out64, _, _ = _run(g, st, 1800.0, fp64=True)
    for n in range(st.ntr):
        assert relerr(out32[n], out64[n]) < 1e-6


def test_monotone_limiter_bounds():
    # a sharp step tracer: the monotone option must not create new extrema
    g, st = small_case(nxp=6, nlev=12, ntr=2, dtlm=3600.0, seed=3, jet=60.0)
    tr = st.tracers.copy()
    lat = np.radians(g.glatw)
    tr[0] = np.where(lat[:, None] > 0.2, 1.0, 0.0).astype(np.float32)
    tr[1] = tr[0]
    tr[:, 0] = 0

    class S:
        pass
    s2 = S()
    s2.__dict__.update(st.__dict__)
    s2.tracers = tr
    plain, _, _ = _run(g, s2, 3600.0)
    mono, _, _ = _run(g, s2, 3600.0, iscal_monot=1)
    pd, _, _ = _run(g, s2, 3600.0, iscal_monot=2)
    assert plain[0, 1:, 1:].min() < -1e-4 or plain[0, 1:, 1:].max() > 1 + 1e-4
    assert mono[0, 1:, 1:].min() > -1e-5 and mono[0, 1:, 1:].max() < 1 + 1e-5
    assert pd[0, 1:, 1:].min() > -1e-6


def test_implicit_columns_engage():
    # strong vertical mass flux drives the vertical CFL above one: the
    # implicit columns must switch on and the result stay finite and bounded
    g, st = small_case(nxp=5, nlev=12, ntr=2, dtlm=3600.0, seed=7, w_amp=3.0)
    out, ff, diag = _run(g, st, 3600.0)
    assert (ff > 0).any()
    assert np.isfinite(out).all()
    assert diag.cfl_max > 0.98


def test_golden_fixture():
    path = os.path.join(GOLDEN, "transport_nxp3.npz")
    z = np.load(path)
    from olam_b200.synth.grid import build_grid
    g = build_grid(int(z["nxp"]), z["zz"], seed=int(z["seed"]))

    class S:
        pass
    st = S()
    for k in ("vmasc", "wmasc", "rho_old", "rho", "wc", "tracers", "sct"):
        setattr(st, k, z[k])
    st.ntr = st.tracers.shape[0]
    for nrk, key in ((2, "out_rk2"), (3, "out_rk3")):
        out64, _, _ = _run(g, st, float(z["dtlm"]), fp64=True, nrk_scal=nrk)
        assert relerr(out64, z[key]) < 1e-12


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("order", [2, 3])
def test_oracle_limiters_vs_numpy(case_small, mode, order):
    # RK2: numpy plain stage 1, then the monotonic / positive-definite stage
    from numpy_ref import limited_last_stage, plain_stage
    g, st = case_small
    dt = 1800.0
    out64, ff, _ = _run(g, st, dt, fp64=True, iscal_monot=mode, scal_order=order,
                        pdef=np.ones(st.ntr))
    assert ff.max() == 0.0
    rho = st.rho.astype(np.float64)
    for n in range(st.ntr):
        q0 = st.tracers[n].astype(np.float64)
        t0 = st.sct[n].astype(np.float64)
        s1 = plain_stage(g, st.vmasc, st.wmasc, rho, q0.copy(), q0, t0, dt * 0.5, order)
        q0b = q0 + dt * t0 / np.where(st.rho_old == 0, 1, st.rho_old)
        ref = limited_last_stage(g, s1, q0b, rho, st.vmasc, st.wmasc, dt, mode, order)
        assert relerr(out64[n][1:], ref[1:]) < 1e-12
