"""GPU parity of scalar_transport_rk through the C-ABI against the oracle."""
import numpy as np
import pytest

import oracle_lib
from conftest import relerr, small_case
from olam_b200 import abi
from olam_b200.lib import HostState, OlamGpu

pytestmark = pytest.mark.gpu

TOL64 = 1e-5   # field error bound against the FP64 oracle
TOL32 = 1e-5   # against the FP32 oracle (same inputs, same precision)


def run_gpu(g, st, opts, form, coherence=abi.SYNC_EACH_CALL, pdef=None, steps=1):
    fg = abi.FortranGrid(g)
    hs = HostState(vmasc=st.vmasc, wmasc=st.wmasc, rho=st.rho, wc=st.wc)
    dev = OlamGpu(fg, opts, hs)
    try:
        dev.set_transport_form(form)
        dev.set_coherence(coherence)
        var_p = [np.ascontiguousarray(t.copy()) for t in st.tracers]
        var_t = [np.ascontiguousarray(t.copy()) for t in st.sct]
        dev.register_scalars(var_p, var_t, pdef=pdef)
        diag = None
        for _ in range(steps):
            diag = dev.scalar_transport_rk(st.rho_old, want_diag=True)
        if coherence == abi.RESIDENT:
            dev.sync_to_host(abi.F_SCALARS)
        return np.stack(var_p), diag
    finally:
        dev.close()


CASES = [
    dict(),
    dict(nrk_scal=3),
    dict(scal_order=3),
    dict(nrk_scal=3, scal_order=3),
    dict(iscal_monot=1),
    dict(iscal_monot=2),
    dict(iscal_monot=1, scal_order=3, nrk_scal=3),
]


FORMS = [abi.TRANSPORT_FUSED, abi.TRANSPORT_PLAIN, abi.TRANSPORT_FUSED_COLUMN]


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("kw", CASES)
def test_transport_parity_small(form, kw):
    g, st = small_case(nxp=6, nlev=12, ntr=6)
    opts = abi.make_opts(1800.0, **kw)
    fg = abi.FortranGrid(g)
    pdef = np.array([1, 0, 1, 1, 0, 1])
    ref32, ff, d32 = oracle_lib.scalar_transport(fg, opts, st.tracers, st.sct, st, pdef=pdef,
                                                 want_ff=True)
    ref64 = oracle_lib.scalar_transport(fg, opts, st.tracers, st.sct, st, fp64=True, pdef=pdef)
    out, diag = run_gpu(g, st, opts, form, pdef=pdef)
    for n in range(st.ntr):
        assert relerr(out[n], ref64[n]) < TOL64, (n, relerr(out[n], ref64[n]))
        assert relerr(out[n], ref32[n]) < TOL32, (n, relerr(out[n], ref32[n]))
    assert abs(diag.cfl_max - d32.cfl_max) <= 1e-5 * d32.cfl_max
    assert (diag.cfl_k, diag.cfl_iwglobe) == (d32.cfl_k, d32.cfl_iwglobe)


@pytest.mark.parametrize("form", FORMS)
def test_transport_parity_implicit(form):
    # vertical CFL > 1: implicit columns in every stage
    g, st = small_case(nxp=5, nlev=12, ntr=4, dtlm=3600.0, seed=7, w_amp=3.0)
    for kw in (dict(), dict(nrk_scal=3), dict(iscal_monot=1)):
        opts = abi.make_opts(3600.0, **kw)
        fg = abi.FortranGrid(g)
        ref64, ff, _ = oracle_lib.scalar_transport(fg, opts, st.tracers, st.sct, st, fp64=True,
                                                   want_ff=True)
        assert (ff > 0).any()
        out, _ = run_gpu(g, st, opts, form)
        for n in range(st.ntr):
            assert relerr(out[n], ref64[n]) < TOL64, (kw, n, relerr(out[n], ref64[n]))


def test_transport_parity_config1_size():
    # NXP=20, 30 levels (4002 columns), 1 cosine-bell tracer, 300 s steps
    from olam_b200.synth.grid import build_grid, stretched_levels
    from olam_b200.synth.state import transport_state
    g = build_grid(20, stretched_levels(30, 100.0, 30000.0), seed=1)
    st = transport_state(g, 300.0, 1, tracer_kind="bell", solid=True, jet_amp=20.0,
                         t_sfc=250.0, lapse=0.0, seed=1)
    opts = abi.make_opts(300.0)
    fg = abi.FortranGrid(g)
    ref64 = oracle_lib.scalar_transport(fg, opts, st.tracers, st.sct, st, fp64=True)
    for form in (abi.TRANSPORT_FUSED, abi.TRANSPORT_PLAIN):
        out, _ = run_gpu(g, st, opts, form)
        assert relerr(out[0], ref64[0]) < TOL64


def test_resident_multistep_matches_oracle():
    g, st = small_case(nxp=6, nlev=12, ntr=6)
    opts = abi.make_opts(1800.0)
    fg = abi.FortranGrid(g)
    tr = st.tracers.copy()
    for _ in range(3):
        tr = oracle_lib.scalar_transport(fg, opts, tr, st.sct, st, fp64=True).astype(np.float32)
    out, _ = run_gpu(g, st, opts, abi.TRANSPORT_FUSED, coherence=abi.RESIDENT, steps=3)
    for n in range(st.ntr):
        assert relerr(out[n], tr[n]) < 3 * TOL64


@pytest.mark.parametrize("ntr,order", [(40, 2), (130, 2), (130, 3), (64, 3)])
def test_fused_forms_agree_many_tracers(ntr, order):
    # 40 tracers: one ragged 64-tracer group; 130: two full groups and a
    # ragged one; the tiled, per-column and plain forms agree
    g, st = small_case(nxp=8, nlev=16, ntr=ntr, seed=21)
    opts = abi.make_opts(1800.0, scal_order=order)
    a, _ = run_gpu(g, st, opts, abi.TRANSPORT_FUSED)
    b, _ = run_gpu(g, st, opts, abi.TRANSPORT_PLAIN)
    c, _ = run_gpu(g, st, opts, abi.TRANSPORT_FUSED_COLUMN)
    for n in range(st.ntr):
        assert relerr(a[n], b[n]) < 1e-6, (n, relerr(a[n], b[n]))
        assert relerr(c[n], b[n]) < 1e-6, (n, relerr(c[n], b[n]))


def test_per_call_step_in_tracer_groups():
    # more than 64 tracers in the per-call (SYNC_EACH_CALL) mode: the tiled
    # step runs group by group with the copies in and out overlapped; the
    # result is the device-resident step's, bit for bit, and the oracle's
    g, st = small_case(nxp=5, nlev=10, ntr=70)
    opts = abi.make_opts(1800.0)
    sync, _ = run_gpu(g, st, opts, abi.TRANSPORT_FUSED, coherence=abi.SYNC_EACH_CALL, steps=2)
    res, _ = run_gpu(g, st, opts, abi.TRANSPORT_FUSED, coherence=abi.RESIDENT, steps=2)
    assert np.array_equal(sync[:, 1:], res[:, 1:])
    fg = abi.FortranGrid(g)
    sel = [0, 63, 64, 69]
    ref64 = oracle_lib.scalar_transport(fg, opts, [st.tracers[i] for i in sel], [st.sct[i] for i in sel], st,
                                        fp64=True)
    one, _ = run_gpu(g, st, opts, abi.TRANSPORT_FUSED, coherence=abi.SYNC_EACH_CALL, steps=1)
    for j, i in enumerate(sel):
        assert relerr(one[i], ref64[j]) < TOL64, (i, relerr(one[i], ref64[j]))
