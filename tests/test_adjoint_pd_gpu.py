"""GPU adjoint of scalar_transport_rk with the positive-definite limiter
(iscal_monot = 2; omodel/scalar_transport_rk.F90:1085-1472 and :297-314)
through the C-ABI, at a forward state where the limiter is active: against
the FP64 oracle's adjoint of the same step, and the dot-product test
<J x, y> = <x, J^T y> with J x the oracle's exact tangent-linear (FP64) and
J^T y the GPU adjoint (FP32).  Then the checkpointed window with the
limiter against the same window run step by step."""
import numpy as np
import pytest

import oracle_lib
from conftest import relerr
from olam_b200 import abi
from olam_b200.lib import HostState, OlamGpu
from test_oracle_limiter_adjoint import direction, pd_case

pytestmark = pytest.mark.gpu

TOL = 1e-5


def gpu_adjoint(g, st, opts, tr, sct, y, pdef=None):
    fg = abi.FortranGrid(g)
    dev = OlamGpu(fg, opts, HostState(vmasc=st.vmasc, wmasc=st.wmasc, rho=st.rho, wc=st.wc))
    try:
        # the registered tracers and tendencies are the forward step's inputs
        var_p = [np.ascontiguousarray(np.asarray(t, np.float32).copy()) for t in tr]
        var_t = [np.ascontiguousarray(np.asarray(t, np.float32).copy()) for t in sct]
        dev.register_scalars(var_p, var_t, pdef=pdef)
        return dev.scalar_transport_rk_adjoint(y, rho_old=st.rho_old)
    finally:
        dev.close()


@pytest.mark.parametrize("kw", [dict(zeros=False), dict(zeros=False, nrk=3), dict(zeros=False, order=3),
                                dict(zeros=False, dt=7200.0, w_amp=3.0)])
def test_limited_adjoint_matches_oracle(kw):
    g, st, tr, sct, opts = pd_case(**kw)
    fg = abi.FortranGrid(g)
    y = direction(g, 3)
    # the oracle at the forward state of the FP32 inputs the GPU sees
    tr32 = [np.asarray(t, np.float32) for t in tr]
    sct32 = [np.asarray(t, np.float32) for t in sct]
    r0, rs = oracle_lib.scalar_transport_adjoint_pd(fg, opts, y, st, tr32, sct32, fp64=True)
    l0, ls = gpu_adjoint(g, st, opts, tr32, sct32, y)
    for n in range(2):
        assert relerr(l0[n], r0[n]) < TOL, (n, relerr(l0[n], r0[n]))
        assert relerr(ls[n], rs[n]) < TOL, (n, relerr(ls[n], rs[n]))


@pytest.mark.parametrize("zeros", [False, True])
def test_limited_adjoint_dot_product(zeros):
    g, st, tr, sct, opts = pd_case(zeros=zeros)
    fg = abi.FortranGrid(g)
    tr32 = [np.asarray(t, np.float32).astype(np.float64) for t in tr]
    sct32 = [np.asarray(t, np.float32).astype(np.float64) for t in sct]
    dx, ds, y = direction(g, 1), direction(g, 2), direction(g, 3)
    _, jv = oracle_lib.scalar_transport_tl(fg, opts, tr32, sct32, dx, ds, st)
    l0, ls = gpu_adjoint(g, st, opts, tr32, sct32, y)
    lhs = sum(float(np.dot(jv[n].ravel(), y[n].ravel())) for n in range(2))
    rhs = sum(float(np.dot(dx[n].ravel(), l0[n].astype(np.float64).ravel())
                    + np.dot(ds[n].ravel(), ls[n].astype(np.float64).ravel())) for n in range(2))
    assert abs(lhs - rhs) / abs(lhs) < TOL, (lhs, rhs)


def test_mixed_pdef_tracers():
    # a limited and an unlimited tracer in one call
    g, st, tr, sct, opts = pd_case(zeros=False)
    fg = abi.FortranGrid(g)
    y = direction(g, 3)
    tr32 = [np.asarray(t, np.float32) for t in tr]
    sct32 = [np.asarray(t, np.float32) for t in sct]
    pdef = [1, 0]
    r0, rs = oracle_lib.scalar_transport_adjoint_pd(fg, opts, y, st, tr32, sct32, pdef=pdef, fp64=True)
    l0, ls = gpu_adjoint(g, st, opts, tr32, sct32, y, pdef=pdef)
    for n in range(2):
        assert relerr(l0[n], r0[n]) < TOL, (n, relerr(l0[n], r0[n]))
        assert relerr(ls[n], rs[n]) < TOL, (n, relerr(ls[n], rs[n]))


def test_limited_window_equals_stepwise_chain():
    from test_window_gpu import NTR, case, receptors
    g, ds, tr, emis = case(seed=12)
    opts = abi.make_opts(600.0, nacoust=4, nrk_scal=2, iscal_monot=2)
    lam = receptors(g, seed=4)
    fg = abi.FortranGrid(g)
    arrays = oracle_lib.dyn_arrays(g, ds)

    def new_device():
        hs = HostState(**{k: np.array(v, copy=True) for k, v in arrays.items()})
        dev = OlamGpu(fg, opts, hs)
        var_p = [t.copy() for t in tr]
        var_t = [np.zeros_like(t) for t in tr]
        dev.register_scalars(var_p, var_t)
        dev.set_surface_emission(emis)
        dev.set_coherence(abi.RESIDENT)
        return dev, hs, var_p, var_t

    nsteps, nchk = 4, 3
    dev, hs, var_p, _ = new_device()
    try:
        dev.window_forward(nsteps, nchk, abi.TS_GRAPH)
        g0, gs = dev.window_adjoint(lam)
    finally:
        dev.close()
    # step by step: the winds and the tracers before every step read back
    dev, hs, var_p, var_t = new_device()
    steps = []
    try:
        rho_prev = hs["rho"].copy()
        for _ in range(nsteps):
            dev.sync_to_host(abi.F_SCALARS)
            before = [t.copy() for t in var_p]
            dev.timestep(0)
            dev.sync_to_host(abi.F_VMASC | abi.F_WMASC | abi.F_RHO | abi.F_WC)
            steps.append(dict(vmasc=hs["vmasc"].copy(), wmasc=hs["wmasc"].copy(), rho=hs["rho"].copy(),
                              rho_old=rho_prev.astype(np.float32), wc=hs["wc"].copy(), tracers=before))
            rho_prev = hs["rho"].copy()
        dev.set_coherence(abi.SYNC_EACH_CALL)
        # the step's tendencies: zero but the emission at lpw
        for n in range(NTR):
            var_t[n][...] = 0.0
            var_t[n][np.arange(1, g.mwa), g.lpw[1:] - 1] = emis[n][1:]
        l = [x.copy() for x in lam]
        ls_sum = [np.zeros_like(x) for x in lam]
        for w in reversed(steps):
            for k in ("vmasc", "wmasc", "rho", "wc"):
                hs[k][...] = w[k]
            for n in range(NTR):
                var_p[n][...] = w["tracers"][n]
            l, ls = dev.scalar_transport_rk_adjoint(l, rho_old=w["rho_old"])
            ls_sum = [a + b for a, b in zip(ls_sum, ls)]
    finally:
        dev.close()
    for n in range(NTR):
        assert relerr(g0[n][1:], l[n][1:]) < 1e-6, n
        assert relerr(gs[n][1:], ls_sum[n][1:]) < 1e-6, n
