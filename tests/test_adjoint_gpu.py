"""GPU adjoint of scalar_transport_rk through the C-ABI: against the
oracle's FP64 adjoint on the same inputs, and the dot-product test
<F x, y> = <x, F^T y> between the GPU forward step and the GPU adjoint."""
import numpy as np
import pytest

import oracle_lib
from conftest import relerr, small_case
from olam_b200 import abi
from olam_b200.lib import HostState, OlamGpu, OlamGpuError

pytestmark = pytest.mark.gpu

TOL_ORACLE = 1e-5   # normwise, FP32 adjoint against the FP64 oracle adjoint
TOL_DOT = 1e-5      # dot-product identity in FP32


def _device(g, st, opts, tracers, sct):
    fg = abi.FortranGrid(g)
    hs = HostState(vmasc=st.vmasc, wmasc=st.wmasc, rho=st.rho, wc=st.wc)
    dev = OlamGpu(fg, opts, hs)
    var_p = [np.ascontiguousarray(np.asarray(t, np.float32).copy()) for t in tracers]
    var_t = [np.ascontiguousarray(np.asarray(t, np.float32).copy()) for t in sct]
    dev.register_scalars(var_p, var_t)
    return dev, var_p


def _weights(g, ntr, seed):
    rng = np.random.default_rng(seed)
    y = [rng.standard_normal((g.mwa, g.mza)) for _ in range(ntr)]
    for a in y:
        a[0] = 0.0
    return y


def _adjoint_vs_oracle(g, st, opts, ntr, seed=2):
    y = _weights(g, ntr, seed)
    dev, _ = _device(g, st, opts, st.tracers[:ntr], st.sct[:ntr])
    try:
        l0, ls = dev.scalar_transport_rk_adjoint(y, rho_old=st.rho_old)
    finally:
        dev.close()
    r0, rs = oracle_lib.scalar_transport_adjoint(abi.FortranGrid(g), opts, y, st, fp64=True)
    for n in range(ntr):
        assert relerr(l0[n], r0[n]) < TOL_ORACLE, (n, relerr(l0[n], r0[n]))
        assert relerr(ls[n], rs[n]) < TOL_ORACLE, (n, relerr(ls[n], rs[n]))


CASES = [dict(), dict(nrk_scal=3), dict(scal_order=3), dict(nrk_scal=3, scal_order=3)]


@pytest.mark.parametrize("kw", CASES)
def test_adjoint_matches_oracle(kw):
    g, st = small_case(nxp=6, nlev=12, ntr=3)
    _adjoint_vs_oracle(g, st, abi.make_opts(1800.0, **kw), 3)


def test_adjoint_matches_oracle_implicit_columns():
    # vertical CFL > 1: implicit columns in every stage
    g, st = small_case(nxp=5, nlev=12, ntr=4, dtlm=3600.0, seed=7, w_amp=3.0)
    for kw in (dict(), dict(nrk_scal=3)):
        opts = abi.make_opts(3600.0, **kw)
        _, ff, _ = oracle_lib.scalar_transport(abi.FortranGrid(g), opts, st.tracers, st.sct, st,
                                               fp64=True, want_ff=True)
        assert (ff > 0).any()
        _adjoint_vs_oracle(g, st, opts, 4)


@pytest.mark.parametrize("ntr", [5, 32, 36, 70])
def test_adjoint_matches_oracle_ragged_tracer_groups(ntr):
    # 5: one partial group of 64 tracers (ntp = 8); 70: a full and a ragged group
    g, st = small_case(nxp=5, nlev=10, ntr=ntr, seed=4)
    _adjoint_vs_oracle(g, st, abi.make_opts(1800.0, scal_order=3), ntr, seed=9)


@pytest.mark.parametrize("kw", [dict(), dict(nrk_scal=3, scal_order=3)])
def test_adjoint_dot_product_against_gpu_forward(kw):
    g, st = small_case(nxp=6, nlev=12, ntr=2, seed=5)
    opts = abi.make_opts(1800.0, **kw)
    rng = np.random.default_rng(6)
    shape = (g.mwa, g.mza)
    x0 = [rng.standard_normal(shape) for _ in range(2)]
    xs = [1e-4 * rng.standard_normal(shape) for _ in range(2)]
    for a in x0 + xs:
        a[0] = 0.0
        a[:, 0] = 0.0
    y = _weights(g, 2, 8)
    dev, var_p = _device(g, st, opts, x0, xs)
    try:
        dev.scalar_transport_rk(st.rho_old)
        fwd = [v.astype(np.float64) for v in var_p]
        l0, ls = dev.scalar_transport_rk_adjoint(y, rho_old=st.rho_old)
    finally:
        dev.close()
    lhs = sum(float(np.dot(fwd[n].ravel(), y[n].ravel())) for n in range(2))
    rhs = sum(float(np.dot(np.asarray(x0[n], np.float32).astype(np.float64).ravel(), l0[n].ravel().astype(np.float64))
                    + np.dot(np.asarray(xs[n], np.float32).astype(np.float64).ravel(), ls[n].ravel().astype(np.float64)))
              for n in range(2))
    assert abs(lhs - rhs) / abs(lhs) < TOL_DOT, (lhs, rhs)


def test_adjoint_rejects_limited_transport():
    g, st = small_case(nxp=5, nlev=10, ntr=1)
    dev, _ = _device(g, st, abi.make_opts(1800.0, iscal_monot=1), st.tracers, st.sct)
    try:
        with pytest.raises(OlamGpuError) as e:
            dev.scalar_transport_rk_adjoint(_weights(g, 1, 1), rho_old=st.rho_old)
        assert e.value.rc == abi.E_UNSUPPORTED
    finally:
        dev.close()
