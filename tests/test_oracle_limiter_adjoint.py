"""CPU checks of the oracle's adjoint of scalar_transport_rk with the
positive-definite limiter (iscal_monot = 2, update_scalar_pd,
omodel/scalar_transport_rk.F90:1085-1472) at a forward state where the
limiter is active: the exact tangent-linear (forward-mode dual numbers
through the oracle's own step) against central finite differences of the
FP64 step, and the dot-product test <J x, y> = <x, J^T y> of the adjoint
against that tangent-linear (FP64 to 1e-12, FP32 to 1e-5)."""
import numpy as np
import pytest

import oracle_lib
from conftest import small_case
from olam_b200 import abi


def pd_case(seed=21, nrk=2, order=2, dt=3600.0, w_amp=0.05, zeros=True):
    """Tracers with sharp contrasts under a strong flow: the outflow of many
    cells exceeds their mass, so the limiter scales it.  With ``zeros`` the
    fields are zero in about half the cells (the limiter then also sits on
    its clamps, where the step has kinks); otherwise they are strictly
    positive (exp(3 N(0,1))), where the step is differentiable."""
    g, st = small_case(nxp=5, nlev=10, ntr=1, dtlm=dt, seed=3, w_amp=w_amp)
    rng = np.random.default_rng(seed)
    shape = (g.mwa, g.mza)
    if zeros:
        tr = [np.maximum(rng.standard_normal(shape), 0.0) ** 2 for _ in range(2)]
    else:
        tr = [np.exp(3.0 * rng.standard_normal(shape)) for _ in range(2)]
    sct = [1e-5 * np.abs(rng.standard_normal(shape)) for _ in range(2)]   # emissions
    for a in tr + sct:
        a[0] = 0.0
        a[:, 0] = a[:, 1]
    opts = abi.make_opts(dt, nrk_scal=nrk, scal_order=order, iscal_monot=2)
    return g, st, tr, sct, opts


def direction(g, seed, n=2):
    rng = np.random.default_rng(seed)
    out = [rng.standard_normal((g.mwa, g.mza)) for _ in range(n)]
    for a in out:
        a[0] = 0.0
        a[:, 0] = 0.0
    return out


@pytest.mark.parametrize("zeros", [True, False])
def test_limiter_is_active_in_the_case(zeros):
    g, st, tr, sct, opts = pd_case(zeros=zeros)
    fg = abi.FortranGrid(g)
    lim = oracle_lib.scalar_transport(fg, opts, tr, sct, st, fp64=True)
    free = oracle_lib.scalar_transport(fg, abi.make_opts(3600.0, iscal_monot=0), tr, sct, st, fp64=True)
    assert np.abs(lim - free).max() > 1e-3 * np.abs(free).max()


@pytest.mark.parametrize("kw", [dict(), dict(nrk=3), dict(order=3)])
def test_tangent_linear_matches_central_differences(kw):
    # at a state where the step is differentiable (no field on a limiter clamp)
    g, st, tr, sct, opts = pd_case(zeros=False, **kw)
    fg = abi.FortranGrid(g)
    # perturbations relative to the fields, so none reaches a kink near the state
    dx = [a * b for a, b in zip(tr, direction(g, 1))]
    ds = [a * b for a, b in zip(sct, direction(g, 2))]
    _, jv = oracle_lib.scalar_transport_tl(fg, opts, tr, sct, dx, ds, st)
    h = 1e-6
    fp = oracle_lib.scalar_transport(fg, opts, [a + h * b for a, b in zip(tr, dx)],
                                     [a + h * b for a, b in zip(sct, ds)], st, fp64=True)
    fm = oracle_lib.scalar_transport(fg, opts, [a - h * b for a, b in zip(tr, dx)],
                                     [a - h * b for a, b in zip(sct, ds)], st, fp64=True)
    fd = (fp - fm) / (2 * h)
    err = np.abs(fd - jv).max() / np.abs(jv).max()
    assert err < 1e-6, err


@pytest.mark.parametrize("kw", [dict(), dict(nrk=3), dict(order=3), dict(dt=7200.0, w_amp=3.0)])
def test_limiter_adjoint_dot_product_fp64(kw):
    g, st, tr, sct, opts = pd_case(**kw)
    fg = abi.FortranGrid(g)
    dx, ds, y = direction(g, 1), direction(g, 2), direction(g, 3)
    _, jv = oracle_lib.scalar_transport_tl(fg, opts, tr, sct, dx, ds, st)
    la, ls = oracle_lib.scalar_transport_adjoint_pd(fg, opts, y, st, tr, sct, fp64=True)
    lhs = sum(float(np.dot(jv[n].ravel(), y[n].ravel())) for n in range(2))
    rhs = sum(float(np.dot(dx[n].ravel(), la[n].ravel()) + np.dot(ds[n].ravel(), ls[n].ravel())) for n in range(2))
    assert abs(lhs - rhs) / abs(lhs) < 1e-12, (lhs, rhs)


def test_limiter_adjoint_dot_product_fp32():
    g, st, tr, sct, opts = pd_case()
    fg = abi.FortranGrid(g)
    dx, ds, y = direction(g, 1), direction(g, 2), direction(g, 3)
    _, jv = oracle_lib.scalar_transport_tl(fg, opts, tr, sct, dx, ds, st)
    la, ls = oracle_lib.scalar_transport_adjoint_pd(fg, opts, y, st, tr, sct, fp64=False)
    lhs = sum(float(np.dot(jv[n].ravel(), y[n].ravel())) for n in range(2))
    rhs = sum(float(np.dot(dx[n].ravel(), la[n].astype(np.float64).ravel())
                    + np.dot(ds[n].ravel(), ls[n].astype(np.float64).ravel())) for n in range(2))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5, (lhs, rhs)


def test_adjoint_without_pdef_is_the_unlimited_one():
    # tracers without pdef take the unlimited step even with iscal_monot = 2
    g, st, tr, sct, opts = pd_case()
    fg = abi.FortranGrid(g)
    y = direction(g, 3)
    la, ls = oracle_lib.scalar_transport_adjoint_pd(fg, opts, y, st, tr, sct, pdef=[0, 0], fp64=True)
    lu, lsu = oracle_lib.scalar_transport_adjoint(fg, abi.make_opts(3600.0), y, st, fp64=True)
    assert np.abs(la - lu).max() <= 1e-14 * np.abs(lu).max()
    assert np.abs(ls - lsu).max() <= 1e-14 * np.abs(lsu).max()
