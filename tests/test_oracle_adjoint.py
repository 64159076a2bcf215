"""CPU checks of the oracle's adjoint of scalar_transport_rk: the dot-product
test <L x, y> = <x, L^T y> for the linear step (x = old tracer and
tendency, y = a weight on the new tracer), in FP64 and FP32, with and
without implicit columns, RK2 and RK3, horizontal order 2 and 3."""
import numpy as np
import pytest

import oracle_lib
from conftest import small_case
from olam_b200 import abi


def _dot_test(g, st, opts, fp64, seed=5):
    rng = np.random.default_rng(seed)
    fg = abi.FortranGrid(g)
    ntr = 2
    shape = (g.mwa, g.mza)
    x0 = [rng.standard_normal(shape) for _ in range(ntr)]
    xs = [1e-4 * rng.standard_normal(shape) for _ in range(ntr)]
    y = [rng.standard_normal(shape) for _ in range(ntr)]
    for a in x0 + xs + y:
        a[0] = 0.0          # the dummy column
        a[:, 0] = 0.0       # the level below ground
    fwd = oracle_lib.scalar_transport(fg, opts, x0, xs, st, fp64=fp64)
    l0, ls = oracle_lib.scalar_transport_adjoint(fg, opts, y, st, fp64=fp64)
    lhs = sum(float(np.dot(fwd[n].ravel(), y[n].ravel())) for n in range(ntr))
    rhs = sum(float(np.dot(x0[n].ravel(), l0[n].ravel()) + np.dot(xs[n].ravel(), ls[n].ravel()))
              for n in range(ntr))
    return abs(lhs - rhs) / abs(lhs)


CASES = [dict(), dict(nrk_scal=3), dict(scal_order=3), dict(nrk_scal=3, scal_order=3)]


@pytest.mark.parametrize("kw", CASES)
def test_adjoint_dot_product_fp64(kw):
    g, st = small_case(nxp=5, nlev=10, ntr=1, seed=3)
    opts = abi.make_opts(1800.0, **kw)
    assert _dot_test(g, st, opts, True) < 1e-12


@pytest.mark.parametrize("kw", CASES)
def test_adjoint_dot_product_fp32(kw):
    g, st = small_case(nxp=5, nlev=10, ntr=1, seed=3)
    opts = abi.make_opts(1800.0, **kw)
    assert _dot_test(g, st, opts, False) < 1e-5


def test_adjoint_dot_product_implicit_columns():
    # vertical CFL > 1: implicit columns in every stage
    g, st = small_case(nxp=5, nlev=12, ntr=4, dtlm=3600.0, seed=7, w_amp=3.0)
    for kw in (dict(), dict(nrk_scal=3)):
        opts = abi.make_opts(3600.0, **kw)
        _, ff, _ = oracle_lib.scalar_transport(abi.FortranGrid(g), opts, st.tracers, st.sct, st,
                                               fp64=True, want_ff=True)
        assert (ff > 0).any()
        assert _dot_test(g, st, opts, True) < 1e-12


def test_adjoint_matches_finite_differences():
    # FP64 central differences of the forward along seeded directions
    g, st = small_case(nxp=5, nlev=10, ntr=1, seed=3)
    opts = abi.make_opts(1800.0)
    fg = abi.FortranGrid(g)
    rng = np.random.default_rng(11)
    shape = (g.mwa, g.mza)
    base = [1.0 + 0.1 * rng.random(shape)]
    sct0 = [np.zeros(shape)]
    w = rng.standard_normal(shape)
    w[0] = 0.0
    l0, _ = oracle_lib.scalar_transport_adjoint(fg, opts, [w], st, fp64=True)
    for _ in range(5):
        d = rng.standard_normal(shape)
        d[0] = 0.0
        d[:, 0] = 0.0
        h = 1e-3
        fp = oracle_lib.scalar_transport(fg, opts, [base[0] + h * d], sct0, st, fp64=True)
        fm = oracle_lib.scalar_transport(fg, opts, [base[0] - h * d], sct0, st, fp64=True)
        fd = float(np.sum(w * (fp[0] - fm[0]))) / (2 * h)
        ad = float(np.sum(l0[0] * d))
        assert abs(fd - ad) <= 1e-9 * max(1.0, abs(ad)), (fd, ad)


def test_adjoint_rejects_limiters():
    g, st = small_case(nxp=4, nlev=8, ntr=1)
    opts = abi.make_opts(1800.0, iscal_monot=1)
    with pytest.raises(AssertionError):
        oracle_lib.scalar_transport_adjoint(abi.FortranGrid(g), opts, [np.ones((g.mwa, g.mza))], st)
