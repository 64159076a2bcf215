"""GPU parity of the acoustic step's eddy diffusion (comp_horiz_k,
solve_eddy_diff_heat / _vxe, rayf_mix_top_vxe, horizontal diffusion of thil
and the winds) through the C-ABI against the oracle
(convect/pbl_driver.f90:136-238, 519-742; modules/mem_rayf.f90:177-220;
omodel/prog_wrtv_rk.f90:214-251)."""
import numpy as np
import pytest

import oracle_lib
from conftest import relerr
from olam_b200 import abi
from olam_b200.lib import HostState, OlamGpu
from olam_b200.synth.state import eddy_inputs
from test_dynamics_gpu import check_fields, dyn_case

pytestmark = pytest.mark.gpu

EDDY_CASES = [
    dict(),
    dict(akmin=1.0, idiffk=2),
    dict(rayf_mix=True),
]


def _copy(d):
    return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}


def _oracle(fg, opts, arrays, d, nsteps, fp64):
    o = oracle_lib.DynOracle(fg, opts, arrays, fp64=fp64)
    o.set_eddy(abi.make_eddy(_copy(d)))
    hk = o.comp_horiz_k()
    for _ in range(nsteps):
        o.tend0()
        for jstp in range(1, opts.nacoust + 1):
            o.prog_wrtv_rk(jstp)
        o.timeavg_momsc()
    return o, hk


def _gpu(fg, opts, arrays, d, nsteps, coherence):
    hs = HostState(**{k: np.array(v, copy=True) for k, v in arrays.items()})
    dev = OlamGpu(fg, opts, hs)
    dh = _copy(d)
    e = abi.make_eddy(dh)
    rho_old = np.zeros_like(hs["thil"])
    try:
        dev.set_coherence(coherence)
        dev.set_eddy(e)
        dev.comp_horiz_k()
        for _ in range(nsteps):
            dev.tend0(rho_old)
            for jstp in range(1, opts.nacoust + 1):
                dev.prog_wrtv_rk(jstp)
            dev.timeavg_momsc()
        if coherence == abi.RESIDENT:
            dev.sync_to_host(abi.F_ALL)
        return hs, dh
    finally:
        dev.close()


@pytest.mark.parametrize("kw", EDDY_CASES)
def test_comp_horiz_k_parity(kw):
    g, ds = dyn_case()
    fg = abi.FortranGrid(g)
    opts = abi.make_opts(600.0, nacoust=4)
    arrays = oracle_lib.dyn_arrays(g, ds)
    d = eddy_inputs(g, ds.rho, ds.thil, ds.press, **kw)
    _, (am, ah, km, kh) = _oracle(fg, opts, arrays, d, 0, False)
    _, dh = _gpu(fg, opts, arrays, d, 0, abi.SYNC_EACH_CALL)
    assert np.array_equal(dh["kmtopv"][1:], km[1:])
    assert np.array_equal(dh["khtopv"][1:], kh[1:])
    # float32 products and a powf of the device's math library: a few ulp
    assert relerr(dh["akmodx"][1:], am[1:]) < 1e-6
    assert relerr(dh["akhodx"][1:], ah[1:]) < 1e-6


@pytest.mark.parametrize("kw", EDDY_CASES)
def test_eddy_long_step_parity_sync(kw):
    g, ds = dyn_case()
    fg = abi.FortranGrid(g)
    opts = abi.make_opts(600.0, nacoust=4)
    arrays = oracle_lib.dyn_arrays(g, ds)
    d = eddy_inputs(g, ds.rho, ds.thil, ds.press, **kw)
    o64, _ = _oracle(fg, opts, arrays, d, 1, True)
    o32, _ = _oracle(fg, opts, arrays, d, 1, False)
    hs, _ = _gpu(fg, opts, arrays, d, 1, abi.SYNC_EACH_CALL)
    check_fields(hs, o32, o64)
    # the eddy terms are active: the step differs from the one without them
    plain = oracle_lib.DynOracle(fg, opts, arrays, fp64=True)
    plain.tend0()
    for jstp in range(1, opts.nacoust + 1):
        plain.prog_wrtv_rk(jstp)
    plain.timeavg_momsc()
    assert relerr(hs["thil"][1:], plain.a["thil"][1:]) > 100 * relerr(hs["thil"][1:], o64.a["thil"][1:])


def test_eddy_long_steps_parity_resident_with_rayleigh():
    # two long steps on the device with the Rayleigh term on thil, which
    # follows the eddy terms in the column set-up
    g, ds = dyn_case(nxp=8, nlev=16, seed=5)
    fg = abi.FortranGrid(g)
    mza = g.mza
    rayf = np.zeros(mza, np.float32)
    rayf[mza - 4:] = 1.0e-3
    zt = g.zt.astype(np.float32)
    th01d = (300.0 * np.exp(zt / 3.0e4)).astype(np.float32)
    dn01d = (1.2 * np.exp(-zt / 8.0e3)).astype(np.float32)
    vc03d = np.zeros((g.mva, mza), np.float32)
    opts = abi.make_opts(600.0, nacoust=4)
    opts.krayf_bot, opts.initial = mza - 3, 1
    opts.rayf_cof, opts.th01d = abi.ptr(rayf, abi.C.c_float), abi.ptr(th01d, abi.C.c_float)
    opts.dn01d, opts.vc03d = abi.ptr(dn01d, abi.C.c_float), abi.ptr(vc03d, abi.C.c_float)
    arrays = oracle_lib.dyn_arrays(g, ds)
    d = eddy_inputs(g, ds.rho, ds.thil, ds.press, rayf_mix=True, seed=11)
    o64, _ = _oracle(fg, opts, arrays, d, 2, True)
    o32, _ = _oracle(fg, opts, arrays, d, 2, False)
    hs, _ = _gpu(fg, opts, arrays, d, 2, abi.RESIDENT)
    check_fields(hs, o32, o64)
