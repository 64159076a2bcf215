"""GPU tests of the checkpointed window adjoint (olamgpu_window_forward /
olamgpu_window_adjoint) and the surface emission of the device long step.

A window of long steps of the whole core (4 acoustic RK3 steps, the tracer
step, the glue) with checkpoints every nchk steps; the loss is a seeded
weighted sum of the tracers after the window at receptor cells in the lowest
three levels; its gradients are taken with respect to the tracers before
the window and the surface emission rate of each tracer.  Checked against
  * the same window without checkpoints: the forward run step by step with
    the winds and densities of every step read back, then the one-step
    adjoint (olamgpu_scalar_transport_rk_adjoint) applied step by step in
    reverse -- the recomputation from checkpoints must give the same;
  * the FP64 oracle's one-step adjoints chained over the same winds, and
    central finite differences of the FP64 oracle's forward chain along 50
    seeded directions of the initial tracers and the emission."""
import numpy as np
import pytest

import oracle_lib
from conftest import relerr
from olam_b200 import abi
from olam_b200.lib import HostState, OlamGpu

pytestmark = pytest.mark.gpu

NTR, NSTEPS, NCHK, DT = 3, 5, 2, 600.0


def case(nxp=8, nlev=12, seed=6):
    from olam_b200.synth.grid import build_grid, stretched_levels
    from olam_b200.synth.state import dynamics_state, fast_lognormal_tracers
    g = build_grid(nxp, stretched_levels(nlev, 100.0, 30000.0), seed=seed)
    ds = dynamics_state(g, seed=seed)
    tr = fast_lognormal_tracers(g, NTR, seed=seed + 1, clip=(0.0, np.inf), zero_frac=0.0, as_list=True)
    rng = np.random.default_rng(seed + 2)
    emis = [(1e-9 * rng.random(g.mwa)).astype(np.float32) for _ in range(NTR)]
    for e in emis:
        e[0] = 0.0
    return g, ds, tr, emis


def receptors(g, seed=9, nrec=20):
    """dJ/d(tracers after the window): seeded weights at nrec receptor cells
    in the lowest three levels of every tracer."""
    rng = np.random.default_rng(seed)
    lam = [np.zeros((g.mwa, g.mza), np.float32) for _ in range(NTR)]
    for n in range(NTR):
        iw = rng.integers(1, g.mwa, nrec)
        k = g.lpw[iw] - 1 + rng.integers(0, 3, nrec)
        np.add.at(lam[n], (iw, k), rng.standard_normal(nrec).astype(np.float32))
    return lam


def new_device(g, ds, tr, emis, opts):
    fg = abi.FortranGrid(g)
    arrays = oracle_lib.dyn_arrays(g, ds)
    hs = HostState(**{k: np.array(v, copy=True) for k, v in arrays.items()})
    dev = OlamGpu(fg, opts, hs)
    var_p = [t.copy() for t in tr]
    var_t = [np.zeros_like(t) for t in tr]
    dev.register_scalars(var_p, var_t)
    dev.set_surface_emission(emis)
    dev.set_coherence(abi.RESIDENT)
    return dev, hs, var_p


@pytest.fixture(scope="module")
def window_runs():
    g, ds, tr, emis = case()
    opts = abi.make_opts(DT, nacoust=4, nrk_scal=2)
    lam = receptors(g)
    # the window with checkpoints
    dev, hs, var_p = new_device(g, ds, tr, emis, opts)
    try:
        dev.window_forward(NSTEPS, NCHK, abi.TS_GRAPH)
        dev.sync_to_host(abi.F_SCALARS)
        after = [t.copy() for t in var_p]
        g0, gs = dev.window_adjoint(lam)
        # the state after the window is back on the device
        dev.sync_to_host(abi.F_SCALARS)
        restored = [t.copy() for t in var_p]
    finally:
        dev.close()
    # the same window step by step, the winds of every step read back
    dev, hs, var_p = new_device(g, ds, tr, emis, opts)
    winds = []
    try:
        rho_prev = hs["rho"].copy()
        for _ in range(NSTEPS):
            dev.timestep(0)
            dev.sync_to_host(abi.F_VMASC | abi.F_WMASC | abi.F_RHO | abi.F_WC)
            winds.append(dict(vmasc=hs["vmasc"].copy(), wmasc=hs["wmasc"].copy(), rho=hs["rho"].copy(),
                              rho_old=rho_prev.astype(np.float32), wc=hs["wc"].copy()))
            rho_prev = hs["rho"].copy()
        dev.sync_to_host(abi.F_SCALARS)
        after_ref = [t.copy() for t in var_p]
        dev.set_coherence(abi.SYNC_EACH_CALL)
        l = [x.copy() for x in lam]
        ls_sum = [np.zeros_like(x) for x in lam]
        for w in reversed(winds):
            for k in ("vmasc", "wmasc", "rho", "wc"):
                hs[k][...] = w[k]
            l, ls = dev.scalar_transport_rk_adjoint(l, rho_old=w["rho_old"])
            ls_sum = [a + b for a, b in zip(ls_sum, ls)]
    finally:
        dev.close()
    return dict(g=g, tr=tr, emis=emis, opts=opts, lam=lam, g0=g0, gs=gs, after=after, restored=restored,
                after_ref=after_ref, winds=winds, ref0=l, refs=ls_sum)


def test_window_forward_equals_stepwise_run(window_runs):
    r = window_runs
    for a, b in zip(r["after"], r["after_ref"]):
        assert np.array_equal(a, b)
    for a, b in zip(r["restored"], r["after"]):
        assert np.array_equal(a, b)


def test_window_adjoint_equals_uncheckpointed_chain(window_runs):
    r = window_runs
    for n in range(NTR):
        assert relerr(r["g0"][n][1:], r["ref0"][n][1:]) < 1e-6, n
        assert relerr(r["gs"][n][1:], r["refs"][n][1:]) < 1e-6, n


def _st(w):
    class St:
        pass
    s = St()
    for k, v in w.items():
        setattr(s, k, v)
    return s


def oracle_chain_forward(r, x, e):
    """FP64 oracle forward over the recorded winds: tracers x, emission e."""
    g, opts = r["g"], r["opts"]
    fg = abi.FortranGrid(g)
    scp = [np.asarray(t, np.float64) for t in x]
    for w in r["winds"]:
        sct = []
        for n in range(NTR):
            s = np.zeros((g.mwa, g.mza))
            s[np.arange(1, g.mwa), g.lpw[1:] - 1] = e[n][1:]
            sct.append(s)
        scp = list(oracle_lib.scalar_transport(fg, opts, scp, sct, _st(w), fp64=True))
    return scp


def test_window_gradient_against_fp64_oracle_and_differences(window_runs):
    r = window_runs
    g, opts = r["g"], r["opts"]
    fg = abi.FortranGrid(g)
    # FP64 oracle adjoint chain over the same winds
    l = [x.astype(np.float64) for x in r["lam"]]
    ls_sum = [np.zeros((g.mwa, g.mza)) for _ in range(NTR)]
    for w in reversed(r["winds"]):
        la, ls = oracle_lib.scalar_transport_adjoint(fg, opts, l, _st(w), fp64=True)
        l = list(la)
        ls_sum = [a + b for a, b in zip(ls_sum, ls)]
    lpw0 = g.lpw - 1
    ge64 = [s[np.arange(g.mwa), lpw0] for s in ls_sum]
    ge32 = [s[np.arange(g.mwa), lpw0] for s in r["gs"]]
    for n in range(NTR):
        assert relerr(r["g0"][n][1:], l[n][1:]) < 1e-5, n
        assert relerr(ge32[n][1:], ge64[n][1:]) < 1e-5, n
    # central differences of the FP64 forward chain along seeded directions
    rng = np.random.default_rng(17)

    def J(scp):
        return sum(float((scp[n] * r["lam"][n].astype(np.float64)).sum()) for n in range(NTR))
    for _ in range(50):
        dx = [rng.standard_normal((g.mwa, g.mza)) * t for t in r["tr"]]
        de = [rng.standard_normal(g.mwa) * e for e in r["emis"]]
        for a in dx:
            a[0] = 0.0
        h = 1e-3
        jp = J(oracle_chain_forward(r, [t + h * d for t, d in zip(r["tr"], dx)],
                                    [e + h * d for e, d in zip(r["emis"], de)]))
        jm = J(oracle_chain_forward(r, [t - h * d for t, d in zip(r["tr"], dx)],
                                    [e - h * d for e, d in zip(r["emis"], de)]))
        fd = (jp - jm) / (2 * h)
        dot64 = sum(float((l[n] * dx[n]).sum() + (ge64[n] * de[n]).sum()) for n in range(NTR))
        dot32 = sum(float((r["g0"][n].astype(np.float64) * dx[n]).sum() + (ge32[n] * de[n]).sum())
                    for n in range(NTR))
        assert abs(fd - dot64) <= 1e-9 * abs(fd), (fd, dot64)
        assert abs(fd - dot32) <= 1e-5 * abs(fd), (fd, dot32)


def test_window_host_checkpoints_and_parts(window_runs):
    """The window with its checkpoints and final state in page-locked host
    memory, a checkpoint every 3 steps, the adjoint holding one step's
    inputs at a time (each step of a segment from its checkpoint again) and
    lean (its lam arrays in the tracer buffers, the tendencies' adjoint
    summed in place): the same gradient of the initial tracers bit for bit
    as device checkpoints every 2 steps reversed a segment at a time with
    the adjoint's own buffers, the emission's to 1e-6 (the sum over the
    steps rounds in another order).  Then the model goes on: one more long
    step (recorded again, the per-tracer arrays allocated anew) equals the
    window's own run continued by one step."""
    r = window_runs
    g, ds, tr, emis = case()
    dev, hs, var_p = new_device(g, ds, tr, emis, r["opts"])
    try:
        with pytest.raises(Exception):
            dev.window_memory(True, 1, NSTEPS, 3)      # no long step yet: sizes unknown
        dev.window_memory(True, 1, lean=True)           # host memory taken by the window itself
        dev.window_forward(NSTEPS, 3, abi.TS_GRAPH)
        lam = [x.copy() for x in r["lam"]]
        g0, gs = dev.window_adjoint(lam, in_place=True)
        assert g0[0] is lam[0]
        dev.sync_to_host(abi.F_SCALARS)
        restored = [t.copy() for t in var_p]
        dev.timestep(abi.TS_GRAPH)
        dev.sync_to_host(abi.F_SCALARS)
        next_step = [t.copy() for t in var_p]
        dev.window_memory(True, 0, NSTEPS, 3)          # sizes known now: reserved at once
    finally:
        dev.close()
    for n in range(NTR):
        assert np.array_equal(g0[n], r["g0"][n]), n
        assert relerr(gs[n][1:], r["gs"][n][1:]) < 1e-6, n
        assert np.array_equal(restored[n], r["after"][n]), n
    dev, hs, var_p = new_device(g, ds, tr, emis, r["opts"])
    try:
        for _ in range(NSTEPS + 1):
            dev.timestep(0)
        dev.sync_to_host(abi.F_SCALARS)
        ref = [t.copy() for t in var_p]
    finally:
        dev.close()
    for n in range(NTR):
        assert np.array_equal(next_step[n], ref[n]), n


def test_window_rewind_runs_the_window_again(window_runs):
    """After the window and its adjoint, olamgpu_window_rewind puts the
    window's start back; with the initial tracers sent again the same long
    steps give the window's own end state bit for bit (the next iteration
    of an inversion runs on the same winds)."""
    r = window_runs
    g, ds, tr, emis = case()
    dev, hs, var_p = new_device(g, ds, tr, emis, r["opts"])
    try:
        dev.window_memory(False, 0, lean=True)
        dev.window_forward(NSTEPS, NCHK, abi.TS_GRAPH)
        dev.window_adjoint(r["lam"])
        dev.window_rewind()
        for t, t0 in zip(var_p, tr):
            t[...] = t0
        dev.sync_to_device(abi.F_SCALARS)
        for _ in range(NSTEPS):
            dev.timestep(abi.TS_GRAPH)
        dev.sync_to_host(abi.F_SCALARS)
        again = [t.copy() for t in var_p]
    finally:
        dev.close()
    for n in range(NTR):
        assert np.array_equal(again[n], r["after"][n]), n


def test_surface_emission_adds_mass():
    g, ds, tr, emis = case()
    opts = abi.make_opts(DT, nacoust=4, nrk_scal=2)
    dev, hs, var_p = new_device(g, ds, tr, emis, opts)
    try:
        ids = list(range(1, NTR + 1))
        m0 = dev.mass_sums(ids)
        dev.timestep(0)
        m1 = dev.mass_sums(ids)
    finally:
        dev.close()
    vol = g.volt[np.arange(1, g.mwa), g.lpw[1:] - 1]
    for n in range(NTR):
        added = DT * float((emis[n][1:].astype(np.float64) * vol).sum())
        assert abs((m1[1 + n] - m0[1 + n]) - added) <= 1e-4 * added, (n, m1[1 + n] - m0[1 + n], added)
