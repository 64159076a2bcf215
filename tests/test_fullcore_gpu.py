"""The whole device long step at the full-dynamics configuration's size:
NXP=100 (100,002 columns), 60 levels, a balanced 35 m/s mid-latitude jet
with a 6.5 K/km lapse and a seeded Gaussian theta perturbation (0.5 K,
500 km), 5 lognormal FP32 tracers (median 1e-8, sigma_ln 1.5), long steps of
120 s with 4 acoustic RK3 steps and RK3 tracer transport.

Two long steps through olamgpu_timestep (replayed as a CUDA graph) against
the oracle's long step in FP64 (tend0, prog_wrtv_rk x nacoust, timeavg_momsc,
scalar_transport_rk, set_scalars_bottom: omodel/timestep.f90:66-319) and in
FP32 (the reference's declared precision).  Prints every field's max and RMS
relative error against FP64 and the FP32 oracle's own spread."""
import json

import numpy as np
import pytest

import oracle_lib
from olam_b200 import abi
from olam_b200.lib import HostState, OlamGpu

pytestmark = pytest.mark.gpu

NXP, NLEV, NTR, DT, NACOUST, NSTEPS = 100, 60, 5, 120.0, 4, 2


def errors(a, b, mask):
    """(max |a - b| / max |b|, sqrt(sum (a - b)^2 / sum b^2)) over mask."""
    a = np.asarray(a, np.float64)[mask]
    b = np.asarray(b, np.float64)[mask]
    d = a - b
    return float(np.abs(d).max() / np.abs(b).max()), float(np.sqrt((d * d).sum() / (b * b).sum()))


def oracle_run(fg, opts, arrays, tracers, lpw, fp64):
    """NSTEPS long steps of the oracle: the dynamics, then the tracer step
    on the time-averaged mass fluxes, then set_scalars_bottom."""
    o = oracle_lib.DynOracle(fg, opts, arrays, fp64=fp64)
    scp = [t.copy() for t in tracers]
    for _ in range(NSTEPS):
        ro = o.tend0()
        for j in range(1, opts.nacoust + 1):
            o.prog_wrtv_rk(j)
        o.timeavg_momsc()

        class St:
            pass
        st = St()
        st.vmasc, st.wmasc = o.a["vmasc"].astype(np.float32), o.a["wmasc"].astype(np.float32)
        st.rho, st.rho_old = o.a["rho"], ro.astype(np.float32)
        st.wc = o.a["wc"].astype(np.float32)
        out = oracle_lib.scalar_transport(fg, opts, scp, [np.zeros_like(scp[0])] * len(scp), st, fp64=fp64)
        scp = [x.astype(np.float64 if fp64 else np.float32) for x in out]
        # set_scalars_bottom (omodel/obnd.f90:7-36): levels below lpw take lpw's value
        kb = lpw.astype(np.int64) - 1
        below = np.arange(o.a["thil"].shape[1])[None, :] < kb[:, None]
        below[0] = False
        for f in scp + [o.a["thil"]]:
            f[below] = np.broadcast_to(f[np.arange(f.shape[0]), kb][:, None], f.shape)[below]
    return o.a, scp


@pytest.fixture(scope="module")
def fullcore():
    from olam_b200.synth.grid import build_grid, stretched_levels
    from olam_b200.synth.state import dynamics_state, fast_lognormal_tracers
    g = build_grid(NXP, stretched_levels(NLEV, 100.0, 30000.0), seed=4)
    ds = dynamics_state(g, seed=4)
    tr = fast_lognormal_tracers(g, NTR, seed=77, clip=(0.0, np.inf), zero_frac=0.0, as_list=True)
    fg = abi.FortranGrid(g)
    opts = abi.make_opts(DT, nacoust=NACOUST, nrk_wrtv=3, nrk_scal=3)
    arrays = oracle_lib.dyn_arrays(g, ds)
    a64, s64 = oracle_run(fg, opts, arrays, tr, g.lpw, True)
    a32, s32 = oracle_run(fg, opts, arrays, tr, g.lpw, False)
    hs = HostState(**{k: np.array(v, copy=True) for k, v in arrays.items()})
    dev = OlamGpu(fg, opts, hs)
    var_p = [t.copy() for t in tr]
    var_t = [np.zeros_like(t) for t in tr]
    try:
        dev.register_scalars(var_p, var_t)
        dev.set_coherence(abi.RESIDENT)
        for _ in range(NSTEPS):
            dev.timestep(abi.TS_GRAPH)
        dev.sync_to_host(abi.F_ALL)
    finally:
        dev.close()
    return g, hs, var_p, a64, s64, a32, s32


# thermodynamic fields and tracers are held to 1e-5 against FP64; the
# momentum fields (u: vmc, vc; w: wmc, wc) to 5x the reference precision's
# own distance from FP64 (the FP32 oracle), floored at 1e-5
THERMO = ("rho", "thil", "press")
MOMENTUM = ("vmc", "vc", "wmc", "wc")


def test_full_core_two_long_steps_against_fp64(fullcore):
    g, hs, var_p, a64, s64, a32, s32 = fullcore
    kk = np.arange(g.mza)[None, :]
    wmask = kk >= (g.lpw.astype(np.int64)[:, None] - 1)
    wmask[0] = False
    vmask = kk >= (g.lpv.astype(np.int64)[:, None] - 1)
    vmask[0] = False
    # the vertical mass flux lives on faces lpw-1 .. mza-1 (top and bottom are zero)
    report = {}
    for n in THERMO + MOMENTUM:
        m = vmask if n in ("vmc", "vc") else wmask
        if n in ("wmc", "wc"):
            m = m.copy()
            m[:, -1] = False
        report[n] = dict(zip(("max_rel", "rms_rel"), errors(hs[n], a64[n], m)),
                         fp32_oracle=dict(zip(("max_rel", "rms_rel"), errors(a32[n], a64[n], m))))
    for i in range(NTR):
        report[f"tracer{i}"] = dict(zip(("max_rel", "rms_rel"), errors(var_p[i], s64[i], wmask)),
                                    fp32_oracle=dict(zip(("max_rel", "rms_rel"), errors(s32[i], s64[i], wmask))))
    print("FULLCORE_REPORT " + json.dumps(report))
    for n in THERMO:
        assert report[n]["max_rel"] < 1e-5, (n, report[n])
    for n in MOMENTUM:
        bound = max(1e-5, 5.0 * report[n]["fp32_oracle"]["max_rel"])
        assert report[n]["max_rel"] < bound, (n, report[n], bound)
    for i in range(NTR):
        r = report[f"tracer{i}"]
        assert r["max_rel"] < 1e-5, (i, r)
