"""GPU tests of the long step on the device: olamgpu_timestep against the
same sequence of single calls, its recorded graph against the unrecorded
step, and the glue around the hot path -- set_scalars_bottom
(omodel/obnd.f90:7-36), diagvel_t3d (omodel/vel_t3d.f90:7-35),
tracer_maxmin and the mass sums (outils/check_nans.F90:164-550) -- against
numpy restatements (tests/numpy_ref.py)."""
import numpy as np
import pytest

import numpy_ref
import oracle_lib
from olam_b200 import abi
from olam_b200.lib import HostState, OlamGpu
from olam_b200.synth.state import eddy_inputs, fast_lognormal_tracers
from test_dynamics_gpu import dyn_case

pytestmark = pytest.mark.gpu

STATE_FIELDS = ("rho", "press", "thil", "wc", "wmc", "vxe", "vye", "vze", "vmc", "vc", "vmasc", "wmasc")


def _case(nxp=6, nlev=12, ntr=8, seed=4):
    g, ds = dyn_case(nxp, nlev, seed)
    arrays = oracle_lib.dyn_arrays(g, ds)
    tr = fast_lognormal_tracers(g, ntr, seed=seed, as_list=True)
    for q in tr:
        q[1:, 0] = -1.0      # below ground: set_scalars_bottom overwrites it
    return g, ds, arrays, tr


class Dev:
    """A library context on copies of the case's arrays."""

    def __init__(self, g, arrays, tr, opts, coherence=abi.RESIDENT):
        self.fg = abi.FortranGrid(g)
        self.hs = HostState(**{k: np.array(v, copy=True) for k, v in arrays.items()})
        self.dev = OlamGpu(self.fg, opts, self.hs)
        self.p = [q.copy() for q in tr]
        self.t = [np.zeros_like(q) for q in tr]
        self.dev.register_scalars(self.p, self.t)
        self.dev.set_coherence(coherence)

    def host(self):
        self.dev.sync_to_host(abi.F_ALL)
        return {**{n: self.hs[n].copy() for n in STATE_FIELDS}, "scp": np.stack(self.p)}

    def close(self):
        self.dev.close()


def _same(a, b):
    for n in a:
        assert np.array_equal(a[n], b[n], equal_nan=True), n


def test_timestep_matches_single_calls():
    g, _, arrays, tr = _case()
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
    # below-ground tracer levels took the lowest level's value
    assert np.array_equal(out[1]["scp"][:, 1:, 0], out[1]["scp"][:, 1:, 1])


@pytest.mark.parametrize("eddy", [False, True])
def test_timestep_graph_replays_the_step(eddy):
    g, ds, arrays, tr = _case()
    opts = abi.make_opts(600.0, nacoust=4)
    flags = abi.TS_HORIZ_K if eddy else 0
    out, launches = [], []
    for graph in (False, True):
        d = Dev(g, arrays, tr, opts)
        try:
            if eddy:
                e = abi.make_eddy(eddy_inputs(g, ds.rho, ds.thil, ds.press, rayf_mix=True))
                d.dev.set_eddy(e)
            d.dev.profile(True, reset=True)
            d.dev.launch_count(reset=True)
            for _ in range(6):
                d.dev.timestep(flags | (abi.TS_GRAPH if graph else 0))
            launches.append(d.dev.launch_count())
            prof = d.dev.profile_read()
            d.dev.profile(False)
            out.append(d.host())
            if graph:
                # first step unrecorded, then one recording per buffer
                # rotation (3), then replays
                assert prof.get("timestep_graph", (0, 0))[1] == 5, prof
            else:
                assert "timestep_graph" not in prof
        finally:
            d.close()
    _same(out[0], out[1])
    assert launches[0] == launches[1] > 0


def test_timestep_graph_after_host_sync():
    # the host rewrites the tracers between recorded steps: the replay must
    # start from the new values
    g, _, arrays, tr = _case()
    opts = abi.make_opts(600.0, nacoust=4)
    out = []
    for graph in (False, True):
        d = Dev(g, arrays, tr, opts)
        try:
            for step in range(7):
                d.dev.timestep(abi.TS_GRAPH if graph else 0)
                if step == 4:
                    d.dev.sync_to_host(abi.F_SCALARS)
                    for q in d.p:
                        q *= np.float32(0.5)
                    d.dev.sync_to_device(abi.F_SCALARS)
            out.append(d.host())
        finally:
            d.close()
    _same(out[0], out[1])


def test_timestep_diagnostics():
    g, _, arrays, tr = _case(ntr=40)
    opts = abi.make_opts(600.0, nacoust=4)
    d = Dev(g, arrays, tr, opts)
    try:
        ids = [1, 7, 40]
        for _ in range(5):
            d.dev.timestep(abi.TS_GRAPH | abi.TS_MAXMIN | abi.TS_MASS, mass_ids=ids)
        smax, sums = d.dev.timestep_diag(len(tr), len(ids))
        h = d.host()
    finally:
        d.close()
    mm = numpy_ref.tracer_maxmin(h["scp"], g.lpw)
    assert np.array_equal(smax, mm)
    ref = numpy_ref.mass_sums(h["rho"], g.volt, [h["scp"][i - 1] for i in ids], g.lpw)
    assert np.allclose(sums, ref, rtol=1e-12, atol=0)


def test_glue_single_calls_sync():
    g, _, arrays, tr = _case(ntr=5)
    opts = abi.make_opts(600.0, nacoust=4)
    d = Dev(g, arrays, tr, opts, coherence=abi.SYNC_EACH_CALL)
    try:
        # set_scalars_bottom on the host arrays (thil too)
        d.hs["thil"][1:, 0] = -5.0
        d.dev.set_scalars_bottom()
        for q in d.p:
            assert np.array_equal(q[1:, 0], q[1:, 1])
        assert np.array_equal(d.hs["thil"][1:, 0], d.hs["thil"][1:, 1])
        # diagvel_t3d rebuilds vxe, vye, vze from wc and vc: after a short
        # step (which ends with the same computation) it changes nothing
        d.dev.tend0(np.zeros_like(d.hs["thil"]))
        d.dev.prog_wrtv_rk(1)
        keep = {n: d.hs[n].copy() for n in ("vxe", "vye", "vze")}
        for n in keep:
            d.hs[n][1:, 1:] = 0.0
        d.dev.diagvel_t3d()
        for n in keep:
            assert np.array_equal(d.hs[n][1:, 1:], keep[n][1:, 1:]), n
        # tracer_maxmin and mass sums of the host arrays
        mm = d.dev.tracer_maxmin(len(tr))
        assert np.array_equal(mm, numpy_ref.tracer_maxmin(np.stack(d.p), g.lpw))
        s1 = d.dev.mass_sums([2, 5])
        s2 = d.dev.mass_sums([2, 5])
        assert np.array_equal(s1, s2)        # fixed-order sums repeat bit for bit
        ref = numpy_ref.mass_sums(d.hs["rho"], g.volt, [d.p[1], d.p[4]], g.lpw)
        assert np.allclose(s1, ref, rtol=1e-12, atol=0)
        with pytest.raises(Exception):
            d.dev.mass_sums([6])
    finally:
        d.close()
