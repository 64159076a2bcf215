"""GPU edge cases through the C-ABI: no registered tracers, NaN values in the
diagnostics, and plans or arguments the library must reject with a status
(not a fault)."""
import numpy as np
import pytest

from conftest import small_case
from olam_b200 import abi, decomp
from olam_b200.lib import HostState, OlamGpu, OlamGpuError

pytestmark = pytest.mark.gpu


def _dev(g, st, opts=None):
    opts = opts or abi.make_opts(1800.0)
    hs = HostState(vmasc=st.vmasc, wmasc=st.wmasc, rho=st.rho, wc=st.wc)
    return OlamGpu(abi.FortranGrid(g), opts, hs)


def test_no_tracers():
    # num_scalar = 0: the step's loop over scalars never runs (the reference
    # does nothing either); the call succeeds and changes nothing
    g, st = small_case(nxp=5, nlev=8, ntr=1)
    dev = _dev(g, st)
    try:
        dev.register_scalars([], [])
        dev.scalar_transport_rk(st.rho_old)
        dev.set_coherence(abi.RESIDENT)
        dev.scalar_transport_rk(st.rho_old)
    finally:
        dev.close()


def test_maxmin_skips_nan():
    from test_timestep_gpu import Dev, _case
    import numpy_ref
    g, _, arrays, tr = _case(ntr=3)
    tr = [q.copy() for q in tr]
    tr[1][5, 4] = np.nan
    d = Dev(g, arrays, tr, abi.make_opts(600.0, nacoust=4), coherence=abi.SYNC_EACH_CALL)
    try:
        mm = d.dev.tracer_maxmin(3)
    finally:
        d.close()
    assert np.isfinite(mm).all()
    assert np.array_equal(mm, numpy_ref.tracer_maxmin(np.stack(tr), g.lpw))


def test_bad_halo_plans_rejected():
    g, st = small_case(nxp=6, nlev=8, ntr=2)
    loc = decomp.local_grid(g, decomp.bisect(g, 2), 0)

    def hook(ranks, sbuf, rbuf):
        return 0

    hs = HostState(vmasc=loc.v(st.vmasc), wmasc=loc.w(st.wmasc), rho=loc.w(st.rho), wc=loc.w(st.wc))
    dev = OlamGpu(abi.FortranGrid(loc.grid), abi.make_opts(1800.0), hs)
    try:
        # a halo column listed as a column to send
        bad = {r: np.concatenate([v, loc.recv[r][:1]]) for r, v in loc.send.items()}
        with pytest.raises(OlamGpuError):
            dev.set_halo(abi.make_halo(bad, loc.recv, hook))
        # an owned column listed as one to receive
        bad = {r: np.concatenate([v, loc.owned[:1]]) for r, v in loc.recv.items()}
        with pytest.raises(OlamGpuError):
            dev.set_halo(abi.make_halo(loc.send, bad, hook))
        # a hook that fails makes the step fail with a status
        dev.register_scalars([loc.w(t).copy() for t in st.tracers], [loc.w(t).copy() for t in st.sct])
        dev.set_halo(abi.make_halo(loc.send, loc.recv, lambda r, s, q: 3))
        with pytest.raises(OlamGpuError):
            dev.scalar_transport_rk(loc.w(st.rho_old))
        dev.set_halo(None)
    finally:
        dev.close()


def test_timestep_without_resident_mode_is_a_state_error():
    from test_timestep_gpu import Dev, _case
    g, _, arrays, tr = _case(ntr=2)
    d = Dev(g, arrays, tr, abi.make_opts(600.0, nacoust=4), coherence=abi.SYNC_EACH_CALL)
    try:
        with pytest.raises(OlamGpuError):
            d.dev.timestep(0)
        d.dev.set_coherence(abi.RESIDENT)
        d.dev.timestep(0)
        with pytest.raises(OlamGpuError):
            d.dev.timestep(abi.TS_HORIZ_K)      # no eddy inputs registered
    finally:
        d.close()
