"""GPU test of olamgpu_update_scalar_noalloc, the stage entry point that
allocates nothing: two stages through it in a row reproduce one RK2
scalar_transport_rk of the library's plain form, and the two calls leave the
device's free memory unchanged.  Collected last so it also runs after every
other GPU test in the same process."""
import ctypes as C

import numpy as np
import pytest

from conftest import relerr, small_case
from olam_b200 import abi
from olam_b200.lib import HostState, OlamGpu, check

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order,terrain", [(2, 0), (3, 0), (2, 3)])
def test_noalloc_two_stages_match_transport(order, terrain):
    import torch
    g, st = small_case(nxp=6, nlev=12, ntr=1, seed=31)
    if terrain:
        from olam_b200.synth.grid import with_terrain
        g = with_terrain(g, terrain)                   # lpw / lpv floors of a mountain
    opts = abi.make_opts(1800.0, scal_order=order)    # RK2, no limiter
    fg = abi.FortranGrid(g)
    hs = HostState(vmasc=st.vmasc, wmasc=st.wmasc, rho=st.rho, wc=st.wc)
    dev = OlamGpu(fg, opts, hs)
    try:
        dev.set_transport_form(abi.TRANSPORT_PLAIN)
        var_p = [np.ascontiguousarray(st.tracers[0].copy())]
        var_t = [np.ascontiguousarray(st.sct[0].copy())]
        dev.register_scalars(var_p, var_t)
        diag = dev.scalar_transport_rk(st.rho_old, want_diag=True)
        assert diag.cfl_max < 0.9, "case must keep every column explicit"
        ref = var_p[0].copy()

        # device arrays owned by the caller (allocated here, not by the call)
        def dv(a):
            return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()
        scp0, sct = dv(st.tracers[0]), dv(st.sct[0])
        rhos = dv(st.rho.astype(np.float32))           # rhos(:,:,nrk) of RK2 = real(rho)
        vm, wm = dv(st.vmasc), dv(st.wmasc)
        s1, s2 = torch.zeros_like(scp0), torch.zeros_like(scp0)
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        L = dev.lib
        p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        dtl = np.float32(opts.dtlm)

        def stage(src, dtr, dst):
            check(L.olamgpu_update_scalar_noalloc(p(src), p(scp0), p(sct), p(rhos), p(vm), p(wm),
                                                  C.c_float(dtr), p(dst), stream))

        stage(scp0, dtl * np.float32(0.5), s1)         # first call on the device: set-up
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        for _ in range(2):                             # two full passes, each two calls in a row
            stage(scp0, dtl * np.float32(0.5), s1)
            stage(s1, dtl * np.float32(1.0), s2)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0
        out = s2.cpu().numpy()
    finally:
        dev.close()
    e = relerr(out[1:], ref[1:])
    assert e < 1e-6, e


def test_noalloc_rejects_null_arrays():
    g, st = small_case(nxp=4, nlev=8, ntr=1)
    fg = abi.FortranGrid(g)
    dev = OlamGpu(fg, abi.make_opts(1800.0), HostState(vmasc=st.vmasc, wmasc=st.wmasc, rho=st.rho))
    try:
        rc = dev.lib.olamgpu_update_scalar_noalloc(None, None, None, None, None, None, C.c_float(1.0),
                                                   None, None)
        assert rc == abi.E_ARG
    finally:
        dev.close()


def test_noalloc_rejects_a_grid_beyond_the_scratch():
    # NXP = 75 with 60 levels at order 2 needs 50 NXP^2 mza + ... > 16 Mi floats
    from olam_b200.synth.grid import build_grid, stretched_levels
    from olam_b200.synth.state import transport_state
    g = build_grid(75, stretched_levels(60, 100.0, 30000.0), seed=5)
    st = transport_state(g, 600.0, 0, seed=5)
    fg = abi.FortranGrid(g)
    dev = OlamGpu(fg, abi.make_opts(600.0), HostState(vmasc=st.vmasc, wmasc=st.wmasc, rho=st.rho))
    try:
        import torch
        a = torch.zeros(g.mwa * g.mza, dtype=torch.float32, device="cuda")
        v = torch.zeros(g.mva * g.mza, dtype=torch.float32, device="cuda")
        p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        rc = dev.lib.olamgpu_update_scalar_noalloc(p(a), p(a), p(a), p(a), p(v), p(a), C.c_float(1.0),
                                                   p(a), None)
        assert rc == abi.E_ARG
        assert b"scratch" in dev.lib.olamgpu_strerror(rc)
    finally:
        dev.close()
