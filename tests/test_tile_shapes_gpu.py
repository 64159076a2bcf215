"""GPU parity of every shape of the tiled transport kernel (columns per tile
T = 8, 16 or 32, tracers per block G, level chunks per tile KS, tile order)
against the FP64 oracle,
with and without terrain, and the autotuner that picks among them."""
import numpy as np
import pytest

import oracle_lib
from conftest import relerr, small_case
from olam_b200 import abi
from olam_b200.lib import HostState, OlamGpu

pytestmark = pytest.mark.gpu

TOL64 = 1e-5

# order: bit 0 the caller's column order, bit 1 the paired kernel (column
# pairs of 16-column tiles reading each U row once for both)
SHAPES = [(32, 64, 1, 0), (32, 32, 1, 0), (16, 64, 1, 0), (16, 128, 1, 0), (32, 128, 1, 0), (32, 64, 2, 0),
          (32, 32, 3, 1), (16, 128, 2, 1), (32, 128, 2, 1), (32, 64, 1, 1), (16, 128, 1, 2), (16, 128, 1, 3),
          (8, 128, 1, 0), (8, 128, 2, 1)]


def tracers(g, ntr, seed):
    from olam_b200.synth.state import fast_lognormal_tracers
    return fast_lognormal_tracers(g, ntr, seed=seed, as_list=True)


def run(g, st, opts, tr, shape=None, coherence=abi.RESIDENT, steps=1):
    fg = abi.FortranGrid(g)
    dev = OlamGpu(fg, opts, HostState(vmasc=st.vmasc, wmasc=st.wmasc, rho=st.rho, wc=st.wc))
    try:
        dev.set_coherence(coherence)
        if shape is not None:
            dev.set_tile_shape(*shape)
        var_p = [t.copy() for t in tr]
        var_t = [np.zeros_like(t) for t in tr]
        dev.register_scalars(var_p, var_t)
        for _ in range(steps):
            dev.scalar_transport_rk(st.rho_old)
        if coherence == abi.RESIDENT:
            dev.sync_to_host(abi.F_SCALARS)
        used, log = dev.tile_shape()
        return np.stack(var_p), used, log
    finally:
        dev.close()


@pytest.mark.parametrize("terrain", [0, 3])
@pytest.mark.parametrize("shape", SHAPES)
def test_tile_shape_parity(shape, terrain):
    g, st = small_case(nxp=6, nlev=12, ntr=1)
    if terrain:
        from olam_b200.synth.grid import with_terrain
        g = with_terrain(g, terrain)
    tr = tracers(g, 40, seed=5)       # 40 tracers: groups of 32 with a ragged last one
    opts = abi.make_opts(1800.0, nrk_scal=3 if shape[2] > 1 else 2)
    ref = oracle_lib.scalar_transport(abi.FortranGrid(g), opts, tr, [np.zeros_like(t) for t in tr], st, fp64=True)
    out, used, _ = run(g, st, opts, tr, shape)
    assert used == shape
    for n in range(len(tr)):
        assert relerr(out[n][1:], ref[n][1:]) < TOL64, (n, relerr(out[n][1:], ref[n][1:]))


def test_autotuner_picks_a_timed_shape_and_agrees_with_it():
    g, st = small_case(nxp=8, nlev=16, ntr=1)
    tr = tracers(g, 24, seed=8)
    opts = abi.make_opts(1800.0)
    out, used, log = run(g, st, opts, tr, steps=2)
    assert len(log) >= 4
    chosen = [r for r in log if r[4]]
    assert len(chosen) == 1 and chosen[0][:4] == used
    assert chosen[0][5] == min(r[5] for r in log)
    forced, used2, _ = run(g, st, opts, tr, shape=used, steps=2)
    assert used2 == used
    assert np.array_equal(out, forced)


def test_per_call_mode_with_a_tuned_shape():
    # the per-call step (more than 64 tracers) runs its 64-tracer groups with
    # the tuned tile width
    g, st = small_case(nxp=6, nlev=12, ntr=1)
    tr = tracers(g, 72, seed=9)
    opts = abi.make_opts(1800.0)
    ref = oracle_lib.scalar_transport(abi.FortranGrid(g), opts, tr, [np.zeros_like(t) for t in tr], st, fp64=True)
    for shape in ((16, 128, 2, 0), (32, 32, 1, 1)):
        out, used, _ = run(g, st, opts, tr, shape, coherence=abi.SYNC_EACH_CALL)
        for n in range(len(tr)):
            assert relerr(out[n][1:], ref[n][1:]) < TOL64, (shape, n)
