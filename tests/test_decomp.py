"""CPU tests of the decomposition over ranks and the halo plan of the tracer
step (olam_b200/decomp.py): the partition, the local grids' tables, the
pairing of send and receive lists, and a two-rank tracer step over gloo with
one halo exchange per RK stage (omodel/scalar_transport_rk.F90:315-322, 343,
379) that reproduces the single-domain step on every owned column."""
import socket

import numpy as np
import pytest

import numpy_ref
from olam_b200 import decomp

_G = {}


def grid(nxp=8, nlev=10):
    from olam_b200.synth.grid import build_grid, stretched_levels
    if (nxp, nlev) not in _G:
        _G[(nxp, nlev)] = build_grid(nxp, stretched_levels(nlev, 100.0, 30000.0), seed=2)
    return _G[(nxp, nlev)]


@pytest.mark.parametrize("n", [1, 2, 3, 4, 7])
def test_bisect_partition(n):
    g = grid()
    o = decomp.bisect(g, n)
    assert o[0] == -1 and (o[1:] >= 0).all() and (o[1:] < n).all()
    cnt = np.bincount(o[1:], minlength=n)
    # parts are proportional to the ranks they hold: within one column
    # of an even split at every cut
    assert cnt.max() - cnt.min() <= 2
    # each part is compact: its columns' mean distance to their centroid is
    # well below that of the whole sphere
    x = np.asarray(g.xew, np.float64).T
    whole = np.linalg.norm(x[1:] - x[1:].mean(0), axis=1).mean()
    for r in range(n):
        p = x[o == r]
        if n > 1:
            assert np.linalg.norm(p - p.mean(0), axis=1).mean() < whole


@pytest.mark.parametrize("n", [2, 3])
def test_local_grid_tables(n):
    g = grid()
    o = decomp.bisect(g, n)
    for r in range(n):
        loc = decomp.local_grid(g, o, r)
        lg, wm, vm = loc.grid, loc.wmap, loc.vmap
        assert (o[wm[1:1 + loc.nown]] == r).all()
        assert (o[wm[1 + loc.nown:]] != r).all()
        # owned and ring-1 columns see every neighbour and edge locally, with
        # the same global identity and the same coefficients
        core = np.arange(1, lg.mwa)[:loc.nown + 0]
        r1 = np.array([i for i in range(1, lg.mwa)
                       if any(o[g.itab_w_iw[wm[i], k]] == r for k in range(g.npoly[wm[i]]))])
        for i in np.concatenate([core, r1]):
            npl = g.npoly[wm[i]]
            assert lg.npoly[i] == npl
            assert (lg.itab_w_iw[i, :npl] > 0).all()
            assert (wm[lg.itab_w_iw[i, :npl]] == g.itab_w_iw[wm[i], :npl]).all()
            assert (vm[lg.itab_w_iv[i, :npl]] == g.itab_w_iv[wm[i], :npl]).all()
            assert np.array_equal(lg.gxps_coef[i], g.gxps_coef[wm[i]])
        # every edge's W ends are the global ones where they are local
        ends = lg.itab_v_iw[1:]
        ok = ends > 0
        assert (wm[ends[ok]] == g.itab_v_iw[vm[1:]][ok]).all()
        # loop tables: the owned columns, 1-based
        assert np.array_equal(lg.jtw_prog, np.arange(2, loc.nown + 2))


def test_halo_plan_pairs():
    g = grid()
    n = 4
    o = decomp.bisect(g, n)
    locs = [decomp.local_grid(g, o, r) for r in range(n)]
    for q in range(n):
        for r, idx in locs[q].send.items():
            # what q sends to r is exactly what r expects from q, in order
            assert np.array_equal(locs[q].wmap[idx], locs[r].wmap[locs[r].recv[q]])
        for r, idx in locs[q].recv.items():
            assert (o[locs[q].wmap[idx]] == r).all()
        # every halo column is received from its owner
        halo = np.arange(1 + locs[q].nown, locs[q].grid.mwa)
        got = np.concatenate(list(locs[q].recv.values())) if locs[q].recv else np.zeros(0, int)
        assert np.array_equal(np.sort(got), halo)


def _case():
    from olam_b200.synth.state import fast_lognormal_tracers, transport_state
    g = grid()
    st = transport_state(g, 600.0, 0, seed=3)
    tr = fast_lognormal_tracers(g, 3, seed=5)
    sct = (1e-12 * np.random.default_rng(9).standard_normal(tr.shape)).astype(np.float32)
    return g, st, tr, sct


def _rank_main(rank, world, port, q):
    try:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                timeout=timedelta(seconds=120))
        g, st, tr, sct = _case()
        ref = numpy_ref.transport_plain(g, st, tr, sct, 600.0, nrk=2)
        loc = decomp.local_grid(g, decomp.bisect(g, world), rank)
        lg = loc.grid
        vm = loc.v(st.vmasc).astype(np.float64)
        wm = loc.w(st.wmasc).astype(np.float64)
        rhos = loc.w(st.rho).astype(np.float64)
        dtlr = 600.0 * np.array([0.5, 1.0])
        err = 0.0
        for n in range(tr.shape[0]):
            q0 = loc.w(tr[n]).astype(np.float64)
            t0 = loc.w(sct[n]).astype(np.float64)
            s = q0.copy()
            for ist in range(2):
                s = numpy_ref.plain_stage(lg, vm, wm, rhos, s, q0, t0, dtlr[ist])
                decomp.exchange(s, loc, dist)      # border columns for the next stage
            own = loc.owned
            a, b = s[own], ref[n][loc.wmap[own]]
            err = max(err, float(np.abs(a - b).max() / np.abs(b).max()))
            # after the last exchange the halo holds the owners' values too
            h = np.arange(1 + loc.nown, lg.mwa)
            err = max(err, float(np.abs(s[h] - ref[n][loc.wmap[h]]).max() / np.abs(ref[n]).max()))
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, err))
    except Exception as e:  # report to the parent instead of hanging it
        q.put((rank, repr(e)))


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_tracer_step_matches_single_domain(world):
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        assert not isinstance(res[r], str), res[r]
        assert res[r] < 1e-13, (r, res[r])
