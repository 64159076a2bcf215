"""GPU test of the halo exchange of the tracer step (olamgpu_set_halo;
omodel/scalar_transport_rk.F90:315-322, 343, 379): each rank of a two-way
decomposition (olam_b200/decomp.py) runs its part through the library, and
the exchange hook hands it, after every RK stage but the last, the border
values its neighbour computes (taken from the single-domain stages of the
numpy restatement).  Together the ranks' owned columns reproduce the
single-domain GPU step; the columns each rank sends are its own stage
values.  The last test runs the two ranks as two processes on the one GPU,
the hook moving the border columns over gloo."""
import numpy as np
import pytest

import numpy_ref
import oracle_lib
from conftest import relerr, small_case
from olam_b200 import abi, decomp
from olam_b200.lib import HostState, OlamGpu, OlamGpuError
from test_transport_gpu import run_gpu

pytestmark = pytest.mark.gpu


def _stages(g, st, dtlm, nrk):
    """Single-domain stage outputs (float64), [stage][tracer](mwa, mza)."""
    dt = dtlm * (np.array([1 / 3, 0.5, 1.0]) if nrk == 3 else np.array([0.5, 1.0]))
    vm, wm, rho = (st.vmasc.astype(np.float64), st.wmasc.astype(np.float64), st.rho.astype(np.float64))
    out = [[] for _ in range(nrk)]
    for q0, t0 in zip(st.tracers, st.sct):
        q0 = q0.astype(np.float64)
        t0 = t0.astype(np.float64)
        s = q0.copy()
        for k in range(nrk):
            s = numpy_ref.plain_stage(g, vm, wm, rho, s, q0, t0, dt[k])
            out[k].append(s)
    return [np.stack(o) for o in out]


def _rank(g, st, opts, loc, stages, form, nrk):
    ntr = len(st.tracers)
    ntp = (ntr + 3) // 4 * 4
    mza = g.mza
    calls = {"n": 0, "send_err": 0.0}

    def hook(ranks, sbuf, rbuf):
        k = calls["n"]
        calls["n"] += 1
        for r, sv, rv in zip(ranks, sbuf, rbuf):
            if r in loc.send:
                got = sv.reshape(len(loc.send[r]), mza, ntp)[:, :, :ntr]
                want = stages[k][:, loc.wmap[loc.send[r]], :].transpose(1, 2, 0)
                calls["send_err"] = max(calls["send_err"], relerr(got, want))
            if r in loc.recv:
                cols = loc.wmap[loc.recv[r]]
                blk = np.zeros((len(cols), mza, ntp), np.float32)
                blk[:, :, :ntr] = stages[k][:, cols, :].transpose(1, 2, 0)
                rv[:] = blk.ravel()
        return 0

    lg = loc.grid
    fg = abi.FortranGrid(lg)
    hs = HostState(vmasc=loc.v(st.vmasc), wmasc=loc.w(st.wmasc), rho=loc.w(st.rho), wc=loc.w(st.wc))
    dev = OlamGpu(fg, opts, hs)
    try:
        dev.set_transport_form(form)
        var_p = [loc.w(t).copy() for t in st.tracers]
        var_t = [loc.w(t).copy() for t in st.sct]
        dev.register_scalars(var_p, var_t)
        halo = abi.make_halo(loc.send, loc.recv, hook)
        dev.set_halo(halo)
        dev.scalar_transport_rk(loc.w(st.rho_old))
        return np.stack(var_p), calls
    finally:
        dev.close()


@pytest.mark.parametrize("form", [abi.TRANSPORT_FUSED, abi.TRANSPORT_FUSED_COLUMN])
@pytest.mark.parametrize("nrk", [2, 3])
def test_two_ranks_match_one_domain(form, nrk):
    g, st = small_case(nxp=8, nlev=12, ntr=6)
    opts = abi.make_opts(1800.0, nrk_scal=nrk)
    # the restatement has no implicit columns: the case must have none
    _, ff, _ = oracle_lib.scalar_transport(abi.FortranGrid(g), opts, st.tracers, st.sct, st, want_ff=True)
    assert not (ff > 0).any()
    ref, _ = run_gpu(g, st, opts, form)
    stages = _stages(g, st, 1800.0, nrk)
    owner = decomp.bisect(g, 2)
    covered = np.zeros(g.mwa, bool)
    for r in range(2):
        loc = decomp.local_grid(g, owner, r)
        out, calls = _rank(g, st, opts, loc, stages, form, nrk)
        assert calls["n"] == nrk - 1                 # after every stage but the last
        assert calls["send_err"] < 1e-5, calls
        own = loc.owned
        for n in range(len(st.tracers)):
            e = relerr(out[n][own], ref[n][loc.wmap[own]])
            assert e < 1e-5, (r, n, e)
        covered[loc.wmap[own]] = True
    assert covered[1:].all()


@pytest.mark.parametrize("nrk", [2, 3])
def test_device_buffer_hook_matches_one_domain(nrk):
    # the hook gets the library's device buffers and stream (as an NCCL or
    # CUDA-aware MPI exchange would); it checks the packed send columns and
    # writes the neighbour's stage values into the receive buffers with
    # copies ordered on that stream (olam_b200/nccl_halo.py's device views)
    import torch
    from olam_b200.nccl_halo import device_view
    g, st = small_case(nxp=8, nlev=12, ntr=6)
    opts = abi.make_opts(1800.0, nrk_scal=nrk)
    ref, _ = run_gpu(g, st, opts, abi.TRANSPORT_FUSED)
    stages = _stages(g, st, 1800.0, nrk)
    owner = decomp.bisect(g, 2)
    ntr, mza = len(st.tracers), g.mza
    ntp = (ntr + 3) // 4 * 4
    for rank in range(2):
        loc = decomp.local_grid(g, owner, rank)
        calls = {"n": 0, "send_err": 0.0}

        def hook(ranks, sbufs, rbufs, stream):
            k = calls["n"]
            calls["n"] += 1
            with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                for r, (sp, sn), (rp, rn) in zip(ranks, sbufs, rbufs):
                    if sn:
                        got = device_view(sp, sn).cpu().numpy().reshape(len(loc.send[r]), mza, ntp)[:, :, :ntr]
                        want = stages[k][:, loc.wmap[loc.send[r]], :].transpose(1, 2, 0)
                        calls["send_err"] = max(calls["send_err"], relerr(got, want))
                    if rn:
                        cols = loc.wmap[loc.recv[r]]
                        blk = np.zeros((len(cols), mza, ntp), np.float32)
                        blk[:, :, :ntr] = stages[k][:, cols, :].transpose(1, 2, 0)
                        device_view(rp, rn).copy_(torch.from_numpy(blk.ravel()).cuda())
            return 0

        fg = abi.FortranGrid(loc.grid)
        hs = HostState(vmasc=loc.v(st.vmasc), wmasc=loc.w(st.wmasc), rho=loc.w(st.rho), wc=loc.w(st.wc))
        dev = OlamGpu(fg, opts, hs)
        try:
            var_p = [loc.w(t).copy() for t in st.tracers]
            var_t = [loc.w(t).copy() for t in st.sct]
            dev.register_scalars(var_p, var_t)
            dev.set_halo(abi.make_halo_device(loc.send, loc.recv, hook))
            dev.set_coherence(abi.RESIDENT)
            dev.scalar_transport_rk(loc.w(st.rho_old))
            dev.sync_to_host(abi.F_SCALARS)
        finally:
            dev.close()
        assert calls["n"] == nrk - 1
        assert calls["send_err"] < 1e-5, calls
        own = loc.owned
        for n in range(ntr):
            assert relerr(var_p[n][own], ref[n][loc.wmap[own]]) < 1e-5, (rank, n)


def test_halo_needs_the_unlimited_batched_step():
    g, st = small_case(nxp=6, nlev=8, ntr=2)
    loc = decomp.local_grid(g, decomp.bisect(g, 2), 0)
    opts = abi.make_opts(1800.0)
    with pytest.raises(OlamGpuError):
        _rank(g, st, opts, loc, _stages(g, st, 1800.0, 2), abi.TRANSPORT_PLAIN, 2)


def _proc_main(rank, world, port, q, terrain=0):
    """One rank of a decomposed tracer step as its own process: its part of
    the grid through the library, the exchange hook moving the packed border
    columns over gloo (host-staged)."""
    try:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                timeout=timedelta(seconds=120))
        g, st = small_case(nxp=8, nlev=12, ntr=6)
        if terrain:
            from olam_b200.synth.grid import with_terrain
            g = with_terrain(g, terrain, width=2.0)
        opts = abi.make_opts(1800.0, nrk_scal=3)
        loc = decomp.local_grid(g, decomp.bisect(g, world), rank)
        calls = {"n": 0}

        def hook(ranks, sbuf, rbuf):
            calls["n"] += 1
            ops, got = [], []
            for r, sv, rv in zip(ranks, sbuf, rbuf):
                if sv.size:
                    ops.append(dist.P2POp(dist.isend, torch.from_numpy(sv.copy()), r))
                if rv.size:
                    t = torch.empty(rv.size, dtype=torch.float32)
                    got.append((rv, t))
                    ops.append(dist.P2POp(dist.irecv, t, r))
            for req in dist.batch_isend_irecv(ops):
                req.wait()
            for rv, t in got:
                rv[:] = t.numpy()
            return 0

        fg = abi.FortranGrid(loc.grid)
        hs = HostState(vmasc=loc.v(st.vmasc), wmasc=loc.w(st.wmasc), rho=loc.w(st.rho), wc=loc.w(st.wc))
        dev = OlamGpu(fg, opts, hs)
        try:
            var_p = [loc.w(t).copy() for t in st.tracers]
            var_t = [loc.w(t).copy() for t in st.sct]
            dev.register_scalars(var_p, var_t)
            dev.set_halo(abi.make_halo(loc.send, loc.recv, hook))
            dev.scalar_transport_rk(loc.w(st.rho_old))
        finally:
            dev.close()
        own = loc.owned
        q.put((rank, loc.wmap[own], np.stack([p[own] for p in var_p]), calls["n"]))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:   # report to the parent instead of hanging it
        q.put((rank, repr(e), None, None))


@pytest.mark.parametrize("terrain", [0, 4])
def test_two_processes_over_gloo(terrain):
    # two ranks as two processes sharing the GPU: no kernel waits on the
    # other rank (each hook call follows a finished stage on the host), the
    # border columns move over gloo; together the ranks reproduce the
    # one-domain step (flat, and with a mountain across the ranks' border)
    import socket
    import torch.multiprocessing as mp
    g, st = small_case(nxp=8, nlev=12, ntr=6)
    if terrain:
        from olam_b200.synth.grid import with_terrain
        g = with_terrain(g, terrain, width=2.0)
        owner = decomp.bisect(g, 2)
        assert all((g.lpw[1:][owner[1:] == r] > 2).sum() > 50 for r in range(2))
    opts = abi.make_opts(1800.0, nrk_scal=3)
    ref, _ = run_gpu(g, st, opts, abi.TRANSPORT_FUSED)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_proc_main, args=(r, 2, port, q, terrain)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    covered = np.zeros(g.mwa, bool)
    for rank, cols, vals, n in res:
        assert not isinstance(cols, str), cols
        assert n == 2                                  # RK3: after stages 1 and 2
        for t in range(len(st.tracers)):
            e = relerr(vals[t], ref[t][cols])
            assert e < 1e-5, (rank, t, e)
        covered[cols] = True
    assert covered[1:].all()


def _gloo_hook(dist, torch):
    def hook(ranks, sbuf, rbuf):
        ops, got = [], []
        for r, sv, rv in zip(ranks, sbuf, rbuf):
            if sv.size:
                ops.append(dist.P2POp(dist.isend, torch.from_numpy(sv.copy()), r))
            if rv.size:
                t = torch.empty(rv.size, dtype=torch.float32)
                got.append((rv, t))
                ops.append(dist.P2POp(dist.irecv, t, r))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for rv, t in got:
            rv[:] = t.numpy()
        return 0
    return hook


W_OUT = ("rho", "press", "thil", "wc", "wmc", "vxe", "vye", "vze", "wmasc")
V_OUT = ("vmc", "vc", "vmasc")


def _long_case():
    from olam_b200.synth.state import fast_lognormal_tracers
    from test_dynamics_gpu import dyn_case
    g, ds = dyn_case(nxp=8, nlev=12, seed=4)
    arrays = oracle_lib.dyn_arrays(g, ds)
    tr = fast_lognormal_tracers(g, 6, seed=8, as_list=True)
    return g, arrays, tr


def _long_steps(g, arrays, tr, halo=None, nsteps=2):
    opts = abi.make_opts(600.0, nacoust=4)
    hs = HostState(**{k: np.array(v, copy=True) for k, v in arrays.items()})
    dev = OlamGpu(abi.FortranGrid(g), opts, hs)
    p = [q.copy() for q in tr]
    t = [np.zeros_like(q) for q in tr]
    try:
        dev.register_scalars(p, t)
        dev.set_coherence(abi.RESIDENT)
        if halo is not None:
            dev.set_halo(halo)
        for _ in range(nsteps):
            dev.timestep(0)
        dev.sync_to_host(abi.F_ALL)
    finally:
        dev.close()
    return {n: hs[n] for n in W_OUT + V_OUT}, np.stack(p)


def _long_proc(rank, world, port, q):
    try:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                timeout=timedelta(seconds=120))
        g, arrays, tr = _long_case()
        loc = decomp.local_grid(g, decomp.bisect(g, world), rank)
        la = {k: (loc.w(v) if v.shape[0] == g.mwa else loc.v(v)) for k, v in arrays.items()}
        lt = [loc.w(x) for x in tr]
        halo = abi.make_halo(loc.send, loc.recv, _gloo_hook(dist, torch),
                             vm=(loc.send_v, loc.recv_v, loc.send_m, loc.recv_m))
        out, scp = _long_steps(loc.grid, la, lt, halo)
        own = loc.owned
        vown = loc.grid.jtv_prog - 1
        res = {"w": loc.wmap[own], "v": loc.vmap[vown], "scp": scp[:, own]}
        for n in W_OUT:
            res[n] = out[n][own]
        for n in V_OUT:
            res[n] = out[n][vown]
        q.put((rank, res))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:   # report to the parent instead of hanging it
        import traceback
        q.put((rank, repr(e) + traceback.format_exc()[-1500:]))


def test_long_step_two_processes_over_gloo():
    # two long steps of the whole dynamical core (olamgpu_timestep: the
    # acoustic steps with their damping and the tracer step) on a two-way
    # split, as two processes on the one GPU exchanging over gloo, against
    # the one-domain run
    import socket
    import torch.multiprocessing as mp
    g, arrays, tr = _long_case()
    ref, rscp = _long_steps(g, arrays, tr)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_long_proc, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    covw = np.zeros(g.mwa, bool)
    covv = np.zeros(g.mva, bool)
    for rank, r in res:
        assert not isinstance(r, str), r
        for n in W_OUT:
            e = relerr(r[n][:, 1:], ref[n][r["w"]][:, 1:])
            assert e < 1e-6, (rank, n, e)
        for n in V_OUT:
            e = relerr(r[n][:, 1:], ref[n][r["v"]][:, 1:])
            assert e < 1e-6, (rank, n, e)
        e = relerr(r["scp"], rscp[:, r["w"]])
        assert e < 1e-6, (rank, "scp", e)
        covw[r["w"]] = True
        covv[r["v"]] = True
    assert covw[1:].all() and covv[1:].all()
