"""The NCCL halo hook's pairing of sends and receives (olam_b200/nccl_halo.py),
run over gloo on CPU with host buffers: every rank sends each neighbour the
columns the plan lists and receives its own, in one batch per exchange, with
unequal message sizes and a neighbour that only receives."""
import ctypes
import socket

import numpy as np
import pytest


def _rank_main(rank, world, port, q):
    try:
        import contextlib
        from datetime import timedelta

        import torch.distributed as dist

        from olam_b200.nccl_halo import host_view, nccl_exchange
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                timeout=timedelta(seconds=60))
        fn = nccl_exchange(dist, view=host_view, on_stream=lambda s: contextlib.nullcontext())
        # rank r sends (r + 1) * 100 + 10 * peer floats to each peer; rank 0
        # sends nothing to the last rank (which still sends to it)
        def count(src, dst):
            if src == 0 and dst == world - 1 and world > 2:
                return 0
            return (src + 1) * 100 + 10 * dst
        peers = [r for r in range(world) if r != rank]
        sends = [np.full(count(rank, p), rank * 1000.0 + p, np.float32) + np.arange(count(rank, p), dtype=np.float32)
                 for p in peers]
        recvs = [np.zeros(count(p, rank), np.float32) for p in peers]
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p).value or 0   # noqa: E731
        for _ in range(2):   # the hook runs once per stage: twice in a row
            for r in recvs:
                r[...] = 0.0
            rc = fn(peers, [(ptr(a), a.size) for a in sends], [(ptr(a), a.size) for a in recvs], 0)
            assert rc == 0
            for p, r in zip(peers, recvs):
                want = np.full(count(p, rank), p * 1000.0 + rank, np.float32) + np.arange(count(p, rank),
                                                                                             dtype=np.float32)
                assert np.array_equal(r, want), (rank, p)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, "ok"))
    except Exception as e:  # report to the parent instead of hanging it
        q.put((rank, repr(e)))


@pytest.mark.parametrize("world", [2, 3])
def test_hook_pairs_sends_and_receives(world):
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        assert res[r] == "ok", res[r]
