"""Horizontal decomposition of the global grid over ranks (one GPU each) and
the halo plan of the tracer step.

OLAM splits its W columns over MPI ranks and exchanges the border columns of
each tracer between RK stages (omodel/scalar_transport_rk.F90:315-322, 343,
379); its halo is one ring of columns, so update_scalar also exchanges the
reconstruction planes (:416-440).  Here a rank holds two rings of
neighbours, everything one tracer stage of an owned column reads (the
upwind cells of its faces and their gradient stencils), so one exchange of
the tracer values per stage suffices and the gradients of ring 1 are
recomputed locally instead of sent.

* ``bisect`` -- recursive coordinate bisection of the W columns, the scheme
  of omodel/para_decomp.F90:1-568: a group of columns given R ranks is cut
  across its longest Cartesian extent at the column count that gives the
  two parts numbers of columns in proportion to the ranks each keeps
  (R // 2 and the rest); groups split until each holds one rank.  (OLAM
  cuts a binned, area-weighted coordinate; the cut here is exact.)
* ``local_grid`` -- a rank's columns and their two rings as a grid of its
  own: W points owned first, then ring 1, then ring 2 (each part in global
  order); the V points of every edge of owned and ring-1 cells; the M points
  whose three W corners are all local.  Tables point at local indices
  (0, the dummy point, where the neighbour is not local).  jtw_prog lists
  the owned columns, jtv_wadj the edges of owned columns.
* the halo plan -- for every other rank, the local columns it owns that
  this rank holds (``recv``) and this rank's owned columns that it holds
  (``send``), both in global order so that the two sides of a pair agree.

Column arrays of a rank are the global arrays indexed by ``wmap`` / ``vmap``
(``Local.w(a)``, ``Local.v(a)``); after each RK stage every rank sends
``a[send[r]]`` to rank r and writes what it receives into ``a[recv[r]]``.
"""
from __future__ import annotations

import numpy as np

from .synth.grid import Grid

# index tables of the synthetic grid and the point kind their values name
_TABLES = {"itab_w_iv": "v", "itab_w_iw": "w", "itab_w_im": "m", "itab_v_iw": "w", "itab_v_im": "m",
           "itab_m_iv": "v", "itab_m_iw": "w", "itab_m_im": "m"}
# coordinate arrays stored (3, n)
_COORDS = {"xew": "w", "xev": "v", "xem": "m"}


def bisect(g, nparts):
    """Rank (0 .. nparts-1) owning each W point; -1 for the dummy point."""
    if nparts < 1 or nparts > g.mwa - 1:
        raise ValueError(f"cannot split {g.mwa - 1} columns over {nparts} ranks")
    xyz = np.asarray(g.xew, dtype=np.float64).T
    owner = np.full(g.mwa, -1, dtype=np.int32)

    def split(cols, r0, nr):
        if nr == 1:
            owner[cols] = r0
            return
        p = xyz[cols]
        ax = int(np.argmax(p.max(axis=0) - p.min(axis=0)))
        order = cols[np.argsort(p[:, ax], kind="stable")]
        n1 = nr // 2
        ncut = int(round(len(cols) * n1 / nr))
        split(order[:ncut], r0, n1)
        split(order[ncut:], r0 + n1, nr - n1)

    split(np.arange(1, g.mwa), 0, nparts)
    return owner


def _neighbours(g, cells):
    nb = g.itab_w_iw[cells]
    valid = np.arange(nb.shape[1])[None, :] < g.npoly[cells][:, None]
    return np.unique(nb[valid])


def _rings(g, owned):
    own = set(owned.tolist())
    r1 = np.array(sorted(set(_neighbours(g, owned).tolist()) - own), dtype=np.int64)
    r2 = np.array(sorted(set(_neighbours(g, r1).tolist()) - own - set(r1.tolist())), dtype=np.int64)
    return r1, r2


class Local:
    """One rank's part of the grid: ``grid`` (a synth Grid over local
    indices), the maps from local to global array indices, the counts of
    owned and halo columns, and the halo plan."""

    def __init__(self, grid, wmap, vmap, mmap, nown, send, recv):
        self.grid, self.wmap, self.vmap, self.mmap = grid, wmap, vmap, mmap
        self.nown = nown
        self.send, self.recv = send, recv
        # V- and M-point plans of the acoustic step (filled by local_grid)
        self.send_v, self.recv_v, self.send_m, self.recv_m = {}, {}, {}, {}

    def w(self, a):
        """A global W-point array restricted to this rank's points."""
        return np.ascontiguousarray(a[self.wmap])

    def v(self, a):
        return np.ascontiguousarray(a[self.vmap])

    @property
    def owned(self):
        """Local array indices of the owned columns."""
        return np.arange(1, 1 + self.nown)


def local_grid(g, owner, rank):
    """The Local part of rank ``rank`` under the decomposition ``owner``."""
    owned = np.nonzero(owner == rank)[0].astype(np.int64)
    if owned.size == 0:
        raise ValueError(f"rank {rank} owns no column")
    r1, r2 = _rings(g, owned)
    wmap = np.concatenate([[0], owned, r1, r2]).astype(np.int64)
    core = np.concatenate([owned, r1])
    ev = g.itab_w_iv[core]
    valid = np.arange(ev.shape[1])[None, :] < g.npoly[core][:, None]
    vmap = np.concatenate([[0], np.unique(ev[valid])]).astype(np.int64)
    winv = np.zeros(g.mwa, dtype=np.int64)
    winv[wmap[1:]] = np.arange(1, wmap.size)
    vinv = np.zeros(g.mva, dtype=np.int64)
    vinv[vmap[1:]] = np.arange(1, vmap.size)
    cand = np.unique(g.itab_w_im[wmap[1:]])
    cand = cand[cand > 0]
    allw = np.all(winv[g.itab_m_iw[cand]] > 0, axis=1)
    mmap = np.concatenate([[0], cand[allw]]).astype(np.int64)
    minv = np.zeros(g.mma, dtype=np.int64)
    minv[mmap[1:]] = np.arange(1, mmap.size)
    sizes = {"w": g.mwa, "v": g.mva, "m": g.mma}
    if len({g.mwa, g.mva, g.mma, g.mza}) != 4:
        raise ValueError("grid sizes must differ to tell W, V, M and vertical arrays apart")
    maps = {"w": wmap, "v": vmap, "m": mmap}
    invs = {"w": winv, "v": vinv, "m": minv}

    lg = Grid()
    for name, a in vars(g).items():
        if not isinstance(a, np.ndarray):
            setattr(lg, name, a)
            continue
        if name in _COORDS:
            b = a[:, maps[_COORDS[name]]]
        else:
            kind = next((k for k, n in sizes.items() if a.ndim and a.shape[0] == n), None)
            b = a[maps[kind]] if kind else a.copy()
        if name in _TABLES:
            b = invs[_TABLES[name]][b].astype(a.dtype)
        setattr(lg, name, np.ascontiguousarray(b))
    lg.mwa, lg.mva, lg.mma = wmap.size, vmap.size, mmap.size
    # loop tables (1-based, as OLAM's jtab): owned columns and their edges
    lg.jtw_prog = (np.arange(1, 1 + owned.size) + 1).astype(np.int32)
    lg.jtw_wadj = (np.arange(1, 1 + owned.size + r1.size) + 1).astype(np.int32)
    oe = g.itab_w_iv[owned]
    ovalid = np.arange(oe.shape[1])[None, :] < g.npoly[owned][:, None]
    lg.jtv_wadj = (np.sort(vinv[np.unique(oe[ovalid])]) + 1).astype(np.int32)
    # a V point belongs to the rank of its W neighbour iw(mod(iv,2)+1)
    # (para_decomp.F90, V rank from the nearest W) -- global V index parity
    vg = vmap[1:]
    side = (vg + 1) % 2          # Fortran iv = vg + 1; mod(iv, 2) + 1 -> 0-based side
    vowner = owner[g.itab_v_iw[vg, side]]
    lg.jtv_prog = (np.nonzero(vowner == rank)[0] + 2).astype(np.int32)
    mown = np.all(winv[g.itab_m_iw[mmap[1:]]] > 0, axis=1) & (owner[g.itab_m_iw[mmap[1:], 0]] == rank)
    lg.jtm_prog = (np.nonzero(mown)[0] + 2).astype(np.int32)

    # halo plan
    nranks = int(owner.max()) + 1
    halo = np.concatenate([r1, r2])
    send, recv = {}, {}
    for r in range(nranks):
        if r == rank:
            continue
        mine = halo[owner[halo] == r]
        if mine.size:
            recv[r] = winv[np.sort(mine)]
        other = np.nonzero(owner == r)[0]
        h1, h2 = _rings(g, other)
        theirs = np.concatenate([h1, h2])
        theirs = theirs[owner[theirs] == rank]
        if theirs.size:
            send[r] = winv[np.sort(theirs)]
    loc = Local(lg, wmap, vmap, mmap, owned.size, send, recv)
    # V and M points: owned by the rank of a W point (para_decomp.F90: a V
    # point by its W neighbour iw(mod(iv,2)+1), here an M point by its first
    # W corner); the rank that owns one holds it (an edge, or a corner set,
    # of its own columns), so every point held but not owned is received
    # from its owner, in global order on both sides
    vown, mown_all = v_owner(g, owner), m_owner(g, owner)
    for r in range(nranks):
        if r == rank:
            continue
        mine_v = vmap[1:][vown[vmap[1:]] == r]
        if mine_v.size:
            loc.recv_v[r] = vinv[np.sort(mine_v)]
        mine_m = mmap[1:][mown_all[mmap[1:]] == r]
        if mine_m.size:
            loc.recv_m[r] = minv[np.sort(mine_m)]
        ov, om = _held_vm(g, owner, r)
        theirs_v = ov[vown[ov] == rank]
        if theirs_v.size:
            loc.send_v[r] = vinv[np.sort(theirs_v)]
        theirs_m = om[mown_all[om] == rank]
        if theirs_m.size:
            loc.send_m[r] = minv[np.sort(theirs_m)]
    return loc


def v_owner(g, owner):
    """Rank owning each V point (the rank of its W neighbour iw(mod(iv,2)+1),
    iv the 1-based index); -1 for the dummy point."""
    vg = np.arange(g.mva)
    side = (vg + 1) % 2
    o = owner[g.itab_v_iw[vg, side]].astype(np.int32)
    o[0] = -1
    return o


def m_owner(g, owner):
    """Rank owning each M point (the rank of its first W corner)."""
    o = owner[g.itab_m_iw[:, 0]].astype(np.int32)
    o[0] = -1
    return o


def _held_vm(g, owner, r):
    """The V and M points (global indices) that rank r holds."""
    owned = np.nonzero(owner == r)[0].astype(np.int64)
    r1, r2 = _rings(g, owned)
    core = np.concatenate([owned, r1])
    ev = g.itab_w_iv[core]
    valid = np.arange(ev.shape[1])[None, :] < g.npoly[core][:, None]
    vset = np.unique(ev[valid])
    held = np.zeros(g.mwa, bool)
    held[np.concatenate([owned, r1, r2])] = True
    cand = np.unique(g.itab_w_im[np.concatenate([owned, r1, r2])])
    cand = cand[cand > 0]
    mset = cand[np.all(held[g.itab_m_iw[cand]], axis=1)]
    return vset, mset


def exchange(a, loc, dist):
    """Halo exchange of one column array (first axis = local W index) over a
    torch.distributed process group (CPU tensors; gloo): owned columns go to
    the ranks that hold them, halo columns are overwritten with their
    owners' values.  Every rank of the group must call it."""
    import torch
    ops, bufs = [], []
    for r, idx in sorted(loc.send.items()):
        t = torch.from_numpy(np.ascontiguousarray(a[idx]))
        ops.append(dist.P2POp(dist.isend, t, r))
    for r, idx in sorted(loc.recv.items()):
        t = torch.empty((idx.size,) + a.shape[1:], dtype=torch.from_numpy(a[:1]).dtype)
        bufs.append((idx, t))
        ops.append(dist.P2POp(dist.irecv, t, r))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for idx, t in bufs:
        a[idx] = t.numpy()
