"""Synthetic OLAM global hexagonal grid (icosahedral Delaunay -> Voronoi).

This module builds, from the mathematics, the grid tables and metrics that
OLAM's hot path reads.  It is input generation for tests and benchmarks: in a
real run these arrays come from OLAM's own grid file.  It restates:

* icosahedral subdivision (``omodel/icosahedron.f90:1-331``): W points are the
  vertices of the subdivided icosahedron, 10*NXP**2+2 of them; M points are
  the triangles (20*NXP**2); V points are the triangle edges (30*NXP**2).
* ``voronoi`` / ``pcvt`` (``omodel/hex_grid.f90:1-414``): M points at the
  triangle circumcentres so that W cells are Voronoi cells; ``itab_w`` lists
  M/V/W neighbours counter-clockwise with ``dirv = -1`` when the W point is
  ``itab_v%iw(1)`` of the edge (``hex_grid.f90:185-205``).
* ``grid_geometry_hex`` (``hex_grid.f90:418-1125``): V points midway between
  W points, ``dnu/dnv``, normals, quarter-kite areas ``arw0/arm0``, ``farm/farv``,
  polar-stereographic gradient weights ``gxps1/2, gyps1/2``, ``dxps/dyps``,
  and the least-squares ``ecvec_v[xyz]`` coefficients.
* ``ctrlvols_hex_nosfcg`` for flat terrain (``hex_grid.f90:1608-1976``):
  ``arw, arv, volt`` with spherical expansion ``zfacm2, zfact``.
* ``gridset2`` with explicit levels (``omodel/olam_grid.f90:493-733``).
* ``alloc_gridz_other`` / ``alloc_grid_other`` (``modules/mem_grid.f90:350-618``).
* ``alloc_adv`` (``modules/mem_adv.f90:23-357``): vertical quadratic
  coefficients ``a_v/a_w/a_vu/a_wu``, horizontal least-squares ``xy_h/xy_hu``,
  ``xx0_v..yy0_vu``, Laplacian weights ``xx_yy``/``xx_yy_m``.

Index convention: every array keeps OLAM's Fortran layout with the horizontal
index LAST and slot 0 as OLAM's dummy point 1, so Fortran index ``i`` is
array index ``i-1``.  Neighbour tables hold 0-based indices into these arrays
(index 0 = dummy).  Column arrays are ``(n, mza)`` in C order, i.e. the same
bytes as Fortran ``(mza, n)``: k is contiguous.

Geometry is computed in float64 and stored as float32 where OLAM declares
``real`` (``real(r8)`` only for ``volt``), so values agree with OLAM's own
generator to float32 round-off of a restatement, not bit for bit.
"""
from __future__ import annotations

import numpy as np

ERAD = 6371.22e3          # consts_coms.f90 init_consts
ERAD2 = 2.0 * ERAD
F32 = np.float32


# --------------------------------------------------------------------------
# icosahedron and its subdivision
# --------------------------------------------------------------------------

def _icosahedron():
    """Unit icosahedron: 12 vertices (two at the poles) and 20 CCW faces."""
    v = np.zeros((12, 3))
    v[0] = (0.0, 0.0, 1.0)
    v[11] = (0.0, 0.0, -1.0)
    lat = np.arctan(0.5)
    for i in range(5):
        lon = 2.0 * np.pi * i / 5.0
        v[1 + i] = (np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat))
        lon2 = lon + np.pi / 5.0
        v[6 + i] = (np.cos(lat) * np.cos(lon2), np.cos(lat) * np.sin(lon2), -np.sin(lat))
    f = []
    for i in range(5):
        a, b = 1 + i, 1 + (i + 1) % 5
        c, d = 6 + i, 6 + (i + 1) % 5
        f.append((0, a, b))
        f.append((a, c, b))
        f.append((b, c, d))
        f.append((11, d, c))
    f = np.array(f, dtype=np.int64)
    # orient every face counter-clockwise seen from outside
    n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    flip = np.einsum("ij,ij->i", n, v[f].sum(axis=1)) < 0
    f[flip] = f[flip][:, [0, 2, 1]]
    return v, f


def _subdivide(nxp):
    """Return unit W positions (nW,3) and CCW triangles (nT,3) of W ids.

    Each icosahedron face (A,B,C) carries points with integer barycentric
    weights (n-i-j, i, j); a point's position is the normalised weighted sum.
    Shared corner/edge points get one canonical id and one canonical position.
    """
    v, faces = _icosahedron()
    n = nxp
    edges = {}
    for fa in faces:
        for p, q in ((fa[0], fa[1]), (fa[1], fa[2]), (fa[2], fa[0])):
            key = (min(p, q), max(p, q))
            if key not in edges:
                edges[key] = len(edges)
    nint = (n - 1) * (n - 2) // 2
    base_edge = 12
    base_face = 12 + 30 * (n - 1)
    nw = base_face + 20 * nint
    pos = np.zeros((nw, 3))
    pos[:12] = v
    for (a, b), e in edges.items():
        m = np.arange(1, n)
        pts = (n - m)[:, None] * v[a] + m[:, None] * v[b]
        pos[base_edge + e * (n - 1) + (m - 1)] = pts
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    ok = ii + jj <= n
    ii, jj = ii[ok], jj[ok]
    lid = -np.ones((n + 1, n + 1), dtype=np.int64)
    tris = []
    # interior local enumeration
    intmask = (ii >= 1) & (jj >= 1) & (ii + jj <= n - 1)
    intidx = -np.ones((n + 1, n + 1), dtype=np.int64)
    intidx[ii[intmask], jj[intmask]] = np.arange(intmask.sum())
    for fidx, (A, B, C) in enumerate(faces):
        c0 = n - ii - jj
        coefs = np.stack([c0, ii, jj], axis=1)
        corners = np.array([A, B, C])
        gid = np.empty(ii.size, dtype=np.int64)
        nz = (coefs > 0).sum(axis=1)
        # corners
        sel = nz == 1
        gid[sel] = corners[np.argmax(coefs[sel], axis=1)]
        # edges
        sel = nz == 2
        for s in np.nonzero(sel)[0]:
            idx = np.nonzero(coefs[s])[0]
            p, q = corners[idx[0]], corners[idx[1]]
            cp, cq = coefs[s, idx[0]], coefs[s, idx[1]]
            a, b = (p, q) if p < q else (q, p)
            mb = cq if p < q else cp
            gid[s] = base_edge + edges[(a, b)] * (n - 1) + (mb - 1)
        sel = nz == 3
        loc = intidx[ii[sel], jj[sel]]
        gid[sel] = base_face + fidx * nint + loc
        pos[gid[sel]] = (coefs[sel, 0:1] * v[A] + coefs[sel, 1:2] * v[B]
                         + coefs[sel, 2:3] * v[C])
        lid[ii, jj] = gid
        # up triangles (i,j),(i+1,j),(i,j+1) and down (i+1,j),(i+1,j+1),(i,j+1)
        i0, j0 = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        up = i0 + j0 <= n - 1
        tris.append(np.stack([lid[i0[up], j0[up]], lid[i0[up] + 1, j0[up]],
                              lid[i0[up], j0[up] + 1]], axis=1))
        dn = i0 + j0 <= n - 2
        tris.append(np.stack([lid[i0[dn] + 1, j0[dn]], lid[i0[dn] + 1, j0[dn] + 1],
                              lid[i0[dn], j0[dn] + 1]], axis=1))
    pos /= np.linalg.norm(pos, axis=1)[:, None]
    tris = np.concatenate(tris)
    nrm = np.cross(pos[tris[:, 1]] - pos[tris[:, 0]], pos[tris[:, 2]] - pos[tris[:, 0]])
    flip = np.einsum("ij,ij->i", nrm, pos[tris].sum(axis=1)) < 0
    tris[flip] = tris[flip][:, [0, 2, 1]]
    return pos, tris


def _locality_order(pos, block=8):
    """Order W points so that nearby cells get nearby ids.

    Cells are binned on the 6 faces of a cube circumscribing the sphere and
    sorted by a Morton (Z-order) key inside each face.  Kernels schedule work
    by id, so this keeps concurrently running blocks on compact patches.
    """
    ax = np.argmax(np.abs(pos), axis=1)
    sgn = np.sign(pos[np.arange(len(pos)), ax])
    face = ax * 2 + (sgn > 0)
    u = np.empty(len(pos))
    w = np.empty(len(pos))
    for a in range(3):
        s = ax == a
        o = [b for b in range(3) if b != a]
        u[s] = pos[s, o[0]] / np.abs(pos[s, a])
        w[s] = pos[s, o[1]] / np.abs(pos[s, a])
    q = 1 << 15
    iu = np.clip(((u + 1) * 0.5 * q).astype(np.int64), 0, q - 1)
    iv = np.clip(((w + 1) * 0.5 * q).astype(np.int64), 0, q - 1)
    key = np.zeros(len(pos), dtype=np.int64)
    for b in range(15):
        key |= ((iu >> b) & 1) << (2 * b)
        key |= ((iv >> b) & 1) << (2 * b + 1)
    key |= face.astype(np.int64) << 31
    return np.argsort(key, kind="stable")


# --------------------------------------------------------------------------
# polar-stereographic helpers (outils/map_proj_ps.f90:562-608, map_proj.f90:228-254)
# --------------------------------------------------------------------------

def _cossin_lonlat(xe, ye, ze):
    ra = np.sqrt(xe ** 2 + ye ** 2)
    sinlat = ze / ERAD
    coslat = ra / ERAD
    big = ra >= 1.0e2
    sinlon = np.where(big, ye / np.where(big, ra, 1.0), 0.0)
    coslon = np.where(big, xe / np.where(big, ra, 1.0), 1.0)
    return coslon, sinlon, coslat, sinlat


def _de_ps(dxe, dye, dze, coslat, sinlat, coslon, sinlon):
    xq = -sinlon * dxe + coslon * dye
    yq = coslat * dze - sinlat * (coslon * dxe + sinlon * dye)
    zq = sinlat * dze + coslat * (coslon * dxe + sinlon * dye)
    t = ERAD2 / np.maximum(1.0, ERAD2 + zq)
    return xq * t, yq * t


# --------------------------------------------------------------------------
# vertical grid (olam_grid.f90 gridset2, ndz == 1 branch + smoothing)
# --------------------------------------------------------------------------

def stretched_levels(nlev, dz0, ztop):
    """zz(1..nlev+1): surface at 0, first layer dz0, geometric to ztop."""
    lo, hi = 1.0 + 1e-9, 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        tot = dz0 * (r ** nlev - 1.0) / (r - 1.0)
        if tot > ztop:
            hi = r
        else:
            lo = r
    r = 0.5 * (lo + hi)
    dz = dz0 * r ** np.arange(nlev)
    zz = np.concatenate([[0.0], np.cumsum(dz)])
    zz[-1] = ztop
    return zz


def gridset2(zz):
    """Return zm, zt, dzm, dzt (float32, length mza) from explicit levels zz."""
    zz = np.asarray(zz, dtype=F32)
    nza = zz.size
    zmvec = np.zeros(nza + 2, dtype=F32)
    ztvec = np.zeros(nza + 2, dtype=F32)
    zmvec[0] = F32(2.0) * zz[0] - zz[1]
    zmvec[1:nza + 1] = zz
    zmvec[nza + 1] = F32(2.0) * zmvec[nza] - zmvec[nza - 1]
    ztvec[1] = F32(0.5) * (zmvec[0] + zmvec[1])
    for k in range(2, nza + 1):
        dzr = np.sqrt(np.sqrt((zmvec[k + 1] - zmvec[k]) / (zmvec[k - 1] - zmvec[k - 2])))
        ztvec[k] = zmvec[k - 1] + (zmvec[k] - zmvec[k - 1]) / (F32(1.0) + dzr)
    ztvec[nza + 1] = F32(0.5) * (zmvec[nza] + zmvec[nza + 1])
    dzrvec = np.zeros(nza + 2, dtype=F32)
    dzrtmp = np.zeros(nza + 2, dtype=F32)
    for _ in range(5):
        for k in range(3, nza + 2):
            dzrvec[k] = (zmvec[k] - zmvec[k - 1]) / (zmvec[k - 1] - zmvec[k - 2])
        dzrtmp[3] = dzrvec[3]
        for k in range(4, nza + 1):
            dzrtmp[k] = F32(0.3) * dzrvec[k + 1] + F32(0.4) * dzrvec[k] + F32(0.3) * dzrvec[k - 1]
        dzrtmp[nza + 1] = dzrvec[nza + 1]
        for k in range(3, nza + 2):
            zmvec[k] = zmvec[k - 1] + dzrtmp[k] * (zmvec[k - 1] - zmvec[k - 2])
        rdzr = F32(1.0)
        for k in range(3, nza + 1):
            rdzr = np.sqrt(np.sqrt((zmvec[k + 1] - zmvec[k]) / (zmvec[k - 1] - zmvec[k - 2])))
            ztvec[k] = zmvec[k - 1] + (zmvec[k] - zmvec[k - 1]) / (F32(1.0) + rdzr)
        ztvec[nza + 1] = ztvec[nza] + (zmvec[nza + 1] - zmvec[nza]) / (F32(1.0) + rdzr)
    zm = zmvec[1:nza + 1].copy()
    zt = ztvec[1:nza + 1].copy()
    dzm = (ztvec[2:nza + 2] - ztvec[1:nza + 1]).astype(F32)
    dzt = (zmvec[1:nza + 1] - zmvec[0:nza]).astype(F32)
    return zm, zt, dzm, dzt


# --------------------------------------------------------------------------
# the grid object
# --------------------------------------------------------------------------

class Grid:
    """Container of OLAM-layout grid arrays (attributes named as in OLAM)."""

    def __repr__(self):
        return (f"Grid(nxp={self.nxp}, mza={self.mza}, mwa={self.mwa}, "
                f"mva={self.mva}, mma={self.mma})")


def build_grid(nxp, zz, seed=0, numbering="local"):
    """Build a global hex grid with NXP divisions and explicit levels ``zz``.

    ``zz`` has mza entries (zz[0] = ground).  Edge orientation (which W is
    ``itab_v%iw(1)``) is drawn from ``seed`` so both signs of ``dirv`` occur.
    ``numbering`` orders the W points: "local" (cube-face Z-order, nearby
    cells get nearby ids), "generation" (the order the icosahedral
    subdivision makes them: the icosahedron's triangles one after another,
    row by row inside each, as a mesh generator numbers them) or "random"
    (a seeded random permutation).
    """
    rng = np.random.default_rng(seed)
    g = Grid()
    g.nxp = nxp
    posu, tris = _subdivide(nxp)
    if numbering == "local":
        order = _locality_order(posu)
    elif numbering == "generation":
        order = np.arange(posu.shape[0])
    elif numbering == "random":
        order = np.random.default_rng(seed + 99).permutation(posu.shape[0])
    else:
        raise ValueError(f"unknown numbering {numbering!r}")
    inv = np.empty_like(order)
    inv[order] = np.arange(order.size)
    posu = posu[order]
    tris = inv[tris]
    nw = posu.shape[0]
    ntri = tris.shape[0]
    # array index = Fortran index - 1; slot 0 is the dummy point
    W = tris + 1
    g.mwa = nw + 1
    g.mma = ntri + 1
    xew = np.zeros((g.mwa, 3))
    xew[1:] = posu * ERAD

    # ---- M points: spherical circumcentres, ordered by their lowest W id
    mkey = np.sort(W, axis=1)
    morder = np.lexsort((mkey[:, 2], mkey[:, 1], mkey[:, 0]))
    W = W[morder]
    a, b, c = xew[W[:, 0]], xew[W[:, 1]], xew[W[:, 2]]
    cc = np.cross(b - a, c - a)
    cc /= np.linalg.norm(cc, axis=1)[:, None]
    xem = np.zeros((g.mma, 3))
    xem[1:] = cc * ERAD

    # ---- V points: unique triangle edges
    e = np.concatenate([W[:, [0, 1]], W[:, [1, 2]], W[:, [2, 0]]])
    etri = np.concatenate([np.arange(ntri)] * 3) + 1  # M index of the triangle
    ekey = np.sort(e, axis=1)
    code = ekey[:, 0].astype(np.int64) * g.mwa + ekey[:, 1]
    uniq, first, cnt = np.unique(code, return_index=True, return_counts=True)
    assert np.all(cnt == 2), "every Delaunay edge must border two triangles"
    nv = uniq.size
    g.mva = nv + 1
    srt = np.argsort(code, kind="stable")
    pair_m = etri[srt].reshape(nv, 2)
    pair_w = ekey[srt][::2]
    # random orientation of iw(1) -> iw(2)
    flip = rng.random(nv) < 0.5
    iw1 = np.where(flip, pair_w[:, 1], pair_w[:, 0])
    iw2 = np.where(flip, pair_w[:, 0], pair_w[:, 1])
    # im(2) lies left of the directed segment iw1->iw2 seen from outside
    mA, mB = pair_m[:, 0], pair_m[:, 1]
    vdir = xew[iw2] - xew[iw1]
    mid = 0.5 * (xew[iw1] + xew[iw2])
    left = np.einsum("ij,ij->i", np.cross(mid, vdir), xem[mA] - mid) > 0
    im2 = np.where(left, mA, mB)
    im1 = np.where(left, mB, mA)
    itab_v_iw = np.zeros((g.mva, 2), dtype=np.int32)
    itab_v_im = np.zeros((g.mva, 2), dtype=np.int32)
    itab_v_iw[1:, 0], itab_v_iw[1:, 1] = iw1, iw2
    itab_v_im[1:, 0], itab_v_im[1:, 1] = im1, im2
    edge_of = {}
    code_v = np.minimum(iw1, iw2).astype(np.int64) * g.mwa + np.maximum(iw1, iw2)
    vid_sorted = np.argsort(code_v)
    code_sorted = code_v[vid_sorted]

    def edge_id(wa, wb):
        cd = np.minimum(wa, wb).astype(np.int64) * g.mwa + np.maximum(wa, wb)
        return vid_sorted[np.searchsorted(code_sorted, cd)] + 1

    # ---- W neighbour lists, counter-clockwise
    # for a CCW triangle (p,q,r) at corner p: neighbour q precedes neighbour r
    corner = np.concatenate([W[:, [0, 1, 2]], W[:, [1, 2, 0]], W[:, [2, 0, 1]]])
    ctri = np.concatenate([np.arange(ntri)] * 3) + 1
    cs = np.argsort(corner[:, 0], kind="stable")
    corner, ctri = corner[cs], ctri[cs]
    npoly = np.bincount(corner[:, 0], minlength=g.mwa).astype(np.int32)
    npoly[0] = 0
    assert npoly[1:].min() >= 5 and npoly[1:].max() <= 6
    start = np.concatenate([[0], np.cumsum(npoly)])
    slots = np.full((g.mwa, 6), -1, dtype=np.int64)
    nxt = np.full((g.mwa, 6), -1, dtype=np.int64)
    tri_of = np.zeros((g.mwa, 6), dtype=np.int64)
    local = np.arange(corner.shape[0]) - start[corner[:, 0]]
    slots[corner[:, 0], local] = corner[:, 1]
    nxt[corner[:, 0], local] = corner[:, 2]
    tri_of[corner[:, 0], local] = ctri
    # chain: iw(1) = slots[:,0]; iw(j+1) = nxt of the slot whose first is iw(j)
    nbr_w = np.zeros((g.mwa, 7), dtype=np.int32)
    nbr_m = np.zeros((g.mwa, 7), dtype=np.int32)
    cur = slots[:, 0].copy()
    for j in range(6):
        nbr_w[:, j] = np.where(j < npoly, cur, 0)
        hit = slots == cur[:, None]
        k = np.argmax(hit, axis=1)
        nbr_m[:, j] = np.where(j < npoly, tri_of[np.arange(g.mwa), k], 0)
        cur = nxt[np.arange(g.mwa), k]
    nbr_w[0] = 0
    nbr_m[0] = 0
    # M(j) is the triangle (iw, iw(j), iw(j+1)); edge iv(j) joins M(j-1), M(j)
    rows = np.arange(1, g.mwa)
    nbr_v = np.zeros((g.mwa, 7), dtype=np.int32)
    dirv = np.zeros((g.mwa, 7), dtype=F32)
    for j in range(6):
        valid = j < npoly[rows]
        iv = np.zeros(rows.size, dtype=np.int64)
        iv[valid] = edge_id(rows[valid], nbr_w[rows[valid], j])
        nbr_v[rows, j] = iv
        d = np.where(itab_v_iw[iv, 0] == rows, -1.0, 1.0)
        dirv[rows, j] = np.where(valid, d, 0.0)
    g.npoly = npoly
    g.itab_w_iw, g.itab_w_iv, g.itab_w_im, g.dirv = nbr_w, nbr_v, nbr_m, dirv
    g.itab_v_iw, g.itab_v_im = itab_v_iw, itab_v_im
    g.iwglobe = np.arange(1, g.mwa + 1, dtype=np.int32)

    # M-point neighbour tables (itab_m%iv, iw, im): the three edges/W of a triangle
    itab_m_iw = np.zeros((g.mma, 3), dtype=np.int32)
    itab_m_iw[1:] = W
    itab_m_iv = np.zeros((g.mma, 3), dtype=np.int32)
    itab_m_iv[1:, 0] = edge_id(W[:, 0], W[:, 1])
    itab_m_iv[1:, 1] = edge_id(W[:, 1], W[:, 2])
    itab_m_iv[1:, 2] = edge_id(W[:, 2], W[:, 0])
    itab_m_im = np.zeros((g.mma, 3), dtype=np.int32)
    for j in range(3):
        ivj = itab_m_iv[1:, j]
        a_, b_ = itab_v_im[ivj, 0], itab_v_im[ivj, 1]
        itab_m_im[1:, j] = np.where(a_ == np.arange(1, g.mma), b_, a_)
    g.itab_m_iw, g.itab_m_iv, g.itab_m_im = itab_m_iw, itab_m_iv, itab_m_im

    _horizontal_metrics(g, xew, xem)
    _vertical_and_volumes(g, zz)
    _adv_coefficients(g)
    return g


def _horizontal_metrics(g, xew, xem):
    """grid_geometry_hex (hex_grid.f90:418-1125) restated in float64."""
    iw1, iw2 = g.itab_v_iw[:, 0], g.itab_v_iw[:, 1]
    im1, im2 = g.itab_v_im[:, 0], g.itab_v_im[:, 1]
    xev = 0.5 * (xew[iw1] + xew[iw2])
    xev[1:] *= (ERAD / np.linalg.norm(xev[1:], axis=1))[:, None]
    xev[0] = 0.0
    dnu = np.linalg.norm(xem[im1] - xem[im2], axis=1)
    dnv = np.linalg.norm(xew[iw1] - xew[iw2], axis=1)
    dnu[0] = dnv[0] = 1.0
    un = (xem[im2] - xem[im1]) / dnu[:, None]
    vn = (xew[iw2] - xew[iw1]) / dnv[:, None]
    un[0] = vn[0] = 0.0
    dvm1 = np.linalg.norm(xev - xem[im1], axis=1)
    dvm2 = np.linalg.norm(xev - xem[im2], axis=1)
    qk1 = 0.25 * dvm1 * dnv
    qk2 = 0.25 * dvm2 * dnv
    qk1[0] = qk2[0] = 0.0
    arm0 = np.zeros(g.mma)
    np.add.at(arm0, im1, 2.0 * qk1)
    np.add.at(arm0, im2, 2.0 * qk2)
    arw0 = np.zeros(g.mwa)
    np.add.at(arw0, iw1, qk1 + qk2)
    np.add.at(arw0, iw2, qk1 + qk2)
    arw0[0] = 1.0
    arm0[0] = 1.0
    wn = xew / ERAD
    coslon, sinlon, coslat, sinlat = _cossin_lonlat(xew[:, 0], xew[:, 1], xew[:, 2])

    mw = g.mwa
    npoly = g.npoly
    farm = np.zeros((mw, 7))
    farv = np.zeros((mw, 7))
    gxps1 = np.zeros((mw, 7))
    gxps2 = np.zeros((mw, 7))
    gyps1 = np.zeros((mw, 7))
    gyps2 = np.zeros((mw, 7))
    dxps = np.zeros((g.mva, 2))
    dyps = np.zeros((g.mva, 2))
    rows = np.arange(1, mw)
    arwi = 1.0 / arw0
    for j2 in range(6):
        valid = j2 < npoly[rows]
        r = rows[valid]
        j1 = np.where(j2 == 0, npoly[r] - 1, j2 - 1)
        iv = g.itab_w_iv[r, j2]
        w2 = g.itab_w_iw[r, j2]
        w1 = g.itab_w_iw[r, j1]
        first = g.itab_v_iw[iv, 0] == w1
        farm[r, j1] += np.where(first, qk1[iv], qk2[iv]) * arwi[r]
        farm[r, j2] += np.where(first, qk2[iv], qk1[iv]) * arwi[r]
        farv[r, j2] = (qk1[iv] + qk2[iv]) * arwi[r]
        cl, sl, ct, st = coslon[r], sinlon[r], coslat[r], sinlat[r]
        d = xew[w1] - xew[r]
        xw1, yw1 = _de_ps(d[:, 0], d[:, 1], d[:, 2], ct, st, cl, sl)
        d = xew[w2] - xew[r]
        xw2, yw2 = _de_ps(d[:, 0], d[:, 1], d[:, 2], ct, st, cl, sl)
        d = xev[iv] - xew[r]
        xv, yv = _de_ps(d[:, 0], d[:, 1], d[:, 2], ct, st, cl, sl)
        vmagi = 1.0 / (xw1 * yw2 - xw2 * yw1)
        gxps1[r, j1] = yw2 * vmagi
        gxps2[r, j1] = -yw1 * vmagi
        gyps1[r, j1] = -xw2 * vmagi
        gyps2[r, j1] = xw1 * vmagi
        neg = g.dirv[r, j2] < 0
        dxps[iv[neg], 0] = xv[neg]
        dyps[iv[neg], 0] = yv[neg]
        dxps[iv[~neg], 1] = xv[~neg]
        dyps[iv[~neg], 1] = yv[~neg]
    gxps1 *= farm
    gyps1 *= farm
    gxps2 *= farm
    gyps2 *= farm
    # combined grad_t2d weights (mem_grid.f90 alloc_grid_other)
    gxc = np.zeros((mw, 7))
    gyc = np.zeros((mw, 7))
    for n1 in range(6):
        valid = n1 < npoly
        n2 = np.where(n1 == 0, npoly - 1, n1 - 1)
        n2 = np.clip(n2, 0, 6)
        gxc[:, n1] = np.where(valid, gxps1[:, n1] + gxps2[np.arange(mw), n2], 0.0)
        gyc[:, n1] = np.where(valid, gyps1[:, n1] + gyps2[np.arange(mw), n2], 0.0)

    # ecvec: least-squares correction of the Perot weights (hex_grid.f90:880-1000)
    ecx = np.zeros((mw, 7))
    ecy = np.zeros((mw, 7))
    ecz = np.zeros((mw, 7))
    for npl in (5, 6):
        r = rows[npoly[rows] == npl]
        fo = 2.0 * farv[r, :npl]
        vnv = vn[g.itab_w_iv[r, :npl]]                       # (n, npl, 3)
        w = wn[r]                                            # (n, 3)
        vdotw = np.einsum("njc,nc->nj", vnv, w)
        vps = vnv - vdotw[..., None] * w[:, None, :]
        vps /= np.linalg.norm(vps, axis=2)[..., None]
        wx, wy, wz = w[:, 0:1], w[:, 1:2], w[:, 2:3]
        up = wz >= 0.0
        fact = (wy * vps[..., 0] - wx * vps[..., 1]) / np.where(up, 1.0 + wz, 1.0 - wz)
        s_ = np.where(up, 1.0, -1.0)
        rx = s_ * (vps[..., 0] * wz - vps[..., 2] * wx) + wy * fact
        ry = s_ * (vps[..., 1] * wz - vps[..., 2] * wy) - wx * fact
        A = np.stack([rx * rx, ry * ry, rx * ry], axis=1)    # (n, 3, npl)
        bb = np.stack([1.0 - np.einsum("nj,nj->n", fo, A[:, 0]),
                       1.0 - np.einsum("nj,nj->n", fo, A[:, 1]),
                       -np.einsum("nj,nj->n", fo, A[:, 2])], axis=1)
        AAt = A @ np.transpose(A, (0, 2, 1))
        lam = np.linalg.solve(AAt, bb[..., None])[..., 0]
        x = np.einsum("ncj,nc->nj", A, lam)                 # minimum-norm solution
        cf = x + fo
        good = np.all(cf > 0.03, axis=1) & np.all(cf < 0.7, axis=1)
        cf = np.where(good[:, None], cf, fo)
        ecx[r, :npl] = cf * vps[..., 0]
        ecy[r, :npl] = cf * vps[..., 1]
        ecz[r, :npl] = cf * vps[..., 2]

    # M-point coordinates in the PS plane of each W (for hex_quad)
    xm_ps = np.zeros((mw, 7))
    ym_ps = np.zeros((mw, 7))
    for j in range(6):
        valid = j < npoly
        m = g.itab_w_im[:, j]
        d = xem[m] - xew
        x, y = _de_ps(d[:, 0], d[:, 1], d[:, 2], coslat, sinlat, coslon, sinlon)
        xm_ps[:, j] = np.where(valid, x, 0.0)
        ym_ps[:, j] = np.where(valid, y, 0.0)

    g.xew, g.xev, g.xem = (xew.T.astype(F32).copy(), xev.T.astype(F32).copy(),
                           xem.T.astype(F32).copy())
    g.glatw = np.degrees(np.arctan2(xew[:, 2], np.hypot(xew[:, 0], xew[:, 1]))).astype(F32)
    g.glonw = np.degrees(np.arctan2(xew[:, 1], xew[:, 0])).astype(F32)
    g.glatv = np.degrees(np.arctan2(xev[:, 2], np.hypot(xev[:, 0], xev[:, 1]))).astype(F32)
    g.glonv = np.degrees(np.arctan2(xev[:, 1], xev[:, 0])).astype(F32)
    g.dnu, g.dnv = dnu.astype(F32), dnv.astype(F32)
    g.dniu, g.dniv = (1.0 / dnu).astype(F32), (1.0 / dnv).astype(F32)
    g.unx, g.uny, g.unz = (un[:, i].astype(F32) for i in range(3))
    g.vnx, g.vny, g.vnz = (vn[:, i].astype(F32) for i in range(3))
    g.wnx, g.wny, g.wnz = (wn[:, i].astype(F32) for i in range(3))
    g.arw0, g.arm0 = arw0.astype(F32), arm0.astype(F32)
    g.arw0i = (1.0 / arw0).astype(F32)
    g.farm, g.farv = farm.astype(F32), farv.astype(F32)
    g.dxps, g.dyps = dxps.astype(F32), dyps.astype(F32)
    g.gxps_coef, g.gyps_coef = gxc.astype(F32), gyc.astype(F32)
    g.ecvec_vx, g.ecvec_vy, g.ecvec_vz = ecx.astype(F32), ecy.astype(F32), ecz.astype(F32)
    g._xm_ps, g._ym_ps = xm_ps, ym_ps
    g._arw0_64 = arw0


def _vertical_and_volumes(g, zz):
    """gridset2 + ctrlvols_hex_nosfcg (flat) + mem_grid derived arrays."""
    zm, zt, dzm, dzt = gridset2(zz)
    mza = zm.size
    g.mza = mza
    g.zm, g.zt, g.dzm, g.dzt = zm, zt, dzm, dzt
    g.dzim = (F32(1.0) / dzm).astype(F32)
    g.dzit = (F32(1.0) / dzt).astype(F32)
    zfacm = ((ERAD + zm.astype(np.float64)) / ERAD).astype(F32)
    zfact = ((ERAD + zt.astype(np.float64)) / ERAD).astype(F32)
    g.zfacm, g.zfact = zfacm, zfact
    g.zfacm2 = (zfacm * zfacm).astype(F32)
    g.zfacit = (F32(1.0) / zfact).astype(F32)
    g.zfacim = (F32(1.0) / zfacm).astype(F32)
    # lowest prognostic levels: flat terrain at zm(1) -> 2 (Fortran) everywhere
    g.lpw = np.full(g.mwa, 2, dtype=np.int32)
    g.lpv = np.full(g.mva, 2, dtype=np.int32)
    g.lpm = np.full(g.mma, 2, dtype=np.int32)
    g.lve2 = np.zeros(g.mwa, dtype=np.int32)
    # alloc_gridz_other
    dzt_top = np.zeros(mza, dtype=F32)
    dzt_bot = np.zeros(mza, dtype=F32)
    dzt_top[0] = zm[0] - zt[0]
    dzt_bot[0] = dzt[0] - dzt_top[0]
    dzt_top[1:] = zm[1:] - zt[1:]
    dzt_bot[1:] = zt[1:] - zm[:-1]
    g.dzt_top, g.dzt_bot = dzt_top, dzt_bot
    grav = 9.81
    gravm = np.full(mza, grav, dtype=F32)
    zwgt_top8 = np.zeros(mza)
    zwgt_bot8 = np.zeros(mza)
    zwgt_top8[:-1] = dzt_bot[1:].astype(np.float64) * g.dzim[:-1]
    zwgt_bot8[:-1] = dzt_top[:-1].astype(np.float64) * g.dzim[:-1]
    zwgt_top8[-1] = zwgt_top8[-2]
    zwgt_bot8[-1] = zwgt_bot8[-2]
    g.zwgt_top8, g.zwgt_bot8 = zwgt_top8, zwgt_bot8
    g.gdz_wgtp8 = zwgt_top8 * gravm
    g.gdz_wgtm8 = zwgt_bot8 * gravm
    g.gdz_wgtp = g.gdz_wgtp8.astype(F32)
    g.gdz_wgtm = g.gdz_wgtm8.astype(F32)
    g.zwgt_top = zwgt_top8.astype(F32)
    g.zwgt_bot = zwgt_bot8.astype(F32)
    # control volumes (flat terrain): arw(k) = arw0*zfacm2, arw(mza)=0
    mw, mv = g.mwa, g.mva
    arw = np.zeros((mw, mza), dtype=F32)
    arw[1:, :mza - 1] = (g.arw0[1:, None] * g.zfacm2[None, :mza - 1]).astype(F32)
    arv = np.zeros((mv, mza), dtype=F32)
    arv[1:, 1:] = (g.dnu[1:, None] * dzt[None, 1:] * zfact[None, 1:]).astype(F32)
    volt = np.zeros((mw, mza), dtype=np.float64)
    volt[1:, 1:] = (dzt[None, 1:].astype(np.float64) * g.arw0[1:, None]
                    * zfact[None, 1:].astype(np.float64) ** 2)
    g.arw, g.arv, g.volt = arw, arv, volt
    volti = np.zeros((mw, mza), dtype=F32)
    volti[1:, 1:] = (1.0 / volt[1:, 1:]).astype(F32)
    volwi = np.zeros((mw, mza), dtype=F32)
    volwi[1:, 1:mza - 1] = (1.0 / (volt[1:, 1:mza - 1] + volt[1:, 2:mza])).astype(F32)
    iw1, iw2 = g.itab_v_iw[:, 0], g.itab_v_iw[:, 1]
    volvi = np.zeros((mv, mza), dtype=F32)
    volvi[1:, 1:] = (1.0 / (volt[iw1[1:], 1:] + volt[iw2[1:], 1:])).astype(F32)
    g.volti, g.volwi, g.volvi = volti, volwi, volvi
    g.wnxo2 = (g.wnx * F32(0.5)).astype(F32)
    g.wnyo2 = (g.wny * F32(0.5)).astype(F32)
    g.wnzo2 = (g.wnz * F32(0.5)).astype(F32)


def _adv_coefficients(g):
    """alloc_adv (mem_adv.f90:23-357) restated with exact small solves."""
    mza = g.mza
    dzm = g.dzm.astype(np.float64)
    dzt = g.dzt.astype(np.float64)
    top = g.dzt_top.astype(np.float64)
    bot = g.dzt_bot.astype(np.float64)
    a_v = np.zeros((2, 2, mza))
    a_w = np.zeros((2, 2, mza))
    a_vu = np.zeros((2, 2, mza))
    a_wu = np.zeros((2, 2, mza))
    for k in range(1, mza):
        for bounded in (True, False):
            a0 = (top[k] ** 3 + bot[k] ** 3) / (3.0 * dzt[k]) if bounded else 0.0
            z1 = np.array([-dzm[k - 1], dzm[k]])
            z2 = z1 * z1 - a0
            det = z1[0] * z2[1] - z2[0] * z1[1]
            # fit g*z + h*(z^2-a0) through (z1[0], -ds(k-1)) and (z1[1], ds(k))
            g11 = -z2[0] / det     # coefficient of ds(k)   in g
            g12 = -z2[1] / det     # coefficient of ds(k-1) in g
            h21 = z1[0] / det      # coefficient of ds(k)   in h
            h22 = z1[1] / det      # coefficient of ds(k-1) in h
            av = np.array([[g11, g12], [h21, h22]])
            aw = np.empty((2, 2))
            aw[0, 0] = av[1, 0] * (bot[k] ** 2 - a0) - av[0, 0] * bot[k]
            aw[1, 0] = av[1, 1] * (bot[k] ** 2 - a0) - av[0, 1] * bot[k]
            aw[0, 1] = av[1, 0] * (top[k] ** 2 - a0) + av[0, 0] * top[k]
            aw[1, 1] = av[1, 1] * (top[k] ** 2 - a0) + av[0, 1] * top[k]
            if bounded:
                a_v[:, :, k], a_w[:, :, k] = av, aw
            else:
                a_vu[:, :, k], a_wu[:, :, k] = av, aw
    for arr in (a_v, a_w, a_vu, a_wu):
        arr[:, :, 0] = arr[:, :, 1]
    # stored like Fortran a_w(mza,2,2): C array [2][2][mza] with [i-1][j-1][k]
    g.a_v, g.a_w = a_v.astype(F32), a_w.astype(F32)
    g.a_vu, g.a_wu = a_vu.astype(F32), a_wu.astype(F32)

    mw = g.mwa
    npoly = g.npoly
    xy_h = np.zeros((mw, 7, 5))
    xy_hu = np.zeros((mw, 7, 5))
    xx0 = np.zeros(mw)
    xy0 = np.zeros(mw)
    yy0 = np.zeros(mw)
    xx_yy = np.zeros((mw, 7))
    rows = np.arange(1, mw)
    for npl in (5, 6):
        r = rows[npoly[rows] == npl]
        ivs = g.itab_w_iv[r, :npl]
        neg = g.dirv[r, :npl] < 0
        xw = np.where(neg, g.dxps[ivs, 0], g.dxps[ivs, 1]).astype(np.float64) * 2.0
        yw = np.where(neg, g.dyps[ivs, 0], g.dyps[ivs, 1]).astype(np.float64) * 2.0
        # exact second moments of the PS polygon (Green's theorem); the
        # 2-point Gauss rule of hex_quad is exact for these quadratics too
        x = g._xm_ps[r, :npl]
        y = g._ym_ps[r, :npl]
        xn, yn = np.roll(x, -1, axis=1), np.roll(y, -1, axis=1)
        cr = x * yn - xn * y
        sgn = np.where(cr.sum(axis=1) > 0, 1.0, -1.0)
        ixx = sgn * np.sum(cr * (x * x + x * xn + xn * xn), axis=1) / 12.0
        iyy = sgn * np.sum(cr * (y * y + y * yn + yn * yn), axis=1) / 12.0
        ixy = sgn * np.sum(cr * (x * yn + 2 * x * y + 2 * xn * yn + xn * y), axis=1) / 24.0
        arwi = (1.0 / g._arw0_64[r]).astype(F32)
        xx0[r] = ixx.astype(F32) * arwi
        xy0[r] = ixy.astype(F32) * arwi
        yy0[r] = iyy.astype(F32) * arwi
        A = np.stack([xw, yw, xw * xw - xx0[r, None], xw * yw - xy0[r, None],
                      yw * yw - yy0[r, None]], axis=1)         # (n, 5, npl)
        At = np.transpose(A, (0, 2, 1))
        xy_h[r, :npl, :] = np.transpose(np.linalg.solve(A @ At, A), (0, 2, 1))
        Au = np.stack([xw, yw, xw * xw, xw * yw, yw * yw], axis=1)
        Aut = np.transpose(Au, (0, 2, 1))
        xy_hu[r, :npl, :] = np.transpose(np.linalg.solve(Au @ Aut, Au), (0, 2, 1))
        xx_yy[r, :npl] = (g.dniv[ivs].astype(np.float64) * g.dnu[ivs]
                          * g.arw0i[r, None])
    g.xy_h = xy_h.astype(F32)        # Fortran xy_h(5,7,mwa) -> C [mwa][7][5]
    g.xy_hu = xy_hu.astype(F32)
    g.xx_yy = xx_yy.astype(F32)
    xx_yy_m = np.zeros((g.mma, 3))
    for j in range(3):
        ivn = g.itab_m_iv[1:, j]
        xx_yy_m[1:, j] = g.dnv[ivn].astype(np.float64) * g.dniu[ivn] / g.arm0[1:]
    g.xx_yy_m = xx_yy_m.astype(F32)
    iw1, iw2 = g.itab_v_iw[:, 0], g.itab_v_iw[:, 1]
    dx1, dy1 = g.dxps[:, 0].astype(np.float64), g.dyps[:, 0].astype(np.float64)
    dx2, dy2 = g.dxps[:, 1].astype(np.float64), g.dyps[:, 1].astype(np.float64)
    g.xx0_v = np.stack([dx1 * dx1 - xx0[iw1], dx2 * dx2 - xx0[iw2]], axis=1).astype(F32)
    g.xy0_v = np.stack([dx1 * dy1 - xy0[iw1], dx2 * dy2 - xy0[iw2]], axis=1).astype(F32)
    g.yy0_v = np.stack([dy1 * dy1 - yy0[iw1], dy2 * dy2 - yy0[iw2]], axis=1).astype(F32)
    g.xx0_vu = np.stack([dx1 * dx1, dx2 * dx2], axis=1).astype(F32)
    g.xy0_vu = np.stack([dx1 * dy1, dx2 * dy2], axis=1).astype(F32)
    g.yy0_vu = np.stack([dy1 * dy1, dy2 * dy2], axis=1).astype(F32)
    for arr in (g.xx0_v, g.xy0_v, g.yy0_v, g.xx0_vu, g.xy0_vu, g.yy0_vu):
        arr[0] = 0.0


def with_terrain(g0, hmax=4, width=0.9):
    """A copy of grid g0 with a step-topography mountain centred on W point
    1: lpw rises to 2 + hmax (Fortran levels) within ``width`` radians of
    it; a face's lpv is the higher floor of its two cells, an M point's lpm
    the highest lpv of its three faces (omodel/hex_grid.f90:1446) and a
    column's lve2 the largest lpv - lpw of its faces (hex_grid.f90:1927,
    the shaved-cell levels).  The metric arrays stay those of g0."""
    import copy
    g = copy.copy(g0)
    xyz = np.asarray(g.xew, dtype=np.float64).T
    rad = np.linalg.norm(xyz, axis=1)
    rad[rad == 0] = 1.0
    top = xyz[1] / rad[1]
    ang = np.arccos(np.clip(xyz @ top / rad, -1.0, 1.0))
    lpw = 2 + np.floor(hmax * np.clip(1.0 - ang / width, 0.0, 1.0) ** 0.6).astype(np.int32)
    lpw = np.minimum(lpw, g.mza - 2)
    lpw[0] = 2
    g.lpw = lpw.astype(np.int32)
    g.lpv = np.maximum(lpw[g.itab_v_iw[:, 0]], lpw[g.itab_v_iw[:, 1]]).astype(np.int32)
    g.lpv[0] = 2
    g.lpm = np.max(g.lpv[g.itab_m_iv], axis=1).astype(np.int32)
    g.lpm[0] = 2
    faces = np.arange(g.itab_w_iv.shape[1])[None, :] < g.npoly[:, None]
    g.lve2 = np.where(faces, g.lpv[g.itab_w_iv] - lpw[:, None], 0).max(axis=1).clip(0).astype(np.int32)
    g.lve2[0] = 0
    return g
