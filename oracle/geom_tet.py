"""Voronoi dual of a tetrahedralisation — TEST INFRASTRUCTURE (oracle).

Numpy restatement of ``Tetrahedron::update_tet`` steps 1-5 (src/base/geom_tet.rs:101-293),
evaluated in the reference's operation order. Independent of the product's C++ dual: it takes
tetrahedra from any Delaunay code (the tests use scipy's Qhull) and accumulates face pieces in
the order of the tetrahedra it is given. Small meshes only (vectorised, but holds all pieces).
"""
from __future__ import annotations

import numpy as np

EP = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
FO = [(1, 3, 2), (0, 2, 3), (0, 3, 1), (0, 1, 2)]  # face opposite vertex k, counterclockwise from outside


def _dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1], a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def _scale(s, a):
    return s[..., None] * a


def _len(a):
    return np.sqrt(_dot(a, a))


def circumcircle3(a, b, c):
    """delaunay.rs:207-214"""
    u, v = b - a, c - a
    w = _cross(u, v)
    num = _scale(_dot(u, u), _cross(v, w)) + _scale(_dot(v, v), _cross(w, u))
    return a + _scale(0.5 / _dot(w, w), num)


def circumsphere3(a, b, c, d):
    """delaunay.rs:216-221"""
    u, v, w = b - a, c - a, d - a
    num = (_scale(_dot(u, u), _cross(v, w)) + _scale(_dot(v, v), _cross(w, u))) + _scale(_dot(w, w), _cross(u, v))
    return a + _scale(0.5 / _dot(u, _cross(v, w)), num)


def orient_positive(pos, tets):
    """Reorder vertices so that det[p0-p3; p1-p3; p2-p3] > 0 (the reference's orientation)."""
    t = np.array(tets, dtype=np.int64)
    a, b, c, d = (pos[t[:, i]] for i in range(4))
    det = _dot(a - d, _cross(b - d, c - d))
    neg = det < 0
    t[neg, 0], t[neg, 1] = t[neg, 1].copy(), t[neg, 0].copy()
    return t, np.abs(det)


def build_dual(pos: np.ndarray, tets: np.ndarray, n_pts: int) -> dict:
    pos = np.asarray(pos, np.float64)
    N = pos.shape[0]
    t, _ = orient_positive(pos, tets)
    T = t.shape[0]

    # boundary faces: faces of exactly one tetrahedron (geom_tet.rs:101-116)
    fkeys = np.sort(np.stack([t[:, [(k + 1) % 4, (k + 2) % 4, (k + 3) % 4]] for k in range(4)], axis=1), axis=2)  # (T,4,3)
    flat = fkeys.reshape(-1, 3)
    _, inv, cnt = np.unique(flat, axis=0, return_inverse=True, return_counts=True)
    is_b = (cnt[inv.ravel()] == 1).reshape(T, 4)
    surf = []
    for ti in range(T):
        for k in range(4):
            if is_b[ti, k]:
                surf.append([t[ti, FO[k][0]], t[ti, FO[k][1]], t[ti, FO[k][2]]])
    surf = np.array(surf, np.int64).reshape(-1, 3)
    if np.any(surf < n_pts):
        raise ValueError("boundary face joins an interior point")

    # face pieces (geom_tet.rs:122-171), order (tet, edge, side)
    P = [pos[t[:, i]] for i in range(4)]
    c_t = circumsphere3(P[0], P[1], P[2], P[3])
    keys, areas, cents, mids, pis, pjs, vis, vjs, dists = [], [], [], [], [], [], [], [], []
    for (li, lj) in EP:
        oth = [l for l in range(4) if l not in (li, lj)]
        pi, pj = P[li], P[lj]
        dist = _len(pj - pi)
        e = _scale(1.0 / dist, pj - pi)
        m = _scale(np.full(T, 0.5), pi + pj)
        side_out = []
        for (a, b) in [(oth[0], oth[1]), (oth[1], oth[0])]:
            pa, pb = P[a], P[b]
            c_f = circumcircle3(pi, pj, pa)
            u = (pa - m) - _scale(_dot(pa - m, e), e)
            u = _scale(1.0 / _len(u), u)
            nrm = _cross(e, u)
            flip = _dot(pb - m, nrm) < 0.0
            nrm[flip] = -nrm[flip]
            s1 = _dot(c_f - m, u)
            s2 = _dot(c_t - c_f, nrm)
            area = 0.5 * s1 * s2
            cent = _scale(np.full(T, 1.0 / 3.0), m + (c_f + c_t))
            side_out.append((area, cent))
        keys.append(np.stack([np.minimum(t[:, li], t[:, lj]), np.maximum(t[:, li], t[:, lj])], axis=1))
        areas.append(np.stack([side_out[0][0], side_out[1][0]], axis=1))
        cents.append(np.stack([side_out[0][1], side_out[1][1]], axis=1))
        mids.append(m)
        pis.append(pi)
        pjs.append(pj)
        vis.append(t[:, li])
        vjs.append(t[:, lj])
        dists.append(dist)
    keys = np.stack(keys, axis=1).reshape(-1, 2)          # (T*6, 2)
    areas = np.stack(areas, axis=1).reshape(-1, 2)        # (T*6, 2)
    cents = np.stack(cents, axis=1).reshape(-1, 2, 3)
    mids = np.stack(mids, axis=1).reshape(-1, 3)
    pis = np.stack(pis, axis=1).reshape(-1, 3)
    pjs = np.stack(pjs, axis=1).reshape(-1, 3)
    vis = np.stack(vis, axis=1).reshape(-1)
    vjs = np.stack(vjs, axis=1).reshape(-1)
    dists = np.stack(dists, axis=1).reshape(-1)
    ekeys, eid = np.unique(keys, axis=0, return_inverse=True)
    eid = eid.ravel()
    E = ekeys.shape[0]
    e_area = np.zeros(E)
    e_skew = np.zeros((E, 3))
    cent_sum = np.zeros((N, 3))
    # accumulate strictly in (tet, edge, side) order
    order_eid = np.repeat(eid, 2)
    a_all = areas.reshape(-1)
    c_all = cents.reshape(-1, 3)
    m_all = np.repeat(mids, 2, axis=0)
    np.add.at(e_area, order_eid, a_all)
    np.add.at(e_skew, order_eid, _scale(a_all, c_all - m_all))
    vol = a_all * np.repeat(dists, 2) / 6.0
    vi2, vj2 = np.repeat(vis, 2), np.repeat(vjs, 2)
    pi2, pj2 = np.repeat(pis, 2, axis=0), np.repeat(pjs, 2, axis=0)
    ci_ = _scale(vol * 0.75, c_all - pi2)
    cj_ = _scale(vol * 0.75, c_all - pj2)
    inter = np.empty((2 * ci_.shape[0], 3))
    inter[0::2] = ci_
    inter[1::2] = cj_
    idx = np.empty(2 * vi2.size, np.int64)
    idx[0::2] = vi2
    idx[1::2] = vj2
    np.add.at(cent_sum, idx, inter)

    # neighbour CSR and per-face data (geom_tet.rs:178-206)
    A, B = ekeys[:, 0], ekeys[:, 1]
    pa, pb = pos[A], pos[B]
    dist = _len(pb - pa)
    norm = _scale(1.0 / dist, pb - pa)
    ok = np.abs(e_area) > 1e-12 * dist * dist
    skew = np.zeros((E, 3))
    skew[ok] = _scale(1.0 / e_area[ok], e_skew[ok])
    deg = np.bincount(np.concatenate([A, B]), minlength=N)
    nbr_ptr = np.zeros(N + 1, np.int64)
    nbr_ptr[1:] = np.cumsum(deg)
    # entries in edge order: edge e contributes to A[e] then B[e]; per vertex in edge order
    owner = np.empty(2 * E, np.int64)
    owner[0::2] = A
    owner[1::2] = B
    other = np.empty(2 * E, np.int64)
    other[0::2] = B
    other[1::2] = A
    ent_e = np.repeat(np.arange(E), 2)
    sign = np.tile([1.0, -1.0], E)
    o = np.argsort(owner, kind="stable")
    nbr_idx = other[o].astype(np.int32)
    ee = ent_e[o]
    cvol = np.zeros(N)
    np.add.at(cvol, owner, np.repeat(e_area * dist / 6.0, 2))
    cskew = (cent_sum / cvol[:, None]).T.copy()

    # boundary sub-faces (geom_tet.rs:208-259)
    S = surf.shape[0]
    p0, p1, p2 = pos[surf[:, 0]], pos[surf[:, 1]], pos[surf[:, 2]]
    tn = _cross(p1 - p0, p2 - p0)
    tn = _scale(1.0 / _len(tn), tn)
    cc = circumcircle3(p0, p1, p2)
    sq = [_dot(p2 - p1, p2 - p1), _dot(p0 - p2, p0 - p2), _dot(p1 - p0, p1 - p0)]
    lraw = [sq[0] * (sq[1] + sq[2] - sq[0]), sq[1] * (sq[2] + sq[0] - sq[1]), sq[2] * (sq[0] + sq[1] - sq[2])]
    lsum = lraw[0] + lraw[1] + lraw[2]
    lam = [lraw[i] / lsum for i in range(3)]
    bvid, bj, bk, bar, bnr, bwt = [], [], [], [], [], []
    for loc in range(3):
        vi, vj, vk = surf[:, loc], surf[:, (loc + 1) % 3], surf[:, (loc + 2) % 3]
        pi, pj, pk = pos[vi], pos[vj], pos[vk]
        ar = []
        for (pa_, pb_) in [(pj, pk), (pk, pj)]:
            m = _scale(np.full(S, 0.5), pi + pa_)
            e = pa_ - pi
            ln = _len(e)
            u = (pb_ - m) - _scale(_dot(pb_ - m, e) / (ln * ln), e)
            ar.append(0.25 * ln * _dot(cc - m, _scale(1.0 / _len(u), u)))
        asum = ar[0] + ar[1]
        l0, l1, l2 = lam[loc], lam[(loc + 1) % 3], lam[(loc + 2) % 3]
        cj = np.stack([(1.5 + l0) / 3.0, (0.5 + l1) / 3.0, l2 / 3.0], axis=1)
        ck = np.stack([(1.5 + l0) / 3.0, l1 / 3.0, (0.5 + l2) / 3.0], axis=1)
        okb = np.abs(asum) > 1e-12 * _len(pj - pi) * _len(pk - pi)
        w = np.tile([1.0, 0.0, 0.0], (S, 1))
        w[okb] = _scale(1.0 / asum[okb], _scale(ar[0][okb], cj[okb]) + _scale(ar[1][okb], ck[okb]))
        bvid.append(vi), bj.append(vj), bk.append(vk), bar.append(asum), bnr.append(tn), bwt.append(w)
    # per vertex in surface-triangle order, loc order within a triangle
    bvid = np.stack(bvid, axis=1).reshape(-1)
    bj = np.stack(bj, axis=1).reshape(-1)
    bk = np.stack(bk, axis=1).reshape(-1)
    bar = np.stack(bar, axis=1).reshape(-1)
    bnr = np.stack(bnr, axis=1).reshape(-1, 3)
    bwt = np.stack(bwt, axis=1).reshape(-1, 3)
    ob = np.argsort(bvid, kind="stable")
    bcnt = np.bincount(bvid, minlength=N)
    bnd_ptr = np.zeros(N + 1, np.int64)
    bnd_ptr[1:] = np.cumsum(bcnt)

    # least-squares gradient weights (geom_tet.rs:261-293)
    rows = np.repeat(np.arange(N), deg)
    dvec = pos[nbr_idx] - pos[rows]
    omega = 1.0 / (dvec[:, 0] * dvec[:, 0] + dvec[:, 1] * dvec[:, 1] + dvec[:, 2] * dvec[:, 2])
    M = np.zeros((N, 3, 3))
    for r in range(3):
        for s in range(3):
            np.add.at(M[:, r, s], rows, omega * dvec[:, r] * dvec[:, s])
    m = M
    adj = np.empty_like(M)
    adj[:, 0, 0] = m[:, 1, 1] * m[:, 2, 2] - m[:, 1, 2] * m[:, 2, 1]
    adj[:, 0, 1] = m[:, 0, 2] * m[:, 2, 1] - m[:, 0, 1] * m[:, 2, 2]
    adj[:, 0, 2] = m[:, 0, 1] * m[:, 1, 2] - m[:, 0, 2] * m[:, 1, 1]
    adj[:, 1, 0] = m[:, 1, 2] * m[:, 2, 0] - m[:, 1, 0] * m[:, 2, 2]
    adj[:, 1, 1] = m[:, 0, 0] * m[:, 2, 2] - m[:, 0, 2] * m[:, 2, 0]
    adj[:, 1, 2] = m[:, 0, 2] * m[:, 1, 0] - m[:, 0, 0] * m[:, 1, 2]
    adj[:, 2, 0] = m[:, 1, 0] * m[:, 2, 1] - m[:, 1, 1] * m[:, 2, 0]
    adj[:, 2, 1] = m[:, 0, 1] * m[:, 2, 0] - m[:, 0, 0] * m[:, 2, 1]
    adj[:, 2, 2] = m[:, 0, 0] * m[:, 1, 1] - m[:, 0, 1] * m[:, 1, 0]
    det = m[:, 0, 0] * adj[:, 0, 0] + m[:, 0, 1] * adj[:, 1, 0] + m[:, 0, 2] * adj[:, 2, 0]
    omega2 = 1.0 / _dot(dvec, dvec)
    gw = np.empty((3, rows.size))
    for r in range(3):
        gw[r] = omega2 * (adj[rows, r, 0] * dvec[:, 0] + adj[rows, r, 1] * dvec[:, 1] + adj[rows, r, 2] * dvec[:, 2]) / det[rows]

    return dict(
        nbr_ptr=nbr_ptr, nbr_idx=nbr_idx, dist=dist[ee], area=e_area[ee], norm=(norm[ee] * sign[o][:, None]).T.copy(),
        skew=skew[ee].T.copy(), grad_wgt=gw, cvol=cvol, cskew=cskew, bnd_ptr=bnd_ptr, bnd_j=bj[ob].astype(np.int32),
        bnd_k=bk[ob].astype(np.int32), bnd_area=bar[ob], bnd_norm=bnr[ob].T.copy(), bnd_wgt=bwt[ob].T.copy(),
        n_tet=T, surf=surf,
    )
