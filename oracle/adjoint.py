"""Adjoint gradient of the heat solve — TEST INFRASTRUCTURE (oracle).

J(T) = 0.5 sum_{i in sensors} (T_i - d_i)^2 with A(k) T = b(q) the system of
SteadyHeat::assemble_matrix (src/steady/core/steady_heat.rs:143-171) at zero production.
The reference has no adjoint; this is the oracle for the product's one. It is built differently
from the product's gather kernels: explicit sparse Jacobians (selectors, the least-squares gradient
operator of ScalarDomain::update_grad, src/base/scl_dom.rs:146-164) and scipy's SuperLU for the
transposed solve. `tests/test_oracle.py` pins it against central finite differences of the
oracle's own forward model (oracle.heat_triplets + SuperLU).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle


def _system(prob, k, q):
    d = prob.mesh.dual()
    r, c, v, b = oracle.heat_triplets(d, prob.mesh.n_pts, prob.node_bnd, prob.bnd_order, prob.bnd_kind, k, q, prob.s, prob.T0,
                                      prob.bc_val)
    n = prob.n
    A = sp.csr_matrix((v, (r.astype(np.int64), c.astype(np.int64))), shape=(n, n))  # duplicates summed
    return A, b


def solve_state(prob, k, q, refine: int = 2):
    """T = A^-1 b by SuperLU plus iterative refinement with the residual in long double, so that
    finite differences of J at a step of 1e-6 are not limited by the solve's round-off."""
    A, b = _system(prob, k, q)
    lu = spla.splu(A.tocsc())
    T = lu.solve(b)
    Al = A.astype(np.longdouble)
    bl = b.astype(np.longdouble)
    for _ in range(refine):
        r = bl - Al @ T.astype(np.longdouble)
        T = (T.astype(np.longdouble) + lu.solve(r.astype(np.float64)).astype(np.longdouble)).astype(np.float64)
    return T


def objective(prob, logk, q, sensors, target):
    T = solve_state(prob, np.exp(logk), q)
    r = T[sensors].astype(np.longdouble) - target
    return float(0.5 * (r @ r)), T


def _grad_ops(d, n):
    """Sparse gradient operators G_c (c = x, y, z): (G_c f)_u = sum_loc w_c (f_n - f_u)."""
    owner = np.repeat(np.arange(n), np.diff(d["nbr_ptr"]))
    ops = []
    for c in range(3):
        w = d["grad_wgt"][c]
        G = sp.csr_matrix((w, (owner, d["nbr_idx"].astype(np.int64))), shape=(n, n))
        G = G - sp.diags(np.asarray(G.sum(axis=1)).ravel())
        ops.append(G.tocsr())
    return ops, owner


def gradient(prob, logk, q, sensors, target):
    """(J, dJ/dlog k, dJ/dq, lambda)"""
    n = prob.n
    k = np.exp(logk)
    d = prob.mesh.dual()
    A, b = _system(prob, k, q)
    lu = spla.splu(A.tocsc())
    T = lu.solve(b)
    g = np.zeros(n)
    res = T[sensors] - target
    g[sensors] = res
    lam = spla.splu(A.T.tocsc()).solve(g)
    G, owner = _grad_ops(d, n)
    nb = d["nbr_idx"].astype(np.int64)
    nd = nb.size
    dirichlet = prob.node_bnd >= 0
    dirichlet &= prob.bnd_kind[np.maximum(prob.node_bnd, 0)] == 0
    active = ~dirichlet[owner]                       # faces of rows that carry diffusion
    gk = np.stack([Gc @ k for Gc in G])              # grad k, [3][n]
    kv, kn = k[owner], k[nb]
    ks = kv + kn
    km = np.where(ks != 0, 2.0 * kv * kn / np.where(ks != 0, ks, 1.0), 0.0)
    skew = d["skew"]
    kraw = km + 0.5 * (skew[0] * (gk[0, owner] + gk[0, nb]) + skew[1] * (gk[1, owner] + gk[1, nb]) + skew[2] * (gk[2, owner] + gk[2, nb]))
    branch = (kraw > 0.0) & active
    phi = np.where(active, -lam[owner] * (T[nb] - T[owner]) * d["area"] / d["dist"], 0.0)
    inv2 = np.where(ks != 0, 1.0 / np.where(ks != 0, ks, 1.0) ** 2, 0.0)
    Ev = sp.csr_matrix((np.ones(nd), (np.arange(nd), owner)), shape=(nd, n))
    En = sp.csr_matrix((np.ones(nd), (np.arange(nd), nb)), shape=(nd, n))
    M = sp.diags(2.0 * kn * kn * inv2) @ Ev + sp.diags(2.0 * kv * kv * inv2) @ En
    for c in range(3):
        M = M + sp.diags(np.where(branch, 0.5 * skew[c], 0.0)) @ ((Ev + En) @ G[c])
    dJdk = M.T @ phi
    # dJ/dq = lambda^T db/dq, b_v = -(q_v + grad q_v . cskew_v) vol_v on rows that carry sources
    rows_src = (~dirichlet).astype(float)
    cs = d["cskew"]
    DB = sp.eye(n) + sp.diags(cs[0]) @ G[0] + sp.diags(cs[1]) @ G[1] + sp.diags(cs[2]) @ G[2]
    DB = -sp.diags(d["cvol"] * rows_src) @ DB
    dJdq = DB.T @ lam
    J = 0.5 * float(res @ res)
    return J, k * dJdk, dJdq, lam


def fd_directional(prob, logk, q, sensors, target, dk, dq, h=1e-6):
    """central difference (J(p + h delta) - J(p - h delta)) / 2h along delta = (dk, dq)"""
    jp, _ = objective(prob, logk + h * dk, q + h * dq, sensors, target)
    jm, _ = objective(prob, logk - h * dk, q - h * dq, sensors, target)
    return (jp - jm) / (2.0 * h)
