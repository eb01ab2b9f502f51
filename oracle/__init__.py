"""CPU oracle for the assemble-and-solve path — TEST INFRASTRUCTURE ONLY.

Imported only by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg, always as
the reference answer (never as the thing measured or shipped). Parity is UNPINNED against outputs of the
reference itself (a Rust crate that cannot be built here and ships no golden vectors for this
path); the restatement is pinned to known answers instead — see tests/test_oracle.py.

Modules:
  vfv_oracle.c  assembly in push order, CSC/CSR from triplets, SpMV, GMRES, ILU(0)  (C, ctypes)
  geom_tet.py   the Voronoi dual of a tetrahedralisation (numpy)
  lu.py         FP64 sparse LU solve (scipy SuperLU), the reference's LinearLu role
  ordering.py   ILU(0) orderings (natural dependency levels, greedy multicolour)
  ns_oracle.c   coupled Navier-Stokes assembly: pressure-gradient coefficients, Rhie-Chow flow
                data, triplets of SteadyFlow::assemble_matrix in push order  (C, ctypes)
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class OrcDual(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("n_pts", C.c_int64), ("n_dir", C.c_int64), ("n_bsub", C.c_int64),
        ("np", C.c_void_p), ("ni", C.c_void_p), ("dist", C.c_void_p), ("area", C.c_void_p), ("skew", C.c_void_p),
        ("cvol", C.c_void_p), ("cskew", C.c_void_p), ("bp", C.c_void_p), ("bj", C.c_void_p), ("bk", C.c_void_p),
        ("barea", C.c_void_p), ("bw", C.c_void_p),
    ]


class OrcIlu(C.Structure):
    _fields_ = [("rp", C.c_void_p), ("dg", C.c_void_p), ("ci", C.c_void_p), ("perm", C.c_void_p), ("lu", C.c_void_p)]


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        _lib = C.CDLL(_SO)
        _lib.orc_heat_triplets.restype = C.c_int64
        _lib.orc_transport_triplets.restype = C.c_int64
        _lib.orc_csr_from_triplets.restype = C.c_int64
        _lib.orc_gmres.restype = C.c_int
        _lib.orc_ilu0_factor.restype = C.c_int
        _lib.orc_grad_coeff.restype = C.c_int64
        _lib.orc_ns_triplets.restype = C.c_int64
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def grad(dual: dict, f: np.ndarray) -> np.ndarray:
    n = dual["nbr_ptr"].size - 1
    f = _c(f, np.float64)
    g = np.empty((3, n))
    lib().orc_grad(C.c_int64(n), _p(dual["nbr_ptr"]), _p(dual["nbr_idx"]), _p(dual["grad_wgt"]), C.c_int64(dual["nbr_idx"].size),
                   _p(f), _p(g))
    return g


def _orc_dual(dual: dict, n_pts: int):
    keep = {k: np.ascontiguousarray(v) for k, v in dual.items()}
    d = OrcDual()
    d.n = keep["nbr_ptr"].size - 1
    d.n_pts = n_pts
    d.n_dir = keep["nbr_idx"].size
    d.n_bsub = keep["bnd_j"].size
    for f, k in [("np", "nbr_ptr"), ("ni", "nbr_idx"), ("dist", "dist"), ("area", "area"), ("skew", "skew"), ("cvol", "cvol"),
                 ("cskew", "cskew"), ("bp", "bnd_ptr"), ("bj", "bnd_j"), ("bk", "bnd_k"), ("barea", "bnd_area"), ("bw", "bnd_wgt")]:
        setattr(d, f, keep[k].ctypes.data)
    return d, keep


def heat_triplets(dual: dict, n_pts: int, node_bnd: np.ndarray, bnd_order, bnd_kind, k, q, s, T, bc_val):
    """Triplets (rows, cols, vals) and b of SteadyHeat::assemble_matrix in push order.

    node_bnd: boundary id per vertex (n_tot, -1 for points); bnd_order: boundary ids in
    registration order; bnd_kind[id]: 0 temperature, 1 heat flux."""
    n = dual["nbr_ptr"].size - 1
    d, keep = _orc_dual(dual, n_pts)
    fields = [_c(a, np.float64) for a in (k, q, s, T)]
    gk, gq, gs, gT = (grad(dual, a) for a in fields)
    nb = _c(node_bnd, np.int32)
    order = _c(bnd_order, np.int32)
    kind = _c(bnd_kind, np.int32)
    bc = _c(bc_val, np.float64)
    cap = 2 * dual["nbr_idx"].size + 2 * n
    r = np.empty(cap, np.uint64)
    c = np.empty(cap, np.uint64)
    v = np.empty(cap)
    b = np.empty(n)
    nt = lib().orc_heat_triplets(C.byref(d), _p(nb), C.c_int32(order.size), _p(order), _p(kind), *[_p(a) for a in fields], _p(bc),
                                 _p(gk), _p(gq), _p(gs), _p(gT), _p(r), _p(c), _p(v), _p(b))
    del keep
    return r[:nt].copy(), c[:nt].copy(), v[:nt].copy(), b


def transport_triplets(dual: dict, n_pts: int, node_bnd: np.ndarray, D, vel, dt: float):
    """Triplets of the transient transport operator (time + diffusion + power-law advection) of one
    mesh in push order. vel is [3][n]; gradients come from oracle.grad."""
    n = dual["nbr_ptr"].size - 1
    d, keep = _orc_dual(dual, n_pts)
    D = _c(np.broadcast_to(D, (n,)), np.float64)
    vel = _c(vel, np.float64).reshape(3, n)
    gD = grad(dual, D)
    gvel = _c(np.concatenate([grad(dual, vel[q]) for q in range(3)]), np.float64)
    norm = _c(dual["norm"], np.float64)
    nb = _c(node_bnd, np.int32)
    cap = 4 * dual["nbr_idx"].size + 2 * n
    r = np.empty(cap, np.uint64)
    c = np.empty(cap, np.uint64)
    v = np.empty(cap)
    nt = lib().orc_transport_triplets(C.byref(d), _p(norm), _p(nb), C.c_int32(int(nb.max()) + 1 if nb.size else 0), _p(D), _p(gD),
                                      _p(vel), _p(gvel), C.c_double(dt), _p(r), _p(c), _p(v))
    del keep
    return r[:nt].copy(), c[:nt].copy(), v[:nt].copy()


def csr_from_triplets(n: int, rows, cols, vals):
    rows, cols, vals = _c(rows, np.uint64), _c(cols, np.uint64), _c(vals, np.float64)
    rp = np.empty(n + 1, np.int64)
    ci = np.empty(max(rows.size, 1), np.int32)
    va = np.empty(max(rows.size, 1))
    nnz = lib().orc_csr_from_triplets(C.c_int64(n), C.c_int64(rows.size), _p(rows), _p(cols), _p(vals), _p(rp), _p(ci), _p(va))
    return rp, ci[:nnz].copy(), va[:nnz].copy()


def spmv(rp, ci, va, x):
    rp, ci, va, x = _c(rp, np.int64), _c(ci, np.int32), _c(va, np.float64), _c(x, np.float64)
    y = np.empty(rp.size - 1)
    lib().orc_spmv(C.c_int64(rp.size - 1), _p(rp), _p(ci), _p(va), _p(x), _p(y))
    return y


class Ilu0:
    """ILU(0) of P A P^T (perm: new -> old)."""

    def __init__(self, rp, ci, va, perm):
        n = rp.size - 1
        perm = _c(perm, np.int32)
        iperm = np.empty(n, np.int32)
        iperm[perm] = np.arange(n, dtype=np.int32)
        rows = np.repeat(np.arange(n), np.diff(rp))
        nr = iperm[rows]
        nc = iperm[ci]
        o = np.lexsort((nc, nr))
        self.rp = np.zeros(n + 1, np.int64)
        np.add.at(self.rp, nr + 1, 1)
        self.rp = np.cumsum(self.rp).astype(np.int64)
        self.ci = nc[o].astype(np.int32)
        self.lu = _c(va, np.float64)[o].copy()
        sr = nr[o]
        diag = np.nonzero(self.ci == sr)[0]
        if diag.size != n:
            raise ValueError("ILU(0) needs every diagonal")
        self.dg = diag.astype(np.int64)
        self.perm = perm
        self.n = n
        if lib().orc_ilu0_factor(C.c_int64(n), _p(self.rp), _p(self.ci), _p(self.dg), _p(self.lu)) != 0:
            raise ZeroDivisionError("ILU(0): zero pivot")

    def apply(self, r):
        r = _c(r, np.float64)
        t = np.empty(self.n)
        z = np.empty(self.n)
        lib().orc_ilu0_apply(C.c_int64(self.n), _p(self.rp), _p(self.ci), _p(self.dg), _p(self.lu), _p(self.perm), _p(r), _p(t), _p(z))
        return z

    def sweep_apply(self, r, sweeps: int, half: bool = False):
        """z = M^-1 r with `sweeps` Jacobi sweeps of each factor instead of the exact triangular
        solves (Anzt, Chow & Dongarra, "Iterative sparse triangular solves for preconditioning",
        Euro-Par 2015), on L = I + N, U = D + S of this factor:
            u^0 = y = P r,   u^k = y - N u^(k-1);   w^0 = D^-1 u,   w^k = D^-1 (u - S w^(k-1));
        z = P^T w^sweeps. The iterates do not depend on the numbering (every row of a sweep reads
        only the previous sweep). half: N and S as the mixed solver's half-precision copies of the
        float factor: per row and triangle, the values divided by the row's largest magnitude
        (computed in float), rounded to half, and the row's sum multiplied back by that scale."""
        n = self.n
        rows = np.repeat(np.arange(n), np.diff(self.rp))
        low, up = self.ci < rows, self.ci > rows
        d = self.lu[self.dg]
        vals = self.lu
        if half:
            v32 = self.lu.astype(np.float32)
            vals = np.empty(self.lu.size)
            for mask in (low, up):
                sc = np.zeros(n, np.float32)
                np.maximum.at(sc, rows[mask], np.abs(v32[mask]))
                sc[sc == 0] = 1.0
                h = (v32[mask] / sc[rows[mask]]).astype(np.float16)
                vals[mask] = h.astype(np.float64) * sc[rows[mask]].astype(np.float64)

        def tri(mask, x):
            return np.bincount(rows[mask], weights=vals[mask] * x[self.ci[mask]], minlength=n)

        y = _c(r, np.float64)[self.perm]
        u = y.copy()
        for _ in range(sweeps):
            u = y - tri(low, u)
        w = u / d
        for _ in range(sweeps):
            w = (u - tri(up, w)) / d
        z = np.empty(n)
        z[self.perm] = w
        return z

    def c_struct(self):
        s = OrcIlu()
        s.rp, s.dg, s.ci, s.perm, s.lu = (self.rp.ctypes.data, self.dg.ctypes.data, self.ci.ctypes.data, self.perm.ctypes.data,
                                          self.lu.ctypes.data)
        return s


def gmres(rp, ci, va, b, x0=None, tol=1e-6, restart=50, max_outer=200, precond=1, ilu: Ilu0 | None = None, max_steps=0):
    """Restarted GMRES (precond 0 none, 1 Jacobi, 2 ILU(0)). Returns (x, converged, iters, relres)."""
    rp, ci, va, b = _c(rp, np.int64), _c(ci, np.int32), _c(va, np.float64), _c(b, np.float64)
    n = rp.size - 1
    x = np.zeros(n) if x0 is None else _c(x0, np.float64).copy()
    its = C.c_int()
    rel = C.c_double()
    s = ilu.c_struct() if ilu is not None else None
    rc = lib().orc_gmres(C.c_int64(n), _p(rp), _p(ci), _p(va), _p(b), _p(x), C.c_double(tol), C.c_int(restart), C.c_int(max_outer),
                         C.c_int(precond), C.byref(s) if s is not None else None, C.c_int64(max_steps), C.byref(its), C.byref(rel))
    return x, rc == 0, its.value, rel.value


# ---------------------------------------------------------------- coupled Navier-Stokes (ns_oracle.c)
class OrcNsGeom(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("n_pts", C.c_int64), ("n_dir", C.c_int64), ("n_bsub", C.c_int64),
        ("np", C.c_void_p), ("ni", C.c_void_p), ("dist", C.c_void_p), ("area", C.c_void_p), ("norm", C.c_void_p),
        ("skew", C.c_void_p), ("gw", C.c_void_p), ("cvol", C.c_void_p), ("cskew", C.c_void_p), ("bp", C.c_void_p),
        ("bj", C.c_void_p), ("bk", C.c_void_p), ("barea", C.c_void_p), ("bnorm", C.c_void_p), ("bw", C.c_void_p),
        ("gcp", C.c_void_p), ("gcv", C.c_void_p), ("gcc", C.c_void_p), ("n_gc", C.c_int64),
    ]


class NsGeom:
    """The dual plus its pressure-gradient coefficients (Tetrahedron::grad_coeff) for the NS oracle."""

    def __init__(self, dual: dict, n_pts: int):
        self.keep = {k: np.ascontiguousarray(v) for k, v in dual.items()}
        self.n = self.keep["nbr_ptr"].size - 1
        self.n_pts = n_pts
        g = OrcNsGeom()
        g.n, g.n_pts, g.n_dir, g.n_bsub = self.n, n_pts, self.keep["nbr_idx"].size, self.keep["bnd_j"].size
        for f, k in [("np", "nbr_ptr"), ("ni", "nbr_idx"), ("dist", "dist"), ("area", "area"), ("norm", "norm"), ("skew", "skew"),
                     ("gw", "grad_wgt"), ("cvol", "cvol"), ("cskew", "cskew"), ("bp", "bnd_ptr"), ("bj", "bnd_j"), ("bk", "bnd_k"),
                     ("barea", "bnd_area"), ("bnorm", "bnd_norm"), ("bw", "bnd_wgt")]:
            setattr(g, f, self.keep[k].ctypes.data)
        self.gcp = np.zeros(self.n + 1, np.int64)
        tot = lib().orc_grad_coeff(C.byref(g), _p(self.gcp), None, None, C.c_int64(0))
        self.gcv = np.empty(max(tot, 1), np.int32)
        self.gcc = np.empty((3, max(tot, 1)))
        lib().orc_grad_coeff(C.byref(g), _p(self.gcp), _p(self.gcv), _p(self.gcc), C.c_int64(max(tot, 1)))
        self.n_gc = tot
        g.gcp, g.gcv, g.gcc, g.n_gc = self.gcp.ctypes.data, self.gcv.ctypes.data, self.gcc.ctypes.data, max(tot, 1)
        self.g = g
        self.dual = dual

    def vec_grad(self, vec):
        """[9][n] LSQ gradients of the three components (u_x u_y u_z v_x ... w_z)."""
        vec = np.asarray(vec, np.float64).reshape(3, self.n)
        return np.ascontiguousarray(np.concatenate([grad(self.dual, vec[q]) for q in range(3)]))

    def flow(self, vel, p, den, visc, fce):
        """(rc, flux): Rhie-Chow coefficient V/a_P per vertex and face mass flux per directed face."""
        vel = _c(vel, np.float64).reshape(3, self.n)
        fce = _c(fce, np.float64).reshape(3, self.n)
        den, visc, p = (_c(np.broadcast_to(a, (self.n,)), np.float64) for a in (den, visc, p))
        gvel, gfce = self.vec_grad(vel), self.vec_grad(fce)
        gden, gvisc = grad(self.dual, den), grad(self.dual, visc)
        rc = np.empty(self.n)
        flux = np.empty(self.keep["nbr_idx"].size)
        lib().orc_ns_flow(C.byref(self.g), _p(vel), _p(gvel), _p(p), _p(den), _p(gden), _p(visc), _p(gvisc), _p(fce), _p(gfce), _p(rc),
                          _p(flux))
        return rc, flux

    def triplets(self, node_bnd, bnd_order, bc_vel, pref_vid, pref, vel, p, den, visc, fce):
        """Triplets (rows, cols, vals) and b [4n] of SteadyFlow::assemble_matrix at the state (vel, p)."""
        vel = _c(vel, np.float64).reshape(3, self.n)
        fce = _c(fce, np.float64).reshape(3, self.n)
        den, visc, p = (_c(np.broadcast_to(a, (self.n,)), np.float64) for a in (den, visc, p))
        rc, flux = self.flow(vel, p, den, visc, fce)
        gvel, gfce = self.vec_grad(vel), self.vec_grad(fce)
        gden, gvisc = grad(self.dual, den), grad(self.dual, visc)
        nb, order = _c(node_bnd, np.int32), _c(bnd_order, np.int32)
        bcv = _c(bc_vel, np.float64).reshape(3, self.n)
        args = [_p(nb), C.c_int32(order.size), _p(order), _p(bcv), C.c_int64(pref_vid), C.c_double(pref), _p(vel), _p(gvel), _p(den),
                _p(gden), _p(visc), _p(gvisc), _p(fce), _p(gfce), _p(rc), _p(flux)]
        cap = lib().orc_ns_triplets(C.byref(self.g), *args, None, None, None, None)
        r = np.empty(cap, np.uint64)
        c = np.empty(cap, np.uint64)
        v = np.empty(cap)
        b = np.empty(4 * self.n)
        nt = lib().orc_ns_triplets(C.byref(self.g), *args, _p(r), _p(c), _p(v), _p(b))
        return r[:nt].copy(), c[:nt].copy(), v[:nt].copy(), b
