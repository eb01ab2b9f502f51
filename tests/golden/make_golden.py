"""Generates tests/golden/golden_small.npz: small seeded cases of every assembled system of this
path, computed by the CPU oracle (the reference cannot be built or run here, so these vectors pin
the oracle and the product against a committed record rather than against reference output).

Cases (all meshes are jittered cubes, seed 42 unless stated):
  heat   n=6, heterogeneous k and q, flux 0.3 on the top face, production -0.5: mesh positions,
         CSR (rowptr, colind, values), b, and the FP64 LU solution
  trans  n=5 (mesh seed 11): the transport operator (D=1e-3, u=(sin pi y, sin pi z, sin pi x),
         dt=1e-2) as CSR
  flow   lid-driven cavity n=5: CSR and b at the initial state, and one damped Picard step (LU)

Run from the repository root: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_small.npz")


def heat_case():
    import oracle
    from oracle.lu import lu_solve
    from vfvchem_vfvm3d_b200.problems import steady_heat
    prob = steady_heat(6, hetero=True, flux_top=0.3, prod=-0.5)
    d = prob.mesh.dual()
    r, c, v, b = oracle.heat_triplets(d, prob.mesh.n_pts, prob.node_bnd, prob.bnd_order, prob.bnd_kind, prob.k, prob.q, prob.s, prob.T0,
                                      prob.bc_val)
    rp, ci, va = oracle.csr_from_triplets(prob.n, r, c, v)
    pos, _, _ = prob.mesh.export()
    return dict(heat_pos=pos, heat_rp=rp, heat_ci=ci, heat_va=va, heat_b=b, heat_x=lu_solve(rp, ci, va, b))


def transport_case():
    import oracle
    from vfvchem_vfvm3d_b200 import Mesh
    from vfvchem_vfvm3d_b200.problems import transport_fields
    m = Mesh.jitter_cubes([5], [11])[0]
    vel, _ = transport_fields([m])
    _, nb, _ = m.export()
    node_bnd = np.full(m.n_tot, -1, np.int32)
    node_bnd[m.n_pts:] = nb
    r, c, v = oracle.transport_triplets(m.dual(), m.n_pts, node_bnd, 1e-3, vel, 1e-2)
    rp, ci, va = oracle.csr_from_triplets(m.n_tot, r, c, v)
    return dict(trans_rp=rp, trans_ci=ci, trans_va=va)


def flow_case():
    import oracle
    from oracle.lu import lu_solve
    from vfvchem_vfvm3d_b200.problems import lid_cavity
    prob = lid_cavity(5)
    n = prob.n
    g = oracle.NsGeom(prob.mesh.dual(), prob.mesh.n_pts)
    x0 = prob.initial_state()
    r, c, v, b = g.triplets(prob.node_bnd, prob.bnd_order, prob.bc_vel, prob.pref_vid, prob.pref, x0[:3 * n].reshape(3, n), x0[3 * n:],
                            prob.rho, prob.mu, prob.fce)
    rp, ci, va = oracle.csr_from_triplets(4 * n, r, c, v)
    x1 = 0.2 * x0 + 0.8 * lu_solve(rp, ci, va, b)
    return dict(flow_rp=rp, flow_ci=ci, flow_va=va, flow_b=b, flow_x1=x1)


def build():
    out = {}
    for f in (heat_case, transport_case, flow_case):
        out.update(f())
    return out


if __name__ == "__main__":
    np.savez_compressed(OUT, **build())
    print("wrote", OUT, os.path.getsize(OUT), "bytes")
