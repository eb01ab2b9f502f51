"""Seeded synthetic heat problems on jittered-cube meshes.

* ``steady_heat(n, hetero=False)``: the cube heat problem of the reference's heat examples
  (examples/heat/heat_analytic.rs:9-98 layout): Dirichlet T=0 on bnd_l (x=0) and T=1 on bnd_r
  (x=1), zero flux on the four other faces. With ``hetero=False``: k=1, q=0, s=0 (8,000 vertices
  at n=20). With ``hetero=True``: log k ~ N(0,1) i.i.d. per vertex and q ~ U[0,1] (1,000,000
  vertices at n=100), from numpy's PCG64 generator seeded with ``field_seed``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .mesh import Mesh

# boundary ids of the cube meshes in registration order: l, r, f, k, b, t
HEAT_BND_KIND = np.array([L.BC_TEMP, L.BC_TEMP, L.BC_FLUX, L.BC_FLUX, L.BC_FLUX, L.BC_FLUX], np.int32)
HEAT_BND_ORDER = np.arange(6, dtype=np.int32)


@dataclass
class HeatProblem:
    mesh: Mesh
    k: np.ndarray
    q: np.ndarray
    s: np.ndarray
    T0: np.ndarray        # initial guess (Dirichlet values loaded, zero elsewhere)
    bc_val: np.ndarray    # Dirichlet value or outward flux on nodes, 0 on points
    node_bnd: np.ndarray  # boundary id per vertex, -1 for points
    bnd_kind: np.ndarray = field(default_factory=lambda: HEAT_BND_KIND.copy())
    bnd_order: np.ndarray = field(default_factory=lambda: HEAT_BND_ORDER.copy())

    @property
    def n(self) -> int:
        return self.mesh.n_tot


def heat_fields(node_bnd: np.ndarray, hetero: bool = False, field_seed: int = 7, flux_top: float = 0.0, prod: float = 0.0):
    """(k, q, s, T0, bc_val) of the cube heat problem for a vertex set with boundary ids node_bnd
    (-1 for points); numpy only."""
    N = node_bnd.size
    if hetero:
        rng = np.random.default_rng(field_seed)
        k = np.exp(rng.standard_normal(N))
        q = rng.uniform(0.0, 1.0, N)
    else:
        k = np.ones(N)
        q = np.zeros(N)
    s = np.full(N, float(prod))
    bc = np.zeros(N)
    bc[node_bnd == 1] = 1.0          # T = 1 at x = 1
    bc[node_bnd == 5] = flux_top     # optional outward flux on z = 1
    T0 = np.zeros(N)
    T0[node_bnd == 1] = 1.0           # initial_dirichlet (steady_base.rs:53-57)
    return k, q, s, T0, bc


def steady_heat(n: int, hetero: bool = False, mesh_seed: int = 42, field_seed: int = 7, flux_top: float = 0.0,
                prod: float = 0.0) -> HeatProblem:
    mesh = Mesh.jitter_cube(n, mesh_seed, 0.25)
    N = mesh.n_tot
    _, nb, _ = mesh.export()
    node_bnd = np.full(N, -1, np.int32)
    node_bnd[mesh.n_pts:] = nb
    k, q, s, T0, bc = heat_fields(node_bnd, hetero, field_seed, flux_top, prod)
    return HeatProblem(mesh, k, q, s, T0, bc, node_bnd)


@dataclass
class TransportBatch:
    meshes: list
    n_grid: np.ndarray       # grid points per axis of every mesh
    D: float
    dt: float
    steps: int


def transport_batch(count: int = 256, nmin: int = 2000, nmax: int = 50000, seed: int = 4, D: float = 1e-3, dt: float = 1e-2,
                    steps: int = 100, dual_ctx=None) -> TransportBatch:
    """Transport batch: `count` jittered cubes with vertex counts N_i drawn log-uniform in [nmin, nmax]
    (numpy PCG64, `seed`), n_i = round(N_i^(1/3)) grid points per axis, mesh seeds 1000 + i. With
    `dual_ctx` the Voronoi duals are built on that context's device (same bits as on the host)."""
    rng = np.random.default_rng(seed)
    N = np.exp(rng.uniform(np.log(nmin), np.log(nmax), count))
    n = np.maximum(3, np.rint(np.cbrt(N))).astype(np.int32)
    seeds = 1000 + np.arange(count, dtype=np.uint64)
    meshes = Mesh.jitter_cubes_device_dual(dual_ctx, n, seeds) if dual_ctx is not None else Mesh.jitter_cubes(n, seeds)
    return TransportBatch(meshes, n, D, dt, steps)


def transport_fields(meshes, phase_seed: int = 9):
    """Velocity u = (sin pi y, sin pi z, sin pi x) ([3][n_tot]) and a seeded smooth initial field
    c0 = 1 + 0.5 sin(pi x + a) sin(pi y + b) sin(pi z + c), phases per mesh from PCG64(phase_seed)."""
    rng = np.random.default_rng(phase_seed)
    vel, c0 = [], []
    for m in meshes:
        pos, _, _ = m.export()
        x, y, z = pos[:, 0], pos[:, 1], pos[:, 2]
        vel.append(np.stack([np.sin(np.pi * y), np.sin(np.pi * z), np.sin(np.pi * x)]))
        a, b, c = rng.uniform(0, 2 * np.pi, 3)
        c0.append(1.0 + 0.5 * np.sin(np.pi * x + a) * np.sin(np.pi * y + b) * np.sin(np.pi * z + c))
    return np.concatenate(vel, axis=1), np.concatenate(c0)


@dataclass
class FlowProblem:
    """Steady incompressible flow in the unit cube with velocity boundaries on all six faces and
    the pressure fixed at one node (the layout of the reference's examples/flow/flow_lid.rs)."""
    mesh: Mesh
    rho: np.ndarray       # density per vertex
    mu: np.ndarray        # viscosity per vertex
    fce: np.ndarray       # body force [3][n] (rho g, not g)
    bc_vel: np.ndarray    # boundary velocity [3][n] at nodes, 0 at points
    node_bnd: np.ndarray  # boundary id per vertex, -1 for points
    pref_vid: int         # vertex whose pressure is fixed (node 0 = first node)
    pref: float = 0.0
    bnd_order: np.ndarray = field(default_factory=lambda: HEAT_BND_ORDER.copy())

    @property
    def n(self) -> int:
        return self.mesh.n_tot

    def initial_state(self) -> np.ndarray:
        """x0 = [u | v | w | p] with the boundary velocities loaded (initial_dirichlet)."""
        x = np.zeros(4 * self.n)
        x[:3 * self.n] = self.bc_vel.reshape(-1)
        return x


def lid_cavity(n: int, mesh_seed: int = 42, rho: float = 1.0, mu: float = 0.01, lid=(1.0, 0.0, 0.0), gravity: float = 0.0) -> FlowProblem:
    """Lid-driven cavity: u = lid on bnd_t (z = 1), no-slip on the other faces, p = 0 at node 0;
    rho = 1, mu = 0.01 (Re = 100 with U = L = 1) by default. ``gravity`` adds the body force
    (0, 0, -rho g)."""
    mesh = Mesh.jitter_cube(n, mesh_seed, 0.25)
    N = mesh.n_tot
    _, nb, _ = mesh.export()
    node_bnd = np.full(N, -1, np.int32)
    node_bnd[mesh.n_pts:] = nb
    bc = np.zeros((3, N))
    top = node_bnd == 5
    for q in range(3):
        bc[q, top] = lid[q]
    fce = np.zeros((3, N))
    fce[2, :] = -rho * gravity
    return FlowProblem(mesh, np.full(N, float(rho)), np.full(N, float(mu)), fce, bc, node_bnd, mesh.n_pts)
