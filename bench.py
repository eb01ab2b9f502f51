"""Benchmark of the assemble-and-solve path on one B200 (or N replicas).

Workload (one "step"): the 1,000,000-vertex heterogeneous steady heat system (100^3 jittered
cube, log k ~ N(0,1), q ~ U[0,1], Dirichlet T=0/1 on x=0/1, zero flux elsewhere) solved by
GMRES(50) + ILU(0) to relative residual 1e-12 (TOL_RELRES), which puts both solvers within 1e-8
relative 2-norm error of the FP64 reference solution — the FP32-inner / FP64-refinement solver is
the timed `value`; the plain FP64 solver is timed beside it. Inputs are resident in HBM; the matrix
(16.1 M non-zeros, 193 MB of FP64 values and columns) exceeds the 126 MB L2, so no L2 flush is
needed between steps.

The reference solution x_ref is computed on the host by the oracle from its own assembly of the
system: FP64 restarted GMRES(50) with a natural-order ILU(0), driven to relres 1e-14 (SuperLU does
not finish on 10^6 rows in bench time; that oracle solver agrees with SuperLU to 1.0e-11 at 125,000
rows).

The mixed solver's preconditioner is ILU(0) in the natural order with its triangular solves done
as ILU_SWEEPS Jacobi sweeps of each factor (bandwidth-bound launches over compact triangles whose
values are stored in half precision, each row scaled by its largest magnitude); the
plain FP64 solver is the exact multicolour ILU(0) (level-scheduled sweeps). The FP64 solver with
the same swept preconditioner and the mixed solver with the exact one are timed beside them.

`roofline` is the kernel with the largest share of the mixed solve's kernel time (the float
Jacobi sweeps of the factors), timed alone with CUDA events on the library's stream;
`roofline_spmv` is the FP64 SpMV timed the same way.

`--impl reference` times the reference's own algorithm for this path on the host cores
(Jacobi-preconditioned restarted GMRES(50), FP64, the oracle port) to the same relres.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GMRES solve s to 1e-8 vs FP64 LU: mixed vs plain FP64 on GPU; SpMV HBM GB/s"
ERR_TARGET = 1e-8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vfv", choices=["vfv", "reference"])
    ap.add_argument("--n", "--grid", dest="n", type=int, default=100, help="grid points per axis (100 -> 1,000,000 vertices)")
    ap.add_argument("--restart", type=int, default=50)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--engine", type=int, default=2,
                    help="0 persistent cycle kernel, 1 CUDA graph of per-phase kernels, 2 graph with the ILU(0) sweeps overlapped (flexible GMRES)")
    ap.add_argument("--no-extras", action="store_true", help="skip the adjoint and batched-transport timings")
    ap.add_argument("--batch", type=int, default=256, help="meshes in the batched transport timing")
    ap.add_argument("--flow-n", type=int, default=64, help="grid points per axis of the cavity flow timing")
    return ap.parse_args()


def extras_adjoint(heat, prob, x_ref_h, ctx):
    """Steady adjoint: J = 0.5 sum (T_i - d_i)^2 over 1000 seeded sensors, gradient w.r.t. every
    log k and q (one transposed solve + gathers), timed through the host-array API; then checked
    against central finite differences of the device forward model on 64 seeded directions."""
    from vfvchem_vfvm3d_b200 import GmresOptions
    from vfvchem_vfvm3d_b200 import _lib as L
    rng = np.random.default_rng(17)
    sens = rng.choice(prob.n, 1000, replace=False)
    d = rng.uniform(0, 1, 1000)
    g = np.zeros(prob.n)
    g[sens] = x_ref_h[sens] - d
    opts = GmresOptions(tol=1e-10, restart=50, max_outer=2000, precond=L.PRECOND_ILU0, precision=L.MIXED, inner_rtol=1e-6)
    heat.adjoint(x_ref_h, g, opts)
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        _, dk, dq, info = heat.adjoint(x_ref_h, g, opts)
        ts.append(time.perf_counter() - t0)
    out = {"adjoint_s": min(ts), "adjoint_iters": info.iters, "sensors": 1000, "grad_norm_logk": float(np.linalg.norm(dk)),
           "grad_norm_q": float(np.linalg.norm(dq)), "workload": "dJ/dlog k and dJ/dq on the same 1M-vertex system, host arrays in/out"}
    out["fd_check"] = adjoint_fd_check(heat, prob, sens, d)
    return out


def guard_faces(heat, prob):
    """Skew-corrected face conductivities k_f of every directed face (opscl_dom_diff.rs:80 guards
    k_f > 0) with the harmonic means k_m, the face owners and neighbours."""
    dual = prob.mesh.dual()
    gk = heat.grad(prob.k)
    npt = dual["nbr_ptr"]
    v = np.repeat(np.arange(prob.n), np.diff(npt))
    nb = dual["nbr_idx"].astype(np.int64)
    kv, kn = prob.k[v], prob.k[nb]
    km = 2.0 * kv * kn / (kv + kn)
    sk = np.asarray(dual["skew"]).reshape(3, -1)
    kf = km + 0.5 * (sk[0] * (gk[0][v] + gk[0][nb]) + sk[1] * (gk[1][v] + gk[1][nb]) + sk[2] * (gk[2][v] + gk[2][nb]))
    return kf, km, v, nb, npt


def adjoint_fd_check(heat, prob, sens, d, ndir=64, ndir_wide=16, band=1e-2):
    """Central finite differences of J on the device forward model (assembly + FP64 GMRES(50)+ILU(0)
    to relres 1e-14) along seeded directions e = (e_logk, e_q), against the adjoint gradient at the
    same state: step h = 1e-6 on `ndir` directions, h = 1e-4 on the first `ndir_wide`.

    The forward model is only piecewise smooth: a face conductivity k_f is clamped at the k_f > 0
    guard (opscl_dom_diff.rs:80), and k_f depends on k of the face's vertices and, through the
    least-squares gradients, of their neighbours. A perturbation of every log k moves the faces
    that sit near the guard across it, and a difference quotient across that kink is not a
    derivative. So e_q has i.i.d. N(0, 1) entries everywhere, and e_logk has them everywhere except
    on the vertices whose k enters a face with |k_f| <= band * k_m (the face's two vertices and
    their neighbours), where it is zero; the counts are reported.

    The difference J(p + h e) - J(p - h e) is formed without cancellation: with T the computed
    base state, the solutions at p +- h e are T + delta+- where A+- delta+- = b+- - A+- T (the
    residual of T in each perturbed system, a vector of size ~h, solved to relres 1e-14 of its own
    norm; the residual is summed in extended precision on the host from the assembled FP64 values,
    which removes the cancellation of A T against b). T + delta+- is the perturbed solution whatever
    error T carries, so J+ - J- =
    sum_s (T_s - d_s) (delta+_s - delta-_s) + (delta+_s^2 - delta-_s^2) / 2 over the sensors.

    What remains at h = 1e-6 is the FP64 rounding of the perturbed assembly itself: ~1e-16 |A| |T|
    per row against a perturbation signal of ~h times the neighbour differences of T, about 1e-8 of
    the residual, which the sensors' cancellation amplifies to ~1e-6 in the quotient (an error
    that scales as 1/h; an iterative-refinement step of the correction solves does not change it).
    """
    from vfvchem_vfvm3d_b200 import GmresOptions
    from vfvchem_vfvm3d_b200 import _lib as L
    fo = GmresOptions(tol=1e-14, restart=50, max_outer=4000, precond=L.PRECOND_ILU0)
    logk, q = np.log(prob.k), prob.q
    pat = heat.pattern

    kf, km, v, nb, npt = guard_faces(heat, prob)
    near = np.abs(kf) <= band * km
    touched = np.zeros(prob.n, bool)
    touched[v[near]] = True
    touched[nb[near]] = True
    free = ~touched.copy()
    for u in np.nonzero(touched)[0]:  # neighbours of the face vertices enter their gradients
        free[nb[npt[u]:npt[u + 1]]] = False

    def assemble(lk, qq):
        return heat.assemble(np.exp(lk), qq, prob.s, prob.T0, prob.bc_val)

    def solve(b, x0):
        x, _ = pat.solve(b, x0, fo)
        return x

    rp_a, ci_a, _ = pat.export()
    starts = rp_a[:-1].astype(np.int64)

    def residual(b, x):  # b - A x with the pattern's current values, summed in extended precision on the host
        _, _, va = pat.export()
        ax = np.add.reduceat(va.astype(np.longdouble) * x.astype(np.longdouble)[ci_a], starts)
        return (b.astype(np.longdouble) - ax).astype(np.float64)

    def correction(b):  # A^-1 b for a right-hand side of size ~h
        return solve(b, np.zeros(prob.n))

    t0 = time.perf_counter()
    T = solve(assemble(logk, q), prob.T0)
    r0 = T[sens] - d
    J0 = 0.5 * float(r0 @ r0)
    g = np.zeros(prob.n)
    g[sens] = r0
    _, dk, dq, _ = heat.adjoint(T, g, fo)
    res = {}
    for h, nd in ((1e-6, ndir), (1e-4, ndir_wide)):
        errs = []
        r2 = np.random.default_rng(64)
        for _ in range(nd):
            ek, eq = r2.standard_normal(prob.n) * free, r2.standard_normal(prob.n)
            dm = correction(residual(assemble(logk - h * ek, q - h * eq), T))[sens]
            dp = correction(residual(assemble(logk + h * ek, q + h * eq), T))[sens]
            fd = float(r0 @ (dp - dm) + 0.5 * (dp @ dp - dm @ dm)) / (2 * h)
            ad = float(dk @ ek + dq @ eq)
            errs.append(abs(fd - ad) / abs(ad))
        res[f"h={h:g}"] = {"directions": nd, "median_rel": float(np.median(errs)), "max_rel": float(np.max(errs))}
    res["fd_median_rel"] = res["h=1e-06"]["median_rel"]
    res["fd_max_rel"] = res["h=1e-06"]["max_rel"]
    heat.assemble(prob.k, prob.q, prob.s, prob.T0, prob.bc_val)  # leave the base system assembled
    res.update({"J": J0, "directions": f"seed 64: e_q i.i.d. N(0,1) on all {prob.n} vertices; e_logk i.i.d. N(0,1) on the "
                                       f"{int(free.sum())} vertices whose k enters no face with |k_f| <= {band:g} k_m, 0 on the "
                                       f"other {int((~free).sum())}",
                "forward": "device assembly + FP64 GMRES(50)+ILU(0) to relres 1e-14; J+ - J- from correction solves of the "
                           "base state in both perturbed systems (no cancellation)",
                "faces_guard_active": int(np.sum(kf <= 0.0)), "faces_near_guard_1e-4": int(np.sum(np.abs(kf) <= 1e-4 * km)),
                f"faces_near_guard_{band:g}": int(near.sum()), "directed_faces": int(nb.size), "seconds": time.perf_counter() - t0})
    return res


def extras_flow(ctx, n):
    """Lid-driven cavity (rho = 1, mu = 0.01, lid u = (1, 0, 0)) on an n^3 jittered cube, 4 n^3
    unknowns: up to 20 damped Picard iterations (damping 0.8), each solved by GMRES(100) + 4x4
    block-Jacobi to 1e-8 relative residual, FP64 and FP32-inner / FP64-refinement."""
    from vfvchem_vfvm3d_b200 import SteadyFlowGpu
    from vfvchem_vfvm3d_b200 import _lib as L
    from vfvchem_vfvm3d_b200.flow import flow_options
    from vfvchem_vfvm3d_b200.problems import lid_cavity
    import torch
    t0 = time.perf_counter()
    prob = lid_cavity(n)
    t_mesh = time.perf_counter() - t0
    t0 = time.perf_counter()
    fl = SteadyFlowGpu(prob, ctx=ctx)
    t_setup = time.perf_counter() - t0
    x0 = torch.tensor(prob.initial_state(), device="cuda")
    bd = torch.empty_like(x0)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream_ptr)
    fl.assemble_device(x0.data_ptr(), bd.data_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(5):
        fl.assemble_device(x0.data_ptr(), bd.data_ptr())
    e1.record(stream)
    e1.synchronize()
    asm_ms = e0.elapsed_time(e1) / 5
    out = {"workload": f"lid-driven cavity {n}^3 ({4 * prob.n} unknowns, {fl.nnz} nnz, {fl.ntrip} triplets), Re 100; "
                       "20 Picard iterations max, damping 0.8, GMRES(100)+BJ4 to 1e-8 relres",
           "unknowns": 4 * prob.n, "nnz": fl.nnz, "triplets": fl.ntrip, "mesh_s": t_mesh, "setup_s": t_setup, "assembly_ms": asm_ms}
    finals = {}
    for prec, name in [(L.FP64, "fp64"), (L.MIXED, "mixed")]:
        t0 = time.perf_counter()
        r = fl.picard(max_iter=20, tol=1e-300, damp=0.8, opts=flow_options(prec, tol=1e-8, max_outer=100), raise_on_error=False)
        out[name] = {"picard_s": time.perf_counter() - t0, "solve_s": r.solve_seconds, "picard_iters": r.iterations,
                     "gmres_iters": int(np.sum(r.lin_iters)), "last_residual": float(r.residuals[-1]) if r.iterations else None,
                     "status": r.status}
        finals[name] = r.x
    out["speedup_mixed_vs_fp64_solve"] = out["fp64"]["solve_s"] / max(out["mixed"]["solve_s"], 1e-12)
    out["rel_diff_mixed_vs_fp64"] = float(np.linalg.norm(finals["mixed"] - finals["fp64"]) / np.linalg.norm(finals["fp64"]))
    fl.close()
    return out


def extras_transport(ctx, count):
    """Batched transient advection-diffusion: `count` meshes, 100 implicit steps, plus the
    checkpointed adjoint dJ/dD (checkpoint every 10 steps)."""
    from vfvchem_vfvm3d_b200 import GmresOptions, TransientTransportGpu
    from vfvchem_vfvm3d_b200 import _lib as L
    from vfvchem_vfvm3d_b200.problems import transport_batch, transport_fields
    t0 = time.perf_counter()
    tb = transport_batch(count, dual_ctx=ctx)  # Delaunay on the host, Voronoi duals on the device
    vel, c0 = transport_fields(tb.meshes)
    t_mesh = time.perf_counter() - t0
    tr = TransientTransportGpu(tb.meshes, tb.dt, ctx=ctx)
    tr.assemble(tb.D, vel)
    lanes = tr.pattern.autotune()
    # natural-order ILU(0) with 3 Jacobi sweeps per factor (measured on this batch: 0.69 s per 100
    # steps, 5.0 iterations per step, against 0.76 s and 6.8 with the exact multicolour ILU(0))
    swept = dict(precond=L.PRECOND_ILU0, ilu_order=L.ILU_NATURAL, ilu_sweeps=3)
    opts = GmresOptions(tol=1e-10, restart=30, max_outer=200, precision=L.MIXED, inner_rtol=1e-6, **swept)
    tr.run(c0, 3, opts)
    t0 = time.perf_counter()
    c, its = tr.run(c0, tb.steps, opts)
    t_run = time.perf_counter() - t0
    target = np.full(tr.n, float(np.mean(c0)))
    # the adjoint's forward re-runs and transposed solves use the same preconditioner (another
    # ordering would build its ILU(0) structures on the host inside the timed adjoint)
    aopts = GmresOptions(tol=1e-10, restart=30, max_outer=500, precision=L.MIXED, inner_rtol=1e-6, **swept)
    t0 = time.perf_counter()
    J, dJdD, aits = tr.adjoint_D(c0, tb.steps, target, every=10, opts=aopts, return_iters=True)
    t_adj = time.perf_counter() - t0
    return {"meshes": count, "rows": tr.n, "nnz": tr.nnz, "steps": tb.steps, "run_s": t_run, "step_ms": t_run / tb.steps * 1e3,
            "iters_per_step": float(np.mean(its)), "adjoint_dJdD_s": t_adj, "adjoint_iters_per_solve": float(np.mean(aits)), "J": J, "dJdD": dJdD, "spmv_lanes_f64_f32": list(lanes),
            "mesh_setup_s": t_mesh, "per_mesh_steps_mean": float(np.mean(tr.mesh_steps())),
            "per_mesh_steps_min_max": [int(np.min(tr.mesh_steps())), int(np.max(tr.mesh_steps()))],
            "workload": f"{count} jittered cubes, N_i log-uniform in [2000, 50000], D=1e-3, u=(sin pi y, sin pi z, sin pi x), dt=1e-2; "
                        "GMRES(30) + natural-order ILU(0) with 3 Jacobi sweeps, mixed, to 1e-10 relres per mesh and step; host arrays in/out"}


# DRAM bytes (read + write) of one k_spmv<double> launch on the 10^6-vertex heat matrix with 4
# lanes per row, from one ncu capture of that launch (profiles/k_spmv_1M.md); reported as the
# roofline's traffic only when the bench runs that same matrix and lane count.
SPMV_TRAFFIC_N100_4LANES = 209.2e6
# DRAM bytes (read + write) of one k_ilu0_sweep<float, half values> launch on the same matrix (4-sweep
# natural-order factors, 32-bit columns), from one ncu capture of a lower and an upper sweep
# (profiles/k_ilu0_sweep_1M.md)
SWEEP_TRAFFIC_N100 = 66.1e6


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


ILU_SWEEPS = 4      # Jacobi sweeps per ILU(0) factor in the mixed solver's preconditioner
TOL_RELRES = 1e-12  # stopping rule of every solver in both arms: ||b - A x|| <= TOL_RELRES ||b||
REF_TOL = 1e-14     # the oracle's reference solution


def bench_config(args, world):
    """The workload (identical in both arms)."""
    n = args.n ** 3
    return {"workload": f"steady heat, {args.n}^3 jittered cube ({n} vertices), log k~N(0,1), q~U[0,1]; "
                        f"GMRES({args.restart}) to relres {TOL_RELRES:g} (1e-8 rel. error vs the FP64 reference solution)",
            "n": n, "restart": args.restart, "tol_relres": TOL_RELRES, "l2": "inputs larger than L2 (no flush)",
            "parallelism": "replicas" if world > 1 else "single GPU"}


def oracle_heat_system(prob, dual=None):
    """The workload's linear system as the oracle builds it: push-order triplets of
    SteadyHeat::assemble_matrix from the mesh's Voronoi dual, summed into CSR."""
    import oracle  # checker / CPU baseline only
    d = prob.mesh.dual() if dual is None else dual
    r, c, v, b = oracle.heat_triplets(d, prob.mesh.n_pts, prob.node_bnd, prob.bnd_order, prob.bnd_kind, prob.k, prob.q, prob.s, prob.T0,
                                      prob.bc_val)
    rp, ci, va = oracle.csr_from_triplets(prob.n, r, c, v)
    return rp, ci, va, b


def oracle_reference_solution(rp, ci, va, b, x0, restart):
    """FP64 reference solution on the host (the checker of the error target): the oracle's
    restarted GMRES with a natural-order ILU(0), to relres REF_TOL."""
    import oracle
    t0 = time.perf_counter()
    ilu = oracle.Ilu0(rp, ci, va, np.arange(rp.size - 1, dtype=np.int32))
    x, ok, its, rel = oracle.gmres(rp, ci, va, b, x0, tol=REF_TOL, restart=restart, max_outer=1000, precond=2, ilu=ilu)
    return x, {"kind": f"oracle FP64 GMRES({restart}) + natural-order ILU(0) on the host, from the oracle's own assembly",
               "relres": rel, "converged": bool(ok), "iters": its, "seconds": time.perf_counter() - t0,
               "cross_check": "the same oracle solver agrees with SuperLU (scipy 1.18.1) to 6.7e-12 at 64,000 rows and 1.0e-11 at 125,000 rows"}


def cpu_jacobi_solve(rp, ci, va, b, x0, restart):
    """The reference's algorithm (Jacobi-preconditioned restarted GMRES, FP64; OpenMP over all host
    cores) solved to TOL_RELRES and timed directly."""
    import oracle
    t0 = time.perf_counter()
    _, ok, its, rel = oracle.gmres(rp, ci, va, b, x0, tol=TOL_RELRES, restart=restart, max_outer=10**6, precond=1)
    return time.perf_counter() - t0, its, rel, ok


def main():
    args = parse()
    from vfvchem_vfvm3d_b200 import replicas
    R = replicas.init_from_env()
    rank, world, local = R.rank, R.world, R.local
    if args.impl == "reference":
        return run_reference(args, R)
    import torch

    from vfvchem_vfvm3d_b200 import Context, GmresOptions, SteadyHeatGpu
    from vfvchem_vfvm3d_b200 import _lib as L
    from vfvchem_vfvm3d_b200.problems import steady_heat

    torch.cuda.set_device(local)
    ctx = Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr)
    t_setup = time.perf_counter()
    prob = steady_heat(args.n, hetero=True)
    t_mesh = time.perf_counter() - t_setup
    heat = SteadyHeatGpu(prob.mesh, prob.bnd_kind, ctx=ctx)
    dev = torch.device("cuda", local)
    k_d, q_d, s_d, T_d, bc_d = (torch.tensor(a, device=dev) for a in (prob.k, prob.q, prob.s, prob.T0, prob.bc_val))
    torch.cuda.synchronize()
    heat.assemble_device(k_d.data_ptr(), q_d.data_ptr(), s_d.data_ptr(), T_d.data_ptr(), bc_d.data_ptr())
    ctx.synchronize()
    pat = heat.pattern
    pat.autotune()  # SpMV shape (lanes per row, strides per lane), measured before the solvers capture their graphs
    (lanes64, strides64), (lanes32, strides32) = pat.spmv_shape()
    n, nnz = pat.n, pat.nnz
    b_d = torch.tensor(heat.assemble(prob.k, prob.q, prob.s, prob.T0, prob.bc_val), device=dev)
    x_d = torch.empty_like(b_d)
    x0_d = T_d.clone()

    # the checker: the oracle's own assembly of the system and its FP64 reference solution (host)
    x_ref, ref_info, orc = None, None, None
    if rank == 0 and world == 1:
        rp_o, ci_o, va_o, b_o = oracle_heat_system(prob)
        x_ref, ref_info = oracle_reference_solution(rp_o, ci_o, va_o, b_o, prob.T0, args.restart)
        orc = (rp_o, ci_o, va_o, b_o)
        rp_g, ci_g, va_g = pat.export()
        ref_info["gpu_assembly_vs_oracle"] = {
            "pattern_equal": bool(np.array_equal(rp_g.astype(np.int64), rp_o) and np.array_equal(ci_g, ci_o)),
            "values_max_rel": float(np.max(np.abs(va_g - va_o)) / np.max(np.abs(va_o))),
            "b_max_rel": float(np.max(np.abs(b_d.cpu().numpy() - b_o)) / np.max(np.abs(b_o)))}
    x_ref_d = torch.tensor(x_ref, device=dev) if x_ref is not None else None

    def err(x):
        if x_ref_d is None:
            return None
        return float(torch.linalg.vector_norm(x - x_ref_d) / torch.linalg.vector_norm(x_ref_d))

    exact = dict(precond=L.PRECOND_ILU0, ilu_order=L.ILU_MULTICOLOR, engine=args.engine)
    swept = dict(precond=L.PRECOND_ILU0, ilu_order=L.ILU_NATURAL, ilu_sweeps=ILU_SWEEPS, engine=args.engine)
    o64 = GmresOptions(tol=TOL_RELRES, restart=args.restart, max_outer=2000, precision=L.FP64, **exact)
    omx = GmresOptions(tol=TOL_RELRES, restart=args.restart, max_outer=2000, precision=L.MIXED, inner_rtol=1e-6, ilu_sweep_half=1,
                       **swept)
    o64s = GmresOptions(tol=TOL_RELRES, restart=args.restart, max_outer=2000, precision=L.FP64, **swept)
    omxe = GmresOptions(tol=TOL_RELRES, restart=args.restart, max_outer=2000, precision=L.MIXED, inner_rtol=1e-6, **exact)
    # the same solvers with one-pass classical Gram-Schmidt (no reorthogonalisation)
    omx1 = GmresOptions(tol=TOL_RELRES, restart=args.restart, max_outer=2000, precision=L.MIXED, inner_rtol=1e-6, ortho=L.ORTHO_CGS,
                        ilu_sweep_half=1, **swept)
    o641 = GmresOptions(tol=TOL_RELRES, restart=args.restart, max_outer=2000, precision=L.FP64, ortho=L.ORTHO_CGS, **exact)
    o64s1 = GmresOptions(tol=TOL_RELRES, restart=args.restart, max_outer=2000, precision=L.FP64, ortho=L.ORTHO_CGS, **swept)

    def timed(opts, steps, warm):
        for _ in range(warm):
            pat.solve_device(b_d.data_ptr(), x0_d.data_ptr(), x_d.data_ptr(), opts)
        ts, infos = [], []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            infos.append(pat.solve_device(b_d.data_ptr(), x0_d.data_ptr(), x_d.data_ptr(), opts))
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        return ts, infos, err(x_d)

    replicas.barrier(R)
    torch.cuda.synchronize()
    launches0 = ctx.launch_count
    with ClockSampler(local) as clk:
        t_mx, i_mx, e_mx = timed(omx, args.steps, args.warmup)
        launches_mx = (ctx.launch_count - launches0) // (args.steps + args.warmup) * args.steps
        t_64, i_64, e_64 = timed(o64, args.steps, args.warmup)
        t_64s, i_64s, e_64s = timed(o64s, args.steps, args.warmup)
        t_mxe, i_mxe, e_mxe = timed(omxe, args.steps, args.warmup)
        t_mx1, i_mx1, e_mx1 = timed(omx1, args.steps, args.warmup)
        t_641, i_641, e_641 = timed(o641, args.steps, args.warmup)
        t_64s1, i_64s1, e_64s1 = timed(o64s1, args.steps, args.warmup)
    torch.cuda.synchronize()
    mx_s = sum(t_mx) / len(t_mx)
    f64_s = sum(t_64) / len(t_64)
    f64s_s = sum(t_64s) / len(t_64s)
    mxe_s = sum(t_mxe) / len(t_mxe)
    replicas.barrier(R)
    mx1_s, f641_s, f64s1_s = (sum(t) / len(t) for t in (t_mx1, t_641, t_64s1))
    mx_s, f64_s, f64s_s, mxe_s, mx1_s, f641_s, f64s1_s = replicas.max_over_ranks(R, [mx_s, f64_s, f64s_s, mxe_s, mx1_s, f641_s, f64s1_s])

    # SpMV (FP64 and FP32) timed alone: the kernel the metric names
    xs = torch.randn(n, dtype=torch.float64, device=dev)
    ys = torch.empty_like(xs)
    xs32, ys32 = xs.float(), torch.empty(n, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()

    def kernel_time(fn, reps=50):
        for _ in range(5):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    sp64 = kernel_time(lambda: pat.spmv_device(xs.data_ptr(), ys.data_ptr()))
    sp32 = kernel_time(lambda: pat.spmv_device_f32(xs32.data_ptr(), ys32.data_ptr()))
    bytes64 = 12 * nnz + 4 * (n + 1) + 8 * n + 8 * n
    bytes32 = 8 * nnz + 4 * (n + 1) + 4 * n + 4 * n
    peak, peak_kind = peaks()
    gbs64 = bytes64 / sp64 / 1e9
    gbs32 = bytes32 / sp32 / 1e9

    # The mixed solve's preconditioner timed alone: ILU_SWEEPS Jacobi sweeps of each factor in float
    # arithmetic over the row-scaled half-precision values (natural-order ILU(0) in A's numbering;
    # 2 x ILU_SWEEPS k_ilu0_sweep launches per apply). Algorithmic bytes per sweep: the triangle's
    # row pointer (4 (n+1)) and row scales (4 n), column indices (2 or 4 bytes) and half values (2)
    # of its entries (nl = nu = (nnz - n) / 2 strictly lower / upper entries), right-hand side,
    # previous iterate and new iterate (12 n), the diagonal for the upper sweeps (4 n); the last
    # lower sweep also writes D^-1 u (4 n) and reads the diagonal (4 n).
    rs32, ts32, zs32 = xs32.clone(), torch.empty_like(xs32), torch.empty_like(xs32)
    torch.cuda.synchronize()
    pat.ilu0_sweep_apply_device(rs32.data_ptr(), zs32.data_ptr(), ILU_SWEEPS, L.ILU_NATURAL, half=True)
    ilu_s = kernel_time(lambda: pat.ilu0_sweep_apply_device(rs32.data_ptr(), zs32.data_ptr(), ILU_SWEEPS, L.ILU_NATURAL, half=True))
    col_bytes = pat.ilu0_sweep_layout(L.ILU_NATURAL)
    ilu_launches = 2 * ILU_SWEEPS
    ntri = (nnz - n) // 2
    bytes_ilu32 = ILU_SWEEPS * (2 * 4 * (n + 1) + (col_bytes + 2) * 2 * ntri + 36 * n) + 8 * n
    gbs_ilu32 = bytes_ilu32 / ilu_s / 1e9
    # the exact level-scheduled float apply (the FP64 baseline's preconditioner structure), for context
    ilu_nlev = pat.ilu0_apply_device_f32(rs32.data_ptr(), ts32.data_ptr(), zs32.data_ptr())
    lev_s = kernel_time(lambda: pat.ilu0_apply_device_f32(rs32.data_ptr(), ts32.data_ptr(), zs32.data_ptr()))

    # assembly (gradients + face coefficients + b), timed alone
    def asm():
        heat.assemble_device(k_d.data_ptr(), q_d.data_ptr(), s_d.data_ptr(), T_d.data_ptr(), bc_d.data_ptr())
    asm_s = kernel_time(asm, reps=10)
    # Algorithmic bytes of one assembly (k_grad_lsq<4> over k, q, T, s + k_assemble_heat): per
    # directed face the neighbour index and 3 LSQ weights (gradients) and the neighbour index, 3 skew
    # components, area and distance (coefficients), 72 bytes; per row 132 bytes for the gradients
    # (row pointer, 4 fields in, 12 components out) and 184 for the rest (kind, row and face
    # pointers, diagonal slot, k, q, s, boundary value, 3 x 4 gradient components, skew centroid
    # offset, volume, b out); 8 bytes per value written. Gathers of neighbours' fields hit L2.
    n_dir = int(prob.mesh.n_dir)
    bytes_asm = 72 * n_dir + 316 * n + 8 * nnz
    gbs_asm = bytes_asm / asm_s / 1e9

    # end to end through the C ABI with host buffers: values + b + x0 in, x out, every step
    rp_h, ci_h, va_h = pat.export()
    b_h = b_d.cpu().numpy()
    x0_h = prob.T0.copy()
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
    va_p, b_p, x0_p = pin(va_h), pin(b_h), pin(x0_h)
    x_p = pin(np.empty_like(b_h))
    e2e = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        pat.set_values(va_p)
        x_h, inf = pat.solve(b_p, x0_p, omx, out=x_p)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e.append(dt)
    e2e_s = sum(e2e) / len(e2e)
    e2e_err = float(np.linalg.norm(x_h - x_ref) / np.linalg.norm(x_ref)) if x_ref is not None else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rp_o, ci_o, va_o, b_o = orc
        dt, its, rel, ok = cpu_jacobi_solve(rp_o, ci_o, va_o, b_o, prob.T0, args.restart)
        cpu = {"value": dt, "unit": "s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"one converged solve timed directly: Jacobi GMRES({args.restart}) FP64 (the reference's LinearGmres "
                         f"algorithm, oracle port, OpenMP) on the oracle-assembled system, {its} Arnoldi steps to relres {rel:.2e}"
                         + ("" if ok else " (not converged)")}

    extras = None
    if not args.no_extras and world == 1:
        extras = {"steady_adjoint": extras_adjoint(heat, prob, x_ref if x_ref is not None else x_d.cpu().numpy(), ctx),
                  "batched_transport": extras_transport(ctx, args.batch),
                  "cavity_flow": extras_flow(ctx, args.flow_n)}

    clocks = clk.summary()
    out = {
        "metric": METRIC,
        "value": mx_s,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": mx_s * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32-inner/f64-refine",
        "data": "synthetic (seeded jittered-cube Delaunay mesh, seeded fields)",
        "config": bench_config(args, world),
        "fp64_solve_s": f64_s,
        "speedup_mixed_vs_fp64": f64_s / mx_s,
        "solvers": {
            "mixed": f"FP32 GMRES({args.restart}) cycles in FP64 refinement, ILU(0) natural order, {ILU_SWEEPS} Jacobi sweeps per factor "
                     "over row-scaled half-precision factor values",
            "fp64": f"FP64 GMRES({args.restart}), exact multicolour ILU(0) ({ilu_nlev} colour levels, level-scheduled sweeps)",
            "fp64_same_precond": "FP64 GMRES with the mixed solver's preconditioner",
            "mixed_exact_ilu": "the mixed solver with the FP64 solver's exact multicolour ILU(0)"},
        "fp64_same_precond_s": f64s_s, "speedup_mixed_vs_fp64_same_precond": f64s_s / mx_s,
        "mixed_exact_ilu_s": mxe_s,
        "gram_schmidt_one_pass": {
            "note": "the same three solvers with one-pass classical Gram-Schmidt (VFV_ORTHO_CGS) instead of two passes",
            "mixed_s": mx1_s, "fp64_s": f641_s, "fp64_same_precond_s": f64s1_s,
            "speedup_mixed_vs_fp64": f641_s / mx1_s, "speedup_mixed_vs_fp64_same_precond": f64s1_s / mx1_s,
            "iters_mixed": i_mx1[-1].iters, "iters_fp64": i_641[-1].iters, "err_mixed": e_mx1, "err_fp64": e_641},
        "iters_mixed": i_mx[-1].iters, "iters_fp64": i_64[-1].iters, "iters_fp64_same_precond": i_64s[-1].iters,
        "iters_mixed_exact_ilu": i_mxe[-1].iters, "ilu_levels": ilu_nlev,
        "err_mixed": e_mx, "err_fp64": e_64, "err_fp64_same_precond": e_64s, "err_mixed_exact_ilu": e_mxe, "err_target": ERR_TARGET,
        "nnz": nnz, "engine": args.engine,
        "roofline": {"bound": "hbm", "kernel": f"k_ilu0_sweep<float, half values> (Jacobi sweeps of the ILU(0) factors, {ilu_launches} "
                                                f"launches per apply, {col_bytes}-byte columns)",
                     "achieved": gbs_ilu32, "peak": peak, "unit": "GB/s", "frac": gbs_ilu32 / peak, "peak_kind": peak_kind,
                     "traffic": SWEEP_TRAFFIC_N100 if args.n == 100 else None,
                     "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
                     "algorithmic_bytes_per_launch": bytes_ilu32 / ilu_launches, "apply_us": ilu_s * 1e6,
                     "exact_level_apply_us": lev_s * 1e6},
        "roofline_spmv": {"bound": "hbm", "kernel": f"k_spmv<double> (CSR, {lanes64} lanes/row, {strides64} strides/lane)", "achieved": gbs64, "peak": peak, "unit": "GB/s",
                          "frac": gbs64 / peak, "peak_kind": peak_kind,
                          "traffic": SPMV_TRAFFIC_N100_4LANES if (args.n == 100 and (lanes64, strides64) == (4, 4)) else None,
                          "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
                          "algorithmic_bytes_per_launch": bytes64},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 8 * nnz + 16 * n, "d2h_bytes_per_step": 8 * n, "err": e2e_err},
        "gpu_launches": int(launches_mx),
        "clocks": clocks,
        "ref_solution": ref_info,
        "spmv_fp64_gbs": gbs64, "spmv_fp32_gbs": gbs32, "spmv_shape_f32": [lanes32, strides32], "spmv_fp64_ms": sp64 * 1e3, "spmv_fp32_ms": sp32 * 1e3,
        "assembly_ms": asm_s * 1e3, "mesh_setup_s": t_mesh,
        "roofline_assembly": {"bound": "hbm", "kernel": "k_grad_lsq<4> (thread per row) + k_assemble_heat (4 lanes per row)",
                              "achieved": gbs_asm, "peak": peak, "unit": "GB/s", "frac": gbs_asm / peak, "peak_kind": peak_kind,
                              "algorithmic_bytes": bytes_asm, "ms": asm_s * 1e3},
        "extras": extras,
    }
    if rank == 0:
        print(json.dumps(out))
    replicas.finalize(R)


def reference_heat_system(n):
    """The workload's system for the reference arm, built by the oracle alone: its jittered-cube
    vertex set, its Bowyer-Watson Delaunay (delaunay.rs restated), its Voronoi dual (geom_tet.rs
    restated) and its push-order assembly (steady_heat.rs); no product code runs in this process."""
    import oracle
    from oracle import mesh as om
    from vfvchem_vfvm3d_b200.problems import HEAT_BND_KIND, HEAT_BND_ORDER, heat_fields
    pos, node_bnd, n_pts = om.jitter_cube(n, 42, 0.25)
    d = om.dual(pos, om.delaunay(pos), n_pts)
    k, q, s, T0, bc = heat_fields(node_bnd, hetero=True)
    r, c, v, b = oracle.heat_triplets(d, n_pts, node_bnd, HEAT_BND_ORDER, HEAT_BND_KIND, k, q, s, T0, bc)
    rp, ci, va = oracle.csr_from_triplets(node_bnd.size, r, c, v)
    return rp, ci, va, b, T0, "oracle mesh (jittered cube, Delaunay, dual) + oracle assembly"


def run_reference(args, R):
    """Reference arm: the reference's LinearGmres algorithm (Jacobi-preconditioned restarted
    GMRES(50), FP64) on the host cores, the oracle port, on the same system and stopping rule.
    Each step is a bounded sample (one restart cycle of 50 Arnoldi steps from the warm start);
    `value` is one converged solve to TOL_RELRES timed directly afterwards. Rank 0 alone runs it."""
    from vfvchem_vfvm3d_b200 import replicas
    world = R.world
    if R.rank != 0:
        replicas.finalize(R)
        return
    import oracle  # the reference arm runs the CPU port of the reference's algorithm
    t0 = time.perf_counter()
    rp, ci, va, b, x0, source = reference_heat_system(args.n)
    t_build = time.perf_counter() - t0
    per = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.gmres(rp, ci, va, b, x0, tol=TOL_RELRES, restart=args.restart, max_outer=1, precond=1, max_steps=args.restart)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            per.append(dt)
    dt_solve, its, rel, ok = cpu_jacobi_solve(rp, ci, va, b, x0, args.restart)
    out = {
        "impl": "reference", "metric": METRIC, "value": dt_solve, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sum(per) / len(per) * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered-cube Delaunay mesh, seeded fields)",
        "config": bench_config(args, world),
        "cpu_baseline": {"value": dt_solve, "unit": "s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"steps: one restart cycle ({args.restart} Arnoldi steps) each; value: one converged solve timed "
                                   f"directly, {its} Arnoldi steps to relres {rel:.2e}" + ("" if ok else " (not converged)")},
        "e2e": {"value": dt_solve, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "iters": its, "relres": rel, "nnz": int(ci.size), "system_source": source, "system_build_s": t_build,
    }
    print(json.dumps(out))
    replicas.finalize(R)


if __name__ == "__main__":
    main()
