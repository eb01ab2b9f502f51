"""Benchmark of the assemble-and-solve path on one B200 (or N replicas).

Workload (one "step"): the 1,000,000-vertex heterogeneous steady heat system (100^3 jittered
cube, log k ~ N(0,1), q ~ U[0,1], Dirichlet T=0/1 on x=0/1, zero flux elsewhere) solved by
GMRES(50) + ILU(0) to 1e-8 relative 2-norm error against a reference solution — the
FP32-inner / FP64-refinement solver is the timed `value`; the plain FP64 solver is timed beside
it. Inputs are resident in HBM; the matrix (16.1 M non-zeros, 193 MB of FP64 values and
columns) exceeds the 126 MB L2, so no L2 flush is needed between steps.

`roofline` is the float ILU(0) level sweeps, the largest share of the mixed solve's kernel time,
timed alone with CUDA events on the library's stream; `roofline_spmv` is the FP64 SpMV timed the
same way.

`--impl reference` times the reference's own algorithm for this path on the host cores
(Jacobi-preconditioned restarted GMRES(50), FP64, the oracle port), on a bounded sample.
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
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="bounded CPU baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--engine", type=int, default=2,
                    help="0 persistent cycle kernel, 1 CUDA graph of per-phase kernels, 2 graph with the ILU(0) sweeps overlapped (flexible GMRES)")
    ap.add_argument("--no-extras", action="store_true", help="skip the adjoint and batched-transport timings")
    ap.add_argument("--batch", type=int, default=256, help="meshes in the batched transport timing")
    ap.add_argument("--flow-n", type=int, default=64, help="grid points per axis of the cavity flow timing")
    return ap.parse_args()


def extras_adjoint(heat, prob, x_ref_h, ctx):
    """Steady adjoint: J = 0.5 sum (T_i - d_i)^2 over 1000 seeded sensors, gradient w.r.t. every
    log k and q (one transposed solve + gathers), timed through the host-array API."""
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
    return {"adjoint_s": min(ts), "adjoint_iters": info.iters, "sensors": 1000, "grad_norm_logk": float(np.linalg.norm(dk)),
            "grad_norm_q": float(np.linalg.norm(dq)), "workload": "dJ/dlog k and dJ/dq on the same 1M-vertex system, host arrays in/out"}


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
    tb = transport_batch(count)
    vel, c0 = transport_fields(tb.meshes)
    t_mesh = time.perf_counter() - t0
    tr = TransientTransportGpu(tb.meshes, tb.dt, ctx=ctx)
    tr.assemble(tb.D, vel)
    lanes = tr.pattern.autotune()
    opts = GmresOptions(tol=1e-10, restart=30, max_outer=200, precond=L.PRECOND_ILU0, precision=L.MIXED, inner_rtol=1e-6)
    tr.run(c0, 3, opts)
    t0 = time.perf_counter()
    c, its = tr.run(c0, tb.steps, opts)
    t_run = time.perf_counter() - t0
    target = np.full(tr.n, float(np.mean(c0)))
    aopts = GmresOptions(tol=1e-10, restart=30, max_outer=500, precond=L.PRECOND_ILU0, precision=L.MIXED, inner_rtol=1e-6)
    t0 = time.perf_counter()
    J, dJdD, aits = tr.adjoint_D(c0, tb.steps, target, every=10, opts=aopts, return_iters=True)
    t_adj = time.perf_counter() - t0
    return {"meshes": count, "rows": tr.n, "nnz": tr.nnz, "steps": tb.steps, "run_s": t_run, "step_ms": t_run / tb.steps * 1e3,
            "iters_per_step": float(np.mean(its)), "adjoint_dJdD_s": t_adj, "adjoint_iters_per_solve": float(np.mean(aits)), "J": J, "dJdD": dJdD, "spmv_lanes_f64_f32": list(lanes),
            "mesh_setup_s": t_mesh,
            "workload": f"{count} jittered cubes, N_i log-uniform in [2000, 50000], D=1e-3, u=(sin pi y, sin pi z, sin pi x), dt=1e-2; "
                        "GMRES(30)+ILU(0) mixed to 1e-10 relres per mesh and step; host arrays in/out"}


# DRAM bytes (read + write) of one k_spmv<double> launch on the 10^6-vertex heat matrix with 4
# lanes per row, from one ncu capture of that launch (profiles/k_spmv_1M.md); reported as the
# roofline's traffic only when the bench runs that same matrix and lane count.
SPMV_TRAFFIC_N100_4LANES = 209.2e6


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


def cpu_baseline_jacobi(rp, ci, va, b, x0, restart, budget_s, steps_needed=None):
    """Reference algorithm on the host cores: Jacobi GMRES(restart), FP64 (oracle port, OpenMP)."""
    import oracle  # CPU-baseline leg only
    lib = oracle.lib()
    t0 = time.perf_counter()
    steps = restart
    _, _, its, _ = oracle.gmres(rp, ci, va, b, x0, tol=1e-300, restart=restart, max_outer=1, precond=1, max_steps=steps)
    dt = time.perf_counter() - t0
    # grow the sample to roughly the time budget
    if dt < budget_s / 3:
        steps = max(restart, int(restart * (budget_s / 2) / max(dt, 1e-3)) // restart * restart)
        t0 = time.perf_counter()
        _, _, its, _ = oracle.gmres(rp, ci, va, b, x0, tol=1e-300, restart=restart, max_outer=10**6, precond=1, max_steps=steps)
        dt = time.perf_counter() - t0
    del lib
    return dt / max(its, 1), its


def main():
    args = parse()
    from vfvchem_vfvm3d_b200 import replicas
    R = replicas.init_from_env()
    rank, world, local = R.rank, R.world, R.local
    import torch

    if args.impl == "reference":
        return run_reference(args, R)

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
    lanes64, lanes32 = pat.autotune()  # SpMV lanes per row, measured before the solvers capture their graphs
    n, nnz = pat.n, pat.nnz
    b_d = torch.tensor(heat.assemble(prob.k, prob.q, prob.s, prob.T0, prob.bc_val), device=dev)
    x_d = torch.empty_like(b_d)
    x0_d = T_d.clone()

    ilu = dict(precond=L.PRECOND_ILU0, ilu_order=L.ILU_MULTICOLOR, engine=args.engine)
    # reference solution: FP64 GMRES driven to round-off
    ref_opts = GmresOptions(tol=1e-14, restart=args.restart, max_outer=4000, **ilu)
    try:
        info_ref = pat.solve_device(b_d.data_ptr(), x0_d.data_ptr(), x_d.data_ptr(), ref_opts)
    except Exception:
        ref_opts.tol = 1e-13
        info_ref = pat.solve_device(b_d.data_ptr(), x0_d.data_ptr(), x_d.data_ptr(), ref_opts)
    x_ref = x_d.clone()

    def err(x):
        return float(torch.linalg.vector_norm(x - x_ref) / torch.linalg.vector_norm(x_ref))

    # residual tolerance giving <= 1e-8 error for the FP64 solver, shared by both solvers
    tol = 1e-9
    for _ in range(5):
        pat.solve_device(b_d.data_ptr(), x0_d.data_ptr(), x_d.data_ptr(), GmresOptions(tol=tol, restart=args.restart, max_outer=2000, **ilu))
        if err(x_d) <= 0.5 * ERR_TARGET:
            break
        tol /= 4
    o64 = GmresOptions(tol=tol, restart=args.restart, max_outer=2000, precision=L.FP64, **ilu)
    omx = GmresOptions(tol=tol, restart=args.restart, max_outer=2000, precision=L.MIXED, inner_rtol=1e-6, **ilu)

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
        launches_mx = ctx.launch_count - launches0
        t_64, i_64, e_64 = timed(o64, args.steps, args.warmup)
    torch.cuda.synchronize()
    mx_s = sum(t_mx) / len(t_mx)
    f64_s = sum(t_64) / len(t_64)
    replicas.barrier(R)
    mx_s, f64_s = replicas.max_over_ranks(R, [mx_s, f64_s])

    # SpMV (FP64 and FP32) timed alone: the kernel the metric names
    xs = torch.randn(n, dtype=torch.float64, device=dev)
    ys = torch.empty_like(xs)
    xs32, ys32 = xs.float(), torch.empty(n, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()

    def spmv_time(fn, reps=50):
        for _ in range(5):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    sp64 = spmv_time(lambda: pat.spmv_device(xs.data_ptr(), ys.data_ptr()))
    sp32 = spmv_time(lambda: pat.spmv_device_f32(xs32.data_ptr(), ys32.data_ptr()))
    bytes64 = 12 * nnz + 4 * (n + 1) + 8 * n + 8 * n
    bytes32 = 8 * nnz + 4 * (n + 1) + 4 * n + 4 * n
    peak, peak_kind = peaks()
    gbs64 = bytes64 / sp64 / 1e9
    gbs32 = bytes32 / sp32 / 1e9

    # ILU(0) sweeps with the float factor, timed alone: the mixed solve's preconditioner, whose
    # 2 x levels launches per apply are the largest share of the solve's kernel time. Algorithmic
    # bytes per apply: L+U values and columns (8 nnz), row pointer, diagonal position and
    # permutation per sweep (2 x 12 n), r in and z out (8 n); the intermediate t stays in L2.
    rs32, ts32, zs32 = xs32.clone(), torch.empty_like(xs32), torch.empty_like(xs32)
    torch.cuda.synchronize()
    ilu_nlev = pat.ilu0_apply_device_f32(rs32.data_ptr(), ts32.data_ptr(), zs32.data_ptr())
    ilu_s = spmv_time(lambda: pat.ilu0_apply_device_f32(rs32.data_ptr(), ts32.data_ptr(), zs32.data_ptr()), reps=20)
    bytes_ilu32 = 8 * nnz + 28 * n
    gbs_ilu32 = bytes_ilu32 / ilu_s / 1e9

    # assembly (gradients + face coefficients + b), timed alone
    def asm():
        heat.assemble_device(k_d.data_ptr(), q_d.data_ptr(), s_d.data_ptr(), T_d.data_ptr(), bc_d.data_ptr())
    asm_s = spmv_time(asm, reps=10)

    # end to end through the C ABI with host buffers: values + b + x0 in, x out, every step
    rp_h, ci_h, va_h = pat.export()
    b_h = b_d.cpu().numpy()
    x0_h = prob.T0.copy()
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
    va_p, b_p, x0_p = pin(va_h), pin(b_h), pin(x0_h)
    e2e = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        pat.set_values(va_p)
        x_h, inf = pat.solve(b_p, x0_p, omx)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e.append(dt)
    e2e_s = sum(e2e) / len(e2e)
    e2e_err = float(np.linalg.norm(x_h - x_ref.cpu().numpy()) / np.linalg.norm(x_ref.cpu().numpy()))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rp64 = rp_h.astype(np.int64)
        per_step, sample_steps = cpu_baseline_jacobi(rp64, ci_h, va_h, b_h, x0_h, args.restart, args.cpu_seconds)
        # steps the reference algorithm needs: Jacobi GMRES on the GPU to the same error
        jac = GmresOptions(tol=tol, restart=args.restart, max_outer=20000, precond=L.PRECOND_JACOBI)
        ij = pat.solve_device(b_d.data_ptr(), x0_d.data_ptr(), x_d.data_ptr(), jac)
        cpu = {"value": per_step * ij.iters, "unit": "s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"{sample_steps} Arnoldi steps of Jacobi GMRES({args.restart}) FP64 on the same system, "
                         f"{per_step * 1e3:.1f} ms/step x {ij.iters} steps (Jacobi GMRES iteration count to the same tolerance)"}

    extras = None
    if not args.no_extras and world == 1:
        extras = {"steady_adjoint": extras_adjoint(heat, prob, x_ref.cpu().numpy(), ctx),
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
        "config": {"workload": f"steady heat, {args.n}^3 jittered cube ({n} vertices, {nnz} nnz), log k~N(0,1), q~U[0,1]; "
                               f"GMRES({args.restart})+ILU(0) multicolour to 1e-8 rel. error",
                   "n": n, "nnz": nnz, "restart": args.restart, "tol_relres": tol, "engine": args.engine, "l2": "inputs larger than L2 (no flush)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "fp64_solve_s": f64_s,
        "speedup_mixed_vs_fp64": f64_s / mx_s,
        "iters_mixed": i_mx[-1].iters, "iters_fp64": i_64[-1].iters, "ilu_levels": i_mx[-1].levels,
        "err_mixed": e_mx, "err_fp64": e_64, "ref_relres": info_ref.relres,
        "spmv_fp64_gbs": gbs64, "spmv_fp32_gbs": gbs32, "spmv_fp64_ms": sp64 * 1e3, "spmv_fp32_ms": sp32 * 1e3,
        "assembly_ms": asm_s * 1e3, "mesh_setup_s": t_mesh,
        "roofline": {"bound": "hbm", "kernel": f"k_ilu0_level<float> ({2 * ilu_nlev} level launches per apply)", "achieved": gbs_ilu32,
                     "peak": peak, "unit": "GB/s", "frac": gbs_ilu32 / peak, "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_apply": bytes_ilu32, "apply_us": ilu_s * 1e6, "launch_us": ilu_s * 1e6 / (2 * ilu_nlev)},
        "roofline_spmv": {"bound": "hbm", "kernel": f"k_spmv<double> (CSR, {lanes64} lanes/row)", "achieved": gbs64, "peak": peak, "unit": "GB/s",
                          "frac": gbs64 / peak, "peak_kind": peak_kind,
                          "traffic": SPMV_TRAFFIC_N100_4LANES if (args.n == 100 and lanes64 == 4) else None,
                          "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
                          "algorithmic_bytes_per_launch": bytes64},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 8 * nnz + 16 * n, "d2h_bytes_per_step": 8 * n, "err": e2e_err},
        "gpu_launches": int(launches_mx),
        "clocks": clocks,
        "extras": extras,
    }
    if rank == 0:
        print(json.dumps(out))
    replicas.finalize(R)


def run_reference(args, R):
    """Reference arm: Jacobi GMRES on the host cores (the reference's LinearGmres algorithm);
    rank 0 alone runs it, the other ranks only join the final barrier."""
    from vfvchem_vfvm3d_b200 import replicas
    world = R.world
    if R.rank != 0:
        replicas.finalize(R)
        return
    import oracle  # the reference arm runs the CPU port of the reference's algorithm
    from vfvchem_vfvm3d_b200.problems import steady_heat
    prob = steady_heat(args.n, hetero=True)
    d = prob.mesh.dual()
    r, c, v, b = oracle.heat_triplets(d, prob.mesh.n_pts, prob.node_bnd, prob.bnd_order, prob.bnd_kind, prob.k, prob.q, prob.s, prob.T0,
                                      prob.bc_val)
    rp, ci, va = oracle.csr_from_triplets(prob.n, r, c, v)
    per = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        _, _, its, _ = oracle.gmres(rp, ci, va, b, prob.T0, tol=1e-300, restart=args.restart, max_outer=1, precond=1,
                                    max_steps=args.restart)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            per.append(dt / max(its, 1))
    per_step = sum(per) / len(per)
    # Jacobi GMRES steps to the target: from the CPU oracle on this system, bounded (extrapolated if capped)
    out = {
        "impl": "reference", "metric": METRIC, "value": None, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": f"steady heat {args.n}^3, Jacobi GMRES({args.restart}) FP64 (reference algorithm)"},
    }
    cap = int(max(args.restart, 60.0 / max(per_step, 1e-4))) // args.restart * args.restart
    x, ok, its, rel = oracle.gmres(rp, ci, va, b, prob.T0, tol=1e-10, restart=args.restart, max_outer=10**6, precond=1, max_steps=cap)
    steps_needed = its if ok else int(its * np.log(1e-10) / np.log(max(rel, 1e-300)))
    val = per_step * steps_needed
    out.update({"value": val, "ms_per_step": val * 1e3,
                "cpu_baseline": {"value": val, "unit": "s", "cores": os.cpu_count(), "kind": "port",
                                 "sample": f"{args.steps} x {args.restart} Arnoldi steps timed ({per_step * 1e3:.1f} ms/step); "
                                           f"{its} steps run to relres {rel:.2e} ({'converged' if ok else 'extrapolated'})"},
                "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(out))
    replicas.finalize(R)


if __name__ == "__main__":
    main()
