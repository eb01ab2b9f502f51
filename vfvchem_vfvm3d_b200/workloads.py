"""Standard workloads of this package, runnable from the command line (for timing and profiling).

    python -m vfvchem_vfvm3d_b200.workloads heat --n 100 --solves 1 --precision mixed --engine 2 --sweeps 4 --half
    python -m vfvchem_vfvm3d_b200.workloads flow --n 32 --picard 2 --precision mixed
    python -m vfvchem_vfvm3d_b200.workloads transport --count 16 --steps 5
    python -m vfvchem_vfvm3d_b200.workloads spmv --n 100 --reps 3 --lanes 4,4

heat: the heterogeneous steady heat system (n^3 jittered cube, log k ~ N(0,1), q ~ U[0,1]) solved
by GMRES(50) + ILU(0) to relres 1e-10 (exact multicolour ILU(0), or --sweeps Jacobi sweeps of the
natural-order factors; --solves 0 assembles only); flow: the lid-driven cavity's damped Picard loop with
GMRES(100) + 4x4 block-Jacobi; transport: the batched transient transport (meshes of 2,000-50,000
vertices); spmv: the heat matrix's SpMV, FP64 then FP32 (lanes per row autotuned unless --lanes gives them;
with --lanes the only k_spmv launches are the timed ones). Each prints one summary line.
"""
from __future__ import annotations

import argparse
import time

import numpy as np


def _ctx():
    from . import Context
    return Context(0)


def heat(args):
    from . import GmresOptions, SteadyHeatGpu
    from . import _lib as L
    from .problems import steady_heat
    ctx = _ctx()
    prob = steady_heat(args.n, hetero=True)
    h = SteadyHeatGpu(prob.mesh, prob.bnd_kind, ctx=ctx)
    b = h.assemble(prob.k, prob.q, prob.s, prob.T0, prob.bc_val)
    h.pattern.autotune()
    opts = GmresOptions(tol=1e-10, restart=50, max_outer=2000, precond=L.PRECOND_ILU0,
                        precision=L.MIXED if args.precision == "mixed" else L.FP64, inner_rtol=1e-6, engine=args.engine,
                        ilu_order=L.ILU_NATURAL if args.sweeps > 0 else L.ILU_MULTICOLOR, ilu_sweeps=args.sweeps,
                        ilu_sweep_half=1 if args.half else 0)
    if args.solves == 0:
        print(f"heat n={prob.n} nnz={h.pattern.nnz}: assembled")
    for _ in range(args.solves):
        t0 = time.perf_counter()
        x, info = h.pattern.solve(b, prob.T0, opts)
        print(f"heat n={prob.n} nnz={h.pattern.nnz} {args.precision} engine={args.engine} sweeps={args.sweeps}: {info.iters} iterations, "
              f"relres {info.relres:.2e}, {time.perf_counter() - t0:.3f} s (host clock)")


def flow(args):
    from . import SteadyFlowGpu
    from . import _lib as L
    from .flow import flow_options
    from .problems import lid_cavity
    ctx = _ctx()
    fl = SteadyFlowGpu(lid_cavity(args.n), ctx=ctx)
    r = fl.picard(max_iter=args.picard, tol=1e-300, damp=0.8,
                  opts=flow_options(L.MIXED if args.precision == "mixed" else L.FP64, tol=1e-8, max_outer=100), raise_on_error=False)
    print(f"flow n={args.n} unknowns={fl.n_unknowns} nnz={fl.nnz}: {r.iterations} Picard iterations, GMRES {list(map(int, r.lin_iters))}, "
          f"solves {r.solve_seconds:.3f} s")


def transport(args):
    from . import TransientTransportGpu
    from .problems import transport_batch, transport_fields
    ctx = _ctx()
    tb = transport_batch(args.count)
    vel, c0 = transport_fields(tb.meshes)
    tr = TransientTransportGpu(tb.meshes, tb.dt, ctx=ctx)
    tr.assemble(tb.D, vel)
    tr.pattern.autotune()
    t0 = time.perf_counter()
    _, its = tr.run(c0, args.steps)
    print(f"transport {args.count} meshes, {tr.n} rows: {args.steps} steps, {float(np.mean(its)):.2f} iterations per step, "
          f"{time.perf_counter() - t0:.3f} s")


def spmv(args):
    import torch
    from . import SteadyHeatGpu
    from .problems import steady_heat
    ctx = _ctx()
    prob = steady_heat(args.n, hetero=True)
    h = SteadyHeatGpu(prob.mesh, prob.bnd_kind, ctx=ctx)
    h.assemble(prob.k, prob.q, prob.s, prob.T0, prob.bc_val)
    p = h.pattern
    if args.lanes:
        lanes = tuple(int(v) for v in args.lanes.split(","))
        p.set_spmv_lanes(*lanes)
    else:
        lanes = p.autotune()
    x = torch.randn(p.n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    x32, y32 = x.float(), torch.empty(p.n, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    for _ in range(args.reps):
        p.spmv_device(x.data_ptr(), y.data_ptr())
    for _ in range(args.reps):
        p.spmv_device_f32(x32.data_ptr(), y32.data_ptr())
    ctx.synchronize()
    print(f"spmv n={p.n} nnz={p.nnz} lanes={lanes}: {args.reps} FP64 then {args.reps} FP32 launches")


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m vfvchem_vfvm3d_b200.workloads")
    sub = ap.add_subparsers(dest="case", required=True)
    a = sub.add_parser("heat")
    a.add_argument("--n", type=int, default=100)
    a.add_argument("--solves", type=int, default=1)
    a.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    a.add_argument("--engine", type=int, default=2)
    a.add_argument("--sweeps", type=int, default=0,
                   help="ILU(0) applied by this many Jacobi sweeps per factor in the natural order (0: exact multicolour ILU(0))")
    a.add_argument("--half", action="store_true", help="mixed + sweeps: the swept factors' values in row-scaled half precision")
    a = sub.add_parser("flow")
    a.add_argument("--n", type=int, default=32)
    a.add_argument("--picard", type=int, default=2)
    a.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    a = sub.add_parser("transport")
    a.add_argument("--count", type=int, default=16)
    a.add_argument("--steps", type=int, default=5)
    a = sub.add_parser("spmv")
    a.add_argument("--n", type=int, default=100)
    a.add_argument("--reps", type=int, default=3)
    a.add_argument("--lanes", default="", help="lanes per row 'f64,f32' instead of the autotuner (e.g. 4,4)")
    args = ap.parse_args(argv)
    {"heat": heat, "flow": flow, "transport": transport, "spmv": spmv}[args.case](args)


if __name__ == "__main__":
    main()
