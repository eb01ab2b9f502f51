"""Context and sparse-pattern handles over the C ABI."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .errors import raise_for


def _check(ctx_handle, code: int) -> None:
    if code != 0:
        lib = L.load()
        msg = lib.vfv_last_error(ctx_handle)
        raise_for(code, msg.decode() if msg else f"status {code}")


@dataclass
class GmresOptions:
    """Options of ``LinearGmres::new_with_options`` (src/linear/linear_gmres.rs:24) plus the GPU
    additions (preconditioner, precision, ILU ordering). Defaults are the reference's."""

    tol: float = 1e-6
    restart: int = 50
    max_outer: int = 200
    precond: int = L.PRECOND_JACOBI
    precision: int = L.FP64
    ilu_order: int = L.ILU_MULTICOLOR
    inner_rtol: float = 0.0
    engine: int = L.ENGINE_GRAPH
    wait_limit: int = 0  # polls before a bounded device wait gives up (0: the library default)
    ilu_sweeps: int = 0  # ILU(0): 0 exact triangular solves, k > 0 k Jacobi sweeps of each factor
    ilu_sweeps_upper: int = 0  # with ilu_sweeps > 0: sweeps of the upper factor (0: ilu_sweeps)
    ortho: int = L.ORTHO_CGS2  # Gram-Schmidt: two passes, a second pass only when needed (DGKS), or one pass
    ilu_sweep_half: int = 0  # mixed + ilu_sweeps: swept factors stored as row-scaled half-precision values

    def to_c(self) -> L.GmresOpts:
        o = L.GmresOpts()
        o.tol, o.restart, o.max_outer = float(self.tol), int(self.restart), int(self.max_outer)
        o.precond, o.precision, o.ilu_order = int(self.precond), int(self.precision), int(self.ilu_order)
        o.inner_rtol = float(self.inner_rtol)
        o.engine = int(self.engine)
        o.wait_limit = int(self.wait_limit)
        o.ilu_sweeps = int(self.ilu_sweeps)
        o.ilu_sweeps_upper = int(self.ilu_sweeps_upper)
        o.ortho = int(self.ortho)
        o.ilu_sweep_half = int(self.ilu_sweep_half)
        return o


@dataclass
class SolveInfo:
    status: int
    iters: int
    cycles: int
    levels: int
    relres: float
    bnorm: float

    @staticmethod
    def from_c(i: L.SolveInfo) -> "SolveInfo":
        return SolveInfo(i.status, i.iters, i.cycles, i.levels, i.relres, i.bnorm)


class Context:
    """A CUDA device and stream owned by the library (``vfv_ctx``)."""

    def __init__(self, device: int = 0):
        lib = L.load()
        h = C.c_void_p()
        _check(None, lib.vfv_ctx_create(int(device), C.byref(h)))
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    @property
    def stream_ptr(self) -> int:
        return L.load().vfv_ctx_stream(self._h) or 0

    @property
    def launch_count(self) -> int:
        return int(L.load().vfv_ctx_launch_count(self._h))

    def synchronize(self) -> None:
        _check(self._h, L.load().vfv_ctx_synchronize(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            L.load().vfv_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class Pattern:
    """A device CSR matrix: pattern fixed at creation, values refreshed per assembly."""

    def __init__(self, ctx: Context, handle, owned: bool = True):
        self.ctx = ctx
        self._h = handle
        self._owned = owned
        n, nnz, nt = C.c_int64(), C.c_int64(), C.c_int64()
        _check(ctx.handle, L.load().vfv_pattern_info(handle, C.byref(n), C.byref(nnz), C.byref(nt)))
        self.n, self.nnz, self.ntrip = n.value, nnz.value, nt.value

    @classmethod
    def from_triplets(cls, ctx: Context, n: int, rows: np.ndarray, cols: np.ndarray) -> "Pattern":
        rows = np.ascontiguousarray(rows, dtype=np.uint64)
        cols = np.ascontiguousarray(cols, dtype=np.uint64)
        if rows.shape != cols.shape:
            raise ValueError("rows and cols differ in length")
        h = C.c_void_p()
        _check(ctx.handle, L.load().vfv_pattern_from_triplets(ctx.handle, int(n), rows.size, L.ptr(rows, C.c_uint64),
                                                             L.ptr(cols, C.c_uint64), C.byref(h)))
        return cls(ctx, h)

    @classmethod
    def from_csr(cls, ctx: Context, rowptr: np.ndarray, colind: np.ndarray) -> "Pattern":
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        colind = np.ascontiguousarray(colind, dtype=np.int32)
        h = C.c_void_p()
        _check(ctx.handle, L.load().vfv_pattern_from_csr(ctx.handle, rowptr.size - 1, L.ptr(rowptr, C.c_int32),
                                                        L.ptr(colind, C.c_int32), C.byref(h)))
        return cls(ctx, h)

    @property
    def handle(self):
        return self._h

    def values_from_triplets(self, vals: np.ndarray) -> None:
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        if vals.size != self.ntrip:
            raise ValueError(f"expected {self.ntrip} triplet values, got {vals.size}")
        _check(self.ctx.handle, L.load().vfv_values_from_triplets(self.ctx.handle, self._h, L.dptr(vals)))

    def set_values(self, vals: np.ndarray) -> None:
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        if vals.size != self.nnz:
            raise ValueError("wrong number of values")
        _check(self.ctx.handle, L.load().vfv_values_set(self.ctx.handle, self._h, vals.ctypes.data_as(C.c_void_p), 0))

    def set_values_device(self, ptr: int) -> None:
        _check(self.ctx.handle, L.load().vfv_values_set(self.ctx.handle, self._h, C.c_void_p(ptr), 1))

    def export(self):
        rp = np.empty(self.n + 1, np.int32)
        ci = np.empty(self.nnz, np.int32)
        va = np.empty(self.nnz, np.float64)
        _check(self.ctx.handle, L.load().vfv_csr_export(self.ctx.handle, self._h, L.ptr(rp, C.c_int32), L.ptr(ci, C.c_int32),
                                                       L.dptr(va)))
        return rp, ci, va

    def solve(self, b: np.ndarray, x0: np.ndarray | None = None, opts: GmresOptions | None = None, out: np.ndarray | None = None):
        """Host-array solve (``vfv_solve``); returns (x, SolveInfo). ``out``: a contiguous float64
        array of n entries to receive x (e.g. in pinned memory), else a new array."""
        opts = opts or GmresOptions()
        b = np.ascontiguousarray(b, dtype=np.float64)
        x0 = np.zeros(self.n) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64)
        if out is None:
            x = np.empty(self.n)
        else:
            if out.dtype != np.float64 or out.shape != (self.n,) or not out.flags.c_contiguous or not out.flags.writeable:
                raise ValueError("out must be a writeable contiguous float64 array of n entries")
            x = out
        info = L.SolveInfo()
        o = opts.to_c()
        code = L.load().vfv_solve(self.ctx.handle, self._h, L.dptr(b), L.dptr(x0), L.dptr(x), C.byref(o), C.byref(info))
        _check(self.ctx.handle, code)
        return x, SolveInfo.from_c(info)

    def solve_device(self, b_ptr: int, x0_ptr: int, x_ptr: int, opts: GmresOptions | None = None) -> SolveInfo:
        """Device-pointer solve (``vfv_solve_device``)."""
        opts = opts or GmresOptions()
        info = L.SolveInfo()
        o = opts.to_c()
        code = L.load().vfv_solve_device(self.ctx.handle, self._h, C.c_void_p(b_ptr), C.c_void_p(x0_ptr), C.c_void_p(x_ptr),
                                          C.byref(o), C.byref(info))
        _check(self.ctx.handle, code)
        return SolveInfo.from_c(info)

    def spmv_device(self, x_ptr: int, y_ptr: int) -> None:
        _check(self.ctx.handle, L.load().vfv_spmv_device(self.ctx.handle, self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr)))

    def spmv_device_f32(self, x_ptr: int, y_ptr: int) -> None:
        _check(self.ctx.handle, L.load().vfv_spmv_device_f32(self.ctx.handle, self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr)))

    def ilu0_apply_device(self, r_ptr: int, z_ptr: int, order: int = L.ILU_MULTICOLOR) -> int:
        lev = C.c_int32()
        _check(self.ctx.handle, L.load().vfv_ilu0_apply_device(self.ctx.handle, self._h, int(order), C.c_void_p(r_ptr),
                                                               C.c_void_p(z_ptr), C.byref(lev)))
        return lev.value

    def ilu0_apply_device_f32(self, r_ptr: int, t_ptr: int, z_ptr: int, order: int = L.ILU_MULTICOLOR) -> int:
        """z = M^-1 r with the float factor, enqueued on the context's stream (no synchronisation);
        t is a float work vector of n entries. Returns the number of colour levels."""
        lev = C.c_int32()
        _check(self.ctx.handle, L.load().vfv_ilu0_apply_device_f32(self.ctx.handle, self._h, int(order), C.c_void_p(r_ptr),
                                                                   C.c_void_p(t_ptr), C.c_void_p(z_ptr), C.byref(lev)))
        return lev.value

    def ilu0_sweep_apply_device(self, r_ptr: int, z_ptr: int, sweeps: int, order: int = L.ILU_MULTICOLOR, f32: bool = False,
                                half: bool = False) -> None:
        """z = M^-1 r with `sweeps` Jacobi sweeps of each ILU(0) factor (double, the float factor
        with f32, its row-scaled half-precision values with half; float vectors for both), enqueued
        on the context's stream (no synchronisation)."""
        lib = L.load()
        fn = lib.vfv_ilu0_sweep_apply_device_f16 if half else lib.vfv_ilu0_sweep_apply_device_f32 if f32 else lib.vfv_ilu0_sweep_apply_device
        _check(self.ctx.handle, fn(self.ctx.handle, self._h, int(order), int(sweeps), C.c_void_p(r_ptr), C.c_void_p(z_ptr)))

    def ilu0_sweep_layout(self, order: int = L.ILU_MULTICOLOR) -> int:
        """bytes per column index of the swept factors (2: 16-bit offsets from the row, 4: absolute)"""
        cb = C.c_int32()
        _check(self.ctx.handle, L.load().vfv_ilu0_sweep_layout(self._h, int(order), C.byref(cb)))
        return cb.value

    def autotune(self):
        """Pick the SpMV lanes per row (double, float) by measurement; call before the first solve."""
        a, b = C.c_int32(), C.c_int32()
        _check(self.ctx.handle, L.load().vfv_pattern_autotune(self.ctx.handle, self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def spmv_shape(self):
        """((lanes, strides) double, (lanes, strides) float) of the SpMV in use."""
        a, b, c, d = (C.c_int32() for _ in range(4))
        _check(self.ctx.handle, L.load().vfv_pattern_spmv_shape(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        return (a.value, b.value), (c.value, d.value)

    def set_spmv_lanes(self, lanes64: int, lanes32: int) -> None:
        _check(self.ctx.handle, L.load().vfv_pattern_set_spmv_lanes(self.ctx.handle, self._h, int(lanes64), int(lanes32)))

    def ilu0_ordering(self, order: int = L.ILU_MULTICOLOR):
        """(perm new->old, lev_ptr) of the ILU(0) factor's symmetric permutation (host only)."""
        nlev = C.c_int32()
        _check(self.ctx.handle, L.load().vfv_ilu0_ordering(self.ctx.handle, self._h, int(order), None, None, C.byref(nlev)))
        perm = np.empty(self.n, np.int32)
        lev = np.empty(nlev.value + 1, np.int32)
        _check(self.ctx.handle, L.load().vfv_ilu0_ordering(self.ctx.handle, self._h, int(order), L.ptr(perm, C.c_int32),
                                                          L.ptr(lev, C.c_int32), C.byref(nlev)))
        return perm, lev

    def close(self) -> None:
        if self._owned and getattr(self, "_h", None):
            L.load().vfv_pattern_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
