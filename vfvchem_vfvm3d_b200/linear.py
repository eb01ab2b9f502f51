"""``LinearGmres`` with the reference's ``LinearBase`` surface, solved on the GPU.

Reference: trait ``LinearBase`` (src/linear/linear_base.rs:5-10) and ``LinearGmres``
(src/linear/linear_gmres.rs:8-85). Same constructor checks and error variants, same call
sequence: ``update_sparse`` once per pattern, ``build_matrix`` per assembly, ``solve_matrix`` with
the previous iterate as warm start. The pattern and the triplet->slot map stay on the device, so
a repeated ``update_sparse`` with an unchanged (row, col) sequence is recognised and skipped
(the reference rebuilds it every time step, src/transient/transient_base.rs:83).
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .core import Context, GmresOptions, Pattern, SolveInfo, default_context
from .errors import (
    LinearGmresNonPositiveMaxOuter,
    LinearGmresNonPositiveRestart,
    LinearGmresNonPositiveThreads,
    LinearGmresNonPositiveTolerance,
)


@dataclass
class Triplet:
    """``faer::sparse::Triplet<usize, usize, f64>``"""

    row: int
    col: int
    val: float


def _as_arrays(a_triplet):
    if isinstance(a_triplet, tuple) and len(a_triplet) == 3:
        r, c, v = a_triplet
        return (np.ascontiguousarray(r, np.uint64), np.ascontiguousarray(c, np.uint64), np.ascontiguousarray(v, np.float64))
    r = np.fromiter((t.row for t in a_triplet), np.uint64, len(a_triplet))
    c = np.fromiter((t.col for t in a_triplet), np.uint64, len(a_triplet))
    v = np.fromiter((t.val for t in a_triplet), np.float64, len(a_triplet))
    return r, c, v


class SparseMatrix:
    """The assembled matrix (``SparseColMat<usize, f64>`` in the reference) resident on the GPU."""

    def __init__(self, pattern: Pattern):
        self.pattern = pattern

    def to_csr(self):
        return self.pattern.export()


class LinearGmres:
    def __init__(self, num_thread: int, tol: float, restart: int, max_outer: int, ctx: Context | None = None, **gpu_opts):
        self.ctx = ctx or default_context()
        self.opts = GmresOptions(tol=tol, restart=restart, max_outer=max_outer, **gpu_opts)
        self.num_thread = num_thread
        self._pattern: Pattern | None = None
        self._key = None
        self.last_info: SolveInfo | None = None

    @classmethod
    def new(cls, num_thread: int, **kw) -> "LinearGmres":
        """``LinearGmres::new`` — defaults tol 1e-6, restart 50, max_outer 200 (linear_gmres.rs:20-22)."""
        return cls.new_with_options(num_thread, 1e-6, 50, 200, **kw)

    @classmethod
    def new_with_options(cls, num_thread: int, tol: float, restart: int, max_outer: int, **kw) -> "LinearGmres":
        if num_thread == 0:
            raise LinearGmresNonPositiveThreads(f"num_thread = {num_thread}")
        if tol != tol or tol <= 0.0:
            raise LinearGmresNonPositiveTolerance(f"tol = {tol}")
        if restart == 0:
            raise LinearGmresNonPositiveRestart(f"restart = {restart}")
        if max_outer == 0:
            raise LinearGmresNonPositiveMaxOuter(f"max_outer = {max_outer}")
        return cls(num_thread, tol, restart, max_outer, **kw)

    # ---- LinearBase
    def update_sparse(self, a_triplet, mat_size: int) -> None:
        r, c, _ = _as_arrays(a_triplet)
        h = hashlib.blake2b(digest_size=16)
        h.update(np.int64(mat_size).tobytes())
        h.update(r.tobytes())
        h.update(c.tobytes())
        key = h.digest()
        if key == self._key and self._pattern is not None:
            return
        self._pattern = Pattern.from_triplets(self.ctx, mat_size, r, c)
        self._key = key

    def build_matrix(self, a_triplet) -> SparseMatrix:
        if self._pattern is None:
            raise ValueError("build_matrix before update_sparse")
        _, _, v = _as_arrays(a_triplet)
        self._pattern.values_from_triplets(v)
        return SparseMatrix(self._pattern)

    def solve_matrix(self, a_mat: SparseMatrix, b_vec: np.ndarray, x_init: np.ndarray, mat_size: int) -> np.ndarray:
        x, info = a_mat.pattern.solve(b_vec, x_init, self.opts)
        self.last_info = info
        return x
