"""FP64 sparse LU solve — TEST INFRASTRUCTURE (oracle).

The reference's ``LinearLu`` (src/linear/linear_lu.rs:57-66) factors with faer 0.24.4's sparse LU,
which is not available here; scipy's SuperLU (scipy 1.18.1, COLAMD ordering, partial pivoting)
plays the same role: an FP64 direct solution the iterative solvers are measured against.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def lu_solve(rp, ci, va, b) -> np.ndarray:
    n = len(rp) - 1
    A = sp.csr_matrix((np.asarray(va, np.float64), np.asarray(ci, np.int64), np.asarray(rp, np.int64)), shape=(n, n)).tocsc()
    lu = spla.splu(A, permc_spec="COLAMD")
    return lu.solve(np.asarray(b, np.float64))
