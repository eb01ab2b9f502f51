"""ILU(0) orderings — TEST INFRASTRUCTURE (oracle). Restates the two orderings the product's
ILU(0) is defined on, from their definitions:

* natural: rows keep their order; level(i) = 1 + max level(k) over pattern neighbours k < i
  (either triangle, i.e. on the symmetrised pattern); rows are grouped by level, ties by index.
  Grouping by level never swaps two coupled rows, so the factor equals ILU(0) of A itself.
* multicolour: greedy colouring in index order, colour(i) = smallest colour not used by a
  symmetrised-pattern neighbour k < i; rows grouped by colour, ties by index.

Both return perm (new -> old) and the level (colour) of every row.
"""
from __future__ import annotations

import numpy as np


def _lower_lists(rp, ci):
    n = rp.size - 1
    lower = [[] for _ in range(n)]
    for i in range(n):
        for k in ci[rp[i]:rp[i + 1]]:
            k = int(k)
            if k < i:
                lower[i].append(k)
            elif k > i:
                lower[k].append(i)
    return lower


def natural(rp, ci):
    n = rp.size - 1
    lower = _lower_lists(rp, ci)
    lev = np.zeros(n, np.int64)
    for i in range(n):
        if lower[i]:
            lev[i] = max(lev[k] for k in lower[i]) + 1
    perm = np.lexsort((np.arange(n), lev)).astype(np.int32)
    return perm, lev


def multicolor(rp, ci):
    n = rp.size - 1
    lower = _lower_lists(rp, ci)
    col = np.zeros(n, np.int64)
    for i in range(n):
        used = {int(col[k]) for k in lower[i]}
        c = 0
        while c in used:
            c += 1
        col[i] = c
    perm = np.lexsort((np.arange(n), col)).astype(np.int32)
    return perm, col
