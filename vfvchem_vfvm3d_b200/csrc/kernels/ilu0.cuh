// ILU(0) preconditioner: level-scheduled factorisation and triangular solves (sm_100a).
//
// The reference has no ILU (its GMRES is Jacobi-preconditioned, src/linear/linear_gmres.rs:79);
// this is the added preconditioner. The factor lives on a symmetric permutation P A P^T of the
// matrix whose rows are grouped into levels (contiguous row ranges): every row depends only on rows
// of earlier levels in the lower factor and of later levels in the upper factor. Two orderings are
// built on the host: the natural order with its dependency levels (the textbook ILU(0) of A) and a
// greedy multicolouring (levels = colours, far fewer launches). Both give an exact ILU(0) of the
// permuted matrix; the multicolour one is a different preconditioner from the natural-order one.
//
// Storage (permuted numbering): CSR lu_rp/lu_ci with columns ascending, lu_diag[i] = slot of the
// diagonal. Lower part = slots before lu_diag (unit diagonal implied), upper = from lu_diag on.
#pragma once
#include "../common.cuh"

namespace vfv {

// One level of the IKJ factorisation: a thread per row. Rows of one level never touch each other.
__global__ void k_ilu0_factor_level(int32_t r0, int32_t r1, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                    const int32_t* __restrict__ dg, double* __restrict__ a, int* __restrict__ bad) {
    const int32_t i = r0 + (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= r1) return;
    const int32_t e_i = rp[i + 1];
    for (int32_t kk = rp[i]; kk < dg[i]; ++kk) {
        const int32_t k = ci[kk];
        const double ukk = a[dg[k]];
        if (ukk == 0.0) {
            *bad = 1;
            return;
        }
        const double lik = a[kk] / ukk;
        a[kk] = lik;
        int32_t p = kk + 1, q = dg[k] + 1;
        const int32_t e_k = rp[k + 1];
        while (p < e_i && q < e_k) {
            const int32_t cp = ci[p], cq = ci[q];
            if (cp == cq) {
                a[p] -= lik * a[q];
                ++p;
                ++q;
            } else if (cp < cq) {
                ++p;
            } else {
                ++q;
            }
        }
    }
    if (a[dg[i]] == 0.0) *bad = 1;
}

// Gather A's values into the permuted factor storage: lu[k] = (T) val[src[k]].
template <typename T>
__global__ void k_gather_vals(int64_t nnz, const int32_t* __restrict__ src, const double* __restrict__ val, T* __restrict__ out) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nnz) out[k] = (T)val[src[k]];
}

template <typename TS, typename TD>
__global__ void k_cast(int64_t n, const TS* __restrict__ in, TD* __restrict__ out) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) out[k] = (TD)in[k];
}

// ---------------------------------------------------------------- level sweeps
// One launch per level, a thread per row. Each level is latency-bound (row range -> indices and
// values -> gather of already solved rows -> store), so the launches are chained with programmatic
// dependent launch: a level kernel first loads everything that does not depend on earlier levels
// (its rows' column indices, factor values, right-hand side), then lets the next level's kernel
// launch (griddepcontrol.launch_dependents) and only then waits for the previous level to finish
// (griddepcontrol.wait) before gathering solved values. The next level's prologue therefore
// overlaps this level's gathers instead of following them.
constexpr int kLevBlock = 128;
constexpr int kLevMinBlocks = 8;   // <= 64 registers: a ~100k-row level (~780 blocks) is one wave
constexpr int kLevK = 16;          // entries of a row held in registers before the wait: rows of the
                                   // late colours hold up to ~15 lower (early colours: upper) entries,
                                   // and every entry left to the loop costs a dependent round trip

__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// LOWER: t[i] = in[perm[i]] - sum_{k < diag} lu[k] t[ci[k]]
// UPPER: t[i] = (t[i] - sum_{k > diag} lu[k] t[ci[k]]) / lu[diag] ; out[perm[i]] = t[i]
template <typename T, bool LOWER>
__global__ void __launch_bounds__(kLevBlock, kLevMinBlocks) k_ilu0_level(int32_t r0, int32_t r1, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                         const int32_t* __restrict__ dg, const T* __restrict__ lu,
                                                         const int32_t* __restrict__ perm, const T* __restrict__ in, T* t, T* out,
                                                         const DevStatus* __restrict__ st) {
    const int32_t i = r0 + (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    int32_t kb = 0, ke = 0, d = 0, pi = 0;
    int32_t c[kLevK];
    T v[kLevK];
    T rhs = T(0), diag = T(1);
    if (i < r1) {
        d = __ldg(dg + i);
        kb = LOWER ? __ldg(rp + i) : d + 1;
        ke = LOWER ? d : __ldg(rp + i + 1);
        pi = __ldg(perm + i);
        if (!LOWER) diag = __ldg(lu + d);
        // the lower sweep's right-hand side is complete before the sweep's first (non-PDL) launch,
        // so it is read before the wait; the upper sweep's comes from the lower sweep (after it)
        if (LOWER) rhs = in[pi];
#pragma unroll
        for (int q = 0; q < kLevK; ++q) {
            c[q] = kb + q < ke ? __ldg(ci + kb + q) : -1;
            v[q] = kb + q < ke ? __ldg(lu + kb + q) : T(0);
        }
    }
    pdl_launch_dependents();
    pdl_wait();
    if (i >= r1 || (st && st->done)) return;
    if (!LOWER) rhs = t[i];
    T s = T(0);
#pragma unroll
    for (int q = 0; q < kLevK; ++q)
        if (c[q] >= 0) s += v[q] * t[c[q]];
    for (int32_t k = kb + kLevK; k < ke; ++k) s += __ldg(lu + k) * t[__ldg(ci + k)];
    if (LOWER) {
        t[i] = rhs - s;
    } else {
        const T x = (rhs - s) / diag;
        t[i] = x;
        out[pi] = x;
    }
}

}  // namespace vfv
