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

// Lower solve for one level: t[i] = rhs[perm[i]] - sum_{k<i} l_ik t[k]   (G lanes per row)
template <typename T, int G>
__global__ void __launch_bounds__(256) k_ilu0_lower(int32_t r0, int32_t r1, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                   const int32_t* __restrict__ dg, const T* __restrict__ lu, const int32_t* __restrict__ perm,
                                                   const T* __restrict__ rhs, T* __restrict__ t, const DevStatus* __restrict__ st) {
    if (st && st->done) return;
    const int lane = threadIdx.x & (G - 1);
    const int32_t i = r0 + (int32_t)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G);
    T s = T(0);
    if (i < r1) {
        const int32_t e = dg[i];
        for (int32_t k = rp[i] + lane; k < e; k += G) s += lu[k] * t[ci[k]];
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, G);
    if (lane == 0 && i < r1) t[i] = rhs[perm[i]] - s;
}

// Upper solve for one level: t[i] = (t[i] - sum_{j>i} u_ij t[j]) / u_ii ; out[perm[i]] = t[i]
template <typename T, int G>
__global__ void __launch_bounds__(256) k_ilu0_upper(int32_t r0, int32_t r1, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                   const int32_t* __restrict__ dg, const T* __restrict__ lu, const int32_t* __restrict__ perm,
                                                   T* __restrict__ t, T* __restrict__ out, const DevStatus* __restrict__ st) {
    if (st && st->done) return;
    const int lane = threadIdx.x & (G - 1);
    const int32_t i = r0 + (int32_t)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G);
    T s = T(0);
    int32_t d = 0;
    if (i < r1) {
        d = dg[i];
        const int32_t e = rp[i + 1];
        for (int32_t k = d + 1 + lane; k < e; k += G) s += lu[k] * t[ci[k]];
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, G);
    if (lane == 0 && i < r1) {
        const T v = (t[i] - s) / lu[d];
        t[i] = v;
        out[perm[i]] = v;
    }
}

}  // namespace vfv
