// Per-mesh Krylov recurrences for a batch of independent meshes (sm_100a).
//
// The reference solves every system on its own (one LinearGmres::solve_matrix per system,
// src/transient/transient_base.rs:83-109). A batch here is the concatenation of the meshes' systems
// into one block-diagonal matrix whose SpMV and ILU(0) sweeps run over all meshes at once (both are
// block-diagonal operations), while every mesh keeps its OWN Krylov recurrence: its own dot
// products and norms, Hessenberg matrix, Givens rotations, residual estimate, stopping test and
// `done` flag. A mesh that has converged (or finished its m steps of the cycle) is masked out of the
// orthogonalisation kernels; the cycle ends once every mesh is done.
//
// Bitwise equality with a mesh solved alone: the vector kernels work on tiles of vec_block_rows<T>()
// rows that start at each mesh's first row (the single-system kernels' blocks, shifted), the residual on
// tiles of kBlk / kSpG rows, and every per-mesh sum uses the single-system kernels' reduction order
// over the mesh's own tiles, so a mesh's iterates do not depend on the rest of the batch.
#pragma once
#include "krylov.cuh"

namespace vfv {

// Per-mesh scalar state of the batched recurrence.
struct MeshStat {
    int32_t done;         // the mesh takes no more Arnoldi steps this cycle
    int32_t steps;        // steps of the current cycle
    int32_t converged;    // its true residual met its tolerance (frozen for the rest of the solve)
    int32_t nonfinite;
    int32_t total_steps;  // Arnoldi steps over the whole solve
    int32_t zero_rhs;     // b_mesh = 0: x_mesh = 0
    double beta0;         // ||r|| at the start of the cycle
    double resid_est;     // |g_{j+1}|
    double bnorm;         // ||b_mesh||
};

struct BatchDev {
    int nm, m;
    int64_t ldv;
    const int64_t* mesh_row;   // [nm+1] first row of each mesh
    const int64_t* tile_row;   // [ntile+1] vector tiles (vec_block_rows<T>() rows, inside one mesh)
    const int32_t* tile_mesh;  // [ntile]
    const int32_t* mesh_tile;  // [nm+1]
    const int64_t* rtile_row;  // [nrtile+1] residual tiles (kBlk / kSpG rows, inside one mesh)
    const int32_t* rtile_mesh; // [nrtile]
    const int32_t* mesh_rtile; // [nm+1]
    int ntile, nrtile;
    double* part;              // [kMaxBasis][ntile] per-tile partial dots
    double* rpart;             // [nrtile] per-tile partial residual norms
    double* hacc;              // [nm][kMaxBasis]
    double* coef;              // [nm][kMaxBasis]
    double* H;                 // [nm][m][m+1] column-major per mesh
    double* cs;                // [nm][m]
    double* sn;                // [nm][m]
    double* g;                 // [nm][m+1]
    double* beta;              // [nm][m+1]
    double* inv_beta;          // [nm][m+1]
    double* y;                 // [nm][m]
    double* tol_abs;           // [nm] tol * ||b_mesh||
    MeshStat* ms;              // [nm]
    unsigned* counter;         // [4] arrival / done counters of the per-mesh finish kernels
    DevStatus* st;             // global: done once every mesh is done
    const double* scal;        // [1]: mixed precision, a mesh's cycle also ends at resid_est <= scal[1] * beta0
};

__device__ __forceinline__ int mesh_of_row(const int64_t* __restrict__ mesh_row, int nm, int64_t row) {
    int lo = 0, hi = nm;  // mesh_row[lo] <= row < mesh_row[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(mesh_row + mid) <= row) lo = mid;
        else hi = mid;
    }
    return lo;
}

// y = (A x) * inv_beta[mesh(row)][j]: the single-system SpMV with the step's scale looked up per row.
template <typename TV, typename TX, typename TY, typename TA, int G, int S = 4>
__global__ void __launch_bounds__(kBlk) k_spmv_seg(int64_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                  const TV* __restrict__ val, const TX* __restrict__ x, TY* __restrict__ y,
                                                  const double* __restrict__ inv_beta, int stride, int j,
                                                  const int64_t* __restrict__ mesh_row, int nm, const DevStatus* __restrict__ st) {
    if (st->done) return;
    const int lane = threadIdx.x & (G - 1);
    const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    TA s = TA(0);
    if (row < n) s = row_dot<TV, TX, TA, G, S>(rp, ci, val, x, row, lane);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, G);
    if (lane == 0 && row < n) {
        const double sc = inv_beta[(int64_t)mesh_of_row(mesh_row, nm, row) * stride + j];
        y[row] = (TY)((double)s * sc);
    }
}

// ||b_mesh||^2 and the mesh tolerance; one CTA per mesh.
__global__ void __launch_bounds__(kBlk) k_bnorm(BatchDev B, const double* __restrict__ b, double tol) {
    __shared__ double red[kBlk / 32];
    const int m = blockIdx.x;
    const int64_t r0 = B.mesh_row[m], r1 = B.mesh_row[m + 1];
    double s = 0.0;
    for (int64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) s += b[i] * b[i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) {
        const double bn = sqrt(s);
        MeshStat& M = B.ms[m];
        M = MeshStat{};
        M.bnorm = bn;
        M.zero_rhs = bn == 0.0 ? 1 : 0;
        M.nonfinite = isfinite(bn) ? 0 : 1;
        B.tol_abs[m] = tol * bn;
    }
}

// x = 0 on meshes whose right-hand side is zero (their solution)
__global__ void k_bzero_x(BatchDev B, double* __restrict__ x) {
    const int64_t n = B.mesh_row[B.nm];
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    if (B.ms[mesh_of_row(B.mesh_row, B.nm, row)].zero_rhs) x[row] = 0.0;
}

// r = b - A x per residual tile (FP64), u0 = r, per-tile ||r||^2 (k_residual's arithmetic).
template <typename T, int G>
__global__ void __launch_bounds__(kBlk) k_bresidual(BatchDev B, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                   const double* __restrict__ val, const double* __restrict__ x,
                                                   const double* __restrict__ b, T* __restrict__ u0) {
    __shared__ double red[kBlk / 32];
    const int t = blockIdx.x;
    const MeshStat& M = B.ms[B.rtile_mesh[t]];
    if (M.converged || M.zero_rhs) return;  // frozen mesh: no residual, no partial (its finish skips it)
    const int lane = threadIdx.x & (G - 1);
    const int64_t row = B.rtile_row[t] + threadIdx.x / G;
    const bool in = row < B.rtile_row[t + 1];
    double s = 0.0;
    if (in) s = row_dot<double, double, double, G>(rp, ci, val, x, row, lane);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, G);
    double r2 = 0.0;
    if (lane == 0 && in) {
        const double r = b[row] - s;
        u0[row] = (T)r;
        r2 = r * r;
    }
    const double bs = block_sum(r2, red);
    if (threadIdx.x == 0) B.rpart[t] = bs;
}

// Arrival of one finish CTA: counts `done` meshes; the last arrival publishes the global flags and
// resets the counters. counter[0] arrivals, [1] done meshes, [2] converged meshes, [3] active meshes.
__device__ __forceinline__ void batch_arrive(const BatchDev& B, bool done, bool conv, bool active, bool cycle_start) {
    __threadfence();
    if (done) atomicAdd(B.counter + 1, 1u);
    if (conv) atomicAdd(B.counter + 2, 1u);
    if (active) atomicAdd(B.counter + 3, 1u);
    __threadfence();
    const unsigned t = atomicAdd(B.counter, 1u);
    if (t == (unsigned)B.nm - 1) {
        __threadfence();
        const unsigned nd = atomicAdd(B.counter + 1, 0u), nc = atomicAdd(B.counter + 2, 0u), na = atomicAdd(B.counter + 3, 0u);
        DevStatus* st = B.st;
        if (cycle_start) {
            st->steps = 0;
            st->converged = nc == (unsigned)B.nm ? 1 : 0;
        } else if (na > 0) {
            st->steps += 1;
            st->total_steps += 1;
        }
        st->done = nd == (unsigned)B.nm ? 1 : 0;
        B.counter[0] = B.counter[1] = B.counter[2] = B.counter[3] = 0u;
        __threadfence();
    }
}

// Start of a cycle per mesh (k_residual's last block): beta0, g, the convergence test. One CTA per mesh.
__global__ void __launch_bounds__(kBlk) k_bresid_finish(BatchDev B) {
    __shared__ double red[kBlk / 32];
    const int m = blockIdx.x;
    MeshStat* M = B.ms + m;
    const bool frozen = M->converged || M->zero_rhs;
    double tot = 0.0;
    if (!frozen) {
        const int t0 = B.mesh_rtile[m], nt = B.mesh_rtile[m + 1] - t0;
        tot = reduce_partials(B.rpart + t0, nt, red);
    }
    if (threadIdx.x != 0) return;
    bool conv = frozen;
    if (!frozen) {
        const int m1 = B.m + 1;
        const double beta0 = sqrt(tot);
        B.beta[(int64_t)m * m1] = beta0;
        B.inv_beta[(int64_t)m * m1] = 1.0 / beta0;
        B.g[(int64_t)m * m1] = beta0;
        M->steps = 0;
        M->beta0 = beta0;
        M->resid_est = beta0;
        const bool fin = isfinite(beta0);
        if (!fin) M->nonfinite = 1;
        conv = fin && beta0 <= B.tol_abs[m];
        M->converged = conv ? 1 : 0;
        M->done = (conv || !fin || beta0 == 0.0) ? 1 : 0;
        if (!fin) B.st->nonfinite = 1;
    } else {
        M->done = 1;
        M->steps = 0;
        M->converged = 1;
    }
    batch_arrive(B, M->done != 0, conv, false, true);
}

// First CGS pass: per-tile partial dots of the mesh's basis with w (k_mdot per tile).
template <typename T>
__global__ void __launch_bounds__(kBlk, kVecMinBlocks) k_bmdot(BatchDev B, const T* __restrict__ V, const T* __restrict__ w, int nvec) {
    if (B.st->done) return;
    const int t = blockIdx.x;
    if (B.ms[B.tile_mesh[t]].done) return;
    __shared__ double red[kMaxBasis][kBlk / 32];
    constexpr int R = kVecRows<T>;
    const int nw = blockDim.x >> 5;
    const int64_t row0 = B.tile_row[t] + (int64_t)R * threadIdx.x, end = B.tile_row[t + 1];
    T wt[R];
    load_chunk(w, row0, end, wt);
    group_dots(V, B.ldv, row0, end, wt, nvec, red);
    __syncthreads();
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) {
        double s = 0.0;
        for (int q = 0; q < nw; ++q) s += red[i][q];
        B.part[(int64_t)i * B.ntile + t] = s;
    }
}

// Per-mesh cross-tile sums (k_dots_finish over the mesh's tiles): one warp per (mesh, vector).
template <bool FIRST>
__global__ void __launch_bounds__(256) k_bdots_finish(BatchDev B, int nvec) {
    if (B.st->done) return;
    const int lane = threadIdx.x & 31;
    const int64_t wgl = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wgl >= (int64_t)B.nm * nvec) return;
    const int m = (int)(wgl / nvec), c = (int)(wgl % nvec);
    if (B.ms[m].done) return;
    const int t0 = B.mesh_tile[m], nt = B.mesh_tile[m + 1] - t0;
    const double* p = B.part + (int64_t)c * B.ntile + t0;
    constexpr int kB = 16;
    double s = 0.0;
    for (int q0 = 0; q0 < nt; q0 += 32 * kB) {
        double v[kB];
#pragma unroll
        for (int k = 0; k < kB; ++k) {
            const int q = q0 + lane + 32 * k;
            v[k] = q < nt ? p[q] : 0.0;
        }
#pragma unroll
        for (int h = kB / 2; h > 0; h >>= 1)
#pragma unroll
            for (int k = 0; k < h; ++k) v[k] += v[k + h];
        s += v[0];
    }
    s = warp_sum(s);
    if (lane == 0) {
        const double ib = B.inv_beta[(int64_t)m * (B.m + 1) + c];
        double* hacc = B.hacc + (int64_t)m * kMaxBasis;
        if (FIRST) hacc[c] = s * ib;
        else hacc[c] += s * ib;
        B.coef[(int64_t)m * kMaxBasis + c] = s * ib * ib;
    }
}

// w <- win - sum_i coef_i u_i per tile; FINAL == false: second-pass partial dots; FINAL == true:
// per-tile ||w||^2 (k_update's arithmetic).
template <typename T, bool FINAL>
__global__ void __launch_bounds__(kBlk, kVecMinBlocks) k_bupdate(BatchDev B, const T* __restrict__ V, const T* win, T* w, int nvec) {
    if (B.st->done) return;
    const int t = blockIdx.x;
    const int m = B.tile_mesh[t];
    if (B.ms[m].done) return;
    __shared__ double red[kMaxBasis][kBlk / 32];
    __shared__ double red2[kBlk / 32];
    __shared__ double s_coef[kMaxBasis];
    constexpr int R = kVecRows<T>;
    const int nw = blockDim.x >> 5;
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) s_coef[i] = B.coef[(int64_t)m * kMaxBasis + i];
    __syncthreads();
    const int64_t row0 = B.tile_row[t] + (int64_t)R * threadIdx.x, end = B.tile_row[t + 1];
    double acc[R];
    group_combine(V, B.ldv, row0, end, s_coef, nvec, acc);
    T wt[R];
    load_chunk(win, row0, end, wt);
#pragma unroll
    for (int r = 0; r < R; ++r) wt[r] = (T)((double)wt[r] - acc[r]);  // rows past the end: 0 - 0
    store_chunk(w, row0, end, wt);
    if (!FINAL) {
        group_dots(V, B.ldv, row0, end, wt, nvec, red);
        __syncthreads();
        for (int i = threadIdx.x; i < nvec; i += blockDim.x) {
            double s = 0.0;
            for (int q = 0; q < nw; ++q) s += red[i][q];
            B.part[(int64_t)i * B.ntile + t] = s;
        }
    } else {
        double s = 0.0;
#pragma unroll
        for (int r = 0; r < R; ++r) s += (double)wt[r] * (double)wt[r];
        s = block_sum(s, red2);
        if (threadIdx.x == 0) B.part[t] = s;
    }
}

// End of Arnoldi step j per mesh (k_update<true>'s last block): norm, Hessenberg column, Givens
// rotation, convergence test. One CTA per mesh.
__global__ void __launch_bounds__(kBlk) k_bstep_finish(BatchDev B, int j) {
    if (B.st->done) return;
    __shared__ double red[kBlk / 32];
    const int m = blockIdx.x;
    MeshStat* M = B.ms + m;
    const bool active = !M->done;
    double tot = 0.0;
    if (active) {
        const int t0 = B.mesh_tile[m], nt = B.mesh_tile[m + 1] - t0;
        tot = reduce_partials(B.part + t0, nt, red);
    }
    if (threadIdx.x != 0) return;
    if (active) {
        const int m1 = B.m + 1;
        double* col = B.H + ((int64_t)m * B.m + j) * m1;
        const double* hacc = B.hacc + (int64_t)m * kMaxBasis;
        double* cs = B.cs + (int64_t)m * B.m;
        double* sn = B.sn + (int64_t)m * B.m;
        double* g = B.g + (int64_t)m * m1;
        const double bnext = sqrt(tot);
        for (int i = 0; i <= j; ++i) col[i] = hacc[i];
        col[j + 1] = bnext;
        B.beta[(int64_t)m * m1 + j + 1] = bnext;
        B.inv_beta[(int64_t)m * m1 + j + 1] = 1.0 / bnext;
        for (int i = 0; i < j; ++i) {
            const double a = col[i], bb = col[i + 1];
            col[i] = cs[i] * a + sn[i] * bb;
            col[i + 1] = -sn[i] * a + cs[i] * bb;
        }
        const double a = col[j], bb = col[j + 1];
        const double rr = hypot(a, bb);
        double c = 1.0, sgn = 0.0;
        if (rr > 0.0) {
            c = a / rr;
            sgn = bb / rr;
        }
        cs[j] = c;
        sn[j] = sgn;
        col[j] = rr;
        col[j + 1] = 0.0;
        const double gj = g[j];
        g[j] = c * gj;
        g[j + 1] = -sgn * gj;
        const double est = fabs(g[j + 1]);
        M->steps = j + 1;
        M->total_steps += 1;
        M->resid_est = est;
        const bool fin = isfinite(est) && isfinite(bnext) && isfinite(rr);
        if (!fin) {
            M->nonfinite = 1;
            B.st->nonfinite = 1;
        }
        const double floor_abs = B.scal[1] * M->beta0;
        const bool stop = !fin || rr == 0.0 || bnext == 0.0 || est <= B.tol_abs[m] || est <= floor_abs || j + 1 >= B.m;
        if (stop) M->done = 1;
    }
    batch_arrive(B, M->done != 0, false, active, false);
}

// Back substitution per mesh (k_backsolve), one thread per mesh.
__global__ void k_bbacksolve(BatchDev B) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= B.nm) return;
    const int k = B.ms[m].converged ? 0 : B.ms[m].steps;
    const int m1 = B.m + 1;
    const double* H = B.H + (int64_t)m * B.m * m1;
    const double* g = B.g + (int64_t)m * m1;
    const double* ib = B.inv_beta + (int64_t)m * m1;
    double* y = B.y + (int64_t)m * B.m;
    for (int i = k - 1; i >= 0; --i) {
        double s = g[i];
        for (int q = i + 1; q < k; ++q) s -= H[(int64_t)q * m1 + i] * y[q];
        y[i] = s / H[(int64_t)i * m1 + i];
    }
    for (int i = 0; i < k; ++i) y[i] *= ib[i];
    for (int i = k; i < B.m; ++i) y[i] = 0.0;
}

// z = sum_i y_i u_i over the mesh's steps of this cycle (k_combine per row). MODE 0: x += z;
// MODE 1: x += dinv .* z; MODE 2: zt = (T)z (to be preconditioned).
template <typename T, int MODE>
__global__ void __launch_bounds__(kBlk) k_bcombine(BatchDev B, const T* __restrict__ V, double* __restrict__ x,
                                                  const double* __restrict__ dinv, T* __restrict__ zt) {
    __shared__ double s_y[kMaxBasis];
    const int t = blockIdx.x;
    const int m = B.tile_mesh[t];
    const int k = B.ms[m].converged ? 0 : B.ms[m].steps;
    for (int i = threadIdx.x; i < k; i += blockDim.x) s_y[i] = B.y[(int64_t)m * B.m + i];
    __syncthreads();
    const int64_t end = B.tile_row[t + 1];
    for (int64_t row = B.tile_row[t] + threadIdx.x; row < end; row += kBlk) {
        double z = 0.0;
        for (int i = 0; i < k; ++i) z += s_y[i] * (double)V[(int64_t)i * B.ldv + row];
        if (MODE == 0) x[row] += z;
        if (MODE == 1) x[row] += dinv[row] * z;
        if (MODE == 2) zt[row] = (T)z;
    }
}

}  // namespace vfv
