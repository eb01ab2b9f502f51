// Krylov-subspace kernels for the restarted GMRES (sm_100a).
//
// The reference solves with faer_gmres::restarted_gmres + JacobiPreconLinOp
// (src/linear/linear_gmres.rs:76-84). Restated here from the published algorithm
// (Saad & Schultz 1986, right preconditioning, Givens least squares) with these device choices:
//   * basis vectors u_i are stored UNNORMALISED, with their norms beta_i in a device array;
//     v_i = u_i / beta_i. The SpMV of step j multiplies by 1/beta_j on the way out, so no separate
//     normalisation pass over the basis is ever made;
//   * orthogonalisation is classical Gram-Schmidt with one re-orthogonalisation (CGS2), which has
//     the stability of modified Gram-Schmidt; each pass is one multi-vector kernel that streams the
//     block's rows of every basis vector once, accumulates per-warp partial dots, and reduces them
//     deterministically (fixed order, no float atomics) in the last block to finish;
//   * the Hessenberg column, the Givens rotation and the residual estimate are finished by that last
//     block, so a whole restart cycle runs without a host synchronisation and is captured in a CUDA
//     graph. Every kernel first reads DevStatus::done and returns at once after convergence.
// Vectors are of type T (double, or float in the mixed-precision inner solve); all dots, norms,
// the Hessenberg matrix and the rotations are double.
#pragma once
#include "../common.cuh"

namespace vfv {

constexpr int kBlk = 256;        // threads per block of the vector kernels
constexpr int kVecMinBlocks = 8; // 32 registers: a full SM of threads for the multi-vector kernels
constexpr int kVecGroup = 2;     // basis vectors whose rows a thread loads before using any of them
constexpr int kMaxBasis = 128;   // m + 1 <= kMaxBasis

// Rows of one 16-byte chunk (4 floats, 2 doubles): a thread of the multi-vector kernels owns one
// chunk, a block kBlk chunks.
template <typename T>
constexpr int kVecRows = 16 / (int)sizeof(T);
template <typename T>
__host__ __device__ constexpr int64_t vec_block_rows() {
    return (int64_t)kBlk * kVecRows<T>;
}

// Per-solve device workspace pointers used by the Krylov kernels.
struct KrylovDev {
    int64_t n;          // rows
    int64_t ldv;        // stride between basis vectors (elements)
    int m;              // restart length
    int nblk;           // blocks of the multi-vector kernels
    double* part;       // [kMaxBasis][nblk] per-block partial dots
    unsigned* counter;  // [4] last-block counters
    double* hacc;       // [kMaxBasis] current Hessenberg column (accumulated over the CGS passes)
    double* coef;       // [kMaxBasis] update coefficients d_i / beta_i^2
    double* coefz;      // [kMaxBasis] both CGS passes' coefficients summed (overlapped engine), or null
    double* H;          // [m][m+1] column-major Hessenberg (rotated in place)
    double* cs;         // [m]
    double* sn;         // [m]
    double* g;          // [m+1]
    double* beta;       // [m+1] norms of the stored basis vectors
    double* inv_beta;   // [m+1]
    double* y;          // [m] least-squares solution scaled by 1/beta_i
    DevStatus* st;
    double* wnorm2;     // [1] ||w||^2 of the vector being orthogonalised (the reorthogonalisation test)
    const double* scal; // [0] tol_abs: converged when ||r|| <= tol_abs
                        // [1] inner_floor_rel: a cycle also stops once resid_est <= inner_floor_rel * beta0
};

// ---------------------------------------------------------------- last-block helper
// Threads that wrote partials fence their own writes before calling this (see publish_partial);
// after the block-wide barrier thread 0 takes a ticket, and the block that takes the last ticket
// reads every block's partials.
__device__ __forceinline__ bool last_block_arrive(unsigned* counter) {
    __shared__ bool s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned t = atomicAdd(counter, 1u);
        s_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) __threadfence();
    return s_last;
}

// store one partial and make it visible device-wide before the block arrives
__device__ __forceinline__ void publish_partial(double* p, double v) {
    *p = v;
    __threadfence();
}

// Sum column c of part[c][0..nblk) with all threads of the block, in a fixed order; valid in thread 0.
__device__ __forceinline__ double reduce_partials(const double* part, int nblk, double* red) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += __ldcg(part + b);
    return block_sum(s, red);
}

// Columns c < cnt of part[c][0..nblk): one warp per column; each lane loads 16 partials at once
// (the last block's reduction is latency-bound, so the loads of a batch must all be in flight),
// sums them pairwise, then a fixed shuffle tree; out(c, sum) is called by lane 0. Deterministic.
template <typename F>
__device__ __forceinline__ void reduce_cols_warp(const double* part, int nblk, int cnt, F out) {
    constexpr int kB = 16;  // partials per lane in flight: one L2 round trip per 512 partials
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int c = wid; c < cnt; c += nw) {
        const double* p = part + (int64_t)c * nblk;
        double s = 0.0;
        for (int q0 = 0; q0 < nblk; q0 += 32 * kB) {
            double v[kB];
#pragma unroll
            for (int k = 0; k < kB; ++k) {
                const int q = q0 + lane + 32 * k;
                v[k] = q < nblk ? __ldcg(p + q) : 0.0;
            }
#pragma unroll
            for (int h = kB / 2; h > 0; h >>= 1)
#pragma unroll
                for (int k = 0; k < h; ++k) v[k] += v[k + h];
            s += v[0];
        }
        s = warp_sum(s);
        if (lane == 0) out(c, s);
    }
}

// ---------------------------------------------------------------- SpMV (CSR, G lanes per row)
constexpr int kSpG = 4;  // lanes per row: rows hold ~16 non-zeros, 4 lanes x 4 loads in flight each

// This lane's share of row `row` of A x. The row's first S*G column indices and values are loaded
// before any x is gathered (S strides per lane, all independent), which keeps several loads in
// flight per lane; rows longer than S*G finish in a tail loop.
template <typename TV, typename TX, typename TA, int G, int S = 4>
__device__ __forceinline__ TA row_dot(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const TV* __restrict__ val,
                                      const TX* __restrict__ x, int64_t row, int lane) {
    const int32_t b = __ldg(rp + row), e = __ldg(rp + row + 1);
    int32_t c[S];
    TV v[S];
#pragma unroll
    for (int t = 0; t < S; ++t) {
        const int32_t k = b + lane + t * G;
        const bool ok = k < e;
        c[t] = ok ? __ldcs(ci + k) : -1;
        v[t] = ok ? __ldcs(val + k) : TV(0);
    }
    TA s = TA(0);
#pragma unroll
    for (int t = 0; t < S; ++t)
        if (c[t] >= 0) s += (TA)v[t] * (TA)__ldg(x + c[t]);
    for (int32_t k = b + lane + S * G; k < e; k += G) s += (TA)__ldcs(val + k) * (TA)__ldg(x + __ldcs(ci + k));
    return s;
}

// y = scale * (A x). Accumulation in TA. `scale` may be null (= 1).
template <typename TV, typename TX, typename TY, typename TA, int G, int S = 4>
__global__ void __launch_bounds__(kBlk) k_spmv(int64_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                              const TV* __restrict__ val, const TX* __restrict__ x, TY* __restrict__ y,
                                              const double* __restrict__ scale, const DevStatus* __restrict__ st) {
    if (st && st->done) return;
    const int lane = threadIdx.x & (G - 1);
    const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    TA s = TA(0);
    if (row < n) s = row_dot<TV, TX, TA, G, S>(rp, ci, val, x, row, lane);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, G);
    if (lane == 0 && row < n) {
        const double sc = scale ? *scale : 1.0;
        y[row] = (TY)((double)s * sc);
    }
}

// ---------------------------------------------------------------- residual r = b - A x (FP64)
// Writes u0 = r (type T), accumulates ||r||^2, and in the last block starts a new cycle:
// beta[0] = ||r||, g = (beta0, 0, ...), done/converged flags.
template <typename T, int G>
__global__ void __launch_bounds__(kBlk) k_residual(KrylovDev K, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                  const double* __restrict__ val, const double* __restrict__ x,
                                                  const double* __restrict__ b, T* __restrict__ u0) {
    __shared__ double red[kBlk / 32];
    const int lane = threadIdx.x & (G - 1);
    const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    double s = 0.0;
    if (row < K.n) s = row_dot<double, double, double, G>(rp, ci, val, x, row, lane);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, G);
    double r2 = 0.0;
    if (lane == 0 && row < K.n) {
        const double r = b[row] - s;
        u0[row] = (T)r;
        r2 = r * r;
    }
    const double bs = block_sum(r2, red);
    if (threadIdx.x == 0) publish_partial(K.part + blockIdx.x, bs);
    if (!last_block_arrive(K.counter)) return;
    const double tot = reduce_partials(K.part, gridDim.x, red);
    if (threadIdx.x == 0) {
        *K.counter = 0u;
        const double beta0 = sqrt(tot);
        K.beta[0] = beta0;
        K.inv_beta[0] = 1.0 / beta0;
        K.g[0] = beta0;
        DevStatus* st = K.st;
        st->steps = 0;
        st->beta0 = beta0;
        st->resid_est = beta0;
        const bool fin = isfinite(beta0);
        st->nonfinite = fin ? 0 : 1;
        const bool conv = fin && beta0 <= K.scal[0];
        st->converged = conv ? 1 : 0;
        st->done = (conv || !fin || beta0 == 0.0) ? 1 : 0;
    }
}

// ---------------------------------------------------------------- grouped multi-vector passes
// A thread owns the kVecRows<T> consecutive rows [row0, row0 + R) of one 16-byte chunk; rows past
// `end` read as zero. A chunk is moved with one 16-byte load or store when it is complete and
// aligned, else row by row: the same values either way, so tiles that start at any row (the
// batched kernels' per-mesh tiles) give the arithmetic of aligned ones. The chunks of kVecGroup
// basis vectors are loaded before any of them is used. Per vector the thread's rows are summed in
// row order, then across the warp (butterfly), the block's warps and the blocks, in fixed orders.
template <typename T>
__device__ __forceinline__ void load_chunk(const T* p, int64_t row0, int64_t end, T (&x)[kVecRows<T>]) {
    constexpr int R = kVecRows<T>;
    if (row0 + R <= end && (reinterpret_cast<uintptr_t>(p + row0) & 15u) == 0) {
        if constexpr (R == 4) {
            const float4 t = *reinterpret_cast<const float4*>(p + row0);
            x[0] = t.x, x[1] = t.y, x[2] = t.z, x[3] = t.w;
        } else {
            const double2 t = *reinterpret_cast<const double2*>(p + row0);
            x[0] = t.x, x[1] = t.y;
        }
    } else {
#pragma unroll
        for (int r = 0; r < R; ++r) x[r] = row0 + r < end ? p[row0 + r] : T(0);
    }
}

template <typename T>
__device__ __forceinline__ void store_chunk(T* p, int64_t row0, int64_t end, const T (&x)[kVecRows<T>]) {
    constexpr int R = kVecRows<T>;
    if (row0 + R <= end && (reinterpret_cast<uintptr_t>(p + row0) & 15u) == 0) {
        if constexpr (R == 4) *reinterpret_cast<float4*>(p + row0) = make_float4(x[0], x[1], x[2], x[3]);
        else *reinterpret_cast<double2*>(p + row0) = make_double2(x[0], x[1]);
    } else {
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (row0 + r < end) p[row0 + r] = x[r];
    }
}

// red[i][warp] = this warp's partial of <u_i, wt> for i < nvec (products in double)
template <typename T>
__device__ __forceinline__ void group_dots(const T* __restrict__ V, int64_t ldv, int64_t row0, int64_t end, const T* wt, int nvec,
                                           double (*red)[kBlk / 32]) {
    constexpr int R = kVecRows<T>;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i = 0; i < nvec; i += kVecGroup) {
        T x[kVecGroup][R];
#pragma unroll
        for (int q = 0; q < kVecGroup; ++q) load_chunk(V + (int64_t)(i + q) * ldv, row0, i + q < nvec ? end : 0, x[q]);
#pragma unroll
        for (int q = 0; q < kVecGroup; ++q) {
            double sq = 0.0;
#pragma unroll
            for (int r = 0; r < R; ++r) sq += (double)x[q][r] * (double)wt[r];
            sq = warp_sum(sq);
            if (lane == 0 && i + q < nvec) red[i + q][wid] = sq;
        }
    }
}

// acc[r] = sum_i coef[i] u_i[row0 + r] for i < nvec, i in order
template <typename T>
__device__ __forceinline__ void group_combine(const T* __restrict__ V, int64_t ldv, int64_t row0, int64_t end, const double* coef, int nvec,
                                              double* acc) {
    constexpr int R = kVecRows<T>;
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0.0;
    for (int i = 0; i < nvec; i += kVecGroup) {
        T x[kVecGroup][R];
#pragma unroll
        for (int q = 0; q < kVecGroup; ++q) load_chunk(V + (int64_t)(i + q) * ldv, row0, i + q < nvec ? end : 0, x[q]);
#pragma unroll
        for (int q = 0; q < kVecGroup; ++q) {
            if (i + q < nvec) {
                const double c = coef[i + q];
#pragma unroll
                for (int r = 0; r < R; ++r) acc[r] += c * (double)x[q][r];
            }
        }
    }
}

// ---------------------------------------------------------------- multi-dot (first CGS pass)
// Per-block partials of d_i = <u_i, w> for i < nvec (k_dots_finish<true> completes them).
// with_norm: also the partials of ||w||^2, as vector nvec (the first pass of the reorthogonalise-
// if-needed scheme); only_reorth: a second pass, skipped unless the first pass asked for it.
template <typename T>
__global__ void __launch_bounds__(kBlk, kVecMinBlocks) k_mdot(KrylovDev K, const T* __restrict__ V, const T* __restrict__ w, int nvec,
                                                               int with_norm, int only_reorth) {
    if (K.st->done || (only_reorth && !K.st->reorth)) return;
    __shared__ double red[kMaxBasis][kBlk / 32];
    constexpr int R = kVecRows<T>;
    const int nw = blockDim.x >> 5;
    const int64_t row0 = (int64_t)blockIdx.x * vec_block_rows<T>() + (int64_t)R * threadIdx.x;
    T wt[R];
    load_chunk(w, row0, K.n, wt);
    group_dots(V, K.ldv, row0, K.n, wt, nvec, red);
    if (with_norm) {
        double sq = 0.0;
#pragma unroll
        for (int r = 0; r < R; ++r) sq += (double)wt[r] * (double)wt[r];
        sq = warp_sum(sq);
        if ((threadIdx.x & 31) == 0) red[nvec][threadIdx.x >> 5] = sq;
    }
    __syncthreads();
    const int nout = nvec + (with_norm ? 1 : 0);
    for (int i = threadIdx.x; i < nout; i += blockDim.x) {
        double s = 0.0;
        for (int q = 0; q < nw; ++q) s += red[i][q];
        K.part[(int64_t)i * K.nblk + blockIdx.x] = s;  // summed by k_dots_finish (the next launch)
    }
}

// Cross-block sums of the multi-dot partials, one warp per basis vector spread over the GPU (a
// last-block reduction here would leave the GPU idle for ~15 µs while one block walks
// nvec x nblk partials). FIRST: hacc_i = d_i / beta_i; else hacc_i += d_i / beta_i; both set
// coef_i = d_i / beta_i^2 for the update that follows.
// with_norm: warp nvec sums the partials of ||w||^2 into wnorm2; only_reorth as in k_mdot.
template <bool FIRST>
__global__ void __launch_bounds__(256) k_dots_finish(KrylovDev K, int nvec, int with_norm, int only_reorth) {
    if (K.st->done || (only_reorth && !K.st->reorth)) return;
    const int lane = threadIdx.x & 31;
    const int c = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (c >= nvec + (with_norm ? 1 : 0)) return;
    const double* p = K.part + (int64_t)c * K.nblk;
    constexpr int kB = 16;
    double s = 0.0;
    for (int q0 = 0; q0 < K.nblk; q0 += 32 * kB) {
        double v[kB];
#pragma unroll
        for (int k = 0; k < kB; ++k) {
            const int q = q0 + lane + 32 * k;
            v[k] = q < K.nblk ? p[q] : 0.0;
        }
#pragma unroll
        for (int h = kB / 2; h > 0; h >>= 1)
#pragma unroll
            for (int k = 0; k < h; ++k) v[k] += v[k + h];
        s += v[0];
    }
    s = warp_sum(s);
    if (lane == 0 && c == nvec) {
        K.wnorm2[0] = s;
        return;
    }
    if (lane == 0) {
        const double ib = K.inv_beta[c];
        if (FIRST) K.hacc[c] = s * ib;
        else K.hacc[c] += s * ib;
        const double cf = s * ib * ib;
        K.coef[c] = cf;
        if (K.coefz) K.coefz[c] = FIRST ? cf : K.coefz[c] + cf;
    }
}

// Completes Arnoldi step j from ||w||^2 (tot): Hessenberg column, norms, the rotation of the new
// column by the previous Givens rotations and a new one, the residual estimate and the stopping
// test. One thread.
__device__ __forceinline__ void finish_column(KrylovDev K, int j, double tot) {
    const int m1 = K.m + 1;
    double* col = K.H + (int64_t)j * m1;
    const double bnext = sqrt(tot);
    for (int i = 0; i <= j; ++i) col[i] = K.hacc[i];
    col[j + 1] = bnext;
    K.beta[j + 1] = bnext;
    K.inv_beta[j + 1] = 1.0 / bnext;
    for (int i = 0; i < j; ++i) {
        const double a = col[i], bb = col[i + 1];
        col[i] = K.cs[i] * a + K.sn[i] * bb;
        col[i + 1] = -K.sn[i] * a + K.cs[i] * bb;
    }
    const double a = col[j], bb = col[j + 1];
    const double rr = hypot(a, bb);
    double c = 1.0, sgn = 0.0;
    if (rr > 0.0) {
        c = a / rr;
        sgn = bb / rr;
    }
    K.cs[j] = c;
    K.sn[j] = sgn;
    col[j] = rr;
    col[j + 1] = 0.0;
    const double gj = K.g[j];
    K.g[j] = c * gj;
    K.g[j + 1] = -sgn * gj;
    const double est = fabs(K.g[j + 1]);
    DevStatus* st = K.st;
    st->steps = j + 1;
    st->total_steps += 1;
    st->resid_est = est;
    const bool fin = isfinite(est) && isfinite(bnext) && isfinite(rr);
    if (!fin) st->nonfinite = 1;
    const double floor_abs = K.scal[1] * st->beta0;
    const bool stop = !fin || rr == 0.0 || bnext == 0.0 || est <= K.scal[0] || est <= floor_abs || j + 1 >= K.m;
    if (stop) st->done = 1;
}

// ---------------------------------------------------------------- update + second pass
// w <- win - sum_i coef_i u_i (win == w except in the overlapped engine). Then, with FINAL == false, the partials of the second CGS pass
// d'_i = <u_i, w> (k_dots_finish<false> adds d'_i/beta_i into hacc and sets coef); with
// FINAL == true, ||w||^2 and the last block finishes the Hessenberg column j, the Givens rotation
// and the convergence test - unless dgks is set and the test asks for a second pass, whose own
// k_update (launched with only_reorth) then finishes the column.
template <typename T, bool FINAL>
__global__ void __launch_bounds__(kBlk, kVecMinBlocks) k_update(KrylovDev K, const T* __restrict__ V, const T* win, T* w, int nvec, int j,
                                                                 int dgks, int only_reorth) {
    if (K.st->done || (only_reorth && !K.st->reorth)) return;
    __shared__ double red[kMaxBasis][kBlk / 32];
    __shared__ double red2[kBlk / 32];
    __shared__ double s_coef[kMaxBasis];
    constexpr int R = kVecRows<T>;
    const int nw = blockDim.x >> 5;
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) s_coef[i] = K.coef[i];
    __syncthreads();
    const int64_t row0 = (int64_t)blockIdx.x * vec_block_rows<T>() + (int64_t)R * threadIdx.x;
    double acc[R];
    group_combine(V, K.ldv, row0, K.n, s_coef, nvec, acc);
    T wt[R];
    load_chunk(win, row0, K.n, wt);
#pragma unroll
    for (int r = 0; r < R; ++r) wt[r] = (T)((double)wt[r] - acc[r]);  // rows past the end: 0 - 0
    store_chunk(w, row0, K.n, wt);
    if (!FINAL) {
        group_dots(V, K.ldv, row0, K.n, wt, nvec, red);
        __syncthreads();
        for (int i = threadIdx.x; i < nvec; i += blockDim.x) {
            double s = 0.0;
            for (int q = 0; q < nw; ++q) s += red[i][q];
            K.part[(int64_t)i * K.nblk + blockIdx.x] = s;  // summed by k_dots_finish<false>
        }
    } else {
        double s = 0.0;
#pragma unroll
        for (int r = 0; r < R; ++r) s += (double)wt[r] * (double)wt[r];
        s = block_sum(s, red2);
        if (threadIdx.x == 0) publish_partial(K.part + blockIdx.x, s);
        if (!last_block_arrive(K.counter + 3)) return;
        const double tot = reduce_partials(K.part, gridDim.x, red2);
        if (threadIdx.x == 0) {
            K.counter[3] = 0u;
            // first pass of the reorthogonalise-if-needed scheme (Daniel, Gragg, Kaufman & Stewart
            // 1976): a second pass only when the projection removed more than half of ||w||^2
            const bool again = dgks && tot < 0.5 * K.wnorm2[0];
            K.st->reorth = again ? 1 : 0;
            if (!again) finish_column(K, j, tot);
        }
    }
}

// ---------------------------------------------------------------- end of cycle
// Back substitution R y = g on the rotated Hessenberg (k = steps), y_i scaled by 1/beta_i.
// Overlapped engine: the preconditioned image of the new basis vector by linearity,
// z_{j+1} = M^-1 (w - sum_i c_i u_i) = q - sum_i c_i z_i with q = M^-1 w computed concurrently
// with the orthogonalisation and c_i the sum of both CGS passes' coefficients.
template <typename T>
__global__ void __launch_bounds__(kBlk, kVecMinBlocks) k_zupdate(KrylovDev K, T* Z, const T* __restrict__ q, int nvec, int j) {
    if (K.st->done) return;
    __shared__ double s_c[kMaxBasis];
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) s_c[i] = K.coefz[i];
    __syncthreads();
    constexpr int R = kVecRows<T>;
    const int64_t row0 = (int64_t)blockIdx.x * vec_block_rows<T>() + (int64_t)R * threadIdx.x;
    double acc[R];
    group_combine(Z, K.ldv, row0, K.n, s_c, nvec, acc);
    T qt[R];
    load_chunk(q, row0, K.n, qt);
#pragma unroll
    for (int r = 0; r < R; ++r) qt[r] = (T)((double)qt[r] - acc[r]);
    store_chunk(Z + (int64_t)(j + 1) * K.ldv, row0, K.n, qt);
}

__global__ void k_backsolve(KrylovDev K) {
    if (threadIdx.x != 0) return;
    const int k = K.st->steps;
    const int m1 = K.m + 1;
    for (int i = k - 1; i >= 0; --i) {
        double s = K.g[i];
        for (int q = i + 1; q < k; ++q) s -= K.H[(int64_t)q * m1 + i] * K.y[q];
        K.y[i] = s / K.H[(int64_t)i * m1 + i];
    }
    for (int i = 0; i < k; ++i) K.y[i] *= K.inv_beta[i];
    for (int i = k; i < K.m; ++i) K.y[i] = 0.0;
}

// z = sum_i y_i u_i (i < steps). MODE 0: x += z; MODE 1: x += dinv .* z; MODE 2: zt = (T)z for a preconditioner.
template <typename T, int MODE>
__global__ void __launch_bounds__(kBlk) k_combine(KrylovDev K, const T* __restrict__ V, double* __restrict__ x,
                                                 const double* __restrict__ dinv, T* __restrict__ zt) {
    __shared__ double s_y[kMaxBasis];
    const int k = K.st->steps;
    for (int i = threadIdx.x; i < k; i += blockDim.x) s_y[i] = K.y[i];
    __syncthreads();
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= K.n) return;
    double z = 0.0;
    for (int i = 0; i < k; ++i) z += s_y[i] * (double)V[(int64_t)i * K.ldv + row];
    if (MODE == 0) x[row] += z;
    if (MODE == 1) x[row] += dinv[row] * z;
    if (MODE == 2) zt[row] = (T)z;
}

template <typename T>
__global__ void k_add_to_x(int64_t n, double* __restrict__ x, const T* __restrict__ z) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += (double)z[i];
}

// ||v||^2 into out (single pass, last-block reduction)
__global__ void __launch_bounds__(kBlk) k_norm2(int64_t n, const double* __restrict__ v, double* part, unsigned* counter, double* out) {
    __shared__ double red[kBlk / 32];
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) s += v[i] * v[i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) publish_partial(part + blockIdx.x, s);
    if (!last_block_arrive(counter)) return;
    const double tot = reduce_partials(part, gridDim.x, red);
    if (threadIdx.x == 0) {
        *counter = 0u;
        *out = tot;
    }
}

// ---------------------------------------------------------------- matrix preparation
// dinv[i] = 1 / a_ii (diag_pos[i] = slot of the diagonal, -1 if absent -> 1)
__global__ void k_jacobi_inv(int64_t n, const int32_t* __restrict__ diag_pos, const double* __restrict__ val, double* __restrict__ dinv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t p = diag_pos[i];
    const double d = p >= 0 ? val[p] : 0.0;
    dinv[i] = d != 0.0 ? 1.0 / d : 1.0;
}

// z = M^-1 r for the 4x4 block-Jacobi preconditioner of a field-major 4-field system: block v
// couples rows {v, nb+v, 2nb+v, 3nb+v}; binv is [16][nb] (row-major 4x4 per block). `in` and `out`
// may alias (each thread reads its four entries before writing them).
template <typename T>
__global__ void __launch_bounds__(256) k_bj4_apply(int64_t nb, const T* __restrict__ binv, const T* in, T* out, const DevStatus* st) {
    if (st && st->done) return;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nb) return;
    T r[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) r[c] = in[c * nb + v];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        T acc = binv[(4 * a) * nb + v] * r[0];
#pragma unroll
        for (int c = 1; c < 4; ++c) acc += binv[(4 * a + c) * nb + v] * r[c];
        out[a * nb + v] = acc;
    }
}

// out[k] = (T)(val[k] * dinv[col[k]])  (right Jacobi scaling folded into the Krylov matrix)
template <typename T>
__global__ void k_scale_cols(int64_t nnz, const int32_t* __restrict__ ci, const double* __restrict__ val,
                             const double* __restrict__ dinv, T* __restrict__ out) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nnz) out[k] = (T)(val[k] * (dinv ? dinv[ci[k]] : 1.0));
}

}  // namespace vfv
