// One restart cycle of GMRES(m) as a single persistent cooperative kernel (sm_100a).
//
// Same algorithm as the kernel-per-phase path in krylov.cuh (right-preconditioned GMRES,
// unnormalised basis with device norms, CGS2, Givens least squares — Saad & Schultz 1986),
// restated so that a whole cycle is ONE launch: all CTAs are co-resident (cooperative launch) and
// separate the phases with grid barriers instead of kernel boundaries. Per Arnoldi step that is
// 2*levels barriers for the ILU(0) sweeps and three reduce-barriers for the CGS2 passes; a kernel
// launch plus drain costs several times a barrier, and a level of the multicolour ILU(0) is only a
// few microseconds of work at 10^6 rows, so the launches dominated the step before.
//
// Row ownership: CTA c owns rows [c*chunk, (c+1)*chunk) for SpMV, the Gram-Schmidt passes, the
// update of x and the residual; ILU levels are spread over every sub-warp of the grid.
// Reductions are deterministic: each CTA writes its partials, the LAST CTA to arrive at the
// barrier sums them in CTA order, finishes the scalar work (Hessenberg column, Givens rotation,
// convergence test) and only then releases the barrier.
// Data written inside the kernel is only read with coherent loads (never the non-coherent
// read-only path); the barrier's fences order it.
// Every wait is bounded: a barrier that does not complete within `spin_limit` polls sets
// DevStatus::timeout and every CTA leaves the kernel.
#pragma once
#include "krylov.cuh"

namespace vfv {

constexpr int kMegaThreads = 512;
constexpr int kMegaWarps = kMegaThreads / 32;
constexpr int kMegaRows = 8;  // rows held in registers per thread per tile

struct CycleArgs {
    int64_t n, ldv;
    int m, chunk;
    int precond;  // 0 none, 1 Jacobi (folded into valK, x += dinv .* z), 2 ILU(0)
    const int32_t* rp;
    const int32_t* ci;
    const void* valK;      // T: Krylov matrix values (Jacobi-scaled copy when precond == 1)
    const double* val64;   // FP64 values for the true residual
    const double* b;
    double* x;
    const double* dinv;
    // ILU(0) on the permuted system
    int nlev;
    const int32_t* lev_ptr;
    const int32_t* lrp;
    const int32_t* lci;
    const int32_t* ldg;
    const void* lu;        // T
    const int32_t* perm;
    void* V;               // T [m+1][ldv]
    void* z;               // T [n] preconditioned vector
    void* t;               // T [n] ILU work vector
    void* zc;              // T [n] combined update before the preconditioner
    double *H, *cs, *sn, *g, *beta, *inv_beta, *y, *hacc, *coef;
    double* part;          // [kMaxBasis][gridDim]
    unsigned* bar;         // [0] arrival count, [kGenOffset] generation (separate cache lines)
    unsigned long long* trace;  // optional [m+2][8] phase timestamps written by CTA 0 (null: off)
    DevStatus* st;
    const double* scal;    // [0] tol_abs, [1] inner floor (relative to beta0)
    long long spin_limit;
};

constexpr int kGenOffset = 32;  // the generation word sits 128 bytes after the arrival counter
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s: far above any real barrier

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void trace_mark(const CycleArgs& A, int step, int phase) {
    if (A.trace && blockIdx.x == 0 && threadIdx.x == 0) A.trace[step * 8 + phase] = globaltimer_ns();
}

struct GridSync {
    unsigned gen;  // generation this CTA expects to be released from (thread 0 only)
};

// Arrive; the last CTA runs `last()` with all its threads before releasing. Returns false on timeout.
template <typename F>
__device__ __forceinline__ bool grid_reduce_barrier(const CycleArgs& A, GridSync& gs, F last) {
    __shared__ int s_last;
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned a = atomicAdd(A.bar, 1u);
        s_last = (a == gridDim.x - 1) ? 1 : 0;
        s_ok = 1;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        last();
        __syncthreads();
        if (threadIdx.x == 0) {
            A.bar[0] = 0u;
            __threadfence();
            atomicAdd(A.bar + kGenOffset, 1u);
            gs.gen += 1u;
        }
    } else if (threadIdx.x == 0) {
        volatile unsigned* genp = A.bar + kGenOffset;
        long long it = 0;
        const unsigned long long t0 = globaltimer_ns();
        while (*genp == gs.gen) {
            if (++it > A.spin_limit || (it % 1024 == 0 && globaltimer_ns() - t0 > kBarrierTimeoutNs)) {
                A.st->timeout = 1;
                s_ok = 0;
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
        gs.gen += 1u;
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_ok && *(volatile int*)&A.st->timeout) s_ok = 0;
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ bool grid_barrier(const CycleArgs& A, GridSync& gs) {
    return grid_reduce_barrier(A, gs, [] {});
}

// Sum part[c][0..gridDim) for c < cnt into out_fn(c, sum); called by all threads of the last CTA.
template <typename F>
__device__ __forceinline__ void reduce_columns(const CycleArgs& A, int cnt, F out_fn) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int c = wid; c < cnt; c += kMegaWarps) {
        const double* p = A.part + (int64_t)c * gridDim.x;
        double s = 0.0;
        for (int q = lane; q < (int)gridDim.x; q += 32) s += __ldcg(p + q);
        s = warp_sum(s);
        if (lane == 0) out_fn(c, s);
    }
}

// Write this CTA's per-warp partial dots red[i][warp] as part[i][blockIdx]
__device__ __forceinline__ void store_partials(const CycleArgs& A, double (*red)[kMegaWarps], int cnt) {
    __syncthreads();
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < kMegaWarps; ++q) s += red[i][q];
        A.part[(int64_t)i * gridDim.x + blockIdx.x] = s;
    }
}

template <typename T>
__device__ __forceinline__ void ilu_sweeps(const CycleArgs& A, GridSync& gs, const T* in, T* out, bool& ok) {
    constexpr int G = 8;
    const T* lu = reinterpret_cast<const T*>(A.lu);
    T* t = reinterpret_cast<T*>(A.t);
    const int lane = threadIdx.x & (G - 1);
    // warp-uniform row loops: a warp handles 32/G consecutive rows per iteration
    const int64_t wbase = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32 * (32 / G);
    const int64_t wstep = (int64_t)gridDim.x * blockDim.x / 32 * (32 / G);
    const int sub = (threadIdx.x & 31) / G;
    for (int l = 0; l < A.nlev && ok; ++l) {
        const int32_t r0 = __ldg(A.lev_ptr + l), r1 = __ldg(A.lev_ptr + l + 1);
        for (int64_t i0 = r0 + wbase; i0 < r1; i0 += wstep) {
            const int64_t i = i0 + sub;
            T s = T(0);
            if (i < r1) {
                const int32_t e = __ldg(A.ldg + i);
                for (int32_t k = __ldg(A.lrp + i) + lane; k < e; k += G) s += __ldg(lu + k) * __ldcg(t + __ldg(A.lci + k));
            }
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, G);
            if (lane == 0 && i < r1) t[i] = __ldcg(in + __ldg(A.perm + i)) - s;
        }
        ok = grid_barrier(A, gs);
    }
    for (int l = A.nlev - 1; l >= 0 && ok; --l) {
        const int32_t r0 = __ldg(A.lev_ptr + l), r1 = __ldg(A.lev_ptr + l + 1);
        for (int64_t i0 = r0 + wbase; i0 < r1; i0 += wstep) {
            const int64_t i = i0 + sub;
            T s = T(0);
            int32_t d = 0;
            if (i < r1) {
                d = __ldg(A.ldg + i);
                const int32_t e = __ldg(A.lrp + i + 1);
                for (int32_t k = d + 1 + lane; k < e; k += G) s += __ldg(lu + k) * __ldcg(t + __ldg(A.lci + k));
            }
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, G);
            if (lane == 0 && i < r1) {
                const T v = (__ldcg(t + i) - s) / __ldg(lu + d);
                t[i] = v;
                out[__ldg(A.perm + i)] = v;
            }
        }
        ok = grid_barrier(A, gs);
    }
}

// y[row] = scale * sum_k val[k] x[col[k]] for this CTA's rows, G lanes per row, warp-uniform loop.
// Returns (in lane 0 of each group) through the callback out(row, value).
template <typename TV, typename TX, typename TA, typename F>
__device__ __forceinline__ void cta_spmv(const int32_t* rp, const int32_t* ci, const TV* val, const TX* x, int64_t r0, int64_t r1, F out) {
    constexpr int G = 8;
    const int lane = threadIdx.x & (G - 1);
    const int sub = (threadIdx.x & 31) / G;
    const int wid = threadIdx.x >> 5;
    for (int64_t base = r0 + (int64_t)wid * (32 / G); base < r1; base += (int64_t)kMegaWarps * (32 / G)) {
        const int64_t row = base + sub;
        TA s = TA(0);
        if (row < r1) {
            const int32_t b0 = __ldg(rp + row), e = __ldg(rp + row + 1);
            for (int32_t k = b0 + lane; k < e; k += G) s += (TA)__ldg(val + k) * (TA)__ldcg(x + __ldg(ci + k));
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, G);
        if (lane == 0 && row < r1) out(row, s);
    }
}

template <typename T>
__global__ void __launch_bounds__(kMegaThreads) k_gmres_cycle(CycleArgs A) {
    __shared__ double red[kMaxBasis][kMegaWarps];
    __shared__ double s_coef[kMaxBasis];
    __shared__ GridSync gs_sh;
    __shared__ double s_tot;
    GridSync& gs = gs_sh;
    if (threadIdx.x == 0) gs.gen = *(volatile unsigned*)(A.bar + kGenOffset);
    __syncthreads();
    T* V = reinterpret_cast<T*>(A.V);
    T* Z = reinterpret_cast<T*>(A.z);
    T* ZC = reinterpret_cast<T*>(A.zc);
    const T* valK = reinterpret_cast<const T*>(A.valK);
    const int lane32 = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int64_t r0 = (int64_t)blockIdx.x * A.chunk;
    const int64_t r1 = min(A.n, r0 + A.chunk);
    const int64_t tile = (int64_t)kMegaRows * blockDim.x;
    bool ok = true;

    for (int j = 0; j < A.m && ok; ++j) {
        if (*(volatile int*)&A.st->done) break;
        trace_mark(A, j, 0);
        const T* uj = V + (int64_t)j * A.ldv;
        T* w = V + (int64_t)(j + 1) * A.ldv;
        const T* zin = uj;
        if (A.precond == 2) {
            ilu_sweeps<T>(A, gs, uj, Z, ok);
            if (!ok) break;
            zin = Z;
        }
        trace_mark(A, j, 1);
        // ---- w = (A z) / beta_j on this CTA's rows (G lanes per row)
        {
            const double sc = __ldcg(A.inv_beta + j);
            cta_spmv<T, T, T>(A.rp, A.ci, valK, zin, r0, r1, [&](int64_t row, T s) { w[row] = (T)((double)s * sc); });
        }
        __syncthreads();
        trace_mark(A, j, 2);
        const int nvec = j + 1;
        // ---- pass 1: d_i = <u_i, w>
        for (int i = threadIdx.x; i < nvec * kMegaWarps; i += blockDim.x) (&red[0][0])[i] = 0.0;
        __syncthreads();
        for (int64_t t0 = r0; t0 < r1; t0 += tile) {
            double wr[kMegaRows];
#pragma unroll
            for (int r = 0; r < kMegaRows; ++r) {
                const int64_t row = t0 + r * blockDim.x + threadIdx.x;
                wr[r] = row < r1 ? (double)w[row] : 0.0;
            }
            for (int i = 0; i < nvec; ++i) {
                const T* u = V + (int64_t)i * A.ldv;
                double s = 0.0;
#pragma unroll
                for (int r = 0; r < kMegaRows; ++r) {
                    const int64_t row = t0 + r * blockDim.x + threadIdx.x;
                    if (row < r1) s += (double)u[row] * wr[r];
                }
                s = warp_sum(s);
                if (lane32 == 0) red[i][wid] += s;
            }
        }
        store_partials(A, red, nvec);
        ok = grid_reduce_barrier(A, gs, [&] {
            reduce_columns(A, nvec, [&](int c, double d) {
                const double ib = __ldcg(A.inv_beta + c);
                A.hacc[c] = d * ib;
                A.coef[c] = d * ib * ib;
            });
        });
        if (!ok) break;
        trace_mark(A, j, 3);
        // ---- pass 2: w -= sum coef_i u_i ; d'_i = <u_i, w>
        for (int i = threadIdx.x; i < nvec; i += blockDim.x) s_coef[i] = __ldcg(A.coef + i);
        for (int i = threadIdx.x; i < nvec * kMegaWarps; i += blockDim.x) (&red[0][0])[i] = 0.0;
        __syncthreads();
        for (int64_t t0 = r0; t0 < r1; t0 += tile) {
            double acc[kMegaRows];
#pragma unroll
            for (int r = 0; r < kMegaRows; ++r) acc[r] = 0.0;
            for (int i = 0; i < nvec; ++i) {
                const T* u = V + (int64_t)i * A.ldv;
                const double c = s_coef[i];
#pragma unroll
                for (int r = 0; r < kMegaRows; ++r) {
                    const int64_t row = t0 + r * blockDim.x + threadIdx.x;
                    if (row < r1) acc[r] += c * (double)u[row];
                }
            }
            double wr[kMegaRows];
#pragma unroll
            for (int r = 0; r < kMegaRows; ++r) {
                const int64_t row = t0 + r * blockDim.x + threadIdx.x;
                if (row < r1) {
                    const T nv = (T)((double)w[row] - acc[r]);
                    w[row] = nv;
                    wr[r] = (double)nv;
                } else {
                    wr[r] = 0.0;
                }
            }
            for (int i = 0; i < nvec; ++i) {
                const T* u = V + (int64_t)i * A.ldv;
                double s = 0.0;
#pragma unroll
                for (int r = 0; r < kMegaRows; ++r) {
                    const int64_t row = t0 + r * blockDim.x + threadIdx.x;
                    if (row < r1) s += (double)u[row] * wr[r];
                }
                s = warp_sum(s);
                if (lane32 == 0) red[i][wid] += s;
            }
        }
        store_partials(A, red, nvec);
        ok = grid_reduce_barrier(A, gs, [&] {
            reduce_columns(A, nvec, [&](int c, double d) {
                const double ib = __ldcg(A.inv_beta + c);
                A.hacc[c] = __ldcg(A.hacc + c) + d * ib;
                A.coef[c] = d * ib * ib;
            });
        });
        if (!ok) break;
        trace_mark(A, j, 4);
        // ---- pass 3: w -= sum coef_i u_i ; ||w||^2 ; Hessenberg column, Givens, convergence
        for (int i = threadIdx.x; i < nvec; i += blockDim.x) s_coef[i] = __ldcg(A.coef + i);
        __syncthreads();
        double nrm = 0.0;
        for (int64_t t0 = r0; t0 < r1; t0 += tile) {
            double acc[kMegaRows];
#pragma unroll
            for (int r = 0; r < kMegaRows; ++r) acc[r] = 0.0;
            for (int i = 0; i < nvec; ++i) {
                const T* u = V + (int64_t)i * A.ldv;
                const double c = s_coef[i];
#pragma unroll
                for (int r = 0; r < kMegaRows; ++r) {
                    const int64_t row = t0 + r * blockDim.x + threadIdx.x;
                    if (row < r1) acc[r] += c * (double)u[row];
                }
            }
#pragma unroll
            for (int r = 0; r < kMegaRows; ++r) {
                const int64_t row = t0 + r * blockDim.x + threadIdx.x;
                if (row < r1) {
                    const T nv = (T)((double)w[row] - acc[r]);
                    w[row] = nv;
                    nrm += (double)nv * (double)nv;
                }
            }
        }
        nrm = warp_sum(nrm);
        if (lane32 == 0) red[0][wid] = nrm;
        store_partials(A, red, 1);
        ok = grid_reduce_barrier(A, gs, [&] {
            reduce_columns(A, 1, [&](int, double d) { s_tot = d; });
            __syncthreads();
            if (threadIdx.x == 0) {
                const int m1 = A.m + 1;
                double* col = A.H + (int64_t)j * m1;
                const double bnext = sqrt(s_tot);
                for (int i = 0; i <= j; ++i) col[i] = __ldcg(A.hacc + i);
                col[j + 1] = bnext;
                A.beta[j + 1] = bnext;
                A.inv_beta[j + 1] = 1.0 / bnext;
                for (int i = 0; i < j; ++i) {
                    const double a = col[i], bb = col[i + 1];
                    const double ci = __ldcg(A.cs + i), si = __ldcg(A.sn + i);
                    col[i] = ci * a + si * bb;
                    col[i + 1] = -si * a + ci * bb;
                }
                const double a = col[j], bb = col[j + 1];
                const double rr = hypot(a, bb);
                double c = 1.0, sg = 0.0;
                if (rr > 0.0) {
                    c = a / rr;
                    sg = bb / rr;
                }
                A.cs[j] = c;
                A.sn[j] = sg;
                col[j] = rr;
                col[j + 1] = 0.0;
                const double gj = __ldcg(A.g + j);
                A.g[j] = c * gj;
                A.g[j + 1] = -sg * gj;
                const double est = fabs(-sg * gj);
                volatile DevStatus* st = A.st;
                st->steps = j + 1;
                st->total_steps = st->total_steps + 1;
                st->resid_est = est;
                const bool fin = isfinite(est) && isfinite(bnext) && isfinite(rr);
                if (!fin) st->nonfinite = 1;
                const bool stop = !fin || rr == 0.0 || bnext == 0.0 || est <= A.scal[0] || est <= A.scal[1] * st->beta0 || j + 1 >= A.m;
                if (stop) st->done = 1;
            }
        });
    }
    if (!ok) return;
    trace_mark(A, A.m, 0);

    // ---- least squares (last CTA) then x update
    ok = grid_reduce_barrier(A, gs, [&] {
        if (threadIdx.x == 0) {
            const int k = *(volatile int*)&A.st->steps;
            const int m1 = A.m + 1;
            for (int i = k - 1; i >= 0; --i) {
                double s = __ldcg(A.g + i);
                for (int q = i + 1; q < k; ++q) s -= __ldcg(A.H + (int64_t)q * m1 + i) * A.y[q];
                A.y[i] = s / __ldcg(A.H + (int64_t)i * m1 + i);
            }
            for (int i = 0; i < k; ++i) A.y[i] *= __ldcg(A.inv_beta + i);
        }
    });
    if (!ok) return;
    const int k = *(volatile int*)&A.st->steps;
    for (int i = threadIdx.x; i < k; i += blockDim.x) s_coef[i] = __ldcg(A.y + i);
    __syncthreads();
    for (int64_t row = r0 + threadIdx.x; row < r1; row += blockDim.x) {
        double zz = 0.0;
        for (int i = 0; i < k; ++i) zz += s_coef[i] * (double)V[(int64_t)i * A.ldv + row];
        if (A.precond == 2) ZC[row] = (T)zz;
        else if (A.precond == 1) A.x[row] += A.dinv[row] * zz;
        else A.x[row] += zz;
    }
    if (A.precond == 2) {
        ok = grid_barrier(A, gs);
        if (!ok) return;
        ilu_sweeps<T>(A, gs, ZC, Z, ok);
        if (!ok) return;
        for (int64_t row = r0 + threadIdx.x; row < r1; row += blockDim.x) A.x[row] += (double)__ldcg(Z + row);
    }
    ok = grid_barrier(A, gs);
    if (!ok) return;
    trace_mark(A, A.m, 1);

    // ---- true residual r = b - A x (FP64) into u_0, ||r||, next-cycle state
    {
        double r2 = 0.0;
        cta_spmv<double, double, double>(A.rp, A.ci, A.val64, A.x, r0, r1, [&](int64_t row, double s) {
            const double r = A.b[row] - s;
            V[row] = (T)r;
            r2 += r * r;
        });
        r2 = warp_sum(r2);
        if (lane32 == 0) red[0][wid] = r2;
        store_partials(A, red, 1);
        grid_reduce_barrier(A, gs, [&] {
            reduce_columns(A, 1, [&](int, double d) { s_tot = d; });
            __syncthreads();
            if (threadIdx.x == 0) {
                const double beta0 = sqrt(s_tot);
                A.beta[0] = beta0;
                A.inv_beta[0] = 1.0 / beta0;
                A.g[0] = beta0;
                volatile DevStatus* st = A.st;
                st->steps = 0;
                st->beta0 = beta0;
                st->resid_est = beta0;
                const bool fin = isfinite(beta0);
                st->nonfinite = fin ? 0 : 1;
                const bool conv = fin && beta0 <= A.scal[0];
                st->converged = conv ? 1 : 0;
                st->done = (conv || !fin || beta0 == 0.0) ? 1 : 0;
            }
        });
    }
    trace_mark(A, A.m, 2);
}

}  // namespace vfv
