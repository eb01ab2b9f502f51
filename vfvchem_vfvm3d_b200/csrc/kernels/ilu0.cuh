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

namespace vfv {

// ---------------------------------------------------------------- both sweeps in one launch
// The level-per-launch sweeps above pay a launch and a drain per level (20 per apply on the
// 10^6-row heat matrix, ~5 µs each), while a level moves only ~8 MB. Here one launch runs both
// sweeps as a dataflow over row tasks: a task is at most kChainThreads rows of one level, lower
// tasks in level order followed by upper tasks in reverse level order, and CTAs claim tasks from a
// global counter in that order. A thread owns one row: it loads the row's indices and factor
// values, then gathers the solved values it needs, waiting (bounded) for each one that is not
// solved yet. Solved values double as the ready flags: the work vectors start filled with a
// sentinel bit pattern (all ones, a NaN no arithmetic produces), a relaxed load that returns
// anything else is the final value, and a stored result that happens to equal the sentinel is
// replaced by the canonical NaN.
//
// Progress: a task waits only on tasks claimed before it (its lower entries are rows of earlier
// levels, its upper entries rows of later levels, whose upper tasks come first, and the upper task
// of row i needs the lower result of row i). The smallest unfinished claim therefore has every
// input solved and finishes, so the sweeps complete for any number of resident CTAs (no cooperative
// launch needed; kernels on other streams may share the GPU). Every wait is bounded anyway: past
// the poll limit (or 2 s) the waiting thread raises `abort`, records the timeout and every CTA
// leaves.
//
// Work vectors: two pairs (t = lower results, u = upper results, permuted numbering) used by
// alternate launches; a launch refills the other pair with the sentinel as it goes (row i resets
// its own entries), so no separate clearing pass is needed. The last CTA to leave resets the claim
// counter and flips the parity for the next launch.
//
// Results are bit-identical to k_ilu0_level: each row sums its entries in the same order.
constexpr int kChainThreads = 128;

struct IluChainState {
    unsigned claim;      // next task index
    unsigned pad0[31];
    unsigned exited;     // CTAs that have left this launch
    unsigned pad1[31];
    unsigned parity;     // work-vector pair of the next launch
    unsigned abort;      // a bounded wait gave up: every CTA leaves at its next check
    long long poll_limit;  // polls before a wait gives up (set by the host)
    unsigned pad2[28];
};

template <typename T> struct ChainWord;
template <> struct ChainWord<float> {
    using U = uint32_t;
    static constexpr U kSentinel = 0xFFFFFFFFu;
    static constexpr U kCanonNaN = 0x7FFFFFFFu;
};
template <> struct ChainWord<double> {
    using U = unsigned long long;
    static constexpr U kSentinel = 0xFFFFFFFFFFFFFFFFull;
    static constexpr U kCanonNaN = 0x7FF8000000000000ull;
};

__device__ __forceinline__ uint32_t ld_relaxed_gpu(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_gpu(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ void st_relaxed_gpu(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_gpu(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ float word_to(uint32_t b) { return __uint_as_float(b); }
__device__ __forceinline__ double word_to(unsigned long long b) { return __longlong_as_double((long long)b); }
__device__ __forceinline__ uint32_t to_word(float v) { return __float_as_uint(v); }
__device__ __forceinline__ unsigned long long to_word(double v) { return (unsigned long long)__double_as_longlong(v); }

__device__ __forceinline__ unsigned long long chain_clock_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Slow path of a gather: poll until the word is solved and return it. Returns the sentinel itself
// (after raising abort and the timeout flag) when the poll limit or 2 s pass, or when another
// thread has aborted.
template <typename U>
__device__ __noinline__ U chain_wait(const U* p, U sentinel, IluChainState* cs, int* timeout_flag, long long poll_limit) {
    const unsigned long long t0 = chain_clock_ns();
    for (long long it = 1;; ++it) {
        __nanosleep(64);
        const U b = ld_relaxed_gpu(p);
        if (b != sentinel) return b;
        if ((it & 63) == 0 && *(volatile unsigned*)&cs->abort) return sentinel;
        if (it >= poll_limit || ((it & 1023) == 0 && chain_clock_ns() - t0 > 2000000000ull)) {
            *(volatile unsigned*)&cs->abort = 1u;
            *(volatile int*)timeout_flag = 1;
            return sentinel;
        }
    }
}

// s += sum over entries [kb, ke) of lu[k] * x[ci[k]], gathering x from the work vector `xw`
// (waiting for unsolved rows). The first K entries were loaded into c/v before any wait.
template <typename T, int K>
__device__ __forceinline__ bool chain_gather(const int32_t* c, const T* v, int32_t kb, int32_t ke, const int32_t* __restrict__ ci,
                                             const T* __restrict__ lu, const typename ChainWord<T>::U* xw, T& s, IluChainState* cs,
                                             int* timeout_flag, long long poll_limit) {
    using W = ChainWord<T>;
    using U = typename W::U;
    constexpr int G = 4;  // gathers in flight before the first use
#pragma unroll
    for (int q0 = 0; q0 < K; q0 += G) {
        U raw[G];
#pragma unroll
        for (int g = 0; g < G; ++g) raw[g] = c[q0 + g] >= 0 ? ld_relaxed_gpu(xw + c[q0 + g]) : U(0);
#pragma unroll
        for (int g = 0; g < G; ++g) {
            if (c[q0 + g] < 0) continue;
            U b = raw[g];
            if (b == W::kSentinel) {
                b = chain_wait(xw + c[q0 + g], W::kSentinel, cs, timeout_flag, poll_limit);
                if (b == W::kSentinel) return false;
            }
            s += v[q0 + g] * word_to(b);
        }
    }
    for (int32_t k = kb + K; k < ke; ++k) {
        const int32_t col = __ldg(ci + k);
        U b = ld_relaxed_gpu(xw + col);
        if (b == W::kSentinel) {
            b = chain_wait(xw + col, W::kSentinel, cs, timeout_flag, poll_limit);
            if (b == W::kSentinel) return false;
        }
        s += __ldg(lu + k) * word_to(b);
    }
    return true;
}

template <typename T> struct ChainCfg;
template <> struct ChainCfg<float> { static constexpr int K = 16, kMinBlocks = 8; };
template <> struct ChainCfg<double> { static constexpr int K = 12, kMinBlocks = 6; };

// z = (LU)^-1 r over the permuted factor; tasks[ntask + 1] = row starts of the tasks (each inside
// one level); work = 4 vectors of n words (t0, t1, u0, u1). `in` and `out` may alias: only row i
// reads in[perm[i]], before the upper task of row i writes out[perm[i]].
template <typename T>
__global__ void __launch_bounds__(kChainThreads, ChainCfg<T>::kMinBlocks)
    k_ilu0_chain(int32_t ntask, const int32_t* __restrict__ tasks, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                 const int32_t* __restrict__ dg, const T* __restrict__ lu, const int32_t* __restrict__ perm, int64_t n, const T* in,
                 T* out, typename ChainWord<T>::U* work, IluChainState* cs, int* timeout_flag, const DevStatus* __restrict__ st) {
    using W = ChainWord<T>;
    using U = typename W::U;
    constexpr int K = ChainCfg<T>::K;
    const long long poll_limit = cs->poll_limit;
    const int total = 2 * ntask;
    __shared__ int s_task[2];
    __shared__ unsigned s_par;
    __shared__ int s_abort;
    if (threadIdx.x == 0) {
        // A CTA that finds the solve already done (or an earlier launch aborted) claims nothing but
        // still counts itself out below. `done` may be set by a kernel running concurrently on
        // another stream, so CTAs can disagree; the CTAs that do claim keep claiming until every
        // task is taken, so a launch either completes every row or (no claims at all) none.
        const bool ab = *(volatile unsigned*)&cs->abort != 0u;
        const bool skip = ab || (st && *(volatile const int32_t*)&st->done);
        s_par = *(volatile unsigned*)&cs->parity;
        s_task[0] = skip ? total : (int)atomicAdd(&cs->claim, 1u);
        s_abort = ab ? 1 : 0;
    }
    __syncthreads();
    const unsigned par = s_par & 1u;
    U* tcur = work + (int64_t)par * n;
    U* tnxt = work + (int64_t)(1u - par) * n;
    U* ucur = work + (int64_t)(2u + par) * n;
    U* unxt = work + (int64_t)(3u - par) * n;
    int cur = 0;
    bool ok = true;
    for (;;) {
        const int task = s_task[cur];
        if (task >= total || s_abort) break;
        if (threadIdx.x == 0) s_task[cur ^ 1] = (int)atomicAdd(&cs->claim, 1u);  // next claim, in flight during this task
        const bool lower = task < ntask;
        const int tk = lower ? task : total - 1 - task;
        const int32_t r0 = __ldg(tasks + tk), r1 = __ldg(tasks + tk + 1);
        const int32_t i = r0 + (int32_t)threadIdx.x;
        if (i < r1 && ok) {
            const int32_t d = __ldg(dg + i);
            const int32_t kb = lower ? __ldg(rp + i) : d + 1;
            const int32_t ke = lower ? d : __ldg(rp + i + 1);
            const int32_t pi = __ldg(perm + i);
            int32_t c[K];
            T v[K];
#pragma unroll
            for (int q = 0; q < K; ++q) {
                c[q] = kb + q < ke ? __ldg(ci + kb + q) : -1;
                v[q] = kb + q < ke ? __ldg(lu + kb + q) : T(0);
            }
            T s = T(0);
            if (lower) {
                const T rhs = in[pi];
                tnxt[i] = W::kSentinel;  // the next launch's pair: nobody reads it during this one
                unxt[i] = W::kSentinel;
                ok = chain_gather<T, K>(c, v, kb, ke, ci, lu, tcur, s, cs, timeout_flag, poll_limit);
                if (ok) {
                    U r = to_word(rhs - s);
                    if (r == W::kSentinel) r = W::kCanonNaN;
                    st_relaxed_gpu(tcur + i, r);
                }
            } else {
                const T diag = __ldg(lu + d);
                U rb = ld_relaxed_gpu(tcur + i);
                if (rb == W::kSentinel) rb = chain_wait(tcur + i, W::kSentinel, cs, timeout_flag, poll_limit);
                ok = rb != W::kSentinel;
                if (ok) ok = chain_gather<T, K>(c, v, kb, ke, ci, lu, ucur, s, cs, timeout_flag, poll_limit);
                if (ok) {
                    const T x = (word_to(rb) - s) / diag;
                    U r = to_word(x);
                    if (r == W::kSentinel) r = W::kCanonNaN;
                    st_relaxed_gpu(ucur + i, r);
                    out[pi] = x;
                }
            }
        }
        if (threadIdx.x == 0 && *(volatile unsigned*)&cs->abort) s_abort = 1;
        __syncthreads();
        cur ^= 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned e = atomicAdd(&cs->exited, 1u);
        if (e == gridDim.x - 1) {  // every CTA has stopped claiming: reset for the next launch
            const unsigned claimed = *(volatile unsigned*)&cs->claim;
            cs->claim = 0u;
            cs->exited = 0u;
            if (claimed > 0u) cs->parity = par ^ 1u;  // every row ran and refilled the other pair
            __threadfence();
        }
    }
}

}  // namespace vfv
