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

#include <cuda_fp16.h>

namespace vfv {

// Programmatic dependent launch: let the next kernel of the stream start its prologue / wait until
// the previous kernel has finished and its writes are visible.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// One level of the IKJ factorisation, a thread per row (rows of one level never touch each other):
// for wide levels (the multicolour ordering's ~10^5-row colours), where a thread per row already
// fills the GPU and the rows are too long for the warp kernel's staging.
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

// The same level, one warp per row, for narrow levels (the natural ordering's ~1,500-row levels).
// Lane l holds entry l of row i. Every pivot row k of row i belongs to an earlier level and is
// final. Before waiting for the previous level, the warp stages the structure of row i's pivot rows
// (upper columns in shared memory) and each lane finds, per pivot row, the entry in its own column
// (the merge of the serial loop, as a column match across the lanes); these cannot change. After
// the wait, one round of independent loads brings the pivots and the matched values, and the
// eliminations run in the serial IKJ order: for each lower entry t in turn, l_it = a_it / u_kk, and
// the later entry matching row k's upper part subtracts l_it times it (a thread per row walking the
// merges was 5x slower on the 692 natural levels of the 10^6-row heat matrix). Rows longer than a
// warp, or with more lower entries or longer pivot rows than the staging holds, run the serial loop
// on lane 0. Levels are chained with programmatic dependent launch.
constexpr int kFacWarps = 8;  // rows per block
constexpr int kFacLow = 16;   // lower entries of a row staged
constexpr int kFacUp = 24;    // upper entries of each pivot row staged

struct FacStage {  // one warp's staging: the pivot rows' indices, diagonal slots, upper lengths and columns
    int32_t col[kFacLow][kFacUp];
    int32_t dk[kFacLow], len[kFacLow], k[kFacLow];
};

__device__ __forceinline__ unsigned ld_relaxed_gpu_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_gpu_u32(unsigned* p, unsigned v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ unsigned long long flow_clock_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Row readiness of the dataflow factorisation (k_ilu0_factor_flow): ready[k] == epoch once row k is
// final. Waits poll with relaxed loads (one fence after the last one, by the caller); a wait gives up
// after poll_limit polls or 2 s, raising *abort (which every waiting warp checks) and *timeout_flag.
struct FlowSync {
    unsigned* ready;
    unsigned epoch;
    unsigned* abort;
    int* timeout_flag;
    long long poll_limit;
    // warp-wide: lane l waits for row k_l when has_l (every lane calls it); each lane that waited
    // fences once after its last poll. False (on every lane) when the waits gave up.
    __device__ bool wait_warp(bool has, int32_t k) const {
        const unsigned full = 0xffffffffu;
        bool rdy = !has || ld_relaxed_gpu_u32(ready + k) == epoch;
        if (!__all_sync(full, rdy)) {
            const unsigned long long t0 = flow_clock_ns();
            for (long long it = 1;; ++it) {
                if (it > 8) __nanosleep(64);
                if (!rdy) rdy = ld_relaxed_gpu_u32(ready + k) == epoch;
                if (__all_sync(full, rdy)) break;
                int give_up = 0;
                if ((threadIdx.x & 31) == 0) {
                    if ((it & 15) == 0 && *(volatile unsigned*)abort) give_up = 1;
                    else if (it >= poll_limit || ((it & 255) == 0 && flow_clock_ns() - t0 > 2000000000ull)) {
                        atomicExch(abort, 1u);
                        *(volatile int*)timeout_flag = 1;
                        give_up = 1;
                    }
                }
                if (__shfl_sync(full, give_up, 0)) return false;
            }
        }
        if (has) fence_acq_rel_gpu();
        __syncwarp(full);
        return true;
    }
    __device__ bool wait(int32_t k) const {
        if (ld_relaxed_gpu_u32(ready + k) == epoch) return true;
        const unsigned long long t0 = flow_clock_ns();
        for (long long it = 1;; ++it) {
            if (it > 8) __nanosleep(64);
            if (ld_relaxed_gpu_u32(ready + k) == epoch) return true;
            if ((it & 15) == 0 && *(volatile unsigned*)abort) return false;
            if (it >= poll_limit || ((it & 255) == 0 && flow_clock_ns() - t0 > 2000000000ull)) {
                atomicExch(abort, 1u);
                *(volatile int*)timeout_flag = 1;
                return false;
            }
        }
    }
};

// Factors row i (one warp). FLOW: lane t waits for pivot row t through fs (values then read from
// L2, past the SM's L1), and the row is published in ready[] when done; otherwise the previous level
// has finished (programmatic dependent launch). False when a wait gave up.
template <bool FLOW>
__device__ __forceinline__ bool factor_row_warp(int32_t i, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                const int32_t* __restrict__ dg, double* a, int* __restrict__ bad, FacStage& sg,
                                                const FlowSync& fs) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    auto piv_ld = [](const double* p) { return FLOW ? __ldcg(p) : *p; };
    const int32_t b = rp[i], e = rp[i + 1], d = dg[i];
    const int32_t len = e - b, nl = d - b;
    bool ok = len <= 32 && nl <= kFacLow;
    if (ok && lane < nl) {
        const int32_t k = ci[b + lane];
        const int32_t dk = dg[k], ul = rp[k + 1] - dk - 1;
        sg.k[lane] = k;
        sg.dk[lane] = dk;
        sg.len[lane] = ul;
        if (ul > kFacUp) ok = false;
    }
    ok = __all_sync(full, ok);
    const int32_t c = ok && lane < len ? ci[b + lane] : -1;
    double v = ok && lane < len ? a[b + lane] : 0.0;
    // slot[t]: the slot of pivot row t's entry in this lane's column (-1: none). Structure only, so
    // it is found before the wait; the eliminations after it are then one division and at most one
    // multiply-subtract per pivot.
    int32_t slot[kFacLow];
#pragma unroll
    for (int t = 0; t < kFacLow; ++t) slot[t] = -1;
    if (ok) {
        __syncwarp(full);
        for (int idx = lane; idx < nl * kFacUp; idx += 32) {
            const int t = idx / kFacUp, u = idx - t * kFacUp;
            if (u < sg.len[t]) sg.col[t][u] = ci[sg.dk[t] + 1 + u];
        }
        __syncwarp(full);
#pragma unroll
        for (int t = 0; t < kFacLow; ++t) {
            if (t < nl && lane > t && lane < len) {
                const int ul = sg.len[t];
                for (int u = 0; u < ul; ++u)
                    if (sg.col[t][u] == c) {
                        slot[t] = sg.dk[t] + 1 + u;
                        break;
                    }
            }
        }
    }
    if constexpr (FLOW) {
        // lane t waits for pivot row t; all pivot loads come after every waiting lane's fence
        const bool has = ok && lane < nl;
        if (!fs.wait_warp(has, has ? sg.k[lane] : 0)) return false;
    } else {
        pdl_launch_dependents();
        pdl_wait();
    }
    if (!ok) {  // the serial IKJ loop on lane 0
        int go = 1;
        if (lane == 0) {
            for (int32_t kk = b; kk < d; ++kk) {
                const int32_t k = ci[kk];
                if (FLOW) {
                    if (!fs.wait(k)) {
                        go = 0;
                        break;
                    }
                    fence_acq_rel_gpu();
                }
                const double ukk = piv_ld(a + dg[k]);
                if (ukk == 0.0) {
                    *bad = 1;
                    break;
                }
                const double lik = a[kk] / ukk;
                a[kk] = lik;
                int32_t p = kk + 1, q = dg[k] + 1;
                const int32_t e_k = rp[k + 1];
                while (p < e && q < e_k) {
                    const int32_t cp = ci[p], cq = ci[q];
                    if (cp == cq) {
                        a[p] -= lik * piv_ld(a + q);
                        ++p;
                        ++q;
                    } else if (cp < cq) {
                        ++p;
                    } else {
                        ++q;
                    }
                }
            }
            if (go && a[d] == 0.0) *bad = 1;
        }
        if (!__shfl_sync(full, go, 0)) return false;
    } else {
        // lane t holds pivot u_kk of pivot row t; every lane its matched pivot-row values (one round
        // of independent loads), then the serial IKJ order: l_it = a_it / u_kk, and the later entry
        // matching row k's upper part subtracts l_it times it
        const double ukk = lane < nl ? piv_ld(a + sg.dk[lane]) : 1.0;
        double mv[kFacLow];
#pragma unroll
        for (int t = 0; t < kFacLow; ++t) mv[t] = slot[t] >= 0 ? piv_ld(a + slot[t]) : 0.0;
        const bool zero = __any_sync(full, lane < nl && ukk == 0.0);
        if (!zero) {
#pragma unroll
            for (int t = 0; t < kFacLow; ++t) {
                if (t < nl) {
                    const double lik = __shfl_sync(full, v, t) / __shfl_sync(full, ukk, t);
                    if (lane == t) v = lik;
                    if (slot[t] >= 0) v -= lik * mv[t];
                }
            }
        }
        if (zero) {
            if (lane == 0) *bad = 1;
        } else {
            if (lane < len) a[b + lane] = v;
            if (lane == nl && v == 0.0) *bad = 1;
        }
    }
    if constexpr (FLOW) {  // publish: the warp's stores, one fence, then the row's flag
        __syncwarp(full);
        if (lane == 0) {
            fence_acq_rel_gpu();
            st_relaxed_gpu_u32(fs.ready + i, fs.epoch);
        }
    }
    return true;
}

__global__ void __launch_bounds__(32 * kFacWarps) k_ilu0_factor_level_warp(int32_t r0, int32_t r1, const int32_t* __restrict__ rp,
                                                                            const int32_t* __restrict__ ci, const int32_t* __restrict__ dg,
                                                                            double* __restrict__ a, int* __restrict__ bad) {
    __shared__ FacStage s_stage[kFacWarps];
    const int w = threadIdx.x >> 5;
    const int32_t i = r0 + (int32_t)blockIdx.x * kFacWarps + w;
    if (i >= r1) return;  // whole warps leave together
    factor_row_warp<false>(i, rp, ci, dg, a, bad, s_stage[w], FlowSync{});
}

// The whole factorisation in one launch, for orderings with many narrow levels (the natural order:
// 692 levels on the 10^6-row heat matrix, ~12 us each as separate launches). Rows are in the
// permuted numbering, where every pivot row of row i has a smaller index. Warp g of the W warps of
// the grid factors rows g, g + W, g + 2W, ... in increasing order and, instead of waiting for a whole
// level, waits only for its row's pivot rows (ready[k] == epoch). Progress needs every warp
// resident (the smallest unfinished row always has all its pivots finished, and its warp has
// finished all its earlier rows), hence a cooperative launch. Each row's arithmetic is
// factor_row_warp's, so the factor is bit-identical to the level-by-level one.
__global__ void __launch_bounds__(32 * kFacWarps) k_ilu0_factor_flow(int32_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                                     const int32_t* __restrict__ dg, double* a, int* __restrict__ bad,
                                                                     FlowSync fs) {
    __shared__ FacStage s_stage[kFacWarps];
    const int w = threadIdx.x >> 5;
    const int32_t nw = (int32_t)gridDim.x * kFacWarps;
    for (int32_t i = (int32_t)blockIdx.x * kFacWarps + w; i < n; i += nw)
        if (!factor_row_warp<true>(i, rp, ci, dg, a, bad, s_stage[w], fs)) return;
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

// ---------------------------------------------------------------- Jacobi sweeps of the factors
// The triangular solves of ILU(0) replaced by a fixed number of Jacobi sweeps of each factor
// (Anzt, Chow & Dongarra, "Iterative sparse triangular solves for preconditioning", Euro-Par 2015):
// with L = I + N (N strictly lower) and U = D + S (S strictly upper),
//     u^0 = y,        u^k = y - N u^(k-1)            (k = 1..sweeps)
//     w^0 = D^-1 u,   w^k = D^-1 (u - S w^(k-1))     (k = 1..sweeps, u = u^sweeps)
// and z = w^sweeps. Every row of a sweep is independent, so a sweep is one bandwidth-bound launch
// over all rows (an SpMV over one triangle) instead of one latency-bound launch per level; the
// operator is linear and fixed, so flexible and plain GMRES both accept it.
//
// Storage: N and S as separate compact CSR arrays (a sweep streams only its own triangle's bytes;
// inside A's rows the two halves share DRAM sectors), columns as 16-bit offsets from the row when
// the pattern's bandwidth allows (TC = int16_t; int32_t absolute columns otherwise), and D apart.
// G lanes per row, sweep_k(G) entries per lane loaded before the programmatic-dependent-launch wait (the
// factor does not change between sweeps); lane partial sums are combined by a butterfly (fixed order).
constexpr int kSwBlock = 256;
__host__ __device__ constexpr int sweep_k(int G) { return G >= 4 ? 2 : 8 / G; }  // ~8 entries of a row held before the wait

template <typename TC>
__device__ __forceinline__ int32_t sweep_col(TC c, int32_t row) {
    if constexpr (sizeof(TC) == 2) return row + (int32_t)c;
    else return (int32_t)c;
}

// LOWER: next[i] = rhs[i] - sum_k val[k] prev[col k]; w0 (if set) also gets next[i] / d[i].
// UPPER: w[i] = (rhs[i] - sum_k val[k] prev[col k]) / d[i], stored to next[i], or to out[perm[i]]
//        (out[i] without perm) on the last sweep (out set).
// TV: the stored value type, T or (for float) __half; half values are stored divided by their row's
// largest magnitude in that triangle, rs[i], and the row's sum is multiplied back by it.
template <typename T>
__device__ __forceinline__ T sweep_val(T v) {
    return v;
}
__device__ __forceinline__ float sweep_val(__half v) { return __half2float(v); }

template <typename T, typename TC, bool LOWER, int G, typename TV = T>
__global__ void __launch_bounds__(kSwBlock) k_ilu0_sweep(int32_t n, const int32_t* __restrict__ rowp, const TC* __restrict__ cols,
                                                         const TV* __restrict__ val, const float* __restrict__ rs, const T* __restrict__ d,
                                                         const int32_t* __restrict__ perm, const T* rhs, const T* prev, T* next, T* w0,
                                                         T* out, const DevStatus* __restrict__ st) {
    const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int32_t i = (int32_t)(gt / G);
    const int lane = (int)(gt & (G - 1));
    int32_t kb = 0, ke = 0;
    constexpr int kSwK = sweep_k(G);
    int32_t c[kSwK];
    T v[kSwK];
    if (i < n) {
        kb = __ldg(rowp + i);
        ke = __ldg(rowp + i + 1);
    }
#pragma unroll
    for (int q = 0; q < kSwK; ++q) {
        const int32_t k = kb + lane + q * G;
        c[q] = k < ke ? sweep_col<TC>(__ldg(cols + k), i) : -1;
        v[q] = k < ke ? (T)sweep_val(__ldg(val + k)) : T(0);
    }
    pdl_launch_dependents();
    pdl_wait();
    if (st && st->done) return;  // uniform over the grid
    T s = T(0);
#pragma unroll
    for (int q = 0; q < kSwK; ++q)
        if (c[q] >= 0) s += v[q] * prev[c[q]];
    for (int32_t k = kb + lane + kSwK * G; k < ke; k += G) s += (T)sweep_val(__ldg(val + k)) * prev[sweep_col<TC>(__ldg(cols + k), i)];
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, G);
    if (i >= n || lane != 0) return;
    if (rs) s *= (T)__ldg(rs + i);
    if (LOWER) {
        const T u = rhs[i] - s;
        next[i] = u;
        if (w0) w0[i] = u / __ldg(d + i);
    } else {
        const T w = (rhs[i] - s) / __ldg(d + i);
        if (out) out[perm ? __ldg(perm + i) : i] = w;
        else next[i] = w;
    }
}

// Values of the compact triangles from the factor's rows (thread per row): the strictly lower
// entries of row i to lv[lrp[i]..], the strictly upper ones to uv[urp[i]..], the diagonal to dv[i].
template <typename T>
__global__ void k_split_vals(int32_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ dg, const T* __restrict__ lu,
                             const int32_t* __restrict__ lrp, const int32_t* __restrict__ urp, T* __restrict__ lv, T* __restrict__ uv,
                             T* __restrict__ dv) {
    const int32_t i = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= n) return;
    const int32_t b = rp[i], dd = dg[i], e = rp[i + 1];
    int32_t o = lrp[i];
    for (int32_t k = b; k < dd; ++k) lv[o++] = lu[k];
    dv[i] = lu[dd];
    o = urp[i];
    for (int32_t k = dd + 1; k < e; ++k) uv[o++] = lu[k];
}

// y[i] = in[perm[i]]: the right-hand side in the factor's numbering (first step of a sweep apply)
template <typename T>
__global__ void k_perm_gather(int32_t n, const int32_t* __restrict__ perm, const T* in, T* __restrict__ y) {
    pdl_launch_dependents();
    const int32_t i = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    if (i < n) y[i] = in[__ldg(perm + i)];
}

// Half-precision copies of the compact triangles' float values, row-scaled: scale[i] = the row's
// largest magnitude in the triangle (1 for an empty or all-zero row), h[k] = half(v[k] / scale[i])
// rounded to nearest, so every stored value lies in [-1, 1] whatever the matrix's scaling.
__global__ void k_half_rows(int32_t n, const int32_t* __restrict__ rowp, const float* __restrict__ v, __half* __restrict__ h,
                            float* __restrict__ scale) {
    const int32_t i = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= n) return;
    const int32_t b = rowp[i], e = rowp[i + 1];
    float m = 0.f;
    for (int32_t k = b; k < e; ++k) m = fmaxf(m, fabsf(v[k]));
    const float sc = m > 0.f ? m : 1.f;
    scale[i] = sc;
    for (int32_t k = b; k < e; ++k) h[k] = __float2half_rn(v[k] / sc);
}

// Factor values back in A's own slot order (natural ordering): out[src[k]] = lu[k].
template <typename T>
__global__ void k_scatter_vals(int64_t nnz, const int32_t* __restrict__ src, const T* __restrict__ lu, T* __restrict__ out) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nnz) out[src[k]] = lu[k];
}

}  // namespace vfv

namespace vfv {

// ---------------------------------------------------------------- both sweeps in one launch
// The level-per-launch sweeps above pay a launch and a drain per level (20 per apply on the
// 10^6-row heat matrix). Here one launch runs both sweeps: a task is at most kChainThreads rows of
// one level; CTAs claim tasks from a global counter, lower tasks in level order, then upper tasks
// in reverse level order. Each level has a completion counter; a task first loads everything that
// does not depend on the sweep (its rows' indices, factor values, right-hand side), then one thread
// of the CTA waits (bounded, with backoff) until the level it depends on has all its tasks counted,
// and then the rows gather their solved neighbours from L2 (ld.global.cg: solved values are written
// during the launch, so no L1 copy may be used). One polling thread per CTA keeps the waiting cheap.
//
// Progress: a task waits only on levels whose tasks were all claimed before it (lower level l on
// lower level l-1; upper level L-1 on lower level L-1, which completes after every lower level;
// upper level l on upper level l+1), so the smallest unfinished claim always has its inputs and
// finishes, whatever number of CTAs is resident (no cooperative launch; kernels on other streams
// may share the GPU). Every wait is bounded anyway: past the poll limit (or 2 s) the waiting thread
// raises `abort`, records the timeout, and every CTA leaves. The last CTA to leave zeroes the
// counters for the next launch.
//
// Results are bit-identical to k_ilu0_level: same work vector use (t in place) and the same
// summation order per row.
constexpr int kChainThreads = 128;

struct IluChainState {
    unsigned claim;        // next task index
    unsigned pad0[31];
    unsigned exited;       // CTAs that have left this launch
    unsigned pad1[31];
    unsigned abort;        // a bounded wait gave up: every CTA leaves at its next check
    unsigned pad2;
    long long poll_limit;  // polls before a wait gives up (set by the host)
    unsigned pad3[28];
    // followed by 2 * nlev completion counters: [phase * nlev + level], phase 0 lower, 1 upper
};

__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ unsigned long long chain_clock_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits until *cnt reaches target (one thread). False when the poll limit or 2 s pass (after
// raising abort and the timeout flag) or when another CTA has aborted.
__device__ __noinline__ bool chain_wait_count(const unsigned* cnt, unsigned target, IluChainState* cs, int* timeout_flag,
                                              long long poll_limit) {
    if (ld_relaxed_u32(cnt) >= target) return true;
    const unsigned long long t0 = chain_clock_ns();
    unsigned sleep = 32;
    for (long long it = 1;; ++it) {
        __nanosleep(sleep);
        if (sleep < 1024) sleep <<= 1;
        if (ld_relaxed_u32(cnt) >= target) return true;
        if ((it & 15) == 0 && ld_relaxed_u32(&cs->abort)) return false;
        if (it >= poll_limit || ((it & 255) == 0 && chain_clock_ns() - t0 > 2000000000ull)) {
            *(volatile unsigned*)&cs->abort = 1u;
            *(volatile int*)timeout_flag = 1;
            return false;
        }
    }
}

template <typename T> struct ChainCfg;
template <> struct ChainCfg<float> { static constexpr int K = 16, kMinBlocks = 8; };
template <> struct ChainCfg<double> { static constexpr int K = 16, kMinBlocks = 6; };

// z = (LU)^-1 r over the permuted factor. tasks[ntask + 1]: row starts of the tasks (each inside
// one level); task_lev[ntask]: their levels; lev_ntask[nlev]: tasks per level. t is the work vector
// (n entries, may not alias r or z; r and z may alias: only row i reads r[perm[i]], before the
// upper task of row i writes z[perm[i]]).
template <typename T>
__global__ void __launch_bounds__(kChainThreads, ChainCfg<T>::kMinBlocks)
    k_ilu0_chain(int32_t ntask, int32_t nlev, const int32_t* __restrict__ tasks, const int32_t* __restrict__ task_lev,
                 const int32_t* __restrict__ lev_ntask, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                 const int32_t* __restrict__ dg, const T* __restrict__ lu, const int32_t* __restrict__ perm, const T* in, T* t, T* out,
                 IluChainState* cs, int* timeout_flag, const DevStatus* __restrict__ st) {
    constexpr int K = ChainCfg<T>::K;
    unsigned* done = reinterpret_cast<unsigned*>(cs + 1);
    const long long poll_limit = cs->poll_limit;
    const int total = 2 * ntask;
    __shared__ int s_task[2];
    __shared__ int s_go;
    if (threadIdx.x == 0) {
        // A CTA that finds the solve already done (or an earlier launch aborted) claims nothing but
        // still counts itself out below. `done` may be set by a kernel running concurrently on
        // another stream, so CTAs can disagree; the CTAs that do claim keep claiming until every
        // task is taken, so a launch completes every row or (no claims at all) none.
        const bool skip = ld_relaxed_u32(&cs->abort) != 0u || (st && *(volatile const int32_t*)&st->done);
        s_task[0] = skip ? total : (int)atomicAdd(&cs->claim, 1u);
    }
    __syncthreads();
    int cur = 0;
    for (;;) {
        const int task = s_task[cur];
        if (task >= total) break;
        if (threadIdx.x == 0) s_task[cur ^ 1] = (int)atomicAdd(&cs->claim, 1u);  // next claim, in flight during this task
        const bool lower = task < ntask;
        const int tk = lower ? task : total - 1 - task;
        const int lev = __ldg(task_lev + tk);
        const int32_t r0 = __ldg(tasks + tk), r1 = __ldg(tasks + tk + 1);
        const int32_t i = r0 + (int32_t)threadIdx.x;
        const bool row = i < r1;
        int32_t kb = 0, ke = 0, d = 0, pi = 0;
        int32_t c[K];
        T v[K];
        T rhs = T(0), diag = T(1);
        if (row) {
            d = __ldg(dg + i);
            kb = lower ? __ldg(rp + i) : d + 1;
            ke = lower ? d : __ldg(rp + i + 1);
            pi = __ldg(perm + i);
            if (lower) rhs = in[pi];
            else diag = __ldg(lu + d);
#pragma unroll
            for (int q = 0; q < K; ++q) {
                c[q] = kb + q < ke ? __ldg(ci + kb + q) : -1;
                v[q] = kb + q < ke ? __ldg(lu + kb + q) : T(0);
            }
        }
        if (threadIdx.x == 0) {
            bool ok = true;
            if (lower && lev > 0) ok = chain_wait_count(done + lev - 1, (unsigned)__ldg(lev_ntask + lev - 1), cs, timeout_flag, poll_limit);
            else if (!lower && lev == nlev - 1) ok = chain_wait_count(done + lev, (unsigned)__ldg(lev_ntask + lev), cs, timeout_flag, poll_limit);
            else if (!lower) ok = chain_wait_count(done + nlev + lev + 1, (unsigned)__ldg(lev_ntask + lev + 1), cs, timeout_flag, poll_limit);
            s_go = ok ? 1 : 0;
        }
        __syncthreads();
        if (!s_go) break;
        if (row) {
            if (!lower) rhs = __ldcg(t + i);
            T s = T(0);
#pragma unroll
            for (int q = 0; q < K; ++q)
                if (c[q] >= 0) s += v[q] * __ldcg(t + c[q]);
            for (int32_t k = kb + K; k < ke; ++k) s += __ldg(lu + k) * __ldcg(t + __ldg(ci + k));
            if (lower) {
                t[i] = rhs - s;
            } else {
                const T x = (rhs - s) / diag;
                t[i] = x;
                out[pi] = x;
            }
        }
        __syncthreads();  // this task's rows are stored (and s_task[cur ^ 1] is visible)
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(done + (lower ? 0 : nlev) + lev, 1u);
        }
        cur ^= 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned e = atomicAdd(&cs->exited, 1u);
        if (e == gridDim.x - 1) {  // every CTA has stopped claiming and counting: reset for the next launch
            cs->claim = 0u;
            cs->exited = 0u;
            for (int l = 0; l < 2 * nlev; ++l) done[l] = 0u;
            __threadfence();
        }
    }
}

}  // namespace vfv
