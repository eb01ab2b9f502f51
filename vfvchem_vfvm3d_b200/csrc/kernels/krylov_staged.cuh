// Gram-Schmidt passes with the basis tile staged in shared memory (sm_100a).
//
// A block owns kStR consecutive rows (one per thread). At the start of a pass every thread issues
// asynchronous copies (cp.async, one element per basis vector) of its row of every basis vector
// into shared memory, so the whole tile of the basis — nvec x kStR values, 26 KB (FP32) / 51 KB
// (FP64) at nvec = 51 — is in flight at once instead of a few loads per thread between dependent
// reductions. The tile is then used from shared memory:
//   * the update w -= sum_i c_i u_i (per row, i in order: the same arithmetic as the register
//     kernels);
//   * the dots <u_i, w> over the tile: warp q of the block owns vectors i = q, q + 4, ...; lane l
//     sums rows l, l + 32, l + 64, l + 96, then a fixed shuffle tree gives the tile's partial, so a
//     pass costs 5 shuffles per vector per warp instead of 5 per vector per thread;
//   * the second CGS pass (update followed by dots) reads the basis from DRAM once, not twice.
// The cross-tile sums are k_dots_finish's (or, for a batch, k_bdots_finish's per mesh).
//
// `Map` gives a block its rows, its coefficient offset and whether it runs at all: one system
// (uniform tiles, global done flag) or a batch of meshes (tiles inside meshes, per-mesh done flags).
#pragma once
#include "krylov_batch.cuh"

namespace vfv {

constexpr int kStR = 128;  // rows per tile = threads per block of the staged passes

struct SingleMap {
    int64_t n;
    const DevStatus* st;
    __device__ __forceinline__ bool block(int b, int64_t& r0, int64_t& r1, int64_t& coff) const {
        if (st->done) return false;
        r0 = (int64_t)b * kStR;
        r1 = r0 + kStR < n ? r0 + kStR : n;
        coff = 0;
        return true;
    }
};

struct BatchMap {
    const int64_t* tile_row;
    const int32_t* tile_mesh;
    const MeshStat* ms;
    const DevStatus* st;
    __device__ __forceinline__ bool block(int b, int64_t& r0, int64_t& r1, int64_t& coff) const {
        if (st->done) return false;
        const int m = tile_mesh[b];
        if (ms[m].done) return false;
        r0 = tile_row[b];
        r1 = tile_row[b + 1];
        coff = (int64_t)m * kMaxBasis;
        return true;
    }
};

template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst_smem, const T* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    if constexpr (sizeof(T) == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// This thread's row of u_0 .. u_{nvec-1} into sU[i][threadIdx.x] (zeros past the last row).
template <typename T>
__device__ __forceinline__ void stage_rows(T* sU, const T* V, int64_t ldv, int nvec, int64_t row, bool in) {
    if (in) {
        for (int i = 0; i < nvec; ++i) cp_async_elem(sU + i * kStR + threadIdx.x, V + (int64_t)i * ldv + row);
    } else {
        for (int i = 0; i < nvec; ++i) sU[i * kStR + threadIdx.x] = T(0);
    }
}

// Tile partial dots <u_i, w> (sW = this tile's w in double, zero past the last row) into part[i][b].
template <typename T>
__device__ __forceinline__ void tile_dots(const T* sU, const double* sW, int nvec, double* part, int nparts, int b) {
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    constexpr int kWarps = kStR / 32;
    for (int i = wq; i < nvec; i += kWarps) {
        const T* u = sU + i * kStR;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < kStR / 32; ++k) s += (double)u[lane + 32 * k] * sW[lane + 32 * k];
        s = warp_sum(s);
        if (lane == 0) part[(int64_t)i * nparts + b] = s;
    }
}

// First CGS pass: partial dots of the basis with w.
template <typename T, typename Map>
__global__ void __launch_bounds__(kStR) k_mdot_s(Map M, const T* __restrict__ V, int64_t ldv, const T* __restrict__ w, int nvec,
                                                 double* __restrict__ part, int nparts) {
    extern __shared__ __align__(16) unsigned char st_smem[];
    __shared__ double sW[kStR];
    int64_t r0, r1, coff;
    if (!M.block(blockIdx.x, r0, r1, coff)) return;
    T* sU = reinterpret_cast<T*>(st_smem);
    const int64_t row = r0 + threadIdx.x;
    const bool in = row < r1;
    stage_rows(sU, V, ldv, nvec, row, in);
    sW[threadIdx.x] = in ? (double)w[row] : 0.0;
    cp_async_wait_all();
    __syncthreads();
    tile_dots(sU, sW, nvec, part, nparts, blockIdx.x);
}

// w <- win - sum_i coef_i u_i, then (FINAL == false) the second pass's partial dots, or
// (FINAL == true) the tile's ||w||^2 into part[b]; with LAST (one system) the last block to finish
// also completes the Hessenberg column, the Givens rotation and the convergence test of step j.
template <typename T, typename Map, bool FINAL, bool LAST>
__global__ void __launch_bounds__(kStR) k_update_s(Map M, KrylovDev K, const T* __restrict__ V, int64_t ldv, const T* win, T* w, int nvec,
                                                   const double* __restrict__ coef, double* part, int nparts, int j) {
    extern __shared__ __align__(16) unsigned char st_smem[];
    __shared__ double sW[kStR];
    __shared__ double s_coef[kMaxBasis];
    __shared__ double red[kStR / 32];
    int64_t r0, r1, coff;
    if (!M.block(blockIdx.x, r0, r1, coff)) return;
    T* sU = reinterpret_cast<T*>(st_smem);
    const int64_t row = r0 + threadIdx.x;
    const bool in = row < r1;
    stage_rows(sU, V, ldv, nvec, row, in);
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) s_coef[i] = coef[coff + i];
    const double wi = in ? (double)win[row] : 0.0;
    cp_async_wait_all();
    __syncthreads();
    double acc = 0.0;
    for (int i = 0; i < nvec; ++i) acc += s_coef[i] * (double)sU[i * kStR + threadIdx.x];
    double nvd = 0.0;
    if (in) {
        const T nv = (T)(wi - acc);
        w[row] = nv;
        nvd = (double)nv;
    }
    if (!FINAL) {
        sW[threadIdx.x] = nvd;
        __syncthreads();
        tile_dots(sU, sW, nvec, part, nparts, blockIdx.x);
        return;
    }
    const double bs = block_sum(nvd * nvd, red);
    if (!LAST) {
        if (threadIdx.x == 0) part[blockIdx.x] = bs;
        return;
    }
    if (threadIdx.x == 0) publish_partial(part + blockIdx.x, bs);
    if (!last_block_arrive(K.counter + 3)) return;
    const double tot = reduce_partials(part, gridDim.x, red);
    if (threadIdx.x == 0) {
        K.counter[3] = 0u;
        finish_column(K, j, tot);
    }
}

}  // namespace vfv
