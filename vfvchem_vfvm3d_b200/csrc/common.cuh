// Shared device helpers for the vfvgpu kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace vfv {

constexpr int kWarp = 32;

// Deterministic block reduction of a double: warp shuffles in a fixed tree, then warp 0 reduces
// the per-warp partials in warp order. Result valid in thread 0. `red` needs blockDim/32 doubles.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double block_sum(double v, double* red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        s = lane < nw ? red[lane] : 0.0;
        s = warp_sum(s);
    }
    return s;
}

template <typename T>
__device__ __forceinline__ T ldg_stream(const T* p) { return __ldcs(p); }

// Status flags the device writes and the host reads once per restart cycle.
struct DevStatus {
    int32_t done;        // 1 once the Krylov cycle has converged or broken down
    int32_t steps;       // Arnoldi steps completed in the current cycle
    int32_t nonfinite;   // a NaN/Inf was seen in a reduction
    int32_t converged;   // the last true residual met the tolerance
    int32_t total_steps; // Arnoldi steps over the whole solve
    int32_t timeout;     // a bounded grid barrier gave up (the kernel left early)
    double resid_est;    // |g_{j+1}|, the residual-norm estimate after the last step
    double beta0;        // ||r_0|| of the current cycle
    int32_t reorth;      // the current Arnoldi step takes a second Gram-Schmidt pass (DGKS test)
    int32_t unused;
};

}  // namespace vfv
