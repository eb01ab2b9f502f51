// Internal declarations shared by the translation units of libvfvgpu (not part of the C ABI):
// the context and pattern structures behind the opaque handles, device buffers, error helpers,
// and the GMRES entry used by the operator handles.
#pragma once
#include "../../include/vfv_gpu.h"
#include "common.cuh"
#include "host/mesh.hpp"

#include <algorithm>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

using namespace vfv;

// ================================================================ errors / buffers
// the last error of calls without a context (thread-local), defined in api.cu
std::string& vfv_thread_error();

struct vfv_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    DevStatus* h_status = nullptr;  // pinned
    double* h_scalar = nullptr;     // pinned scratch for small reads
    int64_t launches = 0;           // kernels launched by this context (graph nodes counted per replay)
};

// Makes a context's device current for the duration of an entry point and gives the calling
// thread its previous device back afterwards, so one host thread can drive contexts on several
// devices (kernels, allocations and streams of a context all live on its device).
struct DeviceGuard {
    int prev = -1;
    bool switched = false;
    explicit DeviceGuard(const vfv_ctx* ctx) {
        if (ctx && cudaGetDevice(&prev) == cudaSuccess && prev != ctx->device && cudaSetDevice(ctx->device) == cudaSuccess)
            switched = true;
    }
    ~DeviceGuard() {
        if (switched) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

inline int set_err(vfv_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    vfv_thread_error() = msg;
    return code;
}

#define CK(call)                                                                                           \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return set_err(ctx, VFV_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
struct DBuf {  // device buffer, freed with its owner
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t count) {
        release();
        n = count;
        if (count == 0) return cudaSuccess;
        return cudaMalloc(&p, count * sizeof(T));
    }
    cudaError_t upload(const T* h, size_t count, cudaStream_t s) {
        cudaError_t e = alloc(count);
        if (e != cudaSuccess || count == 0) return e;
        e = cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return e;
        return cudaStreamSynchronize(s);
    }
};

inline int grid_for(int64_t threads, int block = 256) { return (int)std::max<int64_t>(1, (threads + block - 1) / block); }


// ================================================================ ILU structure (host-built)
struct IluStruct {
    int order = -1;
    int nlev = 0;
    std::vector<int32_t> lev_ptr;  // [nlev+1] row ranges in the permuted numbering
    std::vector<int32_t> h_perm;   // new -> old
    DBuf<int32_t> d_lev_ptr;       // same, on the device (read by the cycle kernel)
    DBuf<int32_t> perm, rp, ci, dg, src;
    DBuf<double> lu64;
    DBuf<float> lu32;
    DBuf<int> bad;
    uint64_t version64 = ~0ull, version32 = ~0ull;

    // dataflow factorisation (k_ilu0_factor_flow): per-row ready flags holding the epoch of the
    // factorisation that finished the row, the abort word and timeout flag of its bounded waits, and
    // the cooperative grid (0: not set up)
    DBuf<unsigned> ready, flow_state;
    unsigned epoch = 0;
    int flow_grid = 0;

    // single-launch sweeps (k_ilu0_chain): row tasks inside levels (row starts, levels, tasks per
    // level), and per precision a work vector for standalone applies and the claim and completion
    // counters
    DBuf<int32_t> tasks, task_lev, lev_ntask;
    int ntask = 0;
    struct Chain {
        DBuf<unsigned char> work;   // n entries of the precision (standalone applies)
        DBuf<unsigned char> state;  // IluChainState + 2 nlev completion counters
        int grid = 0;
    } chain[2];                     // [0] double, [1] float

    // Jacobi-sweep applies (vfv_gmres_opts::ilu_sweeps): the factor's strictly lower and strictly
    // upper parts as compact CSR arrays and its diagonal, in A's own numbering for the natural
    // ordering (nat64/nat32 hold the factor's values scattered back to A's slots) and in the
    // factor's permuted numbering for the multicolour one
    struct Split {
        bool built = false, delta16 = false;  // delta16: columns stored as int16 offsets from the row
        DBuf<int32_t> lrp, urp;
        DBuf<int16_t> lcd, ucd;
        DBuf<int32_t> lci, uci;
        DBuf<double> lv64, uv64, d64;
        DBuf<float> lv32, uv32, d32;
        DBuf<uint16_t> lvh, uvh;  // half-precision copies of lv32 / uv32 divided by their row scales
        DBuf<float> lsc, usc;     // row scales: the largest magnitude of the row in each triangle
        uint64_t version64 = ~0ull, version32 = ~0ull, version_half = ~0ull;
    } split;
    DBuf<double> nat64;
    DBuf<float> nat32;
    DBuf<unsigned char> sweep_work[2];  // 5 n entries per precision ([0] double, [1] float): standalone sweep applies
};

struct SolverBase {
    virtual ~SolverBase() = default;
};

struct vfv_pattern {
    vfv_ctx* ctx = nullptr;
    int64_t n = 0, nnz = 0, ntrip = 0;
    int spmv_lanes[2] = {4, 4};    // lanes per row of the SpMV for double / float values (autotuned; kSpG by default)
    int spmv_strides[2] = {4, 4};  // strides each lane loads before its gathers (autotuned with the lanes)
    std::vector<int32_t> h_rp, h_ci;
    DBuf<int32_t> rp, ci, diag_pos;
    DBuf<double> val;
    DBuf<float> val32;
    uint64_t version = 0, version32 = ~0ull;
    DBuf<int64_t> slot_ptr, slot_trip;
    DBuf<double> trip_vals;
    std::vector<int64_t> blocks;          // row ranges of the diagonal blocks of a block-diagonal system (may be empty)
    const vfv_pattern* same_as = nullptr;  // a pattern with identical rows/columns (ILU orderings are shared)
    std::map<int, std::unique_ptr<IluStruct>> ilu;
    // solvers by (precision, preconditioner, ILU ordering + 16 x ILU sweeps, restart, engine + 16 if batched)
    std::map<std::tuple<int, int, int, int, int>, std::unique_ptr<SolverBase>> solvers;
    DBuf<double> tmp_b, tmp_x;  // staging for host-pointer solves
};

struct vfv_mesh {
    Mesh m;
    Dual d;
};

// GMRES solve on device arrays (the solver of vfv_solve): cached per pattern and options. batched:
// the pattern's diagonal blocks (p->blocks) are independent meshes, each with its own Krylov
// recurrence and stopping test.
int solve_dev(vfv_ctx* ctx, vfv_pattern* p, const double* b, const double* x0, double* x, const vfv_gmres_opts* o, vfv_solve_info* info,
              bool batched = false);
// the key of the solver cache for these options
std::tuple<int, int, int, int, int> solver_key(const vfv_gmres_opts& o, bool batched);
// per-mesh Arnoldi steps of the last batched solve with these options
bool batch_mesh_steps(const vfv_pattern* p, const vfv_gmres_opts* o, std::vector<int32_t>& steps);
// the Voronoi dual of a mesh's tetrahedra computed on the device of ctx (same arrays, bit for bit,
// as the host build_dual); "" on success (csrc/kernels/dual.cu)
namespace vfv {
std::string build_dual_device(vfv_ctx* ctx, const Mesh& mesh, Dual& d);
}
// argument checks of the reference's LinearGmres constructor and solve options
int check_opts(vfv_ctx* ctx, const vfv_gmres_opts* o);
// transpose of a pattern (tmap: slot in A of every entry of A^T) and the gather of A's values into it
int make_transpose(vfv_ctx* ctx, const vfv_pattern* p, vfv_pattern** out, DBuf<int32_t>& tmap_d);
int gather_transpose_values(vfv_ctx* ctx, const vfv_pattern* p, vfv_pattern* pt, const int32_t* tmap);
