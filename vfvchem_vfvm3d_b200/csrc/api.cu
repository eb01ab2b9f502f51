// C ABI of libvfvgpu: contexts, sparse patterns, ILU(0) orderings and the graph-captured GMRES
// driver. The operator handles live in heat_api.cu, transport_api.cu, flow_api.cu and mesh_api.cu;
// host orchestration only, the kernels live in kernels/*.
//
// Reference interfaces mirrored (src/linear/linear_base.rs:5-10, src/linear/linear_gmres.rs:8-85):
//   update_sparse -> vfv_pattern_from_triplets (sorted de-duplicated pattern + slot map, once)
//   build_matrix  -> vfv_values_from_triplets  (device scatter summing duplicates in push order)
//   solve_matrix  -> vfv_solve                 (restarted right-preconditioned GMRES, warm start)
#include "internal.cuh"
#include "kernels/adjoint.cuh"
#include "kernels/assemble.cuh"
#include "kernels/ilu0.cuh"
#include "kernels/gmres_cycle.cuh"
#include "kernels/krylov.cuh"
#include "kernels/krylov_batch.cuh"
#include "kernels/ns.cuh"
#include "host/ns_setup.hpp"
#include "host/sort.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

// ================================================================ errors / buffers
std::string& vfv_thread_error() {
    static thread_local std::string e;
    return e;
}

// ================================================================ GMRES driver
namespace {

// SpMV shapes: G lanes per row, each lane loading its first S strides of the row (indices and
// values) before any gather. The autotuner picks one per pattern and precision; (G, 4) exists for
// every G (the shape vfv_pattern_set_spmv_lanes selects).
#define VFV_SPMV_SHAPES(X) X(2, 4) X(2, 8) X(4, 4) X(4, 6) X(4, 8) X(8, 2) X(8, 3) X(8, 4) X(16, 1) X(16, 2) X(16, 4) X(32, 1) X(32, 4)
constexpr int kSpmvShapes[][2] = {
#define VFV_SHAPE_ENTRY(G, S) {G, S},
    VFV_SPMV_SHAPES(VFV_SHAPE_ENTRY)
#undef VFV_SHAPE_ENTRY
};

template <typename TV, typename TX, typename TY, typename TA>
void launch_spmv(cudaStream_t s, int lanes, int strides, int64_t n, const int32_t* rp, const int32_t* ci, const TV* val, const TX* x,
                 TY* y, const double* scale, const DevStatus* st) {
    switch (lanes * 16 + strides) {
#define VFV_SHAPE_CASE(G, S)                                                                                  \
    case G * 16 + S:                                                                                          \
        k_spmv<TV, TX, TY, TA, G, S><<<grid_for(n * G), kBlk, 0, s>>>(n, rp, ci, val, x, y, scale, st);         \
        return;
        VFV_SPMV_SHAPES(VFV_SHAPE_CASE)
#undef VFV_SHAPE_CASE
        default:
            k_spmv<TV, TX, TY, TA, 4, 4><<<grid_for(n * 4), kBlk, 0, s>>>(n, rp, ci, val, x, y, scale, st);
    }
}

// SpMV of a batched solve: the step's scale 1/beta_j looked up per row from its mesh
template <typename TV, typename TX, typename TY, typename TA>
void launch_spmv_seg(cudaStream_t s, int lanes, int strides, int64_t n, const int32_t* rp, const int32_t* ci, const TV* val, const TX* x,
                     TY* y, const double* inv_beta, int stride, int j, const int64_t* mesh_row, int nm, const DevStatus* st) {
    switch (lanes * 16 + strides) {
#define VFV_SHAPE_CASE(G, S)                                                                                                         \
    case G * 16 + S:                                                                                                                 \
        k_spmv_seg<TV, TX, TY, TA, G, S><<<grid_for(n * G), kBlk, 0, s>>>(n, rp, ci, val, x, y, inv_beta, stride, j, mesh_row, nm, st); \
        return;
        VFV_SPMV_SHAPES(VFV_SHAPE_CASE)
#undef VFV_SHAPE_CASE
        default:
            k_spmv_seg<TV, TX, TY, TA, 4, 4><<<grid_for(n * 4), kBlk, 0, s>>>(n, rp, ci, val, x, y, inv_beta, stride, j, mesh_row, nm, st);
    }
}

// Symmetrised, de-duplicated adjacency of the pattern graph (no self loops) as CSR.
void sym_adjacency(const vfv_pattern* p, std::vector<int64_t>& xadj, std::vector<int32_t>& adj) {
    const int64_t n = p->n;
    const std::vector<int32_t>& rp = p->h_rp;
    const std::vector<int32_t>& ci = p->h_ci;
    xadj.assign(n + 1, 0);
    for (int64_t i = 0; i < n; ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] != i) {
                xadj[i + 1]++;
                xadj[ci[k] + 1]++;
            }
    for (int64_t i = 0; i < n; ++i) xadj[i + 1] += xadj[i];
    adj.resize(xadj[n]);
    std::vector<int64_t> cur(xadj.begin(), xadj.end() - 1);
    for (int64_t i = 0; i < n; ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] != i) {
                adj[cur[i]++] = ci[k];
                adj[cur[ci[k]]++] = (int32_t)i;
            }
    // sort and drop duplicates row by row, compacting in place
    std::vector<int64_t> len(n);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t i = 0; i < n; ++i) {
        int32_t* a = adj.data() + xadj[i];
        const int64_t m = xadj[i + 1] - xadj[i];
        std::sort(a, a + m);
        len[i] = std::unique(a, a + m) - a;
    }
    int64_t w = 0;
    for (int64_t i = 0; i < n; ++i) {
        const int64_t r0 = xadj[i];
        for (int64_t k = 0; k < len[i]; ++k) adj[w + k] = adj[r0 + k];
        xadj[i] = w;
        w += len[i];
    }
    xadj[n] = w;
    adj.resize(w);
}

// Greedy colouring: colour(v) = smallest colour unused by the already coloured neighbours,
// visiting the vertices in `order` (which must list every vertex whose colour is reset to -1).
int greedy_colour(const std::vector<int32_t>& order, const int64_t* xadj, const int32_t* adj, int32_t* col, std::vector<int64_t>& mark) {
    for (int32_t v : order) col[v] = -1;
    std::fill(mark.begin(), mark.end(), -1);
    int nc = 0;
    for (int64_t t = 0; t < (int64_t)order.size(); ++t) {
        const int32_t v = order[t];
        for (int64_t k = xadj[v]; k < xadj[v + 1]; ++k) {
            const int32_t c = col[adj[k]];
            if (c >= 0) {
                if (c >= (int32_t)mark.size()) mark.resize(c + 1, -1);
                mark[c] = t;
            }
        }
        int32_t c = 0;
        while (c < (int32_t)mark.size() && mark[c] == t) ++c;
        col[v] = c;
        nc = std::max(nc, c + 1);
    }
    return nc;
}

// Stable counting sort of `order` by key[col[v]] (keys in [0, nkey)).
void sort_by_class(std::vector<int32_t>& order, const int32_t* col, const std::vector<int32_t>& key, int nkey, std::vector<int32_t>& tmp) {
    std::vector<int64_t> start(nkey + 1, 0);
    for (int32_t v : order) start[key[col[v]] + 1]++;
    for (int k = 0; k < nkey; ++k) start[k + 1] += start[k];
    tmp.resize(order.size());
    for (int32_t v : order) tmp[start[key[col[v]]]++] = v;
    order.swap(tmp);
}

// Multicolour ordering with few colours (each colour is a level of both ILU sweeps) of the
// vertices [r0, r1), which must have no edge leaving the range: greedy in index order, then
// iterated greedy (Culberson: re-running greedy with the vertices grouped by colour class never
// needs more colours), then single-neighbour recolouring that tries to empty the last class.
// Deterministic.
int multicolor_range(int64_t r0, int64_t r1, const int64_t* xadj, const int32_t* adj, int32_t* col) {
    const int64_t n = r1 - r0;
    if (n <= 0) return 0;
    std::vector<int32_t> order(n), tmp;
    for (int64_t i = 0; i < n; ++i) order[i] = (int32_t)(r0 + i);
    std::vector<int64_t> mark(64, -1);
    int nc = greedy_colour(order, xadj, adj, col, mark);
    std::vector<int32_t> best(col + r0, col + r1);
    for (int it = 0; it < 8; ++it) {
        std::vector<int32_t> key(nc);
        if (it % 2 == 0) {
            for (int c = 0; c < nc; ++c) key[c] = nc - 1 - c;  // largest colour first
        } else {
            std::vector<int64_t> cnt(nc, 0);
            for (int64_t i = r0; i < r1; ++i) cnt[col[i]]++;
            std::vector<int32_t> cls(nc);
            for (int c = 0; c < nc; ++c) cls[c] = c;
            std::stable_sort(cls.begin(), cls.end(), [&](int32_t a, int32_t b) { return cnt[a] != cnt[b] ? cnt[a] > cnt[b] : a < b; });
            for (int r = 0; r < nc; ++r) key[cls[r]] = r;  // most populated class first
        }
        sort_by_class(order, col, key, nc, tmp);
        const int nc2 = greedy_colour(order, xadj, adj, col, mark);
        if (nc2 <= nc) {
            nc = nc2;
            std::copy(col + r0, col + r1, best.begin());
        } else {
            std::copy(best.begin(), best.end(), col + r0);
        }
    }
    std::vector<char> used;
    for (int round = 0; round < 2 && nc > 1; ++round) {
        const int last = nc - 1;
        int64_t left = 0;
        used.assign(last, 0);
        for (int64_t v = r0; v < r1; ++v) {
            if (col[v] != last) continue;
            bool done = false;
            for (int c = 0; c < last && !done; ++c) {
                int cntc = 0;
                int32_t u = -1;
                for (int64_t k = xadj[v]; k < xadj[v + 1]; ++k)
                    if (col[adj[k]] == c) {
                        ++cntc;
                        u = adj[k];
                    }
                if (cntc == 0) {
                    col[v] = c;
                    done = true;
                } else if (cntc == 1) {
                    std::fill(used.begin(), used.end(), 0);
                    for (int64_t k = xadj[u]; k < xadj[u + 1]; ++k)
                        if (adj[k] != v && col[adj[k]] < last) used[col[adj[k]]] = 1;
                    for (int cc = 0; cc < last; ++cc)
                        if (cc != c && !used[cc]) {
                            col[u] = cc;
                            col[v] = c;
                            done = true;
                            break;
                        }
                }
            }
            if (!done) ++left;
        }
        if (left == 0) {
            nc = last;
            break;
        }
    }
    return nc;
}

// Multicolour ordering of the whole pattern; the diagonal blocks p->blocks (row ranges of a
// block-diagonal system) are coloured independently in parallel when no edge couples two blocks.
int multicolor(const vfv_pattern* p, const std::vector<int64_t>& xadj, const std::vector<int32_t>& adj, std::vector<int32_t>& col) {
    const int64_t n = p->n;
    std::vector<int64_t> blk = p->blocks;
    bool ok = blk.size() >= 2 && blk.front() == 0 && blk.back() == n;
    for (size_t b = 0; ok && b + 1 < blk.size(); ++b)
        for (int64_t v = blk[b]; ok && v < blk[b + 1]; ++v)
            for (int64_t k = xadj[v]; k < xadj[v + 1]; ++k)
                if (adj[k] < blk[b] || adj[k] >= blk[b + 1]) {
                    ok = false;
                    break;
                }
    if (!ok) blk = {0, n};
    const int64_t nb = (int64_t)blk.size() - 1;
    int nc = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(max : nc)
    for (int64_t b = 0; b < nb; ++b) nc = std::max(nc, multicolor_range(blk[b], blk[b + 1], xadj.data(), adj.data(), col.data()));
    return nc;
}

int build_ilu_struct(vfv_ctx* ctx, vfv_pattern* p, int order, IluStruct& S) {
    const int64_t n = p->n;
    const std::vector<int32_t>& rp = p->h_rp;
    const std::vector<int32_t>& ci = p->h_ci;
    std::vector<int64_t> xadj;
    std::vector<int32_t> adj;
    sym_adjacency(p, xadj, adj);
    std::vector<int32_t> lev(n, 0);
    int nlev = 0;
    if (order == VFV_ILU_NATURAL) {  // level = 1 + the deepest lower neighbour
        for (int64_t i = 0; i < n; ++i) {
            int32_t l = 0;
            for (int64_t k = xadj[i]; k < xadj[i + 1] && adj[k] < i; ++k) l = std::max(l, lev[adj[k]] + 1);
            lev[i] = l;
            nlev = std::max(nlev, l + 1);
        }
    } else {
        nlev = multicolor(p, xadj, adj, lev);
    }
    std::vector<int64_t>().swap(xadj);
    std::vector<int32_t>().swap(adj);
    std::vector<int32_t> perm(n), iperm(n);
    std::vector<int64_t> cnt(nlev + 1, 0);
    for (int64_t i = 0; i < n; ++i) cnt[lev[i] + 1]++;
    for (int l = 0; l < nlev; ++l) cnt[l + 1] += cnt[l];
    S.lev_ptr.assign(cnt.begin(), cnt.end());
    {
        std::vector<int64_t> cur(cnt.begin(), cnt.end() - 1);
        for (int64_t i = 0; i < n; ++i) {
            const int64_t q = cur[lev[i]]++;
            perm[q] = (int32_t)i;
            iperm[i] = (int32_t)q;
        }
    }
    std::vector<int32_t> nrp(n + 1, 0), nci(p->nnz), nsrc(p->nnz), ndg(n, -1);
    for (int64_t q = 0; q < n; ++q) nrp[q + 1] = nrp[q] + (rp[perm[q] + 1] - rp[perm[q]]);
    std::vector<std::pair<int32_t, int32_t>> row;
    for (int64_t q = 0; q < n; ++q) {
        const int32_t i = perm[q];
        row.clear();
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) row.push_back({iperm[ci[k]], k});
        std::sort(row.begin(), row.end());
        for (size_t t = 0; t < row.size(); ++t) {
            nci[nrp[q] + t] = row[t].first;
            nsrc[nrp[q] + t] = row[t].second;
            if (row[t].first == q) ndg[q] = nrp[q] + (int32_t)t;
        }
        if (ndg[q] < 0) return set_err(ctx, VFV_BAD_INPUT, "ILU(0) needs a diagonal entry in every row of the pattern");
    }
    cudaStream_t s = ctx->stream;
    S.h_perm = perm;
    CK(S.perm.upload(perm.data(), n, s));
    CK(S.d_lev_ptr.upload(S.lev_ptr.data(), S.lev_ptr.size(), s));
    CK(S.rp.upload(nrp.data(), n + 1, s));
    CK(S.ci.upload(nci.data(), p->nnz, s));
    CK(S.dg.upload(ndg.data(), n, s));
    CK(S.src.upload(nsrc.data(), p->nnz, s));
    CK(S.lu64.alloc(p->nnz));
    CK(S.bad.alloc(1));


    S.order = order;
    S.nlev = nlev;
    return VFV_OK;
}

// Copy of the ordering and permuted pattern of an ILU structure built for a pattern with the same
// rows and columns (the numeric factor is recomputed from this pattern's values).
template <typename T>
cudaError_t copy_dbuf(DBuf<T>& to, const DBuf<T>& from, cudaStream_t s) {
    cudaError_t e = to.alloc(from.n);
    if (e != cudaSuccess || from.n == 0) return e;
    return cudaMemcpyAsync(to.p, from.p, from.n * sizeof(T), cudaMemcpyDeviceToDevice, s);
}

int clone_ilu_struct(vfv_ctx* ctx, const IluStruct& F, int64_t nnz, IluStruct& S) {
    cudaStream_t s = ctx->stream;
    S.order = F.order;
    S.nlev = F.nlev;
    S.lev_ptr = F.lev_ptr;
    S.h_perm = F.h_perm;
    CK(copy_dbuf(S.d_lev_ptr, F.d_lev_ptr, s));
    CK(copy_dbuf(S.perm, F.perm, s));
    CK(copy_dbuf(S.rp, F.rp, s));
    CK(copy_dbuf(S.ci, F.ci, s));
    CK(copy_dbuf(S.dg, F.dg, s));
    CK(copy_dbuf(S.src, F.src, s));
    CK(S.lu64.alloc(nnz));
    CK(S.bad.alloc(1));
    CK(cudaStreamSynchronize(s));
    return VFV_OK;
}

// launch attributes: programmatic dependent launch after the previous kernel, stream priority
inline void launch_attrs(cudaLaunchConfig_t& cfg, cudaLaunchAttribute* attr, bool pdl, int prio, bool use_prio) {
    int na = 0;
    if (pdl) {
        attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[na].val.programmaticStreamSerializationAllowed = 1;
        ++na;
    }
    if (use_prio) {
        attr[na].id = cudaLaunchAttributePriority;
        attr[na].val.priority = prio;
        ++na;
    }
    cfg.attrs = na ? attr : nullptr;
    cfg.numAttrs = na;
}

// numeric ILU(0) of the pattern's current values (double), cast to float when asked
// The factorisation as one dataflow launch (k_ilu0_factor_flow) when the ordering has many levels,
// all narrow (the natural order); level by level otherwise, or with VFV_ILU_FACTOR=levels.
constexpr int32_t kFacWideRows = 32768;  // levels this wide run one thread per row
constexpr int kFlowMinLevels = 32;
constexpr long long kDefaultWaitPolls = 20000000LL;  // polls before a bounded device wait gives up (2 s also ends it)

bool ilu_use_flow(const IluStruct& S) {
    if (S.nlev < kFlowMinLevels) return false;
    if (const char* e = getenv("VFV_ILU_FACTOR"))
        if (std::string(e) == "levels") return false;
    for (int l = 0; l < S.nlev; ++l)
        if (S.lev_ptr[l + 1] - S.lev_ptr[l] >= kFacWideRows) return false;
    return true;
}

// k_ilu0_factor_flow over S.lu64 (values already gathered); VFV_TIMEOUT if a bounded wait gave up
// (polls: its poll limit, 0 = default)
int ilu_factor_flow(vfv_ctx* ctx, IluStruct& S, int32_t n, long long polls) {
    cudaStream_t s = ctx->stream;
    if (!S.flow_grid) {
        int per_sm = 0, sms = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ilu0_factor_flow, 32 * kFacWarps, 0));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
        if (per_sm < 1) return set_err(ctx, VFV_CUDA_ERROR, "ILU(0): the dataflow factorisation does not fit an SM");
        CK(S.ready.alloc(std::max<int64_t>(n, 1)));
        CK(cudaMemsetAsync(S.ready.p, 0, S.ready.n * sizeof(unsigned), s));
        CK(S.flow_state.alloc(2));
        CK(cudaMemsetAsync(S.flow_state.p, 0, 2 * sizeof(unsigned), s));
        S.flow_grid = (int)std::min<int64_t>((int64_t)per_sm * sms, std::max<int64_t>(1, ((int64_t)n + kFacWarps - 1) / kFacWarps));
        S.epoch = 0;
    }
    if (++S.epoch == 0) {  // the flags wrapped around: no row may look finished
        CK(cudaMemsetAsync(S.ready.p, 0, S.ready.n * sizeof(unsigned), s));
        S.epoch = 1;
    }
    FlowSync fs{S.ready.p, S.epoch, S.flow_state.p, reinterpret_cast<int*>(S.flow_state.p + 1),
                polls > 0 ? polls : kDefaultWaitPolls};
    const int32_t* rp = S.rp.p;
    const int32_t* ci = S.ci.p;
    const int32_t* dg = S.dg.p;
    double* a = S.lu64.p;
    int* bad = S.bad.p;
    void* args[] = {(void*)&n, (void*)&rp, (void*)&ci, (void*)&dg, (void*)&a, (void*)&bad, (void*)&fs};
    CK(cudaLaunchCooperativeKernel((const void*)k_ilu0_factor_flow, dim3(S.flow_grid), dim3(32 * kFacWarps), args, 0, s));
    unsigned st[2] = {0u, 0u};
    CK(cudaMemcpyAsync(st, S.flow_state.p, sizeof(st), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (st[0] || st[1]) {
        CK(cudaMemsetAsync(S.flow_state.p, 0, 2 * sizeof(unsigned), s));
        CK(cudaStreamSynchronize(s));
        return set_err(ctx, VFV_TIMEOUT, "ILU(0): a bounded device wait of the dataflow factorisation gave up");
    }
    return VFV_OK;
}

// The numeric factor (and its float copy with want32) for the pattern's current values. polls: poll
// limit of the dataflow factorisation's waits (0 = default); without may_alloc the dataflow
// factorisation runs only if its buffers already exist (level by level otherwise).
int ilu_refresh(vfv_ctx* ctx, vfv_pattern* p, IluStruct& S, bool want32, long long polls = 0, bool may_alloc = true) {
    cudaStream_t s = ctx->stream;
    if (S.version64 != p->version) {
        k_gather_vals<double><<<grid_for(p->nnz), 256, 0, s>>>(p->nnz, S.src.p, p->val.p, S.lu64.p);
        CK(cudaMemsetAsync(S.bad.p, 0, sizeof(int), s));
        const bool flow = ilu_use_flow(S) && (may_alloc || S.flow_grid > 0);
        ctx->launches += 1 + (flow ? 1 : S.nlev);
        if (flow) {
            const int rc = ilu_factor_flow(ctx, S, (int32_t)p->n, polls);
            if (rc != VFV_OK) return rc;
        }
        // narrow levels: one warp per row, chained with programmatic dependent launch; wide levels
        // (>= kFacWideRows rows, e.g. multicolour colours): one thread per row, in stream order
        bool prev_warp = false;
        for (int l = 0; l < (flow ? 0 : S.nlev); ++l) {
            const int32_t r0 = S.lev_ptr[l], r1 = S.lev_ptr[l + 1];
            if (r1 - r0 >= kFacWideRows) {
                k_ilu0_factor_level<<<grid_for(r1 - r0, 128), 128, 0, s>>>(r0, r1, S.rp.p, S.ci.p, S.dg.p, S.lu64.p, S.bad.p);
                prev_warp = false;
                continue;
            }
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3((unsigned)((r1 - r0 + kFacWarps - 1) / kFacWarps));
            cfg.blockDim = dim3(32 * kFacWarps);
            cfg.stream = s;
            cudaLaunchAttribute attr[1];
            launch_attrs(cfg, attr, prev_warp, 0, false);  // after the value gather or a wide level: stream order
            CK(cudaLaunchKernelEx(&cfg, k_ilu0_factor_level_warp, r0, r1, (const int32_t*)S.rp.p, (const int32_t*)S.ci.p,
                                  (const int32_t*)S.dg.p, S.lu64.p, S.bad.p));
            prev_warp = true;
        }
        int bad = 0;
        CK(cudaMemcpyAsync(&bad, S.bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        CK(cudaGetLastError());
        if (bad) return set_err(ctx, VFV_NONFINITE, "ILU(0): zero pivot");
        S.version64 = p->version;
    }
    if (want32 && S.version32 != p->version) {
        if (!S.lu32.p) CK(S.lu32.alloc(p->nnz));
        k_cast<double, float><<<grid_for(p->nnz), 256, 0, s>>>(p->nnz, S.lu64.p, S.lu32.p);
        ctx->launches += 1;
        S.version32 = p->version;
    }
    return VFV_OK;
}

// z = (LU)^-1 r: one launch per level, lower levels then upper levels in reverse, chained with
// programmatic dependent launch. `in` and `out` may alias; `t` must not alias either.
template <typename T, bool LOWER>
cudaError_t launch_level(cudaStream_t s, const IluStruct& S, int l, bool pdl, const T* lu, const T* in, T* t, T* out, const DevStatus* st,
                         int prio = 0, bool use_prio = false) {
    const int32_t r0 = S.lev_ptr[l], r1 = S.lev_ptr[l + 1];
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)std::max(1, (r1 - r0 + kLevBlock - 1) / kLevBlock));
    cfg.blockDim = dim3(kLevBlock);
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    int na = 0;
    if (pdl) {
        attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[na].val.programmaticStreamSerializationAllowed = 1;
        ++na;
    }
    if (use_prio) {  // scheduled ahead of concurrently queued blocks of lower priority
        attr[na].id = cudaLaunchAttributePriority;
        attr[na].val.priority = prio;
        ++na;
    }
    cfg.attrs = na ? attr : nullptr;
    cfg.numAttrs = na;
    return cudaLaunchKernelEx(&cfg, k_ilu0_level<T, LOWER>, r0, r1, (const int32_t*)S.rp.p, (const int32_t*)S.ci.p, (const int32_t*)S.dg.p, lu,
                              (const int32_t*)S.perm.p, in, t, out, st);
}

template <typename T>
void ilu_apply_levels(cudaStream_t s, const IluStruct& S, const T* lu, const T* in, T* t, T* out, const DevStatus* st, int prio = 0,
                      bool use_prio = false) {
    for (int l = 0; l < S.nlev; ++l) launch_level<T, true>(s, S, l, l > 0, lu, in, t, out, st, prio, use_prio);
    for (int l = S.nlev - 1; l >= 0; --l) launch_level<T, false>(s, S, l, true, lu, in, t, out, st, prio, use_prio);
}

// the buffer of precision T out of a double / float pair
template <typename T>
DBuf<T>& of_prec(DBuf<double>& d, DBuf<float>& f) {
    if constexpr (std::is_same<T, double>::value) return d;
    else return f;
}

// Compact triangles of the factor for the Jacobi-sweep apply (k_ilu0_sweep): structure once per
// ILU structure (host), values per factor refresh and precision (device). The natural ordering is
// swept in A's own numbering (A's rows with the factor's values scattered back to A's slots), the
// multicolour ordering in its factor's permuted numbering.
template <typename T>
int ilu_split_refresh(vfv_ctx* ctx, vfv_pattern* p, IluStruct& S, bool half = false) {
    cudaStream_t s = ctx->stream;
    const int64_t n = p->n, nnz = p->nnz;
    IluStruct::Split& X = S.split;
    const bool nat = S.order == VFV_ILU_NATURAL;
    if (!X.built) {
        // the factor's structure in its numbering F
        std::vector<int32_t> rp, ci, dg(n);
        if (nat) {
            rp = p->h_rp;
            ci = p->h_ci;
            for (int64_t i = 0; i < n; ++i)
                for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
                    if (ci[k] == i) dg[i] = k;
        } else {
            rp.resize(n + 1);
            ci.resize(nnz);
            CK(cudaMemcpyAsync(rp.data(), S.rp.p, (n + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(ci.data(), S.ci.p, nnz * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(dg.data(), S.dg.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
        }
        int64_t maxd = 0;
        for (int64_t r = 0; r < n; ++r)
            for (int32_t k = rp[r]; k < rp[r + 1]; ++k) maxd = std::max<int64_t>(maxd, std::abs((int64_t)ci[k] - r));
        // 16-bit column offsets when the factor's bandwidth allows. (A reverse Cuthill-McKee
        // renumbering to make them fit on wider patterns was measured slower on the 10^6-row heat
        // factor: the sweeps are latency-bound, and renumbered gathers lose the mesh order's locality.)
        X.delta16 = maxd <= 32767;
        std::vector<int32_t> lrp(n + 1, 0), urp(n + 1, 0), lc, uc;
        lc.reserve(nnz / 2);
        uc.reserve(nnz / 2);
        for (int64_t r = 0; r < n; ++r) {
            for (int32_t k = rp[r]; k < rp[r + 1]; ++k) {
                if (k < dg[r]) lc.push_back(ci[k]);
                else if (k > dg[r]) uc.push_back(ci[k]);
            }
            lrp[r + 1] = (int32_t)lc.size();
            urp[r + 1] = (int32_t)uc.size();
        }
        CK(X.lrp.upload(lrp.data(), n + 1, s));
        CK(X.urp.upload(urp.data(), n + 1, s));
        if (X.delta16) {
            std::vector<int16_t> ld(lc.size()), ud(uc.size());
            for (int64_t r = 0; r < n; ++r) {
                for (int32_t k = lrp[r]; k < lrp[r + 1]; ++k) ld[k] = (int16_t)(lc[k] - r);
                for (int32_t k = urp[r]; k < urp[r + 1]; ++k) ud[k] = (int16_t)(uc[k] - r);
            }
            CK(X.lcd.upload(ld.data(), ld.size(), s));
            CK(X.ucd.upload(ud.data(), ud.size(), s));
        } else {
            CK(X.lci.upload(lc.data(), lc.size(), s));
            CK(X.uci.upload(uc.data(), uc.size(), s));
        }
        X.built = true;
    }
    constexpr bool dbl = std::is_same<T, double>::value;
    uint64_t& ver = dbl ? X.version64 : X.version32;
    const int64_t nlow = X.delta16 ? (int64_t)X.lcd.n : (int64_t)X.lci.n, nup = X.delta16 ? (int64_t)X.ucd.n : (int64_t)X.uci.n;
    if (ver != p->version) {
    const T* lu = of_prec<T>(S.lu64, S.lu32).p;
    const int32_t *rp = S.rp.p, *dg = S.dg.p;
    if (nat) {  // the factor's values back in A's slot order
        DBuf<T>& nv = of_prec<T>(S.nat64, S.nat32);
        if (!nv.p) CK(nv.alloc(nnz));
        k_scatter_vals<T><<<grid_for(nnz), 256, 0, s>>>(nnz, S.src.p, lu, nv.p);
        ctx->launches += 1;
        lu = nv.p;
        rp = p->rp.p;
        dg = p->diag_pos.p;
    }
    DBuf<T>& lv = of_prec<T>(X.lv64, X.lv32);
    DBuf<T>& uv = of_prec<T>(X.uv64, X.uv32);
    DBuf<T>& dv = of_prec<T>(X.d64, X.d32);
    if (!lv.p) CK(lv.alloc(std::max<int64_t>(nlow, 1)));
    if (!uv.p) CK(uv.alloc(std::max<int64_t>(nup, 1)));
    if (!dv.p) CK(dv.alloc(n));
    k_split_vals<T><<<grid_for(n), 256, 0, s>>>((int32_t)n, rp, dg, lu, X.lrp.p, X.urp.p, lv.p, uv.p, dv.p);
    ctx->launches += 1;
    CK(cudaGetLastError());
    ver = p->version;
    }
    if constexpr (!dbl) {  // the row-scaled half copies of the float values, when asked for
        if (half && X.version_half != p->version) {
            if (!X.lvh.p) CK(X.lvh.alloc(std::max<int64_t>(nlow, 1)));
            if (!X.uvh.p) CK(X.uvh.alloc(std::max<int64_t>(nup, 1)));
            if (!X.lsc.p) CK(X.lsc.alloc(n));
            if (!X.usc.p) CK(X.usc.alloc(n));
            k_half_rows<<<grid_for(n), 256, 0, s>>>((int32_t)n, X.lrp.p, X.lv32.p, reinterpret_cast<__half*>(X.lvh.p), X.lsc.p);
            k_half_rows<<<grid_for(n), 256, 0, s>>>((int32_t)n, X.urp.p, X.uv32.p, reinterpret_cast<__half*>(X.uvh.p), X.usc.p);
            ctx->launches += 2;
            CK(cudaGetLastError());
            X.version_half = p->version;
        }
    }
    return VFV_OK;
}

// Operands of the Jacobi-sweep apply, from the refreshed compact triangles.
template <typename T>
struct SweepOps {
    int32_t n = 0;
    int lanes = 4;  // lanes per row (measured on the 10^6-row heat factor: 1 for float values, 2 for double)
    bool delta16 = false;
    const int32_t *lrp = nullptr, *urp = nullptr, *perm = nullptr;
    const void *lcols = nullptr, *ucols = nullptr;
    const T *lv = nullptr, *uv = nullptr, *d = nullptr;
    // float factors only: the row-scaled half-precision values and their row scales (vfv_gmres_opts::ilu_sweep_half)
    const __half *lvh = nullptr, *uvh = nullptr;
    const float *lsc = nullptr, *usc = nullptr;
};

template <typename T>
SweepOps<T> sweep_ops(const vfv_pattern* p, IluStruct& S, bool half = false) {
    IluStruct::Split& X = S.split;
    SweepOps<T> o;
    if (half && std::is_same<T, float>::value) {
        o.lvh = reinterpret_cast<const __half*>(X.lvh.p);
        o.uvh = reinterpret_cast<const __half*>(X.uvh.p);
        o.lsc = X.lsc.p;
        o.usc = X.usc.p;
    }
    o.n = (int32_t)p->n;
    o.lanes = std::is_same<T, double>::value ? 2 : 1;
    if (const char* e = getenv("VFV_SWEEP_LANES")) {
        const int g = std::atoi(e);
        if (g == 1 || g == 2 || g == 4 || g == 8) o.lanes = g;
    }
    o.delta16 = X.delta16;
    o.lrp = X.lrp.p;
    o.urp = X.urp.p;
    o.lcols = X.delta16 ? (const void*)X.lcd.p : (const void*)X.lci.p;
    o.ucols = X.delta16 ? (const void*)X.ucd.p : (const void*)X.uci.p;
    o.lv = of_prec<T>(X.lv64, X.lv32).p;
    o.uv = of_prec<T>(X.uv64, X.uv32).p;
    o.d = of_prec<T>(X.d64, X.d32).p;
    o.perm = S.order == VFV_ILU_NATURAL ? nullptr : S.perm.p;
    return o;
}


template <typename T, typename TC, bool LOWER, int G>
cudaError_t launch_sweep_g(cudaLaunchConfig_t& cfg, const SweepOps<T>& o, const T* rhs, const T* prev, T* next, T* w0, T* out,
                           const DevStatus* st) {
    cfg.gridDim = dim3((unsigned)grid_for((int64_t)o.n * G, kSwBlock));
    if constexpr (std::is_same<T, float>::value) {
        if (o.lvh)
            return cudaLaunchKernelEx(&cfg, k_ilu0_sweep<T, TC, LOWER, G, __half>, o.n, LOWER ? o.lrp : o.urp,
                                      (const TC*)(LOWER ? o.lcols : o.ucols), LOWER ? o.lvh : o.uvh, LOWER ? o.lsc : o.usc, o.d, o.perm,
                                      rhs, prev, next, w0, out, st);
    }
    return cudaLaunchKernelEx(&cfg, k_ilu0_sweep<T, TC, LOWER, G, T>, o.n, LOWER ? o.lrp : o.urp, (const TC*)(LOWER ? o.lcols : o.ucols),
                              LOWER ? o.lv : o.uv, (const float*)nullptr, o.d, o.perm, rhs, prev, next, w0, out, st);
}

template <typename T, bool LOWER>
cudaError_t launch_sweep(cudaLaunchConfig_t& cfg, const SweepOps<T>& o, const T* rhs, const T* prev, T* next, T* w0, T* out,
                         const DevStatus* st) {
    if (o.delta16) {
        if (o.lanes == 1) return launch_sweep_g<T, int16_t, LOWER, 1>(cfg, o, rhs, prev, next, w0, out, st);
        if (o.lanes == 2) return launch_sweep_g<T, int16_t, LOWER, 2>(cfg, o, rhs, prev, next, w0, out, st);
        if (o.lanes == 8) return launch_sweep_g<T, int16_t, LOWER, 8>(cfg, o, rhs, prev, next, w0, out, st);
        return launch_sweep_g<T, int16_t, LOWER, 4>(cfg, o, rhs, prev, next, w0, out, st);
    }
    if (o.lanes == 1) return launch_sweep_g<T, int32_t, LOWER, 1>(cfg, o, rhs, prev, next, w0, out, st);
    if (o.lanes == 2) return launch_sweep_g<T, int32_t, LOWER, 2>(cfg, o, rhs, prev, next, w0, out, st);
    if (o.lanes == 8) return launch_sweep_g<T, int32_t, LOWER, 8>(cfg, o, rhs, prev, next, w0, out, st);
    return launch_sweep_g<T, int32_t, LOWER, 4>(cfg, o, rhs, prev, next, w0, out, st);
}

// z = M^-1 r by `sweeps` Jacobi sweeps of the lower and `usweeps` of the upper ILU(0) factor: one
// launch per sweep (+1 gather of r
// into the permuted numbering), chained with programmatic dependent launch. buf: 5 work vectors of
// n entries (permuted r, two lower and two upper iterates) aliasing neither r nor z; r and z may
// alias (r is read by the lower sweeps only, z written by the last upper sweep only).
template <typename T>
void ilu_apply_sweeps(cudaStream_t s, const SweepOps<T>& o, int sweeps, int usweeps, const T* in, T* out, T* const* buf, const DevStatus* st,
                      int prio = 0, bool use_prio = false) {
    const T* rhs = in;
    bool pdl = false;
    cudaLaunchAttribute attr[2];
    if (o.perm) {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3((unsigned)grid_for(o.n));
        cfg.blockDim = dim3(256);
        cfg.stream = s;
        launch_attrs(cfg, attr, false, prio, use_prio);
        cudaLaunchKernelEx(&cfg, k_perm_gather<T>, o.n, o.perm, in, buf[0]);
        rhs = buf[0];
        pdl = true;
    }
    cudaLaunchConfig_t cfg{};
    cfg.blockDim = dim3(kSwBlock);
    cfg.stream = s;
    T* const ub[2] = {buf[1], buf[2]};
    T* const wb[2] = {buf[3], buf[4]};
    for (int k = 1; k <= sweeps; ++k) {
        launch_attrs(cfg, attr, pdl, prio, use_prio);
        launch_sweep<T, true>(cfg, o, rhs, k == 1 ? rhs : (const T*)ub[(k - 1) & 1], ub[k & 1], k == sweeps ? wb[0] : (T*)nullptr,
                              (T*)nullptr, st);
        pdl = true;
    }
    const T* u = ub[sweeps & 1];
    for (int k = 1; k <= usweeps; ++k) {
        launch_attrs(cfg, attr, true, prio, use_prio);
        launch_sweep<T, false>(cfg, o, u, (const T*)wb[(k - 1) & 1], wb[k & 1], (T*)nullptr, k == usweeps ? out : (T*)nullptr, st);
    }
}

constexpr int kMaxIluSweeps = 16;

template <typename T>
constexpr int chain_slot() {
    return std::is_same<T, double>::value ? 0 : 1;
}

// Claim counter, completion counters and abort flag cleared, poll limit set: the state of a fresh
// chain (at set-up, and after a wait gave up, which leaves it undefined).
template <typename T>
int chain_reset(vfv_ctx* ctx, IluStruct& S, long long polls) {
    IluStruct::Chain& C = S.chain[chain_slot<T>()];
    cudaStream_t s = ctx->stream;
    IluChainState h{};
    h.poll_limit = polls > 0 ? polls : kDefaultWaitPolls;
    CK(cudaMemsetAsync(C.state.p, 0, C.state.n, s));
    CK(cudaMemcpyAsync(C.state.p, &h, sizeof(h), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    return VFV_OK;
}

// Task table (row ranges of at most kChainThreads rows inside one level, their levels, tasks per
// level) and the chain state of precision T, with a work vector of n entries for standalone
// applies; once per ILU structure and precision.
template <typename T>
int chain_setup(vfv_ctx* ctx, IluStruct& S, int64_t n) {
    IluStruct::Chain& C = S.chain[chain_slot<T>()];
    if (C.grid > 0) return VFV_OK;
    if (!S.tasks.p) {
        std::vector<int32_t> tk, tl, ln(S.nlev, 0);
        for (int l = 0; l < S.nlev; ++l)
            for (int32_t r = S.lev_ptr[l]; r < S.lev_ptr[l + 1]; r += kChainThreads) {
                tk.push_back(r);
                tl.push_back(l);
                ln[l]++;
            }
        tk.push_back(S.lev_ptr[S.nlev]);
        S.ntask = (int)tl.size();
        CK(S.tasks.upload(tk.data(), tk.size(), ctx->stream));
        CK(S.task_lev.upload(tl.data(), tl.size(), ctx->stream));
        CK(S.lev_ntask.upload(ln.data(), ln.size(), ctx->stream));
    }
    CK(C.work.alloc((size_t)n * sizeof(T)));
    CK(C.state.alloc(sizeof(IluChainState) + 2 * (size_t)S.nlev * sizeof(unsigned)));
    int per_sm = 0, sms = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ilu0_chain<T>, kChainThreads, 0));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    C.grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)std::max(per_sm, 1) * sms, 2 * (int64_t)S.ntask));
    return chain_reset<T>(ctx, S, 0);
}

// poll limit of the chain's bounded waits for the launches that follow (enqueued on the stream)
template <typename T>
int chain_set_polls(vfv_ctx* ctx, IluStruct& S, long long polls) {
    IluStruct::Chain& C = S.chain[chain_slot<T>()];
    const long long v = polls > 0 ? polls : kDefaultWaitPolls;  // pageable source: staged before the call returns
    CK(cudaMemcpyAsync(C.state.p + offsetof(IluChainState, poll_limit), &v, sizeof(v), cudaMemcpyHostToDevice, ctx->stream));
    return VFV_OK;
}

// z = (LU)^-1 r in one launch (k_ilu0_chain); t is a work vector of n entries that aliases neither
// r nor z. `timeout_flag` receives 1 if a bounded wait gave up.
template <typename T>
cudaError_t ilu_apply_chain(cudaStream_t s, IluStruct& S, const T* lu, const T* in, T* t, T* out, const DevStatus* st, int* timeout_flag,
                            int prio = 0, bool use_prio = false) {
    IluStruct::Chain& C = S.chain[chain_slot<T>()];
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)C.grid);
    cfg.blockDim = dim3(kChainThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    if (use_prio) {
        attr[0].id = cudaLaunchAttributePriority;
        attr[0].val.priority = prio;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    return cudaLaunchKernelEx(&cfg, k_ilu0_chain<T>, (int32_t)S.ntask, (int32_t)S.nlev, (const int32_t*)S.tasks.p,
                              (const int32_t*)S.task_lev.p, (const int32_t*)S.lev_ntask.p, (const int32_t*)S.rp.p, (const int32_t*)S.ci.p,
                              (const int32_t*)S.dg.p, lu, (const int32_t*)S.perm.p, in, t, out,
                              reinterpret_cast<IluChainState*>(C.state.p), timeout_flag, st);
}

constexpr int kStepsPerIf = 4;  // Arnoldi steps per IF node of a cycle graph

// Sets the IF condition of the next group of Arnoldi steps of a cycle graph: run it unless the solve stopped.
__global__ void k_step_condition(cudaGraphConditionalHandle h, const DevStatus* st) { cudaGraphSetConditional(h, st->done ? 0u : 1u); }

template <typename T>
struct Gmres : SolverBase {
    int64_t n = 0, ldv = 0;
    int m = 0, precond = 0, ilu_order = 0, engine = 0;
    int nblk = 0, mega_grid = 0, mega_chunk = 0;
    int nblk_v = 0;       // blocks of the multi-vector kernels (vec_block_rows<T>() rows each)
    DBuf<T> V, z, z2, zc, valK;
    DBuf<unsigned> bar;
    DBuf<unsigned long long> trace;  // per-phase timestamps of the last cycle (VFV_TRACE_CYCLE=1)
    DBuf<double> part, hacc, coef, H, cs, sn, g, beta, inv_beta, y, dinv, scal, x, b;
    DBuf<double> binv64;  // block-Jacobi inverses [16][n/4]
    DBuf<T> binvK;        // the same in the Krylov precision (aliases binv64 for double)
    DBuf<int> bj_bad;
    DBuf<unsigned> counter;
    DBuf<DevStatus> st;
    KrylovDev K{};
    cudaGraphExec_t exec = nullptr;
    int64_t graph_nodes = 0, step_nodes = 0;
    bool pending_steps = false;
    int steps_seen = 0;
    IluStruct* ilu = nullptr;
    uint64_t bj_version = ~0ull;
    // overlapped engine: preconditioned basis Z, SpMV output a, q = M^-1 a, the second stream
    DBuf<T> Zb, abuf, qbuf;
    DBuf<double> coefz;
    cudaStream_t s2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int ilu_prio = 0;  // greatest stream priority: the sweeps' blocks go first when SM slots free up
    bool ilu_chain = false;  // ILU(0) sweeps as one k_ilu0_chain launch (VFV_ILU_CHAIN=1) instead of one launch per level
    int ortho = VFV_ORTHO_CGS2;  // Gram-Schmidt of the Arnoldi steps (vfv_gmres_opts::ortho)
    bool sweep_half = false;     // float solver: swept factors in row-scaled half precision (vfv_gmres_opts::ilu_sweep_half)
    DBuf<double> wn2;            // ||w||^2 for the reorthogonalisation test
    int sweeps = 0;          // > 0: ILU(0) applied by this many Jacobi sweeps of the lower factor (vfv_gmres_opts::ilu_sweeps)
    int usweeps = 0;         // and this many of the upper factor (ilu_sweeps_upper, or ilu_sweeps when 0)
    DBuf<T> swbuf;           // the sweeps' 5 work vectors
    T* swp[5] = {};
    SweepOps<T> sw_ops{};
    // batch of independent meshes (block-diagonal system), one Krylov recurrence per mesh
    int nm = 0;
    DBuf<int64_t> b_mesh_row, b_tile_row, b_rtile_row;
    DBuf<int32_t> b_tile_mesh, b_mesh_tile, b_rtile_mesh, b_mesh_rtile;
    DBuf<double> b_part, b_rpart, b_hacc, b_coef, b_H, b_cs, b_sn, b_g, b_beta, b_inv_beta, b_y, b_tol;
    DBuf<MeshStat> b_ms;
    DBuf<unsigned> b_counter;
    BatchDev B{};
    std::vector<MeshStat> mesh_stat;  // per-mesh state after the last solve
    long long wait_polls = kDefaultWaitPolls;  // bounded device waits of this solve (vfv_gmres_opts::wait_limit)
    ~Gmres() override {
        if (exec) cudaGraphExecDestroy(exec);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (s2) cudaStreamDestroy(s2);
    }

    int init(vfv_ctx* ctx, vfv_pattern* p, int m_, int precond_, int ilu_order_, int engine_, int sweeps_, int usweeps_, int ortho_,
             bool sweep_half_) {
        n = p->n;
        m = m_;
        precond = precond_;
        ilu_order = ilu_order_;
        engine = engine_;
        sweeps = precond == VFV_PRECOND_ILU0 ? sweeps_ : 0;
        usweeps = sweeps > 0 ? (usweeps_ > 0 ? usweeps_ : sweeps) : 0;
        ortho = ortho_;
        sweep_half = sweep_half_ && sweeps > 0 && !std::is_same<T, double>::value;
        ldv = (n + 63) / 64 * 64;
        nblk_v = (int)((n + vec_block_rows<T>() - 1) / vec_block_rows<T>());
        nblk = nblk_v;  // partial dots per vector
        const int64_t res_blocks = (n * kSpG + kBlk - 1) / kBlk;
        CK(V.alloc((size_t)(m + 1) * ldv));
        CK(cudaMemset(V.p, 0, sizeof(T) * (size_t)(m + 1) * ldv));
        if (precond == VFV_PRECOND_ILU0) {
            CK(z.alloc(n));
            CK(z2.alloc(n));
            CK(zc.alloc(n));
        }
        if (engine == VFV_ENGINE_OVERLAP) {
            CK(Zb.alloc((size_t)(m + 1) * ldv));
            CK(abuf.alloc(n));
            CK(qbuf.alloc(n));
            CK(coefz.alloc(kMaxBasis));
            int lo = 0, hi = 0;
            CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            ilu_prio = hi;
            CK(cudaStreamCreateWithPriority(&s2, cudaStreamNonBlocking, hi));
            CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        }
        if (precond == VFV_PRECOND_BJ4) {
            if (n % 4 != 0) return set_err(ctx, VFV_BAD_INPUT, "block-Jacobi(4) needs a system of 4 fields of equal length");
            CK(z.alloc(n));
            CK(binv64.alloc((size_t)4 * n));
            if (!std::is_same<T, double>::value) CK(binvK.alloc((size_t)4 * n));
            CK(bj_bad.alloc(1));
        }
        if (engine == VFV_ENGINE_PERSISTENT) {
            int per_sm = 0, sms = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gmres_cycle<T>, kMegaThreads, 0));
            CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
            if (per_sm < 1) return set_err(ctx, VFV_CUDA_ERROR, "cycle kernel cannot be resident");
            mega_grid = (int)std::min<int64_t>((int64_t)per_sm * sms, std::max<int64_t>(1, (n + 255) / 256));
            mega_chunk = (int)((n + mega_grid - 1) / mega_grid);
            CK(bar.alloc(2 * kGenOffset));
            CK(cudaMemset(bar.p, 0, 2 * kGenOffset * sizeof(unsigned)));
            if (const char* e = getenv("VFV_TRACE_CYCLE")) {
                if (e[0] == '1') {
                    CK(trace.alloc((size_t)(m + 2) * 8));
                    CK(cudaMemset(trace.p, 0, (size_t)(m + 2) * 8 * sizeof(unsigned long long)));
                }
            }
        }
        CK(part.alloc(std::max<int64_t>((int64_t)kMaxBasis * std::max(nblk, mega_grid), res_blocks) + 16));
        CK(hacc.alloc(kMaxBasis));
        CK(coef.alloc(kMaxBasis));
        CK(H.alloc((size_t)m * (m + 1)));
        CK(cs.alloc(m));
        CK(sn.alloc(m));
        CK(g.alloc(m + 1));
        CK(beta.alloc(m + 1));
        CK(inv_beta.alloc(m + 1));
        CK(y.alloc(m));
        CK(dinv.alloc(n));
        CK(scal.alloc(4));
        CK(x.alloc(n));
        CK(b.alloc(n));
        CK(counter.alloc(8));
        CK(cudaMemset(counter.p, 0, 8 * sizeof(unsigned)));
        CK(st.alloc(1));
        CK(cudaMemset(st.p, 0, sizeof(DevStatus)));
        const bool need_copy = (precond == VFV_PRECOND_JACOBI) || !std::is_same<T, double>::value;
        if (need_copy) CK(valK.alloc(p->nnz));
        K.n = n;
        K.ldv = ldv;
        K.m = m;
        K.nblk = nblk;
        K.part = part.p;
        K.counter = counter.p;
        K.hacc = hacc.p;
        K.coef = coef.p;
        K.H = H.p;
        K.cs = cs.p;
        K.sn = sn.p;
        K.g = g.p;
        K.beta = beta.p;
        K.inv_beta = inv_beta.p;
        K.y = y.p;
        K.st = st.p;
        K.scal = scal.p;
        CK(wn2.alloc(1));
        K.wnorm2 = wn2.p;
        K.coefz = coefz.p;
        if (precond == VFV_PRECOND_ILU0) {
            auto it = p->ilu.find(ilu_order);
            if (it == p->ilu.end()) {
                auto S = std::make_unique<IluStruct>();
                const IluStruct* twin = nullptr;
                if (p->same_as) {
                    auto jt = p->same_as->ilu.find(ilu_order);
                    if (jt != p->same_as->ilu.end()) twin = jt->second.get();
                }
                int rc = twin ? clone_ilu_struct(ctx, *twin, p->nnz, *S) : build_ilu_struct(ctx, p, ilu_order, *S);
                if (rc) return rc;
                it = p->ilu.emplace(ilu_order, std::move(S)).first;
            }
            ilu = it->second.get();
            if (sweeps > 0) {
                CK(swbuf.alloc((size_t)5 * n));
                for (int q = 0; q < 5; ++q) swp[q] = swbuf.p + (size_t)q * n;
            }
            if (const char* e = getenv("VFV_ILU_CHAIN")) ilu_chain = e[0] == '1' && sweeps == 0;
            if (ilu_chain) {
                int rc = chain_setup<T>(ctx, *ilu, n);
                if (rc) return rc;
            }
        }
        return VFV_OK;
    }

    // Tiles of the batched kernels from the mesh row ranges: vector tiles of vec_block_rows<T>() rows and
    // residual tiles of kBlk / kSpG rows, each starting at its mesh's first row.
    int init_batch(vfv_ctx* ctx, const std::vector<int64_t>& rows) {
        nm = (int)rows.size() - 1;
        std::vector<int64_t> tr, rr;
        std::vector<int32_t> tm, mt(nm + 1), rm, mr(nm + 1);
        const int64_t tv = vec_block_rows<T>(), tres = kBlk / kSpG;
        for (int q = 0; q < nm; ++q) {
            mt[q] = (int32_t)tm.size();
            mr[q] = (int32_t)rm.size();
            for (int64_t r = rows[q]; r < rows[q + 1]; r += tv) {
                tr.push_back(r);
                tm.push_back(q);
            }
            for (int64_t r = rows[q]; r < rows[q + 1]; r += tres) {
                rr.push_back(r);
                rm.push_back(q);
            }
        }
        mt[nm] = (int32_t)tm.size();
        mr[nm] = (int32_t)rm.size();
        tr.push_back(rows[nm]);
        rr.push_back(rows[nm]);
        cudaStream_t s = ctx->stream;
        CK(b_mesh_row.upload(rows.data(), rows.size(), s));
        CK(b_tile_row.upload(tr.data(), tr.size(), s));
        CK(b_tile_mesh.upload(tm.data(), tm.size(), s));
        CK(b_mesh_tile.upload(mt.data(), mt.size(), s));
        CK(b_rtile_row.upload(rr.data(), rr.size(), s));
        CK(b_rtile_mesh.upload(rm.data(), rm.size(), s));
        CK(b_mesh_rtile.upload(mr.data(), mr.size(), s));
        const int ntile = (int)tm.size(), nrtile = (int)rm.size();
        CK(b_part.alloc((size_t)kMaxBasis * ntile));
        CK(b_rpart.alloc(nrtile));
        CK(b_hacc.alloc((size_t)nm * kMaxBasis));
        CK(b_coef.alloc((size_t)nm * kMaxBasis));
        CK(b_H.alloc((size_t)nm * m * (m + 1)));
        CK(b_cs.alloc((size_t)nm * m));
        CK(b_sn.alloc((size_t)nm * m));
        CK(b_g.alloc((size_t)nm * (m + 1)));
        CK(b_beta.alloc((size_t)nm * (m + 1)));
        CK(b_inv_beta.alloc((size_t)nm * (m + 1)));
        CK(b_y.alloc((size_t)nm * m));
        CK(b_tol.alloc(nm));
        CK(b_ms.alloc(nm));
        CK(b_counter.alloc(4));
        CK(cudaMemset(b_counter.p, 0, 4 * sizeof(unsigned)));
        B.nm = nm;
        B.m = m;
        B.ldv = ldv;
        B.mesh_row = b_mesh_row.p;
        B.tile_row = b_tile_row.p;
        B.tile_mesh = b_tile_mesh.p;
        B.mesh_tile = b_mesh_tile.p;
        B.rtile_row = b_rtile_row.p;
        B.rtile_mesh = b_rtile_mesh.p;
        B.mesh_rtile = b_mesh_rtile.p;
        B.ntile = ntile;
        B.nrtile = nrtile;
        B.part = b_part.p;
        B.rpart = b_rpart.p;
        B.hacc = b_hacc.p;
        B.coef = b_coef.p;
        B.H = b_H.p;
        B.cs = b_cs.p;
        B.sn = b_sn.p;
        B.g = b_g.p;
        B.beta = b_beta.p;
        B.inv_beta = b_inv_beta.p;
        B.y = b_y.p;
        B.tol_abs = b_tol.p;
        B.ms = b_ms.p;
        B.counter = b_counter.p;
        B.st = st.p;
        B.scal = scal.p;
        return VFV_OK;
    }

    // z = M^-1 r for the ILU(0) preconditioner; `in` and `out` may alias. st: early exit once the
    // solve is done (null: always run).
    void apply_ilu(cudaStream_t s, const T* in, T* out, const DevStatus* stp, int prio = 0, bool use_prio = false) {
        if (sweeps > 0) ilu_apply_sweeps<T>(s, sw_ops, sweeps, usweeps, in, out, swp, stp, prio, use_prio);
        else if (ilu_chain) ilu_apply_chain<T>(s, *ilu, lu_vals(), in, z2.p, out, stp, &st.p->timeout, prio, use_prio);
        else ilu_apply_levels<T>(s, *ilu, lu_vals(), in, z2.p, out, stp, prio, use_prio);
    }

    const T* krylov_vals(vfv_pattern* p) const {
        if (valK.p) return valK.p;
        return reinterpret_cast<const T*>(p->val.p);
    }
    const T* bj_vals() const {
        if constexpr (std::is_same<T, double>::value) return binv64.p;
        else return binvK.p;
    }
    const T* lu_vals() const {
        if constexpr (std::is_same<T, double>::value) return ilu->lu64.p;
        else return ilu->lu32.p;
    }

    // The CGS2 passes of Arnoldi step j on w = A M^-1 u_j (in `win`; the result goes to `w`, which
    // may be the same vector): first-pass dots, update + second-pass dots, update + norm + Givens.
    // VFV_ORTHO_DGKS: first pass with ||w||^2, then a second pass whose three kernels return at once
    // unless the first pass's test asked for it; VFV_ORTHO_CGS: the first pass alone.
    void enqueue_ortho(cudaStream_t s, const T* win, T* w, int j) {
        const int nv = j + 1, fb = grid_for((int64_t)nv * 32), fb1 = grid_for((int64_t)(nv + 1) * 32);
        if (ortho == VFV_ORTHO_CGS2) {
            k_mdot<T><<<nblk, kBlk, 0, s>>>(K, V.p, win, nv, 0, 0);
            k_dots_finish<true><<<fb, 256, 0, s>>>(K, nv, 0, 0);
            k_update<T, false><<<nblk, kBlk, 0, s>>>(K, V.p, win, w, nv, j, 0, 0);
            k_dots_finish<false><<<fb, 256, 0, s>>>(K, nv, 0, 0);
            k_update<T, true><<<nblk, kBlk, 0, s>>>(K, V.p, w, w, nv, j, 0, 0);
            return;
        }
        const int dgks = ortho == VFV_ORTHO_DGKS ? 1 : 0;
        k_mdot<T><<<nblk, kBlk, 0, s>>>(K, V.p, win, nv, dgks, 0);
        k_dots_finish<true><<<dgks ? fb1 : fb, 256, 0, s>>>(K, nv, dgks, 0);
        k_update<T, true><<<nblk, kBlk, 0, s>>>(K, V.p, win, w, nv, j, dgks, 0);
        if (!dgks) return;
        k_mdot<T><<<nblk, kBlk, 0, s>>>(K, V.p, w, nv, 0, 1);
        k_dots_finish<false><<<fb, 256, 0, s>>>(K, nv, 0, 1);
        k_update<T, true><<<nblk, kBlk, 0, s>>>(K, V.p, w, w, nv, j, 0, 1);
    }

    // phase timestamps of the last cycle, averaged over its steps (diagnostics, VFV_TRACE_CYCLE=1)
    void dump_trace(vfv_ctx* ctx, int cycles) {
        std::vector<unsigned long long> h((size_t)(m + 2) * 8);
        if (cudaMemcpy(h.data(), trace.p, h.size() * sizeof(h[0]), cudaMemcpyDeviceToHost) != cudaSuccess) return;
        double ph[5] = {0, 0, 0, 0, 0};
        int steps = 0;
        for (int j = 0; j + 1 < m && h[(j + 1) * 8] != 0; ++j) {
            const unsigned long long* t = &h[j * 8];
            const unsigned long long nxt = h[(j + 1) * 8];
            ph[0] += t[1] - t[0];
            ph[1] += t[2] - t[1];
            ph[2] += t[3] - t[2];
            ph[3] += t[4] - t[3];
            ph[4] += nxt - t[4];
            ++steps;
        }
        if (steps == 0) return;
        fprintf(stderr, "[vfv trace] cycles=%d steps/cycle=%d  per step (us): ilu %.1f spmv %.1f pass1 %.1f pass2 %.1f pass3 %.1f ; "
                        "tail: lsq+update %.1f residual %.1f\n",
                cycles, steps, ph[0] / steps / 1e3, ph[1] / steps / 1e3, ph[2] / steps / 1e3, ph[3] / steps / 1e3, ph[4] / steps / 1e3,
                (h[(m + 0) * 8 + 1] - h[(m + 0) * 8 + 0]) / 1e3, (h[(m + 0) * 8 + 2] - h[(m + 0) * 8 + 1]) / 1e3);
        (void)ctx;
    }

    // Diagnostics (VFV_PROFILE_STEP=1): time the kernels of one Arnoldi step (j = m/2, on the
    // basis left by the last cycle) one group at a time with events, outside the graph.
    void profile_step(vfv_ctx* ctx, vfv_pattern* p) {
        cudaStream_t s = ctx->stream;
        constexpr int G = kSpG;
        const int j = m / 2;
        const T* vk = krylov_vals(p);
        const T* uj = V.p + (int64_t)j * ldv;
        T* w = V.p + (int64_t)(j + 1) * ldv;
        cudaEvent_t ev[6];
        for (auto& e : ev) cudaEventCreate(&e);
        cudaMemsetAsync(st.p, 0, sizeof(DevStatus), s);
        const T* in = uj;
        cudaEventRecord(ev[0], s);
        if (precond == VFV_PRECOND_ILU0) {
            apply_ilu(s, uj, z.p, st.p);
            in = z.p;
        }
        cudaEventRecord(ev[1], s);
        launch_spmv<T, T, T, T>(s, p->spmv_lanes[sizeof(T) == 8 ? 0 : 1], p->spmv_strides[sizeof(T) == 8 ? 0 : 1], n, p->rp.p, p->ci.p, vk, in, w, inv_beta.p + j, st.p);
        cudaEventRecord(ev[2], s);
        enqueue_ortho(s, w, w, j);
        cudaEventRecord(ev[3], s);
        cudaEventSynchronize(ev[3]);
        float t[3];
        for (int q = 0; q < 3; ++q) cudaEventElapsedTime(&t[q], ev[q], ev[q + 1]);
        fprintf(stderr, "[vfv step profile] %s j=%d (us): ilu %.1f spmv %.1f cgs2 passes %.1f\n", sizeof(T) == 4 ? "fp32" : "fp64", j,
                t[0] * 1e3, t[1] * 1e3, t[2] * 1e3);
        for (auto& e : ev) cudaEventDestroy(e);
    }

    CycleArgs cycle_args(vfv_pattern* p) const {
        CycleArgs A{};
        A.n = n;
        A.ldv = ldv;
        A.m = m;
        A.chunk = mega_chunk;
        A.precond = precond;
        A.rp = p->rp.p;
        A.ci = p->ci.p;
        A.valK = krylov_vals(p);
        A.val64 = p->val.p;
        A.b = b.p;
        A.x = x.p;
        A.dinv = dinv.p;
        if (ilu) {
            A.nlev = ilu->nlev;
            A.lev_ptr = ilu->d_lev_ptr.p;
            A.lrp = ilu->rp.p;
            A.lci = ilu->ci.p;
            A.ldg = ilu->dg.p;
            A.lu = lu_vals();
            A.perm = ilu->perm.p;
        }
        A.V = V.p;
        A.z = z.p;
        A.t = z2.p;
        A.zc = zc.p;
        A.H = H.p;
        A.cs = cs.p;
        A.sn = sn.p;
        A.g = g.p;
        A.beta = beta.p;
        A.inv_beta = inv_beta.p;
        A.y = y.p;
        A.hacc = hacc.p;
        A.coef = coef.p;
        A.part = part.p;
        A.bar = bar.p;
        A.trace = trace.p;
        A.st = st.p;
        A.scal = scal.p;
        A.spin_limit = wait_polls;
        return A;
    }

    // One restart cycle = prologue, m Arnoldi steps, epilogue (least squares, update of x, new residual).
    //
    // Overlapped engine (ILU(0) only): flexible GMRES whose preconditioned vectors come by linearity,
    // z_{j+1} = M^-1 w - sum_i c_i z_i, so the latency-bound ILU(0) sweeps of M^-1 w run on a second
    // stream while the bandwidth-bound CGS2 passes orthogonalise w; the correction of x is Z y.
    void enqueue_prologue(cudaStream_t s) {
        if (engine == VFV_ENGINE_OVERLAP) apply_ilu(s, V.p, Zb.p, st.p);  // z_0 = M^-1 u_0
    }

    void enqueue_step(cudaStream_t s, vfv_pattern* p, int j) {
        const T* vk = krylov_vals(p);
        const int lanes = p->spmv_lanes[sizeof(T) == 8 ? 0 : 1], strides = p->spmv_strides[sizeof(T) == 8 ? 0 : 1];
        T* w = V.p + (int64_t)(j + 1) * ldv;
        if (nm > 0) {  // one recurrence per mesh of a batch
            const T* uj = V.p + (int64_t)j * ldv;
            const T* in = uj;
            if (precond == VFV_PRECOND_ILU0) {
                apply_ilu(s, uj, z.p, st.p);
                in = z.p;
            }
            launch_spmv_seg<T, T, T, T>(s, lanes, strides, n, p->rp.p, p->ci.p, vk, in, w, b_inv_beta.p, m + 1, j, b_mesh_row.p, nm, st.p);
            const int nv = j + 1, fb = grid_for((int64_t)nm * nv * 32);
            k_bmdot<T><<<B.ntile, kBlk, 0, s>>>(B, V.p, w, nv);
            k_bdots_finish<true><<<fb, 256, 0, s>>>(B, nv);
            k_bupdate<T, false><<<B.ntile, kBlk, 0, s>>>(B, V.p, w, w, nv);
            k_bdots_finish<false><<<fb, 256, 0, s>>>(B, nv);
            k_bupdate<T, true><<<B.ntile, kBlk, 0, s>>>(B, V.p, w, w, nv);
            k_bstep_finish<<<nm, kBlk, 0, s>>>(B, j);
            return;
        }
        if (engine == VFV_ENGINE_OVERLAP) {
            launch_spmv<T, T, T, T>(s, lanes, strides, n, p->rp.p, p->ci.p, vk, Zb.p + (int64_t)j * ldv, abuf.p, inv_beta.p + j, st.p);
            cudaEventRecord(ev_fork, s);
            cudaStreamWaitEvent(s2, ev_fork, 0);
            apply_ilu(s2, abuf.p, qbuf.p, st.p, ilu_prio, true);
            cudaEventRecord(ev_join, s2);
            enqueue_ortho(s, abuf.p, w, j);
            cudaStreamWaitEvent(s, ev_join, 0);
            k_zupdate<T><<<nblk_v, kBlk, 0, s>>>(K, Zb.p, qbuf.p, j + 1, j);
            return;
        }
        const T* uj = V.p + (int64_t)j * ldv;
        const T* in = uj;
        if (precond == VFV_PRECOND_ILU0) {
            apply_ilu(s, uj, z.p, st.p);
            in = z.p;
        } else if (precond == VFV_PRECOND_BJ4) {
            k_bj4_apply<T><<<grid_for(n / 4), 256, 0, s>>>(n / 4, bj_vals(), uj, z.p, st.p);
            in = z.p;
        }
        launch_spmv<T, T, T, T>(s, lanes, strides, n, p->rp.p, p->ci.p, vk, in, w, inv_beta.p + j, st.p);
        enqueue_ortho(s, w, w, j);
    }

    void enqueue_epilogue(cudaStream_t s, vfv_pattern* p) {
        constexpr int G = kSpG;
        const int sp_blocks = grid_for(n * G);
        const int vb = grid_for(n);
        if (nm > 0) {
            k_bbacksolve<<<grid_for(nm, 128), 128, 0, s>>>(B);
            if (precond == VFV_PRECOND_ILU0) {
                k_bcombine<T, 2><<<B.ntile, kBlk, 0, s>>>(B, V.p, x.p, nullptr, z.p);
                apply_ilu(s, z.p, z.p, nullptr);
                k_add_to_x<T><<<vb, 256, 0, s>>>(n, x.p, z.p);
            } else if (precond == VFV_PRECOND_JACOBI) {
                k_bcombine<T, 1><<<B.ntile, kBlk, 0, s>>>(B, V.p, x.p, dinv.p, nullptr);
            } else {
                k_bcombine<T, 0><<<B.ntile, kBlk, 0, s>>>(B, V.p, x.p, nullptr, nullptr);
            }
            k_bresidual<T, G><<<B.nrtile, kBlk, 0, s>>>(B, p->rp.p, p->ci.p, p->val.p, x.p, b.p, V.p);
            k_bresid_finish<<<nm, kBlk, 0, s>>>(B);
            return;
        }
        k_backsolve<<<1, 32, 0, s>>>(K);
        if (engine == VFV_ENGINE_OVERLAP) {
            k_combine<T, 0><<<vb, kBlk, 0, s>>>(K, Zb.p, x.p, nullptr, nullptr);
        } else if (precond == VFV_PRECOND_ILU0) {
            k_combine<T, 2><<<vb, kBlk, 0, s>>>(K, V.p, x.p, nullptr, z.p);
            apply_ilu(s, z.p, z.p, nullptr);  // in place: row i's upper result is written after row i's input was read
            k_add_to_x<T><<<vb, 256, 0, s>>>(n, x.p, z.p);
        } else if (precond == VFV_PRECOND_BJ4) {
            k_combine<T, 2><<<vb, kBlk, 0, s>>>(K, V.p, x.p, nullptr, z.p);
            k_bj4_apply<T><<<grid_for(n / 4), 256, 0, s>>>(n / 4, bj_vals(), z.p, z.p, nullptr);
            k_add_to_x<T><<<vb, 256, 0, s>>>(n, x.p, z.p);
        } else if (precond == VFV_PRECOND_JACOBI) {
            k_combine<T, 1><<<vb, kBlk, 0, s>>>(K, V.p, x.p, dinv.p, nullptr);
        } else {
            k_combine<T, 0><<<vb, kBlk, 0, s>>>(K, V.p, x.p, nullptr, nullptr);
        }
        k_residual<T, G><<<sp_blocks, kBlk, 0, s>>>(K, p->rp.p, p->ci.p, p->val.p, x.p, b.p, V.p);
    }

    // The whole cycle, captured as one straight graph (every step's kernels return at once once the
    // device `done` flag is set).
    void enqueue_cycle(cudaStream_t s, vfv_pattern* p) {
        enqueue_prologue(s);
        for (int j = 0; j < m; ++j) enqueue_step(s, p, j);
        enqueue_epilogue(s, p);
    }

    // Appends what `fn` enqueues on s to graph g after the nodes `deps`; returns the new frontier.
    template <typename F>
    cudaError_t capture_into(cudaStream_t s, cudaGraph_t g, std::vector<cudaGraphNode_t>& deps, F fn) {
        cudaError_t e = cudaStreamBeginCaptureToGraph(s, g, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                                      cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            if (const char* t = getenv("VFV_TRACE_SOLVE"))
                if (t[0] == '1') fprintf(stderr, "[vfv] begin capture to graph: %s (deps %zu)\n", cudaGetErrorString(e), deps.size());
            return e;
        }
        fn();
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t* nd = nullptr;
        size_t nn = 0;
        cudaError_t e2 = cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &nd, &nn);
        if (e2 != cudaSuccess)
            if (const char* t = getenv("VFV_TRACE_SOLVE"))
                if (t[0] == '1') fprintf(stderr, "[vfv] capture info: %s\n", cudaGetErrorString(e2));
        std::vector<cudaGraphNode_t> front(nd, nd + (e2 == cudaSuccess ? nn : 0));
        cudaGraph_t out = nullptr;
        e = cudaStreamEndCapture(s, &out);
        if (e2 != cudaSuccess) return e2;
        if (e != cudaSuccess) return e;
        deps.swap(front);
        return cudaSuccess;
    }

    // The cycle as a graph whose Arnoldi steps sit in IF nodes, kStepsPerIf steps per node: a
    // one-thread kernel before each node sets the condition from the device `done` flag, so the
    // groups after convergence cost one tiny launch each instead of ~25 kernels per step (a step of
    // a running group that finds the solve done still returns at once, as in the straight graph). Returns an error (and leaves no graph) where the
    // CUDA driver cannot build it; the caller then captures the straight graph.
    cudaError_t build_conditional_graph(cudaStream_t s, vfv_pattern* p, cudaGraph_t* out, int64_t* top_nodes, int64_t* step_nodes) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaGraphCreate(&g, 0);
        if (e != cudaSuccess) return e;
        std::vector<cudaGraphNode_t> deps;
        int64_t body_nodes = 0;
        const char* stage = "prologue";
        e = capture_into(s, g, deps, [&] { enqueue_prologue(s); });
        for (int j0 = 0; j0 < m && e == cudaSuccess; j0 += kStepsPerIf) {
            const int j1 = std::min(m, j0 + kStepsPerIf);
            stage = "handle";  // one handle per conditional node
            cudaGraphConditionalHandle h;
            e = cudaGraphConditionalHandleCreate(&h, g, 1u, cudaGraphCondAssignDefault);
            if (e != cudaSuccess) break;
            stage = "condition kernel";
            e = capture_into(s, g, deps, [&] { k_step_condition<<<1, 1, 0, s>>>(h, st.p); });
            if (e != cudaSuccess) break;
            stage = "conditional node";
            cudaGraphNodeParams np{};
            np.type = cudaGraphNodeTypeConditional;
            np.conditional.handle = h;
            np.conditional.type = cudaGraphCondTypeIf;
            np.conditional.size = 1;
            cudaGraphNode_t cn;
            e = cudaGraphAddNode(&cn, g, deps.empty() ? nullptr : deps.data(), deps.size(), &np);
            if (e != cudaSuccess) break;
            cudaGraph_t body = np.conditional.phGraph_out[0];
            std::vector<cudaGraphNode_t> none;
            stage = "step body";
            e = capture_into(s, body, none, [&] {
                for (int j = j0; j < j1; ++j) enqueue_step(s, p, j);
            });
            if (e == cudaSuccess && j0 == 0) {
                size_t bn = 0;
                e = cudaGraphGetNodes(body, nullptr, &bn);
                body_nodes = (int64_t)bn / (j1 - j0);
            }
            deps.assign(1, cn);
        }
        if (e == cudaSuccess) {
            stage = "epilogue";
            e = capture_into(s, g, deps, [&] { enqueue_epilogue(s, p); });
        }
        if (e != cudaSuccess) {
            if (const char* t = getenv("VFV_TRACE_SOLVE"))
                if (t[0] == '1') fprintf(stderr, "[vfv] conditional cycle graph not built (%s, %zu dependencies): %s\n", stage, deps.size(), cudaGetErrorString(e));
            cudaGraphDestroy(g);
            cudaGetLastError();
            return e;
        }
        size_t tn = 0;
        cudaGraphGetNodes(g, nullptr, &tn);
        *out = g;
        *top_nodes = (int64_t)tn;
        *step_nodes = body_nodes;
        return cudaSuccess;
    }

    // A batched solver (nm > 0, a block-diagonal system of independent meshes) runs one Krylov
    // recurrence per mesh and stops when every mesh meets ||b_i - A_i x_i|| <= tol ||b_i||.
    int solve(vfv_ctx* ctx, vfv_pattern* p, const double* d_b, const double* d_x0, double* d_x, const vfv_gmres_opts& o,
              vfv_solve_info* info) {
        cudaStream_t s = ctx->stream;
        constexpr int G = kSpG;
        const bool mixed = !std::is_same<T, double>::value;
        CK(cudaMemcpyAsync(b.p, d_b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(x.p, d_x0, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        wait_polls = o.wait_limit > 0 ? (long long)o.wait_limit : kDefaultWaitPolls;
        if (ilu && ilu_chain) {
            int rc = chain_set_polls<T>(ctx, *ilu, wait_polls);
            if (rc) return rc;
        }
        // matrix preparation for this solve
        if (precond == VFV_PRECOND_JACOBI) {
            k_jacobi_inv<<<grid_for(n), 256, 0, s>>>(n, p->diag_pos.p, p->val.p, dinv.p);
            k_scale_cols<T><<<grid_for(p->nnz), 256, 0, s>>>(p->nnz, p->ci.p, p->val.p, dinv.p, valK.p);
            ctx->launches += 2;
        } else if (valK.p) {
            k_scale_cols<T><<<grid_for(p->nnz), 256, 0, s>>>(p->nnz, p->ci.p, p->val.p, nullptr, valK.p);
            ctx->launches += 1;
        }
        if (precond == VFV_PRECOND_ILU0) {
            int rc = ilu_refresh(ctx, p, *ilu, mixed, wait_polls);
            if (!rc && sweeps > 0) rc = ilu_split_refresh<T>(ctx, p, *ilu, sweep_half);
            if (rc) return rc;
            if (sweeps > 0) sw_ops = sweep_ops<T>(p, *ilu, sweep_half);
        }
        if (precond == VFV_PRECOND_BJ4 && bj_version != p->version) {
            CK(cudaMemsetAsync(bj_bad.p, 0, sizeof(int), s));
            launch_bj4_setup(s, n / 4, p->rp.p, p->ci.p, p->val.p, binv64.p, bj_bad.p);
            if (binvK.p) k_cast<double, T><<<grid_for(4 * n), 256, 0, s>>>(4 * n, binv64.p, binvK.p);
            ctx->launches += binvK.p ? 2 : 1;
            int bad = 0;
            CK(cudaMemcpyAsync(&bad, bj_bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            if (bad) return set_err(ctx, VFV_NONFINITE, "block-Jacobi(4): singular diagonal block");
            bj_version = p->version;
        }
        double bnorm = 0.0, tol_abs = 0.0;
        if (nm > 0) {
            // per-mesh ||b_i||, tolerances and first residuals (meshes with b_i = 0 get x_i = 0)
            const double hs[2] = {0.0, mixed ? std::max(0.0, o.inner_rtol) : 0.0};
            CK(cudaMemcpyAsync(scal.p, hs, 2 * sizeof(double), cudaMemcpyHostToDevice, s));
            CK(cudaMemsetAsync(st.p, 0, sizeof(DevStatus), s));
            k_bnorm<<<nm, kBlk, 0, s>>>(B, b.p, o.tol);
            k_bzero_x<<<grid_for(n), 256, 0, s>>>(B, x.p);
            k_bresidual<T, G><<<B.nrtile, kBlk, 0, s>>>(B, p->rp.p, p->ci.p, p->val.p, x.p, b.p, V.p);
            k_bresid_finish<<<nm, kBlk, 0, s>>>(B);
            ctx->launches += 4;
            if (info) info->levels = ilu ? ilu->nlev : 0;
        } else {
            // ||b|| and the absolute tolerance
            const int nb = std::min(grid_for(n), 1024);
            k_norm2<<<nb, kBlk, 0, s>>>(n, b.p, part.p, counter.p + 4, scal.p + 2);
            ctx->launches += 1;
            CK(cudaMemcpyAsync(ctx->h_scalar, scal.p + 2, sizeof(double), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            CK(cudaGetLastError());
            bnorm = std::sqrt(ctx->h_scalar[0]);
            if (info) {
                info->bnorm = bnorm;
                info->levels = ilu ? ilu->nlev : 0;
            }
            if (!std::isfinite(bnorm)) return set_err(ctx, VFV_NONFINITE, "right-hand side is not finite");
            if (bnorm == 0.0) {
                CK(cudaMemsetAsync(d_x, 0, n * sizeof(double), s));
                CK(cudaStreamSynchronize(s));
                if (info) {
                    info->status = VFV_OK;
                    info->iters = info->cycles = 0;
                    info->relres = 0.0;
                }
                return VFV_OK;
            }
            tol_abs = o.tol * bnorm;
            const double hs[2] = {tol_abs, mixed ? std::max(0.0, o.inner_rtol) : 0.0};
            CK(cudaMemcpyAsync(scal.p, hs, 2 * sizeof(double), cudaMemcpyHostToDevice, s));
            CK(cudaMemsetAsync(st.p, 0, sizeof(DevStatus), s));
            k_residual<T, G><<<grid_for(n * G), kBlk, 0, s>>>(K, p->rp.p, p->ci.p, p->val.p, x.p, b.p, V.p);
            ctx->launches += 1;
        }
        if (engine != VFV_ENGINE_PERSISTENT && !exec) {
            cudaGraph_t graph = nullptr;
            cudaError_t e = cudaErrorUnknown;
            if (!getenv("VFV_STRAIGHT_GRAPH")) {  // conditional steps unless asked for the straight graph
                e = build_conditional_graph(s, p, &graph, &graph_nodes, &step_nodes);
                if (e == cudaSuccess) {
                    e = cudaGraphInstantiate(&exec, graph, 0);
                    cudaGraphDestroy(graph);
                    if (e != cudaSuccess) {
                        if (const char* t = getenv("VFV_TRACE_SOLVE"))
                            if (t[0] == '1') fprintf(stderr, "[vfv] conditional cycle graph not instantiated: %s\n", cudaGetErrorString(e));
                        exec = nullptr;
                        cudaGetLastError();
                    }
                }
            }
            if (e != cudaSuccess) {
                step_nodes = 0;
                CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                enqueue_cycle(s, p);
                CK(cudaStreamEndCapture(s, &graph));
                size_t nodes = 0;
                CK(cudaGraphGetNodes(graph, nullptr, &nodes));
                graph_nodes = (int64_t)nodes;
                e = cudaGraphInstantiate(&exec, graph, 0);
                cudaGraphDestroy(graph);
                CK(e);
            }
        }
        int cycles = 0, rc = VFV_OK;
        steps_seen = 0;
        pending_steps = false;
        DevStatus hst{};
        for (;;) {
            CK(cudaMemcpyAsync(ctx->h_status, st.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            hst = *ctx->h_status;
            if (pending_steps) {
                ctx->launches += step_nodes * (int64_t)(hst.total_steps - steps_seen);
                pending_steps = false;
            }
            steps_seen = hst.total_steps;
            if (hst.timeout) {
                rc = VFV_TIMEOUT;
                // the state of the wait that gave up is undefined: grid barrier, ILU sweep chain
                if (bar.p) CK(cudaMemsetAsync(bar.p, 0, 2 * kGenOffset * sizeof(unsigned), s));
                CK(cudaMemsetAsync(st.p, 0, sizeof(DevStatus), s));
                if (ilu && ilu_chain) {
                    int rc2 = chain_reset<T>(ctx, *ilu, wait_polls);
                    if (rc2) return rc2;
                }
                break;
            }
            if (hst.nonfinite) {
                rc = VFV_NONFINITE;
                break;
            }
            if (hst.converged) break;
            if (cycles >= o.max_outer) {
                rc = VFV_NOT_CONVERGED;
                break;
            }
            if (engine != VFV_ENGINE_PERSISTENT) {
                CK(cudaGraphLaunch(exec, s));
                // straight graph: every node launches; conditional graph: the top-level nodes, plus
                // the bodies of the steps run (counted when the cycle's status comes back)
                ctx->launches += graph_nodes;
                pending_steps = step_nodes > 0;
            } else {
                CycleArgs A = cycle_args(p);
                void* args[] = {&A};
                CK(cudaLaunchCooperativeKernel((const void*)k_gmres_cycle<T>, dim3(mega_grid), dim3(kMegaThreads), args, 0, s));
                ctx->launches += 1;
            }
            ++cycles;
        }
        CK(cudaGetLastError());
        if (trace.p) dump_trace(ctx, cycles);
        if (const char* e = getenv("VFV_PROFILE_STEP")) {
            if (e[0] == '1' && engine == VFV_ENGINE_GRAPH && nm == 0) profile_step(ctx, p);
        }

        CK(cudaMemcpyAsync(d_x, x.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        double relres = bnorm > 0.0 ? hst.beta0 / bnorm : 0.0;
        if (nm > 0) {  // the batch's relative residual is its worst mesh's
            mesh_stat.resize(nm);
            CK(cudaMemcpyAsync(mesh_stat.data(), b_ms.p, nm * sizeof(MeshStat), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            relres = 0.0;
            for (const MeshStat& M : mesh_stat) {
                bnorm = std::max(bnorm, M.bnorm);
                if (M.bnorm > 0.0) relres = std::max(relres, M.beta0 / M.bnorm);
            }
            if (info) info->bnorm = bnorm;
        }
        CK(cudaStreamSynchronize(s));
        if (const char* e = getenv("VFV_TRACE_SOLVE")) {  // diagnostics: one line per solve
            if (e[0] == '1')
                fprintf(stderr, "[vfv solve] n=%lld %s cycles=%d iters=%d relres=%.3e bnorm=%.3e tol_abs=%.3e meshes=%d\n", (long long)n,
                        mixed ? "mixed" : "fp64", cycles, hst.total_steps, relres, bnorm, tol_abs, nm);
        }
        if (info) {
            info->status = rc;
            info->iters = hst.total_steps;
            info->cycles = cycles;
            info->relres = relres;
        }
        if (rc == VFV_NOT_CONVERGED)
            return set_err(ctx, rc, "GMRES did not converge in " + std::to_string(o.max_outer) + " restart cycles (relres " +
                                        std::to_string(relres) + ")");
        if (rc == VFV_NONFINITE) return set_err(ctx, rc, "GMRES: non-finite residual");
        if (rc == VFV_TIMEOUT) return set_err(ctx, rc, "GMRES: a bounded device wait gave up (grid barrier or ILU(0) sweep)");
        return VFV_OK;
    }
};

}  // namespace

int check_opts(vfv_ctx* ctx, const vfv_gmres_opts* o) {
    if (!o) return set_err(ctx, VFV_BAD_INPUT, "opts is NULL");
    if (!(o->tol > 0.0)) return set_err(ctx, VFV_BAD_INPUT, "tol must be positive (LinearGmresNonPositiveTolerance)");
    if (o->restart <= 0 || o->restart + 1 > kMaxBasis) return set_err(ctx, VFV_BAD_INPUT, "restart must be in [1, 127]");
    if (o->max_outer <= 0) return set_err(ctx, VFV_BAD_INPUT, "max_outer must be positive (LinearGmresNonPositiveMaxOuter)");
    if (o->precond < VFV_PRECOND_NONE || o->precond > VFV_PRECOND_BJ4) return set_err(ctx, VFV_BAD_INPUT, "unknown preconditioner");
    if (o->precond == VFV_PRECOND_BJ4 && o->engine == VFV_ENGINE_PERSISTENT)
        return set_err(ctx, VFV_BAD_INPUT, "block-Jacobi(4) runs on the graph engine only");
    if (o->precision != VFV_FP64 && o->precision != VFV_MIXED) return set_err(ctx, VFV_BAD_INPUT, "unknown precision");
    if (o->ilu_order != VFV_ILU_MULTICOLOR && o->ilu_order != VFV_ILU_NATURAL) return set_err(ctx, VFV_BAD_INPUT, "unknown ILU ordering");
    if (o->engine != VFV_ENGINE_PERSISTENT && o->engine != VFV_ENGINE_GRAPH && o->engine != VFV_ENGINE_OVERLAP)
        return set_err(ctx, VFV_BAD_INPUT, "unknown engine");
    if (o->engine == VFV_ENGINE_OVERLAP && o->precond != VFV_PRECOND_ILU0)
        return set_err(ctx, VFV_BAD_INPUT, "the overlapped engine needs the ILU(0) preconditioner");
    if (o->wait_limit < 0) return set_err(ctx, VFV_BAD_INPUT, "wait_limit must be >= 0 (0 = default)");
    if (o->ilu_sweeps < 0 || o->ilu_sweeps > kMaxIluSweeps) return set_err(ctx, VFV_BAD_INPUT, "ilu_sweeps must be in [0, 16]");
    if (o->ilu_sweeps_upper < 0 || o->ilu_sweeps_upper > kMaxIluSweeps)
        return set_err(ctx, VFV_BAD_INPUT, "ilu_sweeps_upper must be in [0, 16]");
    if (o->ilu_sweep_half != 0 && (o->precond != VFV_PRECOND_ILU0 || o->ilu_sweeps == 0 || o->precision != VFV_MIXED))
        return set_err(ctx, VFV_BAD_INPUT, "ilu_sweep_half needs the mixed precision and ILU(0) with ilu_sweeps > 0");
    if (o->ortho != VFV_ORTHO_CGS2 && o->ortho != VFV_ORTHO_DGKS && o->ortho != VFV_ORTHO_CGS)
        return set_err(ctx, VFV_BAD_INPUT, "unknown orthogonalisation");
    if (o->ortho != VFV_ORTHO_CGS2 && o->engine == VFV_ENGINE_PERSISTENT)
        return set_err(ctx, VFV_BAD_INPUT, "the persistent engine orthogonalises with CGS2 only");
    if (o->ilu_sweeps > 0 && o->precond == VFV_PRECOND_ILU0 && o->engine == VFV_ENGINE_PERSISTENT)
        return set_err(ctx, VFV_BAD_INPUT, "ILU(0) sweeps run on the graph and overlapped engines only");
    return VFV_OK;
}

int solve_dev(vfv_ctx* ctx, vfv_pattern* p, const double* b, const double* x0, double* x, const vfv_gmres_opts* o, vfv_solve_info* info,
              bool batched) {
    vfv_gmres_opts oo = *o;
    batched = batched && p->blocks.size() > 2;
    if (batched) {
        if (oo.precond == VFV_PRECOND_BJ4) return set_err(ctx, VFV_BAD_INPUT, "block-Jacobi(4) is not offered for batches of meshes");
        oo.engine = VFV_ENGINE_GRAPH;  // the per-mesh recurrences run on the graph engine
    }
    const auto key = solver_key(oo, batched);
    auto it = p->solvers.find(key);
    if (it == p->solvers.end()) {
        std::unique_ptr<SolverBase> sb;
        int rc;
        if (oo.precision == VFV_MIXED) {
            auto g = std::make_unique<Gmres<float>>();
            rc = g->init(ctx, p, oo.restart, oo.precond, oo.ilu_order, oo.engine, oo.ilu_sweeps, oo.ilu_sweeps_upper, batched ? VFV_ORTHO_CGS2 : oo.ortho,
                         oo.ilu_sweep_half != 0);
            if (!rc && batched) rc = g->init_batch(ctx, p->blocks);
            sb = std::move(g);
        } else {
            auto g = std::make_unique<Gmres<double>>();
            rc = g->init(ctx, p, oo.restart, oo.precond, oo.ilu_order, oo.engine, oo.ilu_sweeps, oo.ilu_sweeps_upper, batched ? VFV_ORTHO_CGS2 : oo.ortho,
                         oo.ilu_sweep_half != 0);
            if (!rc && batched) rc = g->init_batch(ctx, p->blocks);
            sb = std::move(g);
        }
        if (rc) return rc;
        it = p->solvers.emplace(key, std::move(sb)).first;
    }
    if (oo.precision == VFV_MIXED) return static_cast<Gmres<float>*>(it->second.get())->solve(ctx, p, b, x0, x, oo, info);
    return static_cast<Gmres<double>*>(it->second.get())->solve(ctx, p, b, x0, x, oo, info);
}

// Per-mesh Arnoldi steps of the last batched solve of this pattern with these options (meshes in
// block order); false when no such solve exists.
std::tuple<int, int, int, int, int> solver_key(const vfv_gmres_opts& o, bool batched) {
    const bool ilu = o.precond == VFV_PRECOND_ILU0;
    const int up = o.ilu_sweeps > 0 ? (o.ilu_sweeps_upper > 0 ? o.ilu_sweeps_upper : o.ilu_sweeps) : 0;
    return std::make_tuple(o.precision, o.precond, ilu ? o.ilu_order + 16 * (o.ilu_sweeps + 32 * up + 1024 * (o.ilu_sweep_half != 0)) : 0,
                           o.restart,
                           (batched ? VFV_ENGINE_GRAPH : o.engine) + (batched ? 16 : 64 * o.ortho));
}

bool batch_mesh_steps(const vfv_pattern* p, const vfv_gmres_opts* o, std::vector<int32_t>& steps) {
    const auto key = solver_key(*o, true);
    auto it = p->solvers.find(key);
    if (it == p->solvers.end()) return false;
    const std::vector<MeshStat>* ms = nullptr;
    if (o->precision == VFV_MIXED) ms = &static_cast<Gmres<float>*>(it->second.get())->mesh_stat;
    else ms = &static_cast<Gmres<double>*>(it->second.get())->mesh_stat;
    steps.resize(ms->size());
    for (size_t i = 0; i < ms->size(); ++i) steps[i] = (*ms)[i].total_steps;
    return !ms->empty();
}

namespace {

int finish_pattern(vfv_ctx* ctx, vfv_pattern* p) {
    const int64_t n = p->n;
    std::vector<int32_t> dpos(n, -1);
    for (int64_t i = 0; i < n; ++i)
        for (int32_t k = p->h_rp[i]; k < p->h_rp[i + 1]; ++k)
            if (p->h_ci[k] == i) dpos[i] = k;
    cudaStream_t s = ctx->stream;
    CK(p->rp.upload(p->h_rp.data(), n + 1, s));
    CK(p->ci.upload(p->h_ci.data(), p->nnz, s));
    CK(p->diag_pos.upload(dpos.data(), n, s));
    CK(p->val.alloc(p->nnz));
    CK(cudaMemsetAsync(p->val.p, 0, p->nnz * sizeof(double), s));
    CK(cudaStreamSynchronize(s));
    return VFV_OK;
}

}  // namespace

// Transpose of a pattern: row j of A^T lists, in ascending order, the rows i of A with an entry in
// column j; tmap[k_t] = slot of that entry in A (values of A^T are a gather of A's).
int make_transpose(vfv_ctx* ctx, const vfv_pattern* p, vfv_pattern** out, DBuf<int32_t>& tmap_d) {
    const int64_t n = p->n, nnz = p->nnz;
    const std::vector<int32_t>& rp = p->h_rp;
    const std::vector<int32_t>& ci = p->h_ci;
    std::vector<int32_t> trp(n + 1, 0), tci(nnz), tmap(nnz);
    for (int64_t k = 0; k < nnz; ++k) trp[ci[k] + 1]++;
    for (int64_t j = 0; j < n; ++j) trp[j + 1] += trp[j];
    std::vector<int32_t> cur(trp.begin(), trp.end() - 1);
    for (int64_t i = 0; i < n; ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
            const int32_t q = cur[ci[k]]++;
            tci[q] = (int32_t)i;
            tmap[q] = k;
        }
    vfv_pattern* pt = nullptr;
    int rc = vfv_pattern_from_csr(ctx, n, trp.data(), tci.data(), &pt);
    if (rc) return rc;
    pt->blocks = p->blocks;
    if (trp == rp && tci == ci) pt->same_as = p;  // structurally symmetric: share the ILU orderings
    *out = pt;
    CK(tmap_d.upload(tmap.data(), nnz, ctx->stream));
    return VFV_OK;
}

// values of A^T into its pattern: a gather of A's through the transpose map
int gather_transpose_values(vfv_ctx* ctx, const vfv_pattern* p, vfv_pattern* pt, const int32_t* tmap) {
    k_gather_vals<double><<<grid_for(p->nnz), 256, 0, ctx->stream>>>(p->nnz, tmap, p->val.p, pt->val.p);
    ctx->launches += 1;
    pt->version++;
    CK(cudaGetLastError());
    return VFV_OK;
}

// ================================================================ C ABI
extern "C" {

void vfv_gmres_default_opts(vfv_gmres_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->tol = 1e-6;
    o->restart = 50;
    o->max_outer = 200;
    o->precond = VFV_PRECOND_JACOBI;
    o->precision = VFV_FP64;
    o->ilu_order = VFV_ILU_MULTICOLOR;
    o->engine = VFV_ENGINE_GRAPH;
    o->inner_rtol = 0.0;
    o->wait_limit = 0;
    o->ilu_sweeps = 0;
    o->ilu_sweeps_upper = 0;
    o->ortho = VFV_ORTHO_CGS2;
    o->ilu_sweep_half = 0;
}

int vfv_ctx_create(int device, vfv_ctx** out) {
    vfv_ctx* ctx = nullptr;
    if (!out) return set_err(nullptr, VFV_BAD_INPUT, "out is NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return set_err(nullptr, VFV_CUDA_ERROR, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (device < 0 || device >= count) return set_err(nullptr, VFV_BAD_INPUT, "device index out of range");
    CK(cudaSetDevice(device));
    ctx = new vfv_ctx();
    ctx->device = device;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMallocHost(&ctx->h_status, sizeof(DevStatus)) != cudaSuccess || cudaMallocHost(&ctx->h_scalar, 64) != cudaSuccess) {
        vfv_ctx_destroy(ctx);
        return set_err(nullptr, VFV_CUDA_ERROR, "context allocation failed");
    }
    *out = ctx;
    return VFV_OK;
}

void vfv_ctx_destroy(vfv_ctx* ctx) {
    DeviceGuard dg_(ctx);
    if (!ctx) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    if (ctx->h_scalar) cudaFreeHost(ctx->h_scalar);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* vfv_last_error(const vfv_ctx* ctx) { return ctx ? ctx->err.c_str() : vfv_thread_error().c_str(); }

int vfv_ctx_synchronize(vfv_ctx* ctx) {
    DeviceGuard dg_(ctx);
    if (!ctx) return set_err(nullptr, VFV_BAD_INPUT, "ctx is NULL");
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaGetLastError());
    return VFV_OK;
}

void* vfv_ctx_stream(vfv_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int64_t vfv_ctx_launch_count(const vfv_ctx* ctx) { return ctx ? ctx->launches : 0; }

int vfv_pattern_from_triplets(vfv_ctx* ctx, int64_t n, int64_t ntrip, const uint64_t* rows, const uint64_t* cols, vfv_pattern** out) {
    DeviceGuard dg_(ctx);
    if (!ctx || !out) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    *out = nullptr;
    if (n <= 0 || n >= (int64_t)1 << 31 || ntrip < 0 || (ntrip > 0 && (!rows || !cols)))
        return set_err(ctx, VFV_BAD_INPUT, "invalid matrix size or triplet arrays");
    std::vector<uint64_t> key(ntrip);
    std::vector<int64_t> idx(ntrip);
    int64_t bad = ntrip;  // first out-of-range triplet
#pragma omp parallel for schedule(static) reduction(min : bad)
    for (int64_t t = 0; t < ntrip; ++t) {
        if (rows[t] >= (uint64_t)n || cols[t] >= (uint64_t)n) {
            bad = std::min(bad, t);
            continue;
        }
        key[t] = rows[t] * (uint64_t)n + cols[t];
        idx[t] = t;
    }
    if (bad < ntrip) return set_err(ctx, VFV_BAD_INPUT, "triplet index out of range at " + std::to_string(bad));
    int bits = 1;
    while (bits < 64 && ((uint64_t)n * (uint64_t)n - 1) >> bits) ++bits;
    radix_sort_pairs(key, idx, bits);
    auto p = std::make_unique<vfv_pattern>();
    p->ctx = ctx;
    p->n = n;
    p->ntrip = ntrip;
    p->h_rp.assign(n + 1, 0);
    std::vector<int64_t> sp;
    sp.reserve(ntrip / 2 + 2);
    for (int64_t t = 0; t < ntrip; ++t) {
        if (t == 0 || key[t] != key[t - 1]) {
            sp.push_back(t);
            p->h_ci.push_back((int32_t)(key[t] % (uint64_t)n));
            p->h_rp[key[t] / (uint64_t)n + 1]++;
        }
    }
    sp.push_back(ntrip);
    for (int64_t i = 0; i < n; ++i) p->h_rp[i + 1] += p->h_rp[i];
    p->nnz = (int64_t)p->h_ci.size();
    if (p->nnz >= (int64_t)1 << 31) return set_err(ctx, VFV_BAD_INPUT, "too many non-zeros for 32-bit indices");
    int rc = finish_pattern(ctx, p.get());
    if (rc) return rc;
    cudaStream_t s = ctx->stream;
    CK(p->slot_ptr.upload(sp.data(), sp.size(), s));
    CK(p->slot_trip.upload(idx.data(), ntrip, s));
    CK(p->trip_vals.alloc(ntrip));
    *out = p.release();
    return VFV_OK;
}

int vfv_pattern_from_csr(vfv_ctx* ctx, int64_t n, const int32_t* rowptr, const int32_t* colind, vfv_pattern** out) {
    DeviceGuard dg_(ctx);
    if (!ctx || !out || !rowptr) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    *out = nullptr;
    if (n <= 0 || n >= (int64_t)1 << 31 || rowptr[0] != 0) return set_err(ctx, VFV_BAD_INPUT, "invalid CSR");
    auto p = std::make_unique<vfv_pattern>();
    p->ctx = ctx;
    p->n = n;
    p->h_rp.assign(rowptr, rowptr + n + 1);
    p->nnz = p->h_rp[n];
    if (p->nnz > 0 && !colind) return set_err(ctx, VFV_BAD_INPUT, "colind is NULL");
    p->h_ci.assign(colind, colind + p->nnz);
    for (int64_t i = 0; i < n; ++i) {
        if (p->h_rp[i + 1] < p->h_rp[i]) return set_err(ctx, VFV_BAD_INPUT, "rowptr not monotone");
        for (int32_t k = p->h_rp[i]; k < p->h_rp[i + 1]; ++k) {
            if (p->h_ci[k] < 0 || p->h_ci[k] >= n) return set_err(ctx, VFV_BAD_INPUT, "column index out of range");
            if (k > p->h_rp[i] && p->h_ci[k] <= p->h_ci[k - 1]) return set_err(ctx, VFV_BAD_INPUT, "columns not strictly ascending");
        }
    }
    int rc = finish_pattern(ctx, p.get());
    if (rc) return rc;
    *out = p.release();
    return VFV_OK;
}

void vfv_pattern_destroy(vfv_pattern* p) {
    if (!p) return;
    if (p->ctx) cudaStreamSynchronize(p->ctx->stream);
    delete p;
}

int vfv_pattern_info(const vfv_pattern* p, int64_t* n, int64_t* nnz, int64_t* ntrip) {
    if (!p) return set_err(nullptr, VFV_BAD_INPUT, "pattern is NULL");
    if (n) *n = p->n;
    if (nnz) *nnz = p->nnz;
    if (ntrip) *ntrip = p->ntrip;
    return VFV_OK;
}

int vfv_values_from_triplets(vfv_ctx* ctx, vfv_pattern* p, const double* vals) {
    DeviceGuard dg_(ctx);
    if (!ctx || !p) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    if (!p->slot_ptr.p && p->ntrip == 0 && p->nnz > 0) return set_err(ctx, VFV_BAD_INPUT, "pattern has no triplet map");
    if (p->ntrip > 0 && !vals) return set_err(ctx, VFV_BAD_INPUT, "vals is NULL");
    cudaStream_t s = ctx->stream;
    if (p->ntrip > 0) CK(cudaMemcpyAsync(p->trip_vals.p, vals, p->ntrip * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_values_from_triplets(s, p->nnz, p->slot_ptr.p, p->slot_trip.p, p->trip_vals.p, p->val.p);
    ctx->launches += 1;
    CK(cudaGetLastError());
    p->version++;
    return VFV_OK;
}

int vfv_values_set(vfv_ctx* ctx, vfv_pattern* p, const double* vals, int on_device) {
    DeviceGuard dg_(ctx);
    if (!ctx || !p || !vals) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    CK(cudaMemcpyAsync(p->val.p, vals, p->nnz * sizeof(double), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
    p->version++;
    return VFV_OK;
}

int vfv_csr_export(vfv_ctx* ctx, const vfv_pattern* p, int32_t* rowptr, int32_t* colind, double* vals) {
    DeviceGuard dg_(ctx);
    if (!ctx || !p) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    if (rowptr) std::memcpy(rowptr, p->h_rp.data(), (p->n + 1) * sizeof(int32_t));
    if (colind) std::memcpy(colind, p->h_ci.data(), p->nnz * sizeof(int32_t));
    if (vals) {
        CK(cudaMemcpyAsync(vals, p->val.p, p->nnz * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return VFV_OK;
}

int vfv_solve_device(vfv_ctx* ctx, vfv_pattern* p, const double* b, const double* x0, double* x, const vfv_gmres_opts* opts,
                     vfv_solve_info* info) {
    DeviceGuard dg_(ctx);
    if (!ctx || !p || !b || !x0 || !x) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    int rc = check_opts(ctx, opts);
    if (rc) return rc;
    if (info) std::memset(info, 0, sizeof(*info));
    return solve_dev(ctx, p, b, x0, x, opts, info);
}

int vfv_solve(vfv_ctx* ctx, vfv_pattern* p, const double* b, const double* x0, double* x, const vfv_gmres_opts* opts,
              vfv_solve_info* info) {
    DeviceGuard dg_(ctx);
    if (!ctx || !p || !b || !x0 || !x) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    int rc = check_opts(ctx, opts);
    if (rc) return rc;
    if (info) std::memset(info, 0, sizeof(*info));
    cudaStream_t s = ctx->stream;
    if (!p->tmp_b.p) {
        CK(p->tmp_b.alloc(p->n));
        CK(p->tmp_x.alloc(p->n));
    }
    CK(cudaMemcpyAsync(p->tmp_b.p, b, p->n * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(p->tmp_x.p, x0, p->n * sizeof(double), cudaMemcpyHostToDevice, s));
    rc = solve_dev(ctx, p, p->tmp_b.p, p->tmp_x.p, p->tmp_x.p, opts, info);
    CK(cudaMemcpyAsync(x, p->tmp_x.p, p->n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return rc;
}

int vfv_spmv_device(vfv_ctx* ctx, const vfv_pattern* p, const double* x, double* y) {
    DeviceGuard dg_(ctx);
    if (!ctx || !p || !x || !y) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    launch_spmv<double, double, double, double>(ctx->stream, p->spmv_lanes[0], p->spmv_strides[0], p->n, p->rp.p, p->ci.p, p->val.p, x, y, nullptr, nullptr);
    ctx->launches += 1;
    CK(cudaGetLastError());
    return VFV_OK;
}

int vfv_spmv_device_f32(vfv_ctx* ctx, vfv_pattern* p, const float* x, float* y) {
    DeviceGuard dg_(ctx);
    if (!ctx || !p || !x || !y) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    if (p->version32 != p->version) {
        if (!p->val32.p) CK(p->val32.alloc(p->nnz));
        k_cast<double, float><<<grid_for(p->nnz), 256, 0, ctx->stream>>>(p->nnz, p->val.p, p->val32.p);
        p->version32 = p->version;
    }
    launch_spmv<float, float, float, float>(ctx->stream, p->spmv_lanes[1], p->spmv_strides[1], p->n, p->rp.p, p->ci.p, p->val32.p, x, y, nullptr, nullptr);
    ctx->launches += 1;
    CK(cudaGetLastError());
    return VFV_OK;
}

}  // extern "C"

namespace {
// Finds or builds the ILU(0) structure of an ordering, refreshes its numeric factor and sets up the
// sweep state of precision T (its work vector serves the standalone double apply).
template <typename T>
int ilu_for_apply(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, IluStruct** out) {
    if (ilu_order != VFV_ILU_MULTICOLOR && ilu_order != VFV_ILU_NATURAL) return set_err(ctx, VFV_BAD_INPUT, "unknown ILU ordering");
    auto it = p->ilu.find(ilu_order);
    if (it == p->ilu.end()) {
        auto S = std::make_unique<IluStruct>();
        int rc = build_ilu_struct(ctx, p, ilu_order, *S);
        if (rc) return rc;
        it = p->ilu.emplace(ilu_order, std::move(S)).first;
    }
    IluStruct& S = *it->second;
    int rc = ilu_refresh(ctx, p, S, !std::is_same<T, double>::value);
    if (rc) return rc;
    rc = chain_setup<T>(ctx, S, p->n);
    if (rc) return rc;
    *out = &S;
    return VFV_OK;
}

// z = M^-1 r with `sweeps` Jacobi sweeps of each factor (the apply of vfv_gmres_opts::ilu_sweeps), in
// double or with the float copy of the factor. Enqueued on the context's stream with no
// synchronisation; calls after the first for a pattern, ordering and precision allocate nothing.
template <typename T>
int sweep_apply(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, int sweeps, const T* r, T* z, bool half = false) {
    if (!ctx || !p || !r || !z) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    if (sweeps < 1 || sweeps > kMaxIluSweeps) return set_err(ctx, VFV_BAD_INPUT, "sweeps must be in [1, 16]");
    IluStruct* S = nullptr;
    int rc = ilu_for_apply<T>(ctx, p, ilu_order, &S);
    if (!rc) rc = ilu_split_refresh<T>(ctx, p, *S, half);
    if (rc) return rc;
    DBuf<unsigned char>& W = S->sweep_work[chain_slot<T>()];
    if (!W.p) CK(W.alloc((size_t)5 * p->n * sizeof(T)));
    T* buf[5];
    for (int q = 0; q < 5; ++q) buf[q] = reinterpret_cast<T*>(W.p) + (size_t)q * p->n;
    const SweepOps<T> o = sweep_ops<T>(p, *S, half);
    ilu_apply_sweeps<T>(ctx->stream, o, sweeps, sweeps, r, z, buf, nullptr);
    ctx->launches += 2 * sweeps + (o.perm ? 1 : 0);
    CK(cudaGetLastError());
    return VFV_OK;
}

}  // namespace

extern "C" {

int vfv_ilu0_apply_device(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, const double* r, double* z, int32_t* levels) {
    DeviceGuard dg_(ctx);
    if (!ctx || !p || !r || !z) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    IluStruct* S = nullptr;
    int rc = ilu_for_apply<double>(ctx, p, ilu_order, &S);
    if (rc) return rc;
    ilu_apply_levels<double>(ctx->stream, *S, S->lu64.p, r, reinterpret_cast<double*>(S->chain[0].work.p), z, nullptr);
    ctx->launches += 2 * S->nlev;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaGetLastError());
    if (levels) *levels = S->nlev;
    return VFV_OK;
}

// z = M^-1 r with the float copy of the factor: the level sweeps the mixed-precision solver runs.
// Enqueued on the context's stream with no synchronisation, so calls after the first (which builds
// the factor) allocate nothing and can be timed back to back.
int vfv_ilu0_apply_device_f32(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, const float* r, float* t, float* z, int32_t* levels) {
    DeviceGuard dg_(ctx);
    if (!ctx || !p || !r || !t || !z) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    if (t == r || t == z) return set_err(ctx, VFV_BAD_INPUT, "the work vector aliases r or z");
    IluStruct* S = nullptr;
    int rc = ilu_for_apply<float>(ctx, p, ilu_order, &S);
    if (rc) return rc;
    ilu_apply_levels<float>(ctx->stream, *S, S->lu32.p, r, t, z, nullptr);
    ctx->launches += 2 * S->nlev;
    CK(cudaGetLastError());
    if (levels) *levels = S->nlev;
    return VFV_OK;
}

int vfv_ilu0_sweep_apply_device(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, int sweeps, const double* r, double* z) {
    DeviceGuard dg_(ctx);
    return sweep_apply<double>(ctx, p, ilu_order, sweeps, r, z);
}

int vfv_ilu0_sweep_apply_device_f32(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, int sweeps, const float* r, float* z) {
    DeviceGuard dg_(ctx);
    return sweep_apply<float>(ctx, p, ilu_order, sweeps, r, z);
}

int vfv_ilu0_sweep_apply_device_f16(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, int sweeps, const float* r, float* z) {
    DeviceGuard dg_(ctx);
    return sweep_apply<float>(ctx, p, ilu_order, sweeps, r, z, true);
}

int vfv_ilu0_sweep_layout(const vfv_pattern* p, int ilu_order, int32_t* col_bytes) {
    if (!p) return set_err(nullptr, VFV_BAD_INPUT, "NULL argument");
    auto it = p->ilu.find(ilu_order);
    if (it == p->ilu.end() || !it->second->split.built)
        return set_err(nullptr, VFV_BAD_INPUT, "no Jacobi-sweep layout for this ordering yet (apply or solve with sweeps first)");
    if (col_bytes) *col_bytes = it->second->split.delta16 ? 2 : 4;
    return VFV_OK;
}

// ---------------------------------------------------------------- ILU(0) apply without allocation
// For callers that may not allocate device memory once they are running: code that drives the
// solver from inside a time-step loop under a fixed memory budget, or from a host framework whose
// allocator owns all device memory, or that must not hit the implicit device-wide synchronisation
// of cudaMalloc/cudaFree in the middle of a step. vfv_ilu0_apply_device allocates its sweep state
// when it first meets a pattern; this variant never allocates: its work vector is one fixed device
// array compiled into the library (the per-level sweeps, which need one work vector and give the
// same bits as the single-launch sweeps).
//
// The array is a file-scope __device__ variable: every GPU that loads the library holds its
// 2 MiB until the process exits. Host code cannot use the variable's name as a device address,
// so the device address is looked up with cudaGetSymbolAddress once per device, with that device
// current, by the first call on that device — make that first call before any stream capture.
// The address is cached per device index (atomically, so threads that race on a first call all
// store the same value); the cache assumes the primary context of each device, which the runtime
// API uses, is never reset while the library is loaded. Every call synchronises the context's
// stream before it returns. Every call shares the array and it keeps the last call's contents;
// nothing in it has to start at zero (the sweeps write every element before reading it). Calls
// that overlap on the GPU, from any context or thread, race on the array.
namespace {
constexpr int64_t kNoAllocMaxRows = 1 << 18;  // 262,144 rows of doubles: 2 MiB
__device__ __align__(256) double g_ilu_scratch[kNoAllocMaxRows];
constexpr int kNoAllocMaxDevices = 64;
std::atomic<double*> g_ilu_scratch_ptr[kNoAllocMaxDevices] = {};
}  // namespace

int vfv_ilu0_apply_device_noalloc(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, const double* r, double* z, int32_t* levels) {
    DeviceGuard dg_(ctx);
    if (!ctx || !p || !r || !z) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    if (ilu_order != VFV_ILU_MULTICOLOR && ilu_order != VFV_ILU_NATURAL) return set_err(ctx, VFV_BAD_INPUT, "unknown ILU ordering");
    if (p->n > kNoAllocMaxRows)
        return set_err(ctx, VFV_BAD_INPUT, "vfv_ilu0_apply_device_noalloc: " + std::to_string(p->n) +
                                               " rows exceed its fixed work array of " + std::to_string(kNoAllocMaxRows) + " rows");
    if (ctx->device < 0 || ctx->device >= kNoAllocMaxDevices) return set_err(ctx, VFV_BAD_INPUT, "device index out of range");
    auto it = p->ilu.find(ilu_order);
    if (it == p->ilu.end())
        return set_err(ctx, VFV_BAD_INPUT,
                       "vfv_ilu0_apply_device_noalloc: the pattern's ILU(0) storage is not set up; call vfv_ilu0_apply_device or an "
                       "ILU(0) solve on it once first (that call allocates)");
    IluStruct& S = *it->second;
    double* scratch = g_ilu_scratch_ptr[ctx->device].load(std::memory_order_acquire);
    if (!scratch) {
        int cur = -1;
        CK(cudaGetDevice(&cur));
        if (cur != ctx->device) CK(cudaSetDevice(ctx->device));
        const cudaError_t e = cudaGetSymbolAddress((void**)&scratch, g_ilu_scratch);
        if (cur != ctx->device) cudaSetDevice(cur);
        if (e != cudaSuccess) return set_err(ctx, VFV_CUDA_ERROR, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_ilu_scratch_ptr[ctx->device].store(scratch, std::memory_order_release);
    }
    int rc = ilu_refresh(ctx, p, S, false, 0, false);  // numeric factor into the storage made at set-up
    if (rc) return rc;
    ilu_apply_levels<double>(ctx->stream, S, S.lu64.p, r, scratch, z, nullptr);
    ctx->launches += 2 * S.nlev;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaGetLastError());
    if (levels) *levels = S.nlev;
    return VFV_OK;
}

// Autotuner: times the SpMV of this pattern (its current values) in every shape of kSpmvShapes
// (2 to 32 lanes per row, 1 to 8 strides loaded per lane before the gathers) in double and in float
// (short rows of a scalar problem favour few lanes, the 2-ring rows of the coupled flow system a
// warp per row), keeps the fastest of each for every later SpMV and solver of the pattern.
// Must run before the pattern's first solve (solvers capture their kernels once).
int vfv_pattern_autotune(vfv_ctx* ctx, vfv_pattern* p, int32_t* lanes64, int32_t* lanes32) {
    DeviceGuard dg_(ctx);
    if (!ctx || !p) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    cudaStream_t s = ctx->stream;
    const int64_t n = p->n;
    DBuf<double> x, y;
    DBuf<float> v32, x32, y32;
    CK(x.alloc(n));
    CK(y.alloc(n));
    CK(x32.alloc(n));
    CK(y32.alloc(n));
    CK(v32.alloc(p->nnz));
    CK(cudaMemsetAsync(x.p, 0, n * sizeof(double), s));
    CK(cudaMemsetAsync(x32.p, 0, n * sizeof(float), s));
    k_cast<double, float><<<grid_for(p->nnz), 256, 0, s>>>(p->nnz, p->val.p, v32.p);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const int nshape = (int)(sizeof(kSpmvShapes) / sizeof(kSpmvShapes[0]));
    for (int prec = 0; prec < 2; ++prec) {
        float best = 1e30f;
        int best_g = kSpG, best_s = 4;
        for (int round = 0; round < 2; ++round)  // two rounds: a shape's time is its better one
            for (int c = 0; c < nshape; ++c) {
                const int g = kSpmvShapes[c][0], st = kSpmvShapes[c][1];
                auto run = [&] {
                    if (prec == 0) launch_spmv<double, double, double, double>(s, g, st, n, p->rp.p, p->ci.p, p->val.p, x.p, y.p, nullptr, nullptr);
                    else launch_spmv<float, float, float, float>(s, g, st, n, p->rp.p, p->ci.p, v32.p, x32.p, y32.p, nullptr, nullptr);
                };
                for (int w = 0; w < 3; ++w) run();
                CK(cudaEventRecord(e0, s));
                for (int r = 0; r < 10; ++r) run();
                CK(cudaEventRecord(e1, s));
                CK(cudaEventSynchronize(e1));
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, e0, e1));
                if (ms < best) {
                    best = ms;
                    best_g = g;
                    best_s = st;
                }
            }
        p->spmv_lanes[prec] = best_g;
        p->spmv_strides[prec] = best_s;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->launches += 2 * 2 * nshape * 13 + 1;
    CK(cudaGetLastError());
    if (lanes64) *lanes64 = p->spmv_lanes[0];
    if (lanes32) *lanes32 = p->spmv_lanes[1];
    return VFV_OK;
}

int vfv_pattern_spmv_shape(const vfv_pattern* p, int32_t* lanes64, int32_t* strides64, int32_t* lanes32, int32_t* strides32) {
    if (!p) return set_err(nullptr, VFV_BAD_INPUT, "pattern is NULL");
    if (lanes64) *lanes64 = p->spmv_lanes[0];
    if (strides64) *strides64 = p->spmv_strides[0];
    if (lanes32) *lanes32 = p->spmv_lanes[1];
    if (strides32) *strides32 = p->spmv_strides[1];
    return VFV_OK;
}

int vfv_pattern_set_spmv_lanes(vfv_ctx* ctx, vfv_pattern* p, int32_t lanes64, int32_t lanes32) {
    DeviceGuard dg_(ctx);
    if (!ctx || !p) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    auto ok = [](int32_t g) { return g == 2 || g == 4 || g == 8 || g == 16 || g == 32; };
    if (!ok(lanes64) || !ok(lanes32)) return set_err(ctx, VFV_BAD_INPUT, "SpMV lanes per row must be 2, 4, 8, 16 or 32");
    p->spmv_lanes[0] = lanes64;
    p->spmv_lanes[1] = lanes32;
    p->spmv_strides[0] = p->spmv_strides[1] = 4;
    return VFV_OK;
}

int vfv_ilu0_ordering(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, int32_t* perm, int32_t* lev_ptr, int32_t* nlev) {
    DeviceGuard dg_(ctx);
    if (!ctx || !p) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    if (ilu_order != VFV_ILU_MULTICOLOR && ilu_order != VFV_ILU_NATURAL) return set_err(ctx, VFV_BAD_INPUT, "unknown ILU ordering");
    auto it = p->ilu.find(ilu_order);
    if (it == p->ilu.end()) {
        auto S = std::make_unique<IluStruct>();
        int rc = build_ilu_struct(ctx, p, ilu_order, *S);
        if (rc) return rc;
        it = p->ilu.emplace(ilu_order, std::move(S)).first;
    }
    const IluStruct& S = *it->second;
    if (nlev) *nlev = S.nlev;
    if (perm) std::memcpy(perm, S.h_perm.data(), S.h_perm.size() * sizeof(int32_t));
    if (lev_ptr) std::memcpy(lev_ptr, S.lev_ptr.data(), S.lev_ptr.size() * sizeof(int32_t));
    return VFV_OK;
}

}  // extern "C"
