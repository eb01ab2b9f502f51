// Mesh handles of libvfvgpu: seeded jittered cubes, meshes from given vertices, and the export of
// the Delaunay tetrahedra and the Voronoi dual (host code: csrc/host/mesh.cpp).
#include "host/write_out.hpp"
#include "internal.cuh"

#include <algorithm>
#include <cmath>

#include <cstdlib>
#include <cstring>
#include <omp.h>

// Budget for the dual's stored face pieces; VFV_DUAL_PIECE_STORE_MB overrides it (0: always
// recompute them), so that tests can check both ways give the same dual.
static double dual_piece_store_bytes() {
    if (const char* e = std::getenv("VFV_DUAL_PIECE_STORE_MB")) return std::atof(e) * 1024.0 * 1024.0;
    return kDualPieceStoreBytes;
}

// Delaunay tetrahedralisation and Voronoi dual of a mesh whose vertices are set; takes ownership.
static int mesh_finish(vfv_mesh* mh, vfv_mesh** out) {
    std::string e = delaunay(mh->m);
    if (e.empty()) e = build_dual(mh->m, mh->d, dual_piece_store_bytes());
    if (!e.empty()) {
        delete mh;
        return set_err(nullptr, VFV_BAD_INPUT, e);
    }
    *out = mh;
    return VFV_OK;
}

extern "C" {

int vfv_mesh_jitter_cube(int n, uint64_t seed, double jitter, vfv_mesh** out) {
    if (!out) return set_err(nullptr, VFV_BAD_INPUT, "out is NULL");
    *out = nullptr;
    if (n < 3 || n > 400) return set_err(nullptr, VFV_BAD_INPUT, "grid size n must be in [3, 400]");
    if (!(jitter >= 0.0 && jitter < 0.5)) return set_err(nullptr, VFV_BAD_INPUT, "jitter must be in [0, 0.5)");
    auto* mh = new vfv_mesh();
    mh->m = make_jitter_cube(n, seed, jitter);
    return mesh_finish(mh, out);
}

int vfv_mesh_from_vertices(int64_t n_pts, int64_t n_nds, const double* pos, const int32_t* node_bnd, vfv_mesh** out) {
    if (!out || !pos || (n_nds > 0 && !node_bnd)) return set_err(nullptr, VFV_BAD_INPUT, "NULL argument");
    *out = nullptr;
    if (n_pts < 0 || n_nds < 0 || n_pts + n_nds < 4) return set_err(nullptr, VFV_BAD_INPUT, "need at least four vertices");
    // The Delaunay predicates are exact for any finite coordinates (integer arithmetic on the 2^-18
    // lattice for the generated cubes, filtered double arithmetic with an exact fallback otherwise);
    // magnitudes are bounded so that the filters' degree-5 products stay finite.
    for (int64_t v = 0; v < n_pts + n_nds; ++v)
        for (int c = 0; c < 3; ++c)
            if (!(std::fabs(pos[3 * v + c]) <= 1e50))
                return set_err(nullptr, VFV_BAD_INPUT, "vertex " + std::to_string(v) + ": coordinates must be finite and within 1e50 in magnitude");
    auto* mh = new vfv_mesh();
    mh->m.n_pts = n_pts;
    mh->m.n_nds = n_nds;
    mh->m.pos.assign(pos, pos + 3 * (n_pts + n_nds));
    mh->m.node_bnd.assign(node_bnd, node_bnd + n_nds);
    return mesh_finish(mh, out);
}

void vfv_mesh_destroy(vfv_mesh* m) { delete m; }

int vfv_mesh_dual_device(vfv_ctx* ctx, vfv_mesh* m) {
    DeviceGuard dg_(ctx);
    if (!ctx || !m) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    if (m->m.tets.empty()) return set_err(ctx, VFV_BAD_INPUT, "mesh has no tetrahedra");
    Dual d;
    const std::string e = build_dual_device(ctx, m->m, d);
    if (!e.empty()) return set_err(ctx, e.rfind("dual on the device", 0) == 0 ? VFV_CUDA_ERROR : VFV_BAD_INPUT, e);
    m->d = std::move(d);
    return VFV_OK;
}

int vfv_mesh_jitter_cubes_device_dual(vfv_ctx* ctx, int count, const int32_t* n, const uint64_t* seeds, double jitter, vfv_mesh** out) {
    DeviceGuard dg_(ctx);
    if (!ctx || count <= 0 || !n || !seeds || !out) return set_err(ctx, VFV_BAD_INPUT, "invalid batch arguments");
    for (int i = 0; i < count; ++i) {
        out[i] = nullptr;
        if (n[i] < 3 || n[i] > 400) return set_err(ctx, VFV_BAD_INPUT, "grid size n must be in [3, 400]");
    }
    if (!(jitter >= 0.0 && jitter < 0.5)) return set_err(ctx, VFV_BAD_INPUT, "jitter must be in [0, 0.5)");
    std::vector<std::string> errs(count);
    std::vector<vfv_mesh*> made(count, nullptr);
    // Delaunay of the meshes in parallel on the host, largest first
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return n[a] > n[b]; });
#pragma omp parallel for schedule(dynamic, 1)
    for (int t = 0; t < count; ++t) {
        const int i = order[t];
        auto* mh = new vfv_mesh();
        mh->m = make_jitter_cube(n[i], seeds[i], jitter);
        errs[i] = delaunay(mh->m);
        made[i] = mh;
    }
    int rc = VFV_OK;
    for (int i = 0; i < count && rc == VFV_OK; ++i) {
        if (!errs[i].empty()) {
            rc = set_err(ctx, VFV_BAD_INPUT, errs[i]);
            break;
        }
        rc = vfv_mesh_dual_device(ctx, made[i]);  // the duals one after the other on the device
    }
    if (rc != VFV_OK) {
        for (vfv_mesh* mh : made) delete mh;
        return rc;
    }
    for (int i = 0; i < count; ++i) out[i] = made[i];
    return VFV_OK;
}

int vfv_mesh_jitter_cubes(int count, const int32_t* n, const uint64_t* seeds, double jitter, vfv_mesh** out) {
    if (count <= 0 || !n || !seeds || !out) return set_err(nullptr, VFV_BAD_INPUT, "invalid batch arguments");
    for (int i = 0; i < count; ++i) {
        out[i] = nullptr;
        if (n[i] < 3 || n[i] > 400) return set_err(nullptr, VFV_BAD_INPUT, "grid size n must be in [3, 400]");
    }
    if (!(jitter >= 0.0 && jitter < 0.5)) return set_err(nullptr, VFV_BAD_INPUT, "jitter must be in [0, 0.5)");
    std::vector<std::string> errs(count);
    // meshes in parallel (largest first); the per-mesh OpenMP loops run serially inside
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return n[a] > n[b]; });
#pragma omp parallel for schedule(dynamic, 1)
    for (int t = 0; t < count; ++t) {
        const int i = order[t];
        auto* mh = new vfv_mesh();
        mh->m = make_jitter_cube(n[i], seeds[i], jitter);
        std::string e = delaunay(mh->m);
        if (e.empty()) e = build_dual(mh->m, mh->d, dual_piece_store_bytes());
        if (!e.empty()) {
            errs[i] = e;
            delete mh;
        } else {
            out[i] = mh;
        }
    }
    for (int i = 0; i < count; ++i)
        if (!errs[i].empty()) {
            for (int j = 0; j < count; ++j) {
                delete out[j];
                out[j] = nullptr;
            }
            return set_err(nullptr, VFV_BAD_INPUT, "mesh " + std::to_string(i) + ": " + errs[i]);
        }
    return VFV_OK;
}

int vfv_mesh_info(const vfv_mesh* m, int64_t* n_pts, int64_t* n_nds, int64_t* n_tet, int64_t* n_dir, int64_t* n_bsub) {
    if (!m) return set_err(nullptr, VFV_BAD_INPUT, "mesh is NULL");
    if (n_pts) *n_pts = m->m.n_pts;
    if (n_nds) *n_nds = m->m.n_nds;
    if (n_tet) *n_tet = m->m.n_tet();
    if (n_dir) *n_dir = m->d.n_dir;
    if (n_bsub) *n_bsub = m->d.bnd_ptr.empty() ? 0 : m->d.bnd_ptr.back();
    return VFV_OK;
}

int vfv_mesh_export(const vfv_mesh* m, double* pos, int32_t* node_bnd, int32_t* tets) {
    if (!m) return set_err(nullptr, VFV_BAD_INPUT, "mesh is NULL");
    if (pos) std::memcpy(pos, m->m.pos.data(), m->m.pos.size() * sizeof(double));
    if (node_bnd) std::memcpy(node_bnd, m->m.node_bnd.data(), m->m.node_bnd.size() * sizeof(int32_t));
    if (tets) std::memcpy(tets, m->m.tets.data(), m->m.tets.size() * sizeof(int32_t));
    return VFV_OK;
}

int vfv_mesh_export_dual(const vfv_mesh* m, int64_t* nbr_ptr, int32_t* nbr_idx, double* dist, double* area, double* norm, double* skew,
                         double* grad_wgt, double* cvol, double* cskew, int64_t* bnd_ptr, int32_t* bnd_j, int32_t* bnd_k,
                         double* bnd_area, double* bnd_norm, double* bnd_wgt) {
    if (!m) return set_err(nullptr, VFV_BAD_INPUT, "mesh is NULL");
    const Dual& d = m->d;
    auto cp = [](auto* dst, const auto& v) {
        if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    cp(nbr_ptr, d.nbr_ptr);
    cp(nbr_idx, d.nbr_idx);
    cp(dist, d.dist);
    cp(area, d.area);
    cp(norm, d.norm);
    cp(skew, d.skew);
    cp(grad_wgt, d.gw);
    cp(cvol, d.cvol);
    cp(cskew, d.cskew);
    cp(bnd_ptr, d.bnd_ptr);
    cp(bnd_j, d.bnd_j);
    cp(bnd_k, d.bnd_k);
    cp(bnd_area, d.bnd_area);
    cp(bnd_norm, d.bnd_norm);
    cp(bnd_wgt, d.bnd_wgt);
    return VFV_OK;
}

// output files (host): argument checks here, the formats in host/write_out.cpp
static int write_rc(const std::string& e, bool io) {
    if (e.empty()) return VFV_OK;
    return set_err(nullptr, io ? VFV_IO_ERROR : VFV_BAD_INPUT, e);
}

int vfv_mesh_write_vtu(const vfv_mesh* m, const double* values, int ncomp, const char* path) {
    if (!m || !path || (ncomp != 1 && ncomp != 3)) return set_err(nullptr, VFV_BAD_INPUT, "invalid argument");
    const Mesh& g = m->m;
    const std::string e = write_vtu_tets(path, g.n_tot(), g.pos.data(), g.n_tet(), g.tets.data(), values, ncomp);
    return write_rc(e, e.rfind("cannot write", 0) == 0);
}

int vfv_mesh_write_csv(const vfv_mesh* m, const double* values, int ncomp, const char* path) {
    if (!m || !path || !values || (ncomp != 1 && ncomp != 3)) return set_err(nullptr, VFV_BAD_INPUT, "invalid argument");
    const Mesh& g = m->m;
    const std::string e = write_csv(path, g.n_tot(), g.pos.data(), values, ncomp);
    return write_rc(e, e.rfind("cannot write", 0) == 0);
}

int vfv_points_write_vtu(int64_t n, const double* pos, const double* values, int ncomp, const char* path) {
    if (!path || n < 0 || (n > 0 && !pos) || (ncomp != 1 && ncomp != 3)) return set_err(nullptr, VFV_BAD_INPUT, "invalid argument");
    const std::string e = write_vtu_points(path, n, pos, values, ncomp);
    return write_rc(e, e.rfind("cannot write", 0) == 0);
}

int vfv_points_write_csv(int64_t n, const double* pos, const double* values, int ncomp, const char* path) {
    if (!path || n < 0 || (n > 0 && (!pos || !values)) || (ncomp != 1 && ncomp != 3)) return set_err(nullptr, VFV_BAD_INPUT, "invalid argument");
    const std::string e = write_csv(path, n, pos, values, ncomp);
    return write_rc(e, e.rfind("cannot write", 0) == 0);
}

}  // extern "C"
