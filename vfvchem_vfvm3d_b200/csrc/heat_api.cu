// Steady heat operator handle of libvfvgpu: device assembly of SteadyHeat::assemble_matrix
// (src/steady/core/steady_heat.rs:143-171) into a CSR pattern, the LSQ gradients, and the adjoint
// (transpose solve plus dR/dk, dR/dq gathers).
#include "internal.cuh"
#include "kernels/adjoint.cuh"
#include "kernels/assemble.cuh"

#include <cstring>
#include <cmath>
#include <vector>

struct vfv_heat {
    vfv_ctx* ctx = nullptr;
    int64_t n = 0, n_dir = 0, n_bsub = 0;
    DBuf<int32_t> np, ni, kind, node_bnd, bp, bj, bk, dloc;
    DBuf<double> area, dist, skew, gw, cvol, cskew, barea, bw;
    DBuf<double> f, grad, b;  // f: [5][n] = k, q, s, T, bc_val ; grad: [4][3][n]
    vfv_pattern* pat = nullptr;
    // adjoint (built on first use): transpose pattern, value map, reverse faces, work arrays
    vfv_pattern* pat_t = nullptr;
    DBuf<int32_t> tmap, rev;
    DBuf<double> adj_work;  // pv, pn [n_dir]; sk [3 n_dir]; gkm [n]; psi [3 n]; T, g, lambda, zero, dlogk, dq [n]
    std::vector<int32_t> h_rev;
    ~vfv_heat() {
        delete pat_t;
        delete pat;
    }
};


extern "C" {

// ---------------------------------------------------------------- heat operator
int vfv_heat_create(vfv_ctx* ctx, const vfv_mesh* mh, int32_t n_bnd, const int32_t* bnd_kind, vfv_heat** out) {
    DeviceGuard dg_(ctx);
    if (!ctx || !mh || !out || (n_bnd > 0 && !bnd_kind)) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    *out = nullptr;
    const Mesh& m = mh->m;
    const Dual& d = mh->d;
    const int64_t n = d.n_tot;
    if (d.n_dir >= (int64_t)1 << 31 || n + d.n_dir >= (int64_t)1 << 31) return set_err(ctx, VFV_BAD_INPUT, "mesh too large for 32-bit indices");
    std::vector<int32_t> kind(n, ROW_POINT), nb(n, -1);
    for (int64_t v = m.n_pts; v < n; ++v) {
        const int32_t b = m.node_bnd[v - m.n_pts];
        if (b < 0 || b >= n_bnd) return set_err(ctx, VFV_BAD_INPUT, "node boundary id without a boundary condition");
        if (bnd_kind[b] != VFV_BC_TEMP && bnd_kind[b] != VFV_BC_FLUX) return set_err(ctx, VFV_BAD_INPUT, "unknown boundary kind");
        kind[v] = bnd_kind[b] == VFV_BC_TEMP ? ROW_DIRICHLET : ROW_FLUX;
        nb[v] = b;
    }
    // matrix pattern: row v = its neighbours and itself (ascending); Dirichlet rows only the diagonal
    std::vector<int32_t> np(n + 1), dloc(n, 0), rp(n + 1, 0), ci;
    ci.reserve(d.n_dir + n);
    for (int64_t v = 0; v < n; ++v) {
        np[v] = (int32_t)d.nbr_ptr[v];
        const int64_t b0 = d.nbr_ptr[v], e0 = d.nbr_ptr[v + 1];
        if (kind[v] == ROW_DIRICHLET) {
            ci.push_back((int32_t)v);
        } else {
            int32_t dl = 0;
            while (b0 + dl < e0 && d.nbr_idx[b0 + dl] < v) ++dl;
            dloc[v] = dl;
            for (int64_t i = b0; i < b0 + dl; ++i) ci.push_back(d.nbr_idx[i]);
            ci.push_back((int32_t)v);
            for (int64_t i = b0 + dl; i < e0; ++i) ci.push_back(d.nbr_idx[i]);
        }
        rp[v + 1] = (int32_t)ci.size();
    }
    np[n] = (int32_t)d.nbr_ptr[n];
    auto h = std::make_unique<vfv_heat>();
    h->ctx = ctx;
    h->n = n;
    h->n_dir = d.n_dir;
    h->n_bsub = d.bnd_ptr[n];
    vfv_pattern* pat = nullptr;
    int rc = vfv_pattern_from_csr(ctx, n, rp.data(), ci.data(), &pat);
    if (rc) return rc;
    h->pat = pat;
    cudaStream_t s = ctx->stream;
    std::vector<int32_t> bp(n + 1);
    for (int64_t v = 0; v <= n; ++v) bp[v] = (int32_t)d.bnd_ptr[v];
    CK(h->np.upload(np.data(), n + 1, s));
    CK(h->ni.upload(d.nbr_idx.data(), d.n_dir, s));
    CK(h->kind.upload(kind.data(), n, s));
    CK(h->node_bnd.upload(nb.data(), n, s));
    CK(h->dloc.upload(dloc.data(), n, s));
    CK(h->bp.upload(bp.data(), n + 1, s));
    CK(h->bj.upload(d.bnd_j.data(), d.bnd_j.size(), s));
    CK(h->bk.upload(d.bnd_k.data(), d.bnd_k.size(), s));
    CK(h->area.upload(d.area.data(), d.area.size(), s));
    CK(h->dist.upload(d.dist.data(), d.dist.size(), s));
    CK(h->skew.upload(d.skew.data(), d.skew.size(), s));
    CK(h->gw.upload(d.gw.data(), d.gw.size(), s));
    CK(h->cvol.upload(d.cvol.data(), d.cvol.size(), s));
    CK(h->cskew.upload(d.cskew.data(), d.cskew.size(), s));
    CK(h->barea.upload(d.bnd_area.data(), d.bnd_area.size(), s));
    CK(h->bw.upload(d.bnd_wgt.data(), d.bnd_wgt.size(), s));
    CK(h->f.alloc(5 * n));
    CK(h->grad.alloc(12 * n));
    CK(h->b.alloc(n));
    h->h_rev.resize(d.n_dir);
    for (int64_t i = 0; i < d.n_dir; ++i) h->h_rev[i] = (int32_t)d.nbr_rev[i];
    *out = h.release();
    return VFV_OK;
}

// Adjoint of the heat assembly (zero production): solve A^T lambda = dJ/dT with the GMRES of
// vfv_solve, then dJ/d(log k) and dJ/dq by the gather kernels of kernels/adjoint.cu. Uses k, q
// and their gradients from the last vfv_heat_assemble call.
int vfv_heat_adjoint(vfv_ctx* ctx, vfv_heat* h, const double* T, const double* dJdT, const vfv_gmres_opts* opts, double* lambda,
                     double* dJdlogk, double* dJdq, vfv_solve_info* info) {
    DeviceGuard dg_(ctx);
    if (!ctx || !h || !T || !dJdT) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    int rc = check_opts(ctx, opts);
    if (rc) return rc;
    if (info) std::memset(info, 0, sizeof(*info));
    const int64_t n = h->n, E = h->n_dir;
    cudaStream_t s = ctx->stream;
    if (!h->pat_t) {
        rc = make_transpose(ctx, h->pat, &h->pat_t, h->tmap);
        if (rc) return rc;
        CK(h->rev.upload(h->h_rev.data(), E, s));
        CK(h->adj_work.alloc((size_t)5 * E + (size_t)10 * n));
    }
    double* w = h->adj_work.p;
    double* pv = w;
    double* pn = w + E;
    double* sk = w + 2 * E;
    double* gkm = w + 5 * E;
    double* psi = gkm + n;
    double* dT = psi + 3 * n;
    double* dg = dT + n;
    double* dl = dg + n;
    double* dzero = dl + n;
    double* ddk = dzero + n;
    double* ddq = ddk + n;
    if ((rc = gather_transpose_values(ctx, h->pat, h->pat_t, h->tmap.p))) return rc;
    ctx->launches += 1;
    h->pat_t->version++;
    CK(cudaMemcpyAsync(dT, T, n * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dg, dJdT, n * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(dzero, 0, n * sizeof(double), s));
    rc = solve_dev(ctx, h->pat_t, dg, dzero, dl, opts, info);
    if (rc) return rc;
    AdjDev D{};
    D.n = n;
    D.n_dir = E;
    D.np = h->np.p;
    D.ni = h->ni.p;
    D.rev = h->rev.p;
    D.kind = h->kind.p;
    D.area = h->area.p;
    D.dist = h->dist.p;
    D.skew = h->skew.p;
    D.gw = h->gw.p;
    D.cvol = h->cvol.p;
    D.cskew = h->cskew.p;
    D.k = h->f.p;
    D.gk = h->grad.p;
    D.T = dT;
    D.lambda = dl;
    D.pv = pv;
    D.pn = pn;
    D.sk = sk;
    D.gkm = gkm;
    D.psi = psi;
    D.dlogk = ddk;
    D.dq = ddq;
    launch_adjoint_partials(s, D);
    ctx->launches += 3;
    CK(cudaGetLastError());
    if (lambda) CK(cudaMemcpyAsync(lambda, dl, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (dJdlogk) CK(cudaMemcpyAsync(dJdlogk, ddk, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (dJdq) CK(cudaMemcpyAsync(dJdq, ddq, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return VFV_OK;
}

void vfv_heat_destroy(vfv_heat* h) {
    if (!h) return;
    if (h->ctx) cudaStreamSynchronize(h->ctx->stream);
    delete h;
}

vfv_pattern* vfv_heat_pattern(vfv_heat* h) { return h ? h->pat : nullptr; }

const double* vfv_heat_rhs_device(vfv_heat* h) { return h ? h->b.p : nullptr; }

int vfv_heat_assemble(vfv_ctx* ctx, vfv_heat* h, const double* k, const double* q, const double* s_, const double* T,
                      const double* bc_val, int on_device, double* b_out) {
    DeviceGuard dg_(ctx);
    if (!ctx || !h || !k || !q || !s_ || !T || !bc_val) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    const int64_t n = h->n;
    cudaStream_t s = ctx->stream;
    const double* src[5] = {k, q, s_, T, bc_val};
    const cudaMemcpyKind kd = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    for (int f = 0; f < 5; ++f) CK(cudaMemcpyAsync(h->f.p + f * n, src[f], n * sizeof(double), kd, s));
    const double* fl[4] = {h->f.p, h->f.p + n, h->f.p + 2 * n, h->f.p + 3 * n};
    launch_grad(s, n, h->np.p, h->ni.p, h->gw.p, h->n_dir, 4, fl, h->grad.p);
    HeatDev H{};
    H.n = n;
    H.n_dir = h->n_dir;
    H.n_bsub = h->n_bsub;
    H.np = h->np.p;
    H.ni = h->ni.p;
    H.area = h->area.p;
    H.dist = h->dist.p;
    H.skew = h->skew.p;
    H.cvol = h->cvol.p;
    H.cskew = h->cskew.p;
    H.kind = h->kind.p;
    H.node_bnd = h->node_bnd.p;
    H.bp = h->bp.p;
    H.bj = h->bj.p;
    H.bk = h->bk.p;
    H.barea = h->barea.p;
    H.bw = h->bw.p;
    H.rp = h->pat->rp.p;
    H.dloc = h->dloc.p;
    H.k = fl[0];
    H.q = fl[1];
    H.s = fl[2];
    H.T = fl[3];
    H.bcv = h->f.p + 4 * n;
    H.gk = h->grad.p;
    H.gq = h->grad.p + 3 * n;
    H.gs = h->grad.p + 6 * n;
    H.gT = h->grad.p + 9 * n;
    H.val = h->pat->val.p;
    H.b = h->b.p;
    launch_assemble_heat(s, H);
    ctx->launches += 2;
    CK(cudaGetLastError());
    h->pat->version++;
    if (b_out) {
        CK(cudaMemcpyAsync(b_out, h->b.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    }
    return VFV_OK;
}

int vfv_update_grad(vfv_ctx* ctx, vfv_heat* h, const double* f, double* grad) {
    DeviceGuard dg_(ctx);
    if (!ctx || !h || !f || !grad) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    const int64_t n = h->n;
    cudaStream_t s = ctx->stream;
    DBuf<double> fd, gd;
    CK(fd.alloc(n));
    CK(gd.alloc(3 * n));
    CK(cudaMemcpyAsync(fd.p, f, n * sizeof(double), cudaMemcpyHostToDevice, s));
    const double* fl[1] = {fd.p};
    launch_grad(s, n, h->np.p, h->ni.p, h->gw.p, h->n_dir, 1, fl, gd.p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(grad, gd.p, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return VFV_OK;
}

}  // extern "C"
