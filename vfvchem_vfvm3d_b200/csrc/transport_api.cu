// Batched transient transport handle of libvfvgpu: many meshes concatenated into one block-diagonal
// advection-diffusion system (time + diffusion + power-law advection), implicit Euler steps with
// per-mesh stopping, and the checkpointed adjoint dJ/dD.
#include "internal.cuh"
#include "kernels/assemble.cuh"

#include <cstring>
#include <algorithm>
#include <cmath>
#include <vector>

// Concatenation of several meshes into one block-diagonal transport system.
struct vfv_transport {
    vfv_ctx* ctx = nullptr;
    int nmesh = 0;
    int64_t n = 0, n_dir = 0;
    double dt = 0.0;
    std::vector<int64_t> row_ptr;  // [nmesh+1] vertex (row) offsets of the meshes
    DBuf<int64_t> d_row_ptr;
    DBuf<int32_t> np, ni, dloc;
    DBuf<double> area, dist, skew, norm, gw, cvol, flux, fields, grads, b, c0, c1;
    vfv_pattern* pat = nullptr;
    // transient adjoint: transpose pattern and work space
    vfv_pattern* pat_t = nullptr;
    DBuf<int32_t> tmap;
    DBuf<double> adj;        // checkpoints, one segment of states, two adjoint vectors, rhs, zero, partials, terms
    DBuf<unsigned> adj_counter;
    std::vector<int64_t> run_mesh_steps;  // Arnoldi steps per mesh summed over the last vfv_transport_run
    TransportDev dev() const {
        TransportDev T{};
        T.n = n;
        T.n_dir = n_dir;
        T.np = np.p;
        T.ni = ni.p;
        T.area = area.p;
        T.dist = dist.p;
        T.skew = skew.p;
        T.norm = norm.p;
        T.cvol = cvol.p;
        T.rp = pat->rp.p;
        T.dloc = dloc.p;
        T.D = fields.p;
        T.gD = grads.p;
        T.vel = fields.p + n;
        T.gvel = grads.p + 3 * n;
        T.flux = flux.p;
        T.dt = dt;
        T.val = pat->val.p;
        return T;
    }
    ~vfv_transport() {
        delete pat_t;
        delete pat;
    }
};


extern "C" {

// ---------------------------------------------------------------- transient transport (batched meshes)
int vfv_transport_create(vfv_ctx* ctx, int nmesh, vfv_mesh* const* meshes, double dt, vfv_transport** out) {
    DeviceGuard dg_(ctx);
    if (!ctx || nmesh <= 0 || !meshes || !out) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    if (!(dt > 0.0)) return set_err(ctx, VFV_BAD_INPUT, "dt must be positive");
    *out = nullptr;
    auto t = std::make_unique<vfv_transport>();
    t->ctx = ctx;
    t->nmesh = nmesh;
    t->dt = dt;
    t->row_ptr.assign(nmesh + 1, 0);
    int64_t ndir = 0;
    for (int i = 0; i < nmesh; ++i) {
        if (!meshes[i]) return set_err(ctx, VFV_BAD_INPUT, "NULL mesh");
        t->row_ptr[i + 1] = t->row_ptr[i] + meshes[i]->d.n_tot;
        ndir += meshes[i]->d.n_dir;
    }
    const int64_t n = t->row_ptr[nmesh];
    if (n + ndir >= (int64_t)1 << 31) return set_err(ctx, VFV_BAD_INPUT, "batch too large for 32-bit indices");
    t->n = n;
    t->n_dir = ndir;
    std::vector<int32_t> np(n + 1, 0), ni(ndir), dloc(n), rp(n + 1, 0), ci;
    std::vector<double> area(ndir), dist(ndir), skew(3 * ndir), norm(3 * ndir), gw(3 * ndir), cvol(n);
    ci.reserve(ndir + n);
    int64_t e0 = 0;
    for (int i = 0; i < nmesh; ++i) {
        const Dual& d = meshes[i]->d;
        const int64_t v0 = t->row_ptr[i], D = d.n_dir;
        for (int64_t v = 0; v < d.n_tot; ++v) {
            const int64_t gv = v0 + v;
            np[gv] = (int32_t)(e0 + d.nbr_ptr[v]);
            cvol[gv] = d.cvol[v];
            const int64_t b = d.nbr_ptr[v], e = d.nbr_ptr[v + 1];
            int32_t dl = 0;
            while (b + dl < e && d.nbr_idx[b + dl] < v) ++dl;
            dloc[gv] = dl;
            for (int64_t k = b; k < b + dl; ++k) ci.push_back((int32_t)(v0 + d.nbr_idx[k]));
            ci.push_back((int32_t)gv);
            for (int64_t k = b + dl; k < e; ++k) ci.push_back((int32_t)(v0 + d.nbr_idx[k]));
            rp[gv + 1] = (int32_t)ci.size();
        }
        for (int64_t k = 0; k < D; ++k) {
            ni[e0 + k] = (int32_t)(v0 + d.nbr_idx[k]);
            area[e0 + k] = d.area[k];
            dist[e0 + k] = d.dist[k];
            for (int c = 0; c < 3; ++c) {
                skew[c * ndir + e0 + k] = d.skew[c * D + k];
                norm[c * ndir + e0 + k] = d.norm[c * D + k];
                gw[c * ndir + e0 + k] = d.gw[c * D + k];
            }
        }
        e0 += D;
    }
    np[n] = (int32_t)ndir;
    vfv_pattern* pat = nullptr;
    int rc = vfv_pattern_from_csr(ctx, n, rp.data(), ci.data(), &pat);
    if (rc) return rc;
    t->pat = pat;
    pat->blocks.assign(t->row_ptr.begin(), t->row_ptr.end());
    cudaStream_t s = ctx->stream;
    CK(t->d_row_ptr.upload(t->row_ptr.data(), nmesh + 1, s));
    CK(t->np.upload(np.data(), n + 1, s));
    CK(t->ni.upload(ni.data(), ndir, s));
    CK(t->dloc.upload(dloc.data(), n, s));
    CK(t->area.upload(area.data(), ndir, s));
    CK(t->dist.upload(dist.data(), ndir, s));
    CK(t->skew.upload(skew.data(), 3 * ndir, s));
    CK(t->norm.upload(norm.data(), 3 * ndir, s));
    CK(t->gw.upload(gw.data(), 3 * ndir, s));
    CK(t->cvol.upload(cvol.data(), n, s));
    CK(t->flux.alloc(ndir));
    CK(t->fields.alloc(4 * n));   // D, u, v, w
    CK(t->grads.alloc(12 * n));   // grad D, grad u, grad v, grad w
    CK(t->b.alloc(n));
    CK(t->c0.alloc(n));
    CK(t->c1.alloc(n));
    *out = t.release();
    return VFV_OK;
}

void vfv_transport_destroy(vfv_transport* t) {
    if (!t) return;
    if (t->ctx) cudaStreamSynchronize(t->ctx->stream);
    delete t;
}

vfv_pattern* vfv_transport_pattern(vfv_transport* t) { return t ? t->pat : nullptr; }

int vfv_transport_info(const vfv_transport* t, int64_t* n_tot, int64_t* nnz, int32_t* nmesh, int64_t* row_ptr) {
    if (!t) return set_err(nullptr, VFV_BAD_INPUT, "transport is NULL");
    if (n_tot) *n_tot = t->n;
    if (nnz) *nnz = t->pat->nnz;
    if (nmesh) *nmesh = t->nmesh;
    if (row_ptr) std::memcpy(row_ptr, t->row_ptr.data(), (t->nmesh + 1) * sizeof(int64_t));
    return VFV_OK;
}

int vfv_transport_assemble(vfv_ctx* ctx, vfv_transport* t, const double* D, const double* vel, int on_device) {
    DeviceGuard dg_(ctx);
    if (!ctx || !t || !D || !vel) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    const int64_t n = t->n;
    cudaStream_t s = ctx->stream;
    const cudaMemcpyKind kd = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CK(cudaMemcpyAsync(t->fields.p, D, n * sizeof(double), kd, s));
    CK(cudaMemcpyAsync(t->fields.p + n, vel, 3 * n * sizeof(double), kd, s));
    const double* f4[4] = {t->fields.p, t->fields.p + n, t->fields.p + 2 * n, t->fields.p + 3 * n};
    launch_grad(s, n, t->np.p, t->ni.p, t->gw.p, t->n_dir, 4, f4, t->grads.p);
    const TransportDev T = t->dev();
    launch_face_flux(s, T);
    launch_assemble_transport(s, T);
    ctx->launches += 3;
    CK(cudaGetLastError());
    t->pat->version++;
    return VFV_OK;
}

// nsteps of implicit Euler from c0 (host) with the current matrix: b = -vol c / dt, one batched GMRES
// per step with the per-mesh stopping rule; the state stays on the device between steps.
int vfv_transport_run(vfv_ctx* ctx, vfv_transport* t, const double* c0, int nsteps, const vfv_gmres_opts* opts, double* c_out,
                      int32_t* iters) {
    DeviceGuard dg_(ctx);
    if (!ctx || !t || !c0 || !c_out || nsteps < 0) return set_err(ctx, VFV_BAD_INPUT, "invalid argument");
    int rc = check_opts(ctx, opts);
    if (rc) return rc;
    const int64_t n = t->n;
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(t->c0.p, c0, n * sizeof(double), cudaMemcpyHostToDevice, s));
    double* cur = t->c0.p;
    double* nxt = t->c1.p;
    t->run_mesh_steps.assign(t->nmesh, 0);
    std::vector<int32_t> ms;
    for (int k = 0; k < nsteps; ++k) {
        launch_transport_rhs(s, n, t->cvol.p, t->dt, cur, t->b.p);
        ctx->launches += 1;
        vfv_solve_info info{};
        rc = solve_dev(ctx, t->pat, t->b.p, cur, nxt, opts, &info, true);
        if (rc) return rc;
        if (iters) iters[k] = info.iters;
        if (t->nmesh > 1 && batch_mesh_steps(t->pat, opts, ms))
            for (int i = 0; i < t->nmesh; ++i) t->run_mesh_steps[i] += ms[i];
        else if (t->nmesh == 1)
            t->run_mesh_steps[0] += info.iters;
        std::swap(cur, nxt);
    }
    CK(cudaMemcpyAsync(c_out, cur, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return VFV_OK;
}

int vfv_transport_mesh_steps(const vfv_transport* t, int64_t* steps) {
    if (!t || !steps) return set_err(nullptr, VFV_BAD_INPUT, "NULL argument");
    if ((int)t->run_mesh_steps.size() != t->nmesh) return set_err(nullptr, VFV_BAD_INPUT, "no vfv_transport_run yet");
    std::memcpy(steps, t->run_mesh_steps.data(), t->nmesh * sizeof(int64_t));
    return VFV_OK;
}

// dJ/dD for J = 0.5 ||c_N - target||^2 after nsteps implicit-Euler steps from c0, for the uniform
// diffusivity D of the last vfv_transport_assemble. Discrete adjoint: A^T lam_N = c_N - target,
// A^T lam_k = M^T lam_{k+1} with M = diag(-vol/dt), dJ/dD = -sum_k lam_{k+1}^T (dA/dD) c_{k+1}.
// The forward states are kept every `every` steps (checkpoints) and the states of one segment are
// recomputed from its checkpoint while the backward sweep crosses it.
int vfv_transport_adjoint_D(vfv_ctx* ctx, vfv_transport* t, const double* c0, int nsteps, int every, const double* target,
                            const vfv_gmres_opts* opts, double* J, double* dJdD, int32_t* adj_iters) {
    if (!ctx || !t || !c0 || !target || nsteps <= 0 || every <= 0) return set_err(ctx, VFV_BAD_INPUT, "invalid argument");
    int rc = check_opts(ctx, opts);
    if (rc) return rc;
    const int64_t n = t->n;
    cudaStream_t s = ctx->stream;
    const int nck = (nsteps + every - 1) / every + 1;
    const int blocks = (int)((n + 255) / 256);
    if (!t->pat_t) {
        rc = make_transpose(ctx, t->pat, &t->pat_t, t->tmap);
        if (rc) return rc;
    }
    const size_t need = (size_t)n * (nck + every + 5) + (size_t)blocks + (size_t)nsteps + 8;
    if (t->adj.n < need) CK(t->adj.alloc(need));
    if (!t->adj_counter.p) {
        CK(t->adj_counter.alloc(1));
        CK(cudaMemset(t->adj_counter.p, 0, sizeof(unsigned)));
    }
    double* ck = t->adj.p;                       // [nck][n] checkpoints c_0, c_every, ...
    double* seg = ck + (size_t)nck * n;          // [every][n] states of one segment
    double* lam = seg + (size_t)every * n;       // adjoint vectors
    double* lam2 = lam + n;
    double* rhs = lam2 + n;
    double* zero = rhs + n;
    double* tmp = zero + n;
    double* part = tmp + n;
    double* terms = part + blocks;               // [nsteps]
    if ((rc = gather_transpose_values(ctx, t->pat, t->pat_t, t->tmap.p))) return rc;
    CK(cudaMemsetAsync(zero, 0, n * sizeof(double), s));
    CK(cudaMemcpyAsync(ck, c0, n * sizeof(double), cudaMemcpyHostToDevice, s));
    const TransportDev T = t->dev();
    auto step = [&](const double* cin, double* cout) -> int {
        launch_transport_rhs(s, n, t->cvol.p, t->dt, cin, t->b.p);
        vfv_solve_info info{};
        return solve_dev(ctx, t->pat, t->b.p, cin, cout, opts, &info, true);
    };
    // forward sweep, keeping checkpoints
    CK(cudaMemcpyAsync(t->c0.p, ck, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    double* cur = t->c0.p;
    double* nxt = t->c1.p;
    for (int k = 0; k < nsteps; ++k) {
        if ((rc = step(cur, nxt))) return rc;
        std::swap(cur, nxt);
        if ((k + 1) % every == 0 && (k + 1) / every < nck) CK(cudaMemcpyAsync(ck + (size_t)((k + 1) / every) * n, cur, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    // J and lam_N
    std::vector<double> hc(n), ht(target, target + n);
    CK(cudaMemcpyAsync(hc.data(), cur, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    double jsum = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double r = hc[i] - ht[i];
        jsum += r * r;
        hc[i] = r;
    }
    if (J) *J = 0.5 * jsum;
    CK(cudaMemcpyAsync(rhs, hc.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
    vfv_solve_info info{};
    if ((rc = solve_dev(ctx, t->pat_t, rhs, zero, lam, opts, &info, true))) return rc;
    if (adj_iters) adj_iters[nsteps - 1] = info.iters;
    // backward sweep over the segments, last first
    for (int k = nsteps - 1; k >= 0; --k) {
        const int j = k / every;  // segment of state c_{k+1}: c_{j every + 1 .. j every + every}
        if (k == nsteps - 1 || (k + 1) % every == 0) {
            const int last = std::min(nsteps, j * every + every);
            const double* from = ck + (size_t)j * n;
            for (int q = j * every; q < last; ++q) {
                double* to = seg + (size_t)(q - j * every) * n;
                if ((rc = step(q == j * every ? from : seg + (size_t)(q - 1 - j * every) * n, to))) return rc;
            }
        }
        const double* c_k1 = seg + (size_t)(k - j * every) * n;
        launch_transport_dAdD_dot(s, T, lam, c_k1, part, t->adj_counter.p, terms + k);
        if (k > 0) {
            launch_transport_rhs(s, n, t->cvol.p, t->dt, lam, rhs);  // M^T lam = -vol lam / dt
            if ((rc = solve_dev(ctx, t->pat_t, rhs, lam, lam2, opts, &info, true))) return rc;
            if (adj_iters) adj_iters[k - 1] = info.iters;
            std::swap(lam, lam2);
        }
    }
    std::vector<double> ht2(nsteps);
    CK(cudaMemcpyAsync(ht2.data(), terms, nsteps * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    CK(cudaGetLastError());
    double g = 0.0;
    for (int k = 0; k < nsteps; ++k) g -= ht2[k];
    if (dJdD) *dJdD = g;
    (void)tmp;
    return VFV_OK;
}

}  // extern "C"
