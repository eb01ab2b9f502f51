// Coupled Navier-Stokes handle of libvfvgpu (the reference's SteadyFlow): symbolic set-up on the
// host, device assembly (kernels/ns.cu), and the damped Picard loop around the GMRES of vfv_solve.
#include "internal.cuh"
#include "host/ns_setup.hpp"
#include "kernels/assemble.cuh"
#include "kernels/ns.cuh"

#include <cstring>
#include <cmath>
#include <vector>

// ================================================================ coupled Navier-Stokes (SteadyFlow)
// Field-major [u | v | w | p] system of SteadyFlow::assemble_matrix (src/steady/core/steady_flow.rs:
// 255-303) for one domain whose six faces are velocity boundaries, with the pressure fixed at one
// vertex: assembled on the device from the flow data (flow_helper.rs) and solved by the GMRES of
// vfv_solve (GMRES(m) + 4x4 block-Jacobi for the lid-driven cavity) inside the damped
// Picard loop of SteadyBase::solve (src/steady/steady_base.rs:70-112).
struct vfv_flow {
    vfv_ctx* ctx = nullptr;
    int64_t n = 0, n_pts = 0, n_dir = 0, n_bsub = 0, n_gc = 0, ntrip = 0, pref_vid = 0;
    double pref = 0.0, rho_max = 0.0;
    DBuf<int32_t> np, ni, bp, bj, bk, gcp, gcv, div_off, pst_off, sub_off, slot_loc;
    DBuf<double> dist, area, norm, skew, gw, cvol, cskew, barea, bnorm, bw, gcc;
    DBuf<double> den, visc, fce, bc_vel, gfix, gvel, rc, mom, flux, tv, b, x, xu;
    DBuf<double> xo, rpart;  // previous Picard state and the partials of its scaled change (device)
    DBuf<int64_t> trip_ptr, slot_ptr;
    vfv_pattern* pat = nullptr;
    ~vfv_flow() {
        if (pat) vfv_pattern_destroy(pat);
    }
    NsDev dev(const double* xs) const {
        NsDev D{};
        D.n = n;
        D.n_pts = n_pts;
        D.n_dir = n_dir;
        D.n_bsub = n_bsub;
        D.n_gc = n_gc;
        D.pref_vid = pref_vid;
        D.pref = pref;
        D.np = np.p;
        D.ni = ni.p;
        D.dist = dist.p;
        D.area = area.p;
        D.norm = norm.p;
        D.skew = skew.p;
        D.gw = gw.p;
        D.cvol = cvol.p;
        D.cskew = cskew.p;
        D.bp = bp.p;
        D.bj = bj.p;
        D.bk = bk.p;
        D.barea = barea.p;
        D.bnorm = bnorm.p;
        D.bw = bw.p;
        D.gcp = gcp.p;
        D.gcv = gcv.p;
        D.gcc = gcc.p;
        D.den = den.p;
        D.visc = visc.p;
        D.fce = fce.p;
        D.bc_vel = bc_vel.p;
        D.x = xs;
        D.gvel = gvel.p;
        D.gden = gfix.p;
        D.gvisc = gfix.p + 3 * n;
        D.gfce = gfix.p + 6 * n;
        D.rc = rc.p;
        D.mom = mom.p;
        D.flux = flux.p;
        D.trip_ptr = trip_ptr.p;
        D.div_off = div_off.p;
        D.pst_off = pst_off.p;
        D.sub_off = sub_off.p;
        D.tv = tv.p;
        D.b = b.p;
        D.rp = pat->rp.p;
        D.slot_ptr = slot_ptr.p;
        D.slot_loc = slot_loc.p;
        D.val = pat->val.p;
        return D;
    }
};

namespace {

__global__ void k_damp(int64_t n, double damp, double* __restrict__ x, const double* __restrict__ xu) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = (1.0 - damp) * x[i] + damp * xu[i];
}

// Picard change measure of scaled_residual (src/base/scaling.rs:113-136), on the device: for the
// pressure field the scale is max(range p, rho_max |u|max^2) with a round-off dead band of
// 1e-11 max|p|, for the velocity field max |u| (ranges and maxima over the old and the new state);
// the measure is the larger of the two RMS changes over their scales, NaN if the new state is not
// finite. Four small kernels: per-block extrema, their reduction, per-block sums of squared
// changes, their reduction into out[0]. Extrema are exact in any order; the sums are summed in a
// fixed block order.
constexpr int kResBlocks = 296;  // two per SM
struct ResPart { double vmax, pmin, pmax, pabs, sp, sv; int32_t nonfinite, pad; };

__global__ void __launch_bounds__(256) k_res_extrema(int64_t n, const double* __restrict__ xo, const double* __restrict__ xn,
                                                    ResPart* part) {
    __shared__ double sv[4][8];
    __shared__ int snf;
    if (threadIdx.x == 0) snf = 0;
    __syncthreads();
    double vmax = 0.0, pmin = 1e308, pmax = -1e308, pabs = 0.0;
    int nf = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        for (int st = 0; st < 2; ++st) {
            const double* x = st ? xn : xo;
            const double a = x[i], b = x[n + i], c = x[2 * n + i], p = x[3 * n + i];
            vmax = fmax(vmax, sqrt(a * a + b * b + c * c));
            pmin = fmin(pmin, p);
            pmax = fmax(pmax, p);
            pabs = fmax(pabs, fabs(p));
            if (st && !(isfinite(a) && isfinite(b) && isfinite(c) && isfinite(p))) nf = 1;
        }
    }
    if (nf) snf = 1;
    for (int o = 16; o > 0; o >>= 1) {
        vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        pmin = fmin(pmin, __shfl_xor_sync(0xffffffffu, pmin, o));
        pmax = fmax(pmax, __shfl_xor_sync(0xffffffffu, pmax, o));
        pabs = fmax(pabs, __shfl_xor_sync(0xffffffffu, pabs, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sv[0][wid] = vmax;
        sv[1][wid] = pmin;
        sv[2][wid] = pmax;
        sv[3][wid] = pabs;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ResPart r{};
        r.vmax = sv[0][0];
        r.pmin = sv[1][0];
        r.pmax = sv[2][0];
        r.pabs = sv[3][0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            r.vmax = fmax(r.vmax, sv[0][w]);
            r.pmin = fmin(r.pmin, sv[1][w]);
            r.pmax = fmax(r.pmax, sv[2][w]);
            r.pabs = fmax(r.pabs, sv[3][w]);
        }
        r.nonfinite = snf;
        part[blockIdx.x] = r;
    }
}

// part[nb] <- the reduced extrema (one thread)
__global__ void k_res_extrema_finish(int nb, ResPart* part) {
    ResPart g = part[0];
    for (int b = 1; b < nb; ++b) {
        const ResPart& r = part[b];
        g.vmax = fmax(g.vmax, r.vmax);
        g.pmin = fmin(g.pmin, r.pmin);
        g.pmax = fmax(g.pmax, r.pmax);
        g.pabs = fmax(g.pabs, r.pabs);
        g.nonfinite |= r.nonfinite;
    }
    part[nb] = g;
}

__global__ void __launch_bounds__(256) k_res_sums(int64_t n, const double* __restrict__ xo, const double* __restrict__ xn, ResPart* part,
                                                 int nb) {
    __shared__ double red[8];
    const double dead = 1e-11 * part[nb].pabs;
    double sp = 0.0, sv = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double dp = fmax(fabs(xn[3 * n + i] - xo[3 * n + i]) - dead, 0.0);
        sp += dp * dp;
        for (int c = 0; c < 3; ++c) {
            const double d = fabs(xn[c * n + i] - xo[c * n + i]);
            sv += d * d;
        }
    }
    sp = block_sum(sp, red);
    __syncthreads();
    sv = block_sum(sv, red);
    if (threadIdx.x == 0) {
        part[blockIdx.x].sp = sp;
        part[blockIdx.x].sv = sv;
    }
}

__global__ void k_res_finish(int64_t n, int nb, double rho_max, const ResPart* part, double* out) {
    const ResPart g = part[nb];
    double sp = 0.0, sv = 0.0;
    for (int b = 0; b < nb; ++b) {
        sp += part[b].sp;
        sv += part[b].sv;
    }
    if (g.nonfinite) {
        out[0] = nan("");
        return;
    }
    const double floor_ = 1e-30;
    const double nn = (double)(n > 1 ? n : 1);
    const double rp = sqrt(sp / nn) / fmax(fmax(g.pmax - g.pmin, rho_max * g.vmax * g.vmax), floor_);
    const double rv = sqrt(sv / nn) / fmax(g.vmax, floor_);
    out[0] = fmax(rp, rv);
}

int flow_assemble(vfv_ctx* ctx, vfv_flow* f, const double* xs) {
    cudaStream_t s = ctx->stream;
    const int64_t n = f->n;
    const double* fv[3] = {xs, xs + n, xs + 2 * n};
    launch_grad(s, n, f->np.p, f->ni.p, f->gw.p, f->n_dir, 3, fv, f->gvel.p);
    launch_ns_assemble(s, f->dev(xs));
    ctx->launches += 8;
    f->pat->version++;
    CK(cudaGetLastError());
    return VFV_OK;
}

}  // namespace

extern "C" {

int vfv_flow_pattern_host(const vfv_mesh* mh, int64_t pref_vid, int64_t* nnz, int64_t* ntrip, int32_t* rowptr, int32_t* colind) {
    if (!mh) return set_err(nullptr, VFV_BAD_INPUT, "NULL mesh");
    NsLayout L;
    const std::string e = build_ns_layout(mh->d, pref_vid, L);
    if (!e.empty()) return set_err(nullptr, VFV_BAD_INPUT, e);
    if (nnz) *nnz = L.nnz();
    if (ntrip) *ntrip = L.ntrip();
    if (rowptr) std::copy(L.rp.begin(), L.rp.end(), rowptr);
    if (colind) std::copy(L.ci.begin(), L.ci.end(), colind);
    return VFV_OK;
}

int vfv_flow_create(vfv_ctx* ctx, const vfv_mesh* mh, const double* rho, const double* mu, const double* fce, const double* bc_vel,
                    int64_t pref_vid, double pref, vfv_flow** out) {
    DeviceGuard dg_(ctx);
    if (!ctx || !mh || !rho || !mu || !fce || !bc_vel || !out) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    *out = nullptr;
    const Dual& d = mh->d;
    const int64_t n = d.n_tot;
    if (n + d.n_dir >= (int64_t)1 << 31) return set_err(ctx, VFV_BAD_INPUT, "mesh too large for 32-bit indices");
    for (int64_t v = mh->m.n_pts; v < n; ++v) {
        const int32_t bnd = mh->m.node_bnd[v - mh->m.n_pts];
        if (bnd < 0 || bnd >= NUM_BND) return set_err(ctx, VFV_BAD_INPUT, "every node must lie on a velocity boundary");
    }
    NsLayout L;
    const std::string e = build_ns_layout(d, pref_vid, L);
    if (!e.empty()) return set_err(ctx, VFV_BAD_INPUT, e);
    auto f = std::make_unique<vfv_flow>();
    f->ctx = ctx;
    f->n = n;
    f->n_pts = d.n_pts;
    f->n_dir = d.n_dir;
    f->n_bsub = d.bnd_ptr[n];
    f->n_gc = (int64_t)L.gcv.size();
    f->ntrip = L.ntrip();
    f->pref_vid = pref_vid;
    f->pref = pref;
    for (int64_t v = 0; v < n; ++v) f->rho_max = std::max(f->rho_max, std::fabs(rho[v]));
    vfv_pattern* pat = nullptr;
    int rc = vfv_pattern_from_csr(ctx, 4 * n, L.rp.data(), L.ci.data(), &pat);
    if (rc) return rc;
    f->pat = pat;
    rc = vfv_pattern_autotune(ctx, pat, nullptr, nullptr);  // rows of 16 to 400 entries: measure the SpMV shape
    if (rc) return rc;
    cudaStream_t s = ctx->stream;
    std::vector<int32_t> np(n + 1), bp(n + 1);
    for (int64_t v = 0; v <= n; ++v) {
        np[v] = (int32_t)d.nbr_ptr[v];
        bp[v] = (int32_t)d.bnd_ptr[v];
    }
    CK(f->np.upload(np.data(), n + 1, s));
    CK(f->ni.upload(d.nbr_idx.data(), d.n_dir, s));
    CK(f->bp.upload(bp.data(), n + 1, s));
    CK(f->bj.upload(d.bnd_j.data(), d.bnd_j.size(), s));
    CK(f->bk.upload(d.bnd_k.data(), d.bnd_k.size(), s));
    CK(f->dist.upload(d.dist.data(), d.dist.size(), s));
    CK(f->area.upload(d.area.data(), d.area.size(), s));
    CK(f->norm.upload(d.norm.data(), d.norm.size(), s));
    CK(f->skew.upload(d.skew.data(), d.skew.size(), s));
    CK(f->gw.upload(d.gw.data(), d.gw.size(), s));
    CK(f->cvol.upload(d.cvol.data(), d.cvol.size(), s));
    CK(f->cskew.upload(d.cskew.data(), d.cskew.size(), s));
    CK(f->barea.upload(d.bnd_area.data(), d.bnd_area.size(), s));
    CK(f->bnorm.upload(d.bnd_norm.data(), d.bnd_norm.size(), s));
    CK(f->bw.upload(d.bnd_wgt.data(), d.bnd_wgt.size(), s));
    CK(f->gcp.upload(L.gcp.data(), L.gcp.size(), s));
    CK(f->gcv.upload(L.gcv.data(), L.gcv.size(), s));
    CK(f->gcc.upload(L.gcc.data(), L.gcc.size(), s));
    CK(f->trip_ptr.upload(L.trip_ptr.data(), L.trip_ptr.size(), s));
    CK(f->div_off.upload(L.div_off.data(), L.div_off.size(), s));
    CK(f->pst_off.upload(L.pst_off.data(), L.pst_off.size(), s));
    CK(f->sub_off.upload(L.sub_off.data(), L.sub_off.size(), s));
    CK(f->slot_ptr.upload(L.slot_ptr.data(), L.slot_ptr.size(), s));
    CK(f->slot_loc.upload(L.slot_loc.data(), L.slot_loc.size(), s));
    CK(f->den.upload(rho, n, s));
    CK(f->visc.upload(mu, n, s));
    CK(f->fce.upload(fce, 3 * n, s));
    CK(f->bc_vel.upload(bc_vel, 3 * n, s));
    CK(f->gfix.alloc(15 * n));
    CK(f->gvel.alloc(9 * n));
    CK(f->rc.alloc(n));
    CK(f->mom.alloc(3 * n));
    CK(f->flux.alloc(d.n_dir));
    CK(f->tv.alloc(f->ntrip));
    CK(f->b.alloc(4 * n));
    CK(f->x.alloc(4 * n));
    CK(f->xu.alloc(4 * n));
    // gradients of the fixed fields: (rho, mu, fce_x, fce_y) and fce_z -> gfix [rho | mu | fce (9)]
    const double* f4[4] = {f->den.p, f->visc.p, f->fce.p, f->fce.p + n};
    launch_grad(s, n, f->np.p, f->ni.p, f->gw.p, f->n_dir, 4, f4, f->gfix.p);
    const double* f1[1] = {f->fce.p + 2 * n};
    launch_grad(s, n, f->np.p, f->ni.p, f->gw.p, f->n_dir, 1, f1, f->gfix.p + 12 * n);
    ctx->launches += 2;
    CK(cudaStreamSynchronize(s));
    CK(cudaGetLastError());
    *out = f.release();
    return VFV_OK;
}

void vfv_flow_destroy(vfv_flow* f) {
    if (!f) return;
    if (f->ctx) cudaStreamSynchronize(f->ctx->stream);
    delete f;
}

vfv_pattern* vfv_flow_pattern(vfv_flow* f) { return f ? f->pat : nullptr; }

int vfv_flow_info(const vfv_flow* f, int64_t* n_unknowns, int64_t* nnz, int64_t* ntrip) {
    if (!f) return set_err(nullptr, VFV_BAD_INPUT, "NULL flow");
    if (n_unknowns) *n_unknowns = 4 * f->n;
    if (nnz) *nnz = f->pat->nnz;
    if (ntrip) *ntrip = f->ntrip;
    return VFV_OK;
}

int vfv_flow_assemble_device(vfv_ctx* ctx, vfv_flow* f, const double* x, double* b) {
    DeviceGuard dg_(ctx);
    if (!ctx || !f || !x) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    int rc = flow_assemble(ctx, f, x);
    if (rc) return rc;
    if (b) CK(cudaMemcpyAsync(b, f->b.p, 4 * f->n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return VFV_OK;
}

int vfv_flow_assemble(vfv_ctx* ctx, vfv_flow* f, const double* x, double* b) {
    DeviceGuard dg_(ctx);
    if (!ctx || !f || !x) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    CK(cudaMemcpyAsync(f->x.p, x, 4 * f->n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    int rc = flow_assemble(ctx, f, f->x.p);
    if (rc) return rc;
    if (b) CK(cudaMemcpyAsync(b, f->b.p, 4 * f->n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return VFV_OK;
}

int vfv_flow_picard(vfv_ctx* ctx, vfv_flow* f, double* x, int max_iter, double tol, double damp, const vfv_gmres_opts* opts,
                    double* res, int32_t* lin_iters, int32_t* iters_done, double* solve_seconds) {
    DeviceGuard dg_(ctx);
    if (!ctx || !f || !x) return set_err(ctx, VFV_BAD_INPUT, "NULL argument");
    if (max_iter <= 0) return set_err(ctx, VFV_BAD_INPUT, "max_iter must be positive (SolverNonPositiveMaxIter)");
    if (!(tol > 0.0)) return set_err(ctx, VFV_BAD_INPUT, "tol must be positive (SolverNonPositiveTolerance)");
    if (!(damp > 0.0 && damp <= 1.0)) return set_err(ctx, VFV_BAD_INPUT, "damping must be in (0, 1] (SolverInvalidDamping)");
    int rc = check_opts(ctx, opts);
    if (rc) return rc;
    cudaStream_t s = ctx->stream;
    const int64_t N4 = 4 * f->n;
    if (!f->xo.p) {
        CK(f->xo.alloc(N4));
        CK(f->rpart.alloc(sizeof(ResPart) / sizeof(double) * (kResBlocks + 1) + 1));
    }
    CK(cudaMemcpyAsync(f->x.p, x, N4 * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(f->xo.p, f->x.p, N4 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    ResPart* rpart = reinterpret_cast<ResPart*>(f->rpart.p);
    double* rout = f->rpart.p + sizeof(ResPart) / sizeof(double) * (kResBlocks + 1);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    double tsolve = 0.0;
    int it = 0;
    bool conv = false;
    for (; it < max_iter && !conv; ++it) {
        if ((rc = flow_assemble(ctx, f, f->x.p))) break;
        CK(cudaEventRecord(e0, s));
        vfv_solve_info info{};
        rc = solve_dev(ctx, f->pat, f->b.p, f->x.p, f->xu.p, opts, &info);
        CK(cudaEventRecord(e1, s));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        tsolve += ms * 1e-3;
        if (lin_iters) lin_iters[it] = info.iters;
        if (rc) break;
        k_damp<<<grid_for(N4), 256, 0, s>>>(N4, damp, f->x.p, f->xu.p);
        k_res_extrema<<<kResBlocks, 256, 0, s>>>(f->n, f->xo.p, f->x.p, rpart);
        k_res_extrema_finish<<<1, 1, 0, s>>>(kResBlocks, rpart);
        k_res_sums<<<kResBlocks, 256, 0, s>>>(f->n, f->xo.p, f->x.p, rpart, kResBlocks);
        k_res_finish<<<1, 1, 0, s>>>(f->n, kResBlocks, f->rho_max, rpart, rout);
        CK(cudaMemcpyAsync(f->xo.p, f->x.p, N4 * sizeof(double), cudaMemcpyDeviceToDevice, s));
        ctx->launches += 5;
        CK(cudaMemcpyAsync(ctx->h_scalar, rout, sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        const double r = ctx->h_scalar[0];
        if (res) res[it] = r;
        if (!std::isfinite(r)) {
            rc = set_err(ctx, VFV_NONFINITE, "Picard: non-finite residual (SteadyNonFiniteResidual)");
            ++it;
            break;
        }
        conv = r < tol;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(cudaMemcpyAsync(x, f->x.p, N4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (iters_done) *iters_done = it;
    if (solve_seconds) *solve_seconds = tsolve;
    if (rc) return rc;
    if (!conv) return set_err(ctx, VFV_NOT_CONVERGED, "Picard iteration did not reach the tolerance (SteadyDidNotConverge)");
    return VFV_OK;
}

}  // extern "C"
