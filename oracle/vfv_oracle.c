/*
 * CPU oracle for the assemble-and-solve path of vfvchem-vfvm3d — TEST INFRASTRUCTURE ONLY.
 *
 * Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the reference answer; the
 * product (libvfvgpu.so) never links or calls it.
 *
 * Parity status: UNPINNED against reference-produced outputs. The reference is Rust (no cargo or
 * rustc here) and ships no golden vectors for this path; its GMRES lives in the un-vendored crate
 * faer_gmres 0.5.0 and its CSC build and LU in faer 0.24.4. This restatement is pinned instead to
 * known answers (tests/test_oracle.py): linear-field exactness of the two-point flux, LSQ
 * gradients exact for linear fields, row sums, symmetry of the point block, the FP64 sparse LU
 * solution (scipy SuperLU) and analytic 1-D slab profiles.
 *
 * Functions restate (file:line in the reference project):
 *   orc_grad            ScalarDomain::update_grad            src/base/scl_dom.rs:146-164
 *   orc_heat_triplets   SteadyHeat::assemble_matrix          src/steady/core/steady_heat.rs:143-171
 *                       with OpSclDomDiffusion               src/operator/core/opscl_dom_diff.rs:40-91
 *                            OpSclDomProduction              src/operator/core/opscl_dom_prod.rs:39-76
 *                            OpSclDomSource                  src/operator/core/opscl_dom_src.rs:37-68
 *                            OpSclBndDirichlet               src/operator/core/opscl_bnd_dir.rs:56-78
 *                            OpSclBndDiffusion               src/operator/core/opscl_bnd_diff.rs:40-96
 *                            OpSclBndProduction              src/operator/core/opscl_bnd_prod.rs:39-81
 *                            OpSclBndSource                  src/operator/core/opscl_bnd_src.rs:37-73
 *                            OpSclBndNeumann                 src/operator/core/opscl_bnd_neu.rs:36-88
 *                       and OperatorBase::add_sclscl_a/add_scl_b src/operator/operator_base.rs:12-34
 *   orc_csr_from_triplets  LinearGmres::update_sparse + build_matrix (linear_gmres.rs:53-74):
 *                       sorted, de-duplicated pattern, duplicates summed in push order (stable
 *                       argsort), explicit zeros kept; returned as CSR (the reference's CSC of A is
 *                       the CSR of A^T, so callers compare canonical sorted forms)
 *   orc_gmres           LinearGmres::solve_matrix (linear_gmres.rs:76-84): restarted GMRES with
 *                       Jacobi (or ILU(0)) right preconditioning, warm start, modified Gram-Schmidt,
 *                       Givens rotations (Saad & Schultz 1986; Saad, Iterative Methods, Alg. 9.5)
 *   orc_ilu0_*          ILU(0) (Saad, Alg. 10.4, IKJ) on a given symmetric permutation — the added
 *                       preconditioner, which has no reference counterpart
 * Compiled with -ffp-contract=off so products and sums round like the reference's Rust scalars.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------ */
void orc_grad(int64_t n, const int64_t* np, const int32_t* ni, const double* gw, int64_t n_dir, const double* f, double* grad) {
    for (int64_t v = 0; v < n; ++v) {
        double gx = 0.0, gy = 0.0, gz = 0.0;
        for (int64_t i = np[v]; i < np[v + 1]; ++i) {
            const double d = f[ni[i]] - f[v];
            gx += gw[i] * d;
            gy += gw[n_dir + i] * d;
            gz += gw[2 * n_dir + i] * d;
        }
        grad[v] = gx;
        grad[n + v] = gy;
        grad[2 * n + v] = gz;
    }
}

/* ------------------------------------------------------------------------------------------ */
typedef struct {
    int64_t n, n_pts, n_dir, n_bsub;
    const int64_t* np;
    const int32_t* ni;
    const double *dist, *area, *skew; /* skew [3][n_dir] */
    const double *cvol, *cskew;       /* cskew [3][n] */
    const int64_t* bp;
    const int32_t *bj, *bk;
    const double *barea, *bw;         /* bw [3][n_bsub] */
} orc_dual;

static int64_t push(uint64_t* r, uint64_t* c, double* v, int64_t t, int64_t row, int64_t col, double val) {
    r[t] = (uint64_t)row;
    c[t] = (uint64_t)col;
    v[t] = val;
    return t + 1;
}

/* diffusion over the neighbours of one vertex (opscl_dom_diff.rs:55-87, opscl_bnd_diff.rs:55-91) */
static int64_t diff_row(const orc_dual* d, int64_t v, const double* k, const double* gk, uint64_t* r, uint64_t* c, double* val, int64_t t) {
    const int64_t N = d->n, D = d->n_dir;
    const double kv = k[v], gxv = gk[v], gyv = gk[N + v], gzv = gk[2 * N + v];
    for (int64_t i = d->np[v]; i < d->np[v + 1]; ++i) {
        const int64_t nb = d->ni[i];
        const double kn = k[nb];
        const double sx = d->skew[i], sy = d->skew[D + i], sz = d->skew[2 * D + i];
        const double km = (kv + kn != 0.0) ? 2.0 * kv * kn / (kv + kn) : 0.0;
        double kf = km + 0.5 * (sx * (gxv + gk[nb]) + sy * (gyv + gk[N + nb]) + sz * (gzv + gk[2 * N + nb]));
        kf = kf > 0.0 ? kf : km;
        const double coeff = kf * d->area[i] / d->dist[i];
        t = push(r, c, val, t, v, nb, coeff);
        t = push(r, c, val, t, v, v, -coeff);
    }
    return t;
}

/* production (opscl_dom_prod.rs:56-73) */
static int64_t prod_row(const orc_dual* d, int64_t v, const double* s, const double* gs, const double* gT, uint64_t* r, uint64_t* c,
                        double* val, int64_t t, double* b) {
    const int64_t N = d->n;
    const double sx = d->cskew[v], sy = d->cskew[N + v], sz = d->cskew[2 * N + v];
    const double vol = d->cvol[v];
    const double prd_v = s[v];
    const double prd_c = prd_v + gs[v] * sx + gs[N + v] * sy + gs[2 * N + v] * sz;
    const double unk_skew = gT[v] * sx + gT[N + v] * sy + gT[2 * N + v] * sz;
    t = push(r, c, val, t, v, v, prd_c * vol);
    b[v] += -prd_v * unk_skew * vol;
    return t;
}

/* source (opscl_dom_src.rs:48-65) */
static void src_row(const orc_dual* d, int64_t v, const double* q, const double* gq, double* b) {
    const int64_t N = d->n;
    const double sx = d->cskew[v], sy = d->cskew[N + v], sz = d->cskew[2 * N + v];
    const double vol = d->cvol[v];
    const double src_c = q[v] + gq[v] * sx + gq[N + v] * sy + gq[2 * N + v] * sz;
    b[v] += -src_c * vol;
}

/*
 * Triplets and b in the push order of SteadyHeat::assemble_matrix. node_bnd[v] is the boundary
 * id of vertex v (-1 for points); bnd_order[] lists boundary ids in registration order and
 * bnd_kind[id] is 0 (temperature) or 1 (heat flux). Dirichlet boundaries are applied first in
 * their registration order, then flux boundaries in theirs (steady_heat.rs:152-161). bc_val[v]
 * is the boundary value of node v. Returns the number of triplets written.
 */
int64_t orc_heat_triplets(const orc_dual* d, const int32_t* node_bnd, int32_t n_bnd, const int32_t* bnd_order, const int32_t* bnd_kind,
                          const double* k, const double* q, const double* s, const double* T, const double* bc_val, const double* gk,
                          const double* gq, const double* gs, const double* gT, uint64_t* r, uint64_t* c, double* val, double* b) {
    const int64_t n = d->n;
    int64_t t = 0;
    (void)T;
    memset(b, 0, sizeof(double) * n);
    /* domain operators: diffusion, production, source over points (steady_heat.rs:145-149) */
    for (int64_t v = 0; v < d->n_pts; ++v) t = diff_row(d, v, k, gk, r, c, val, t);
    for (int64_t v = 0; v < d->n_pts; ++v) t = prod_row(d, v, s, gs, gT, r, c, val, t, b);
    for (int64_t v = 0; v < d->n_pts; ++v) src_row(d, v, q, gq, b);
    /* Dirichlet boundaries (steady_heat.rs:152-154) */
    for (int32_t oi = 0; oi < n_bnd; ++oi) {
        const int32_t bid = bnd_order[oi];
        if (bnd_kind[bid] != 0) continue;
        for (int64_t v = d->n_pts; v < n; ++v) {
            if (node_bnd[v] != bid) continue;
            t = push(r, c, val, t, v, v, 1.0);
            b[v] += bc_val[v];
        }
    }
    /* flux boundaries: diffusion, production, source, Neumann (steady_heat.rs:155-160) */
    for (int32_t oi = 0; oi < n_bnd; ++oi) {
        const int32_t bid = bnd_order[oi];
        if (bnd_kind[bid] != 1) continue;
        for (int64_t v = d->n_pts; v < n; ++v)
            if (node_bnd[v] == bid) t = diff_row(d, v, k, gk, r, c, val, t);
        for (int64_t v = d->n_pts; v < n; ++v)
            if (node_bnd[v] == bid) t = prod_row(d, v, s, gs, gT, r, c, val, t, b);
        for (int64_t v = d->n_pts; v < n; ++v)
            if (node_bnd[v] == bid) src_row(d, v, q, gq, b);
        for (int64_t v = d->n_pts; v < n; ++v) {
            if (node_bnd[v] != bid) continue;
            const double fv = bc_val[v];
            for (int64_t sb = d->bp[v]; sb < d->bp[v + 1]; ++sb) {
                const int64_t j = d->bj[sb], kk = d->bk[sb];
                const double fj = node_bnd[j] == bid ? bc_val[j] : fv;
                const double fk = node_bnd[kk] == bid ? bc_val[kk] : fv;
                const double area = d->barea[sb];
                b[v] += area * (d->bw[sb] * fv + d->bw[d->n_bsub + sb] * fj + d->bw[2 * d->n_bsub + sb] * fk);
            }
        }
    }
    return t;
}

/* ------------------------------------------------------------------------------------------ */
/*
 * Transient advection-diffusion for one mesh, in push order per operator: time
 * (OpSclDomTimeUnity::apply_time, opscl_dom_timeunity.rs:32-58) over points, diffusion
 * (opscl_dom_diff.rs:55-87) over points, advection (OpSclDomAdvection, opscl_dom_adv.rs:49-125)
 * over points, then the boundary twins (opscl_bnd_timeunity, opscl_bnd_diff, opscl_bnd_adv) for
 * the nodes of each zero-flux boundary in boundary order. Face mass flux from
 * flow_helper::update_flux (flow_helper.rs:72-179) with zero pressure and body force, density and
 * species weight 1. gvel is [9][n] (du/dx, du/dy, du/dz, dv/dx, ...). Returns the triplet count.
 */
static int64_t transport_row_time(const orc_dual* d, int64_t v, double dt, uint64_t* r, uint64_t* c, double* val, int64_t t) {
    return push(r, c, val, t, v, v, -d->cvol[v] / dt);
}

static double face_df(const orc_dual* d, int64_t v, int64_t i, const double* D, const double* gD) {
    const int64_t N = d->n, E = d->n_dir;
    const int64_t nb = d->ni[i];
    const double dv = D[v], dn = D[nb];
    const double sx = d->skew[i], sy = d->skew[E + i], sz = d->skew[2 * E + i];
    const double dm = (dv + dn != 0.0) ? 2.0 * dv * dn / (dv + dn) : 0.0;
    double df = dm + 0.5 * (sx * (gD[v] + gD[nb]) + sy * (gD[N + v] + gD[N + nb]) + sz * (gD[2 * N + v] + gD[2 * N + nb]));
    return df > 0.0 ? df : dm;
}

static double face_flux(const orc_dual* d, const double* norm, int64_t v, int64_t i, const double* vel, const double* gvel) {
    const int64_t N = d->n, E = d->n_dir;
    const int64_t nb = d->ni[i];
    const double sx = d->skew[i], sy = d->skew[E + i], sz = d->skew[2 * E + i];
    const double nx = norm[i], ny = norm[E + i], nz = norm[2 * E + i];
    const double den_f = 0.5 * (1.0 + 1.0) + 0.5 * (sx * (0.0 + 0.0) + sy * (0.0 + 0.0) + sz * (0.0 + 0.0));
    double uf[3];
    for (int q = 0; q < 3; ++q) {
        const double* g = gvel + 3 * q * N;
        uf[q] = 0.5 * (vel[q * N + v] + vel[q * N + nb]) + 0.5 * (sx * (g[v] + g[nb]) + sy * (g[N + v] + g[N + nb]) + sz * (g[2 * N + v] + g[2 * N + nb]));
    }
    return den_f * (uf[0] * nx + uf[1] * ny + uf[2] * nz + 0.0) * d->area[i];
}

static int64_t transport_row_diff(const orc_dual* d, int64_t v, const double* D, const double* gD, uint64_t* r, uint64_t* c, double* val,
                                  int64_t t) {
    for (int64_t i = d->np[v]; i < d->np[v + 1]; ++i) {
        const double cond = face_df(d, v, i, D, gD) * d->area[i] / d->dist[i];
        t = push(r, c, val, t, v, d->ni[i], cond);
        t = push(r, c, val, t, v, v, -cond);
    }
    return t;
}

static int64_t transport_row_adv(const orc_dual* d, const double* norm, int64_t v, const double* D, const double* gD, const double* vel,
                                 const double* gvel, uint64_t* r, uint64_t* c, double* val, int64_t t) {
    for (int64_t i = d->np[v]; i < d->np[v + 1]; ++i) {
        const int64_t E = d->n_dir;
        const double sx = d->skew[i], sy = d->skew[E + i], sz = d->skew[2 * E + i];
        const double wgt_f = 0.5 * (1.0 + 1.0) + 0.5 * (sx * (0.0 + 0.0) + sy * (0.0 + 0.0) + sz * (0.0 + 0.0));
        const double den_f = wgt_f;
        const double cond = face_df(d, v, i, D, gD) * d->area[i] / d->dist[i];
        const double flux = den_f != 0.0 ? wgt_f / den_f * face_flux(d, norm, v, i, vel, gvel) : 0.0;
        const double pe = cond != 0.0 ? flux / cond : 0.0;
        double x = 1.0 - 0.1 * fabs(pe);
        x = x > 0.0 ? x : 0.0;
        const double x2 = x * x;
        const double coeff = cond * (x2 * x2 * x - 1.0) + (-flux > 0.0 ? -flux : 0.0);
        t = push(r, c, val, t, v, d->ni[i], coeff);
        t = push(r, c, val, t, v, v, -coeff);
    }
    return t;
}

int64_t orc_transport_triplets(const orc_dual* d, const double* norm, const int32_t* node_bnd, int32_t n_bnd, const double* D,
                               const double* gD, const double* vel, const double* gvel, double dt, uint64_t* r, uint64_t* c,
                               double* val) {
    int64_t t = 0;
    for (int64_t v = 0; v < d->n_pts; ++v) t = transport_row_time(d, v, dt, r, c, val, t);
    for (int64_t v = 0; v < d->n_pts; ++v) t = transport_row_diff(d, v, D, gD, r, c, val, t);
    for (int64_t v = 0; v < d->n_pts; ++v) t = transport_row_adv(d, norm, v, D, gD, vel, gvel, r, c, val, t);
    for (int32_t b = 0; b < n_bnd; ++b) {
        for (int64_t v = d->n_pts; v < d->n; ++v)
            if (node_bnd[v] == b) t = transport_row_time(d, v, dt, r, c, val, t);
        for (int64_t v = d->n_pts; v < d->n; ++v)
            if (node_bnd[v] == b) t = transport_row_diff(d, v, D, gD, r, c, val, t);
        for (int64_t v = d->n_pts; v < d->n; ++v)
            if (node_bnd[v] == b) t = transport_row_adv(d, norm, v, D, gD, vel, gvel, r, c, val, t);
    }
    return t;
}

/* ------------------------------------------------------------------------------------------ */
/* stable sort of triplet indices by (row, col): counting sort on col, then on row */
static void stable_order(int64_t n, int64_t nt, const uint64_t* r, const uint64_t* c, int64_t* ord) {
    int64_t* cnt = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    int64_t* tmp = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nt > 0 ? nt : 1));
    for (int64_t t = 0; t < nt; ++t) cnt[c[t] + 1]++;
    for (int64_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
    for (int64_t t = 0; t < nt; ++t) tmp[cnt[c[t]]++] = t;
    memset(cnt, 0, sizeof(int64_t) * ((size_t)n + 1));
    for (int64_t t = 0; t < nt; ++t) cnt[r[t] + 1]++;
    for (int64_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
    for (int64_t q = 0; q < nt; ++q) {
        const int64_t t = tmp[q];
        ord[cnt[r[t]]++] = t;
    }
    free(cnt);
    free(tmp);
}

/* CSR of A from triplets: rp[n+1], ci[nnz], va[nnz]; returns nnz. ci/va need room for nt. */
int64_t orc_csr_from_triplets(int64_t n, int64_t nt, const uint64_t* r, const uint64_t* c, const double* v, int64_t* rp, int32_t* ci,
                              double* va) {
    int64_t* ord = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nt > 0 ? nt : 1));
    stable_order(n, nt, r, c, ord);
    memset(rp, 0, sizeof(int64_t) * ((size_t)n + 1));
    int64_t nnz = 0;
    for (int64_t q = 0; q < nt; ++q) {
        const int64_t t = ord[q];
        if (q > 0 && r[ord[q - 1]] == r[t] && c[ord[q - 1]] == c[t]) {
            va[nnz - 1] += v[t];
        } else {
            ci[nnz] = (int32_t)c[t];
            va[nnz] = v[t];
            rp[r[t] + 1]++;
            ++nnz;
        }
    }
    for (int64_t i = 0; i < n; ++i) rp[i + 1] += rp[i];
    free(ord);
    return nnz;
}

/* ------------------------------------------------------------------------------------------ */
void orc_spmv(int64_t n, const int64_t* rp, const int32_t* ci, const double* va, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) s += va[k] * x[ci[k]];
        y[i] = s;
    }
}

/* ILU(0) in place on a CSR whose columns ascend per row (IKJ variant). dg[i] = diagonal slot. */
int orc_ilu0_factor(int64_t n, const int64_t* rp, const int32_t* ci, const int64_t* dg, double* a) {
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t kk = rp[i]; kk < dg[i]; ++kk) {
            const int64_t k = ci[kk];
            const double ukk = a[dg[k]];
            if (ukk == 0.0) return 1;
            const double lik = a[kk] / ukk;
            a[kk] = lik;
            int64_t p = kk + 1, qq = dg[k] + 1;
            while (p < rp[i + 1] && qq < rp[k + 1]) {
                if (ci[p] == ci[qq]) {
                    a[p] -= lik * a[qq];
                    ++p;
                    ++qq;
                } else if (ci[p] < ci[qq]) {
                    ++p;
                } else {
                    ++qq;
                }
            }
        }
        if (a[dg[i]] == 0.0) return 1;
    }
    return 0;
}

/* z = (LU)^-1 r on the permuted system: rhs_i = r[perm[i]], out z[perm[i]] = x_i */
void orc_ilu0_apply(int64_t n, const int64_t* rp, const int32_t* ci, const int64_t* dg, const double* a, const int32_t* perm,
                    const double* r, double* t, double* z) {
    for (int64_t i = 0; i < n; ++i) {
        double s = r[perm[i]];
        for (int64_t k = rp[i]; k < dg[i]; ++k) s -= a[k] * t[ci[k]];
        t[i] = s;
    }
    for (int64_t i = n - 1; i >= 0; --i) {
        double s = t[i];
        for (int64_t k = dg[i] + 1; k < rp[i + 1]; ++k) s -= a[k] * t[ci[k]];
        t[i] = s / a[dg[i]];
        z[perm[i]] = t[i];
    }
}

/* ------------------------------------------------------------------------------------------ */
static double dotp(int64_t n, const double* a, const double* b) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

typedef struct {
    /* optional ILU(0) on a permutation (precond == 2) */
    const int64_t *rp, *dg;
    const int32_t *ci, *perm;
    const double* lu;
} orc_ilu;

/*
 * Restarted GMRES(m), right preconditioning M^-1 (precond 0: none, 1: Jacobi, 2: ILU(0)),
 * modified Gram-Schmidt Arnoldi, Givens least squares. Stops when ||b - A x|| <= tol ||b|| (the
 * Arnoldi estimate inside a cycle, the true residual at each restart) or after max_outer cycles.
 * x holds the warm start on entry. Returns 0 converged, 1 not converged; iters/relres out.
 * max_steps > 0 caps the total number of Arnoldi steps (a bounded sample for timing).
 */
int orc_gmres(int64_t n, const int64_t* rp, const int32_t* ci, const double* va, const double* b, double* x, double tol, int m,
              int max_outer, int precond, const orc_ilu* ilu, int64_t max_steps, int* iters_out, double* relres_out) {
    double* V = (double*)malloc(sizeof(double) * (size_t)n * (m + 1));
    double* Hm = (double*)calloc((size_t)(m + 1) * m, sizeof(double));
    double *cs = (double*)malloc(sizeof(double) * m), *sn = (double*)malloc(sizeof(double) * m);
    double *g = (double*)malloc(sizeof(double) * (m + 1)), *y = (double*)malloc(sizeof(double) * m);
    double *w = (double*)malloc(sizeof(double) * n), *z = (double*)malloc(sizeof(double) * n);
    double *tmp = (double*)malloc(sizeof(double) * n), *dinv = (double*)malloc(sizeof(double) * n);
    for (int64_t i = 0; i < n; ++i) {
        double dd = 0.0;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) dd = va[k];
        dinv[i] = dd != 0.0 ? 1.0 / dd : 1.0;
    }
    const double bnorm = sqrt(dotp(n, b, b));
    int its = 0, conv = 0;
    double rel = 0.0;
    if (bnorm == 0.0) {
        memset(x, 0, sizeof(double) * n);
        conv = 1;
        goto done;
    }
    for (int outer = 0; outer <= max_outer; ++outer) {
        orc_spmv(n, rp, ci, va, x, w);
        for (int64_t i = 0; i < n; ++i) w[i] = b[i] - w[i];
        const double beta = sqrt(dotp(n, w, w));
        rel = beta / bnorm;
        if (beta <= tol * bnorm) {
            conv = 1;
            break;
        }
        if (outer == max_outer || (max_steps > 0 && its >= max_steps)) break;
        for (int64_t i = 0; i < n; ++i) V[i] = w[i] / beta;
        memset(g, 0, sizeof(double) * (m + 1));
        g[0] = beta;
        int j = 0;
        for (; j < m; ++j) {
            double* vj = V + (int64_t)j * n;
            const double* pin = vj;
            if (precond == 1) {
                for (int64_t i = 0; i < n; ++i) z[i] = dinv[i] * vj[i];
                pin = z;
            } else if (precond == 2) {
                orc_ilu0_apply(n, ilu->rp, ilu->ci, ilu->dg, ilu->lu, ilu->perm, vj, tmp, z);
                pin = z;
            }
            orc_spmv(n, rp, ci, va, pin, w);
            double* h = Hm + (int64_t)j * (m + 1);
            for (int i = 0; i <= j; ++i) {
                const double* vi = V + (int64_t)i * n;
                h[i] = dotp(n, w, vi);
#pragma omp parallel for schedule(static)
                for (int64_t q = 0; q < n; ++q) w[q] -= h[i] * vi[q];
            }
            h[j + 1] = sqrt(dotp(n, w, w));
            if (h[j + 1] != 0.0) {
                double* vn = V + (int64_t)(j + 1) * n;
                for (int64_t q = 0; q < n; ++q) vn[q] = w[q] / h[j + 1];
            }
            for (int i = 0; i < j; ++i) {
                const double a0 = h[i], a1 = h[i + 1];
                h[i] = cs[i] * a0 + sn[i] * a1;
                h[i + 1] = -sn[i] * a0 + cs[i] * a1;
            }
            const double rr = hypot(h[j], h[j + 1]);
            cs[j] = rr > 0.0 ? h[j] / rr : 1.0;
            sn[j] = rr > 0.0 ? h[j + 1] / rr : 0.0;
            h[j] = rr;
            h[j + 1] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            ++its;
            if (fabs(g[j + 1]) <= tol * bnorm || rr == 0.0 || (max_steps > 0 && its >= max_steps)) {
                ++j;
                break;
            }
        }
        if (j > m) j = m;
        for (int i = j - 1; i >= 0; --i) {
            double s = g[i];
            for (int q = i + 1; q < j; ++q) s -= Hm[(int64_t)q * (m + 1) + i] * y[q];
            y[i] = s / Hm[(int64_t)i * (m + 1) + i];
        }
        memset(w, 0, sizeof(double) * n);
        for (int i = 0; i < j; ++i) {
            const double* vi = V + (int64_t)i * n;
#pragma omp parallel for schedule(static)
            for (int64_t q = 0; q < n; ++q) w[q] += y[i] * vi[q];
        }
        if (precond == 1) {
            for (int64_t q = 0; q < n; ++q) x[q] += dinv[q] * w[q];
        } else if (precond == 2) {
            orc_ilu0_apply(n, ilu->rp, ilu->ci, ilu->dg, ilu->lu, ilu->perm, w, tmp, z);
            for (int64_t q = 0; q < n; ++q) x[q] += z[q];
        } else {
            for (int64_t q = 0; q < n; ++q) x[q] += w[q];
        }
    }
done:
    if (iters_out) *iters_out = its;
    if (relres_out) *relres_out = rel;
    free(V);
    free(Hm);
    free(cs);
    free(sn);
    free(g);
    free(y);
    free(w);
    free(z);
    free(tmp);
    free(dinv);
    return conv ? 0 : 1;
}
