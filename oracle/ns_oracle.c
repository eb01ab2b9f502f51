/*
 * CPU oracle for the coupled Navier-Stokes assembly (lid-driven cavity) — TEST INFRASTRUCTURE ONLY.
 *
 * Used by tests/ as the reference answer; the product (libvfvgpu.so) never links or calls it.
 * Parity UNPINNED against reference outputs (the reference is Rust and cannot be built here); the
 * restatement is pinned to known answers in tests/test_oracle_ns.py (pressure-gradient
 * coefficients exact for linear fields and zero for constants, the LU solution of the assembled
 * system).
 *
 * Functions restate (file:line in the reference project):
 *   orc_grad_coeff   Tetrahedron::update_tet step 6, pressure gradient coefficients
 *                    src/base/geom_tet.rs:295-347 (stable sort by vertex, merge in push order)
 *   orc_ns_flow      flow_helper::update_flow + update_flux   src/operator/core/flow_helper.rs:3-179
 *   orc_ns_triplets  SteadyFlow::assemble_matrix              src/steady/core/steady_flow.rs:255-303
 *                    for one domain with velocity boundaries only and a reference pressure:
 *                    OpVecDomAdvection   opvec_dom_adv.rs:49-117     OpVecDomGradient  opvec_dom_grad.rs:41-71
 *                    OpVecDomDiffusion   opvec_dom_diff.rs:40-95     OpVecDomTranspose opvec_dom_dtrn.rs:40-114
 *                    OpVecDomDilatatory  opvec_dom_ddil.rs:41-113    OpVecDomSource    opvec_dom_src.rs:38-73
 *                    OpSclDomDivergence  opscl_dom_div.rs:45-154     OpSclDomPressureStabilizer opscl_dom_pstab.rs:51-152
 *                    OpVecBndDirichlet   opvec_bnd_dir.rs:55-83      OpSclBndDivergence opscl_bnd_div.rs:45-187
 *                    OpSclBndPressureStabilizer opscl_bnd_pstab.rs:51-154
 *                    OpSclDomPressureReference  opscl_dom_pref.rs:40-64 (replaces its row, last)
 *                    with the field-major unknown layout [u | v | w | p] of
 *                    OperatorBase::add_vecvec_a / add_vecscl_a / add_sclvec_a (operator_base.rs:37-94)
 * Compiled with -ffp-contract=off; every expression keeps the reference's evaluation order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int64_t n, n_pts, n_dir, n_bsub;
    const int64_t* np;
    const int32_t* ni;
    const double *dist, *area, *norm, *skew, *gw; /* norm, skew, gw: [3][n_dir] */
    const double *cvol, *cskew;                   /* cskew [3][n] */
    const int64_t* bp;
    const int32_t *bj, *bk;
    const double *barea, *bnorm, *bw;             /* bnorm, bw: [3][n_bsub] */
    const int64_t* gcp;                           /* grad_coeff CSR (orc_grad_coeff) */
    const int32_t* gcv;
    const double* gcc;                            /* [3][n_gc] */
    int64_t n_gc;
} orc_ns_geom;

/* ------------------------------------------------------------------ grad_coeff (geom_tet.rs:295-347) */
typedef struct {
    int64_t vid;
    double c[3];
    int64_t seq;
} gc_ent;

static int gc_cmp(const void* a, const void* b) {
    const gc_ent* x = (const gc_ent*)a;
    const gc_ent* y = (const gc_ent*)b;
    if (x->vid != y->vid) return x->vid < y->vid ? -1 : 1;
    return x->seq < y->seq ? -1 : (x->seq > y->seq); /* stable: push order */
}

static int64_t gc_vertex(const orc_ns_geom* g, int64_t v, gc_ent* buf) {
    const int64_t D = g->n_dir, B = g->n_bsub;
    int64_t t = 0;
#define GC_PUSH(VID, CX, CY, CZ)          \
    do {                                  \
        buf[t].vid = (VID);               \
        buf[t].c[0] = (CX);               \
        buf[t].c[1] = (CY);               \
        buf[t].c[2] = (CZ);               \
        buf[t].seq = t;                   \
        ++t;                              \
    } while (0)
    for (int64_t i = g->np[v]; i < g->np[v + 1]; ++i) {
        const int64_t nb = g->ni[i];
        const double area = g->area[i];
        const double nx = g->norm[i], ny = g->norm[D + i], nz = g->norm[2 * D + i];
        const double sx = g->skew[i], sy = g->skew[D + i], sz = g->skew[2 * D + i];
        GC_PUSH(v, 0.5 * area * nx, 0.5 * area * ny, 0.5 * area * nz);
        GC_PUSH(nb, 0.5 * area * nx, 0.5 * area * ny, 0.5 * area * nz);
        const int64_t ss[2] = {v, nb};
        for (int q = 0; q < 2; ++q) {
            const int64_t s = ss[q];
            for (int64_t k = g->np[s]; k < g->np[s + 1]; ++k) {
                const double wx = g->gw[k], wy = g->gw[D + k], wz = g->gw[2 * D + k];
                const double w_skew = 0.5 * (wx * sx + wy * sy + wz * sz) * area;
                GC_PUSH(g->ni[k], w_skew * nx, w_skew * ny, w_skew * nz);
                GC_PUSH(s, -w_skew * nx, -w_skew * ny, -w_skew * nz);
            }
        }
    }
    for (int64_t b = g->bp[v]; b < g->bp[v + 1]; ++b) {
        const double area = g->barea[b];
        const double nx = g->bnorm[b], ny = g->bnorm[B + b], nz = g->bnorm[2 * B + b];
        const double wv = g->bw[b], wj = g->bw[B + b], wk = g->bw[2 * B + b];
        GC_PUSH(v, wv * area * nx, wv * area * ny, wv * area * nz);
        GC_PUSH(g->bj[b], wj * area * nx, wj * area * ny, wj * area * nz);
        GC_PUSH(g->bk[b], wk * area * nx, wk * area * ny, wk * area * nz);
    }
#undef GC_PUSH
    qsort(buf, (size_t)t, sizeof(gc_ent), gc_cmp);
    int64_t w = 0;
    for (int64_t r = 0; r < t; ++r) {
        if (w > 0 && buf[w - 1].vid == buf[r].vid) {
            buf[w - 1].c[0] += buf[r].c[0];
            buf[w - 1].c[1] += buf[r].c[1];
            buf[w - 1].c[2] += buf[r].c[2];
        } else {
            buf[w++] = buf[r];
        }
    }
    return w;
}

/* gcp[n+1] always written; gcv/gcc (capacity cap) written when non-NULL. Returns the total count. */
int64_t orc_grad_coeff(const orc_ns_geom* g, int64_t* gcp, int32_t* gcv, double* gcc, int64_t cap) {
    int64_t maxp = 0;
    for (int64_t v = 0; v < g->n; ++v) {
        int64_t c = 0;
        for (int64_t i = g->np[v]; i < g->np[v + 1]; ++i) {
            const int64_t nb = g->ni[i];
            c += 2 + 2 * (g->np[v + 1] - g->np[v]) + 2 * (g->np[nb + 1] - g->np[nb]);
        }
        c += 3 * (g->bp[v + 1] - g->bp[v]);
        if (c > maxp) maxp = c;
    }
    gc_ent* buf = (gc_ent*)malloc(sizeof(gc_ent) * (size_t)(maxp > 0 ? maxp : 1));
    int64_t tot = 0;
    gcp[0] = 0;
    for (int64_t v = 0; v < g->n; ++v) {
        const int64_t m = gc_vertex(g, v, buf);
        if (gcv && gcc && tot + m <= cap) {
            for (int64_t k = 0; k < m; ++k) {
                gcv[tot + k] = (int32_t)buf[k].vid;
                gcc[tot + k] = buf[k].c[0];
                gcc[cap + tot + k] = buf[k].c[1];
                gcc[2 * cap + tot + k] = buf[k].c[2];
            }
        }
        tot += m;
        gcp[v + 1] = tot;
    }
    free(buf);
    return tot;
}

/* ------------------------------------------------------------------ flow data (flow_helper.rs) */
static double pow5(double x) {
    const double x2 = x * x;
    return x2 * x2 * x;
}

static double face_visc(const orc_ns_geom* g, int64_t v, int64_t i, const double* visc, const double* gvisc) {
    const int64_t N = g->n, D = g->n_dir;
    const int64_t nb = g->ni[i];
    const double mv = visc[v], mn = visc[nb];
    const double sx = g->skew[i], sy = g->skew[D + i], sz = g->skew[2 * D + i];
    const double vm = (mv + mn != 0.0) ? 2.0 * mv * mn / (mv + mn) : 0.0;
    const double vf = vm + 0.5 * (sx * (gvisc[v] + gvisc[nb]) + sy * (gvisc[N + v] + gvisc[N + nb]) + sz * (gvisc[2 * N + v] + gvisc[2 * N + nb]));
    return vf > 0.0 ? vf : vm;
}

static double face_den(const orc_ns_geom* g, int64_t v, int64_t i, const double* den, const double* gden) {
    const int64_t N = g->n, D = g->n_dir;
    const int64_t nb = g->ni[i];
    const double sx = g->skew[i], sy = g->skew[D + i], sz = g->skew[2 * D + i];
    return 0.5 * (den[v] + den[nb]) + 0.5 * (sx * (gden[v] + gden[nb]) + sy * (gden[N + v] + gden[N + nb]) + sz * (gden[2 * N + v] + gden[2 * N + nb]));
}

/* vel [3][n], gvel [9][n] (component-major: u_x u_y u_z v_x ...), p [n], den/visc [n] with grads
 * [3][n], fce [3][n] with gfce [9][n]. Outputs rc [n] and flux [n_dir]. */
void orc_ns_flow(const orc_ns_geom* g, const double* vel, const double* gvel, const double* p, const double* den, const double* gden,
                 const double* visc, const double* gvisc, const double* fce, const double* gfce, double* rc, double* flux) {
    const int64_t N = g->n, D = g->n_dir;
    for (int64_t v = 0; v < N; ++v) {
        double cp = 0.0;
        for (int64_t i = g->np[v]; i < g->np[v + 1]; ++i) {
            const int64_t nb = g->ni[i];
            const double face = g->area[i], dist = g->dist[i];
            const double nx = g->norm[i], ny = g->norm[D + i], nz = g->norm[2 * D + i];
            const double den_f = face_den(g, v, i, den, gden);
            const double visc_f = face_visc(g, v, i, visc, gvisc);
            const double cond = visc_f * face / dist;
            const double fl = den_f * 0.5 * ((vel[v] + vel[nb]) * nx + (vel[N + v] + vel[N + nb]) * ny + (vel[2 * N + v] + vel[2 * N + nb]) * nz) * face;
            const double pe = cond != 0.0 ? fl / cond : 0.0;
            double x = 1.0 - 0.1 * fabs(pe);
            x = x > 0.0 ? x : 0.0;
            cp += cond * pow5(x) + (fl > 0.0 ? fl : 0.0);
        }
        rc[v] = cp > 0.0 ? g->cvol[v] / cp : 0.0;
    }
    double* mom = (double*)malloc(sizeof(double) * 3 * (size_t)N);
    for (int64_t v = 0; v < N; ++v) {
        const double cx = g->cskew[v], cy = g->cskew[N + v], cz = g->cskew[2 * N + v];
        const double vol = g->cvol[v];
        double px = 0.0, py = 0.0, pz = 0.0;
        for (int64_t k = g->gcp[v]; k < g->gcp[v + 1]; ++k) {
            const double pm = p[g->gcv[k]];
            px += g->gcc[k] * pm / vol;
            py += g->gcc[g->n_gc + k] * pm / vol;
            pz += g->gcc[2 * g->n_gc + k] * pm / vol;
        }
        double fc[3];
        for (int q = 0; q < 3; ++q)
            fc[q] = fce[q * N + v] + gfce[(3 * q) * N + v] * cx + gfce[(3 * q + 1) * N + v] * cy + gfce[(3 * q + 2) * N + v] * cz;
        mom[v] = rc[v] * (px - fc[0]);
        mom[N + v] = rc[v] * (py - fc[1]);
        mom[2 * N + v] = rc[v] * (pz - fc[2]);
    }
    for (int64_t v = 0; v < N; ++v) {
        for (int64_t i = g->np[v]; i < g->np[v + 1]; ++i) {
            const int64_t nb = g->ni[i];
            const double face = g->area[i], dist = g->dist[i];
            const double nx = g->norm[i], ny = g->norm[D + i], nz = g->norm[2 * D + i];
            const double sx = g->skew[i], sy = g->skew[D + i], sz = g->skew[2 * D + i];
            const double den_f = face_den(g, v, i, den, gden);
            double uf[3];
            for (int q = 0; q < 3; ++q) {
                const double* gq = gvel + 3 * q * N;
                uf[q] = 0.5 * (vel[q * N + v] + vel[q * N + nb]) +
                        0.5 * (sx * (gq[v] + gq[nb]) + sy * (gq[N + v] + gq[N + nb]) + sz * (gq[2 * N + v] + gq[2 * N + nb]));
            }
            const double fce_e = 0.5 * (nx * (fce[v] + fce[nb]) + ny * (fce[N + v] + fce[N + nb]) + nz * (fce[2 * N + v] + fce[2 * N + nb]));
            const double mom_e = 0.5 * (nx * (mom[v] + mom[nb]) + ny * (mom[N + v] + mom[N + nb]) + nz * (mom[2 * N + v] + mom[2 * N + nb]));
            const double vel_rc = -0.5 * (rc[v] + rc[nb]) * ((p[nb] - p[v]) / dist - fce_e) + mom_e;
            flux[i] = den_f * (uf[0] * nx + uf[1] * ny + uf[2] * nz + vel_rc) * face;
        }
    }
    free(mom);
}

/* ------------------------------------------------------------------ assembly */
typedef struct {
    uint64_t* r;
    uint64_t* c;
    double* v;
    int64_t t;
} trip_buf;

static void tpush(trip_buf* tb, int64_t row, int64_t col, double val) {
    if (tb->r) {
        tb->r[tb->t] = (uint64_t)row;
        tb->c[tb->t] = (uint64_t)col;
        tb->v[tb->t] = val;
    }
    tb->t++;
}

typedef struct {
    const double *vel, *gvel, *den, *gden, *visc, *gvisc, *fce, *gfce, *rc, *flux;
} ns_fields;

static void force_centroid(const orc_ns_geom* g, const ns_fields* f, int64_t v, double out[3]) {
    const int64_t N = g->n;
    const double cx = g->cskew[v], cy = g->cskew[N + v], cz = g->cskew[2 * N + v];
    for (int q = 0; q < 3; ++q)
        out[q] = f->fce[q * N + v] + f->gfce[(3 * q) * N + v] * cx + f->gfce[(3 * q + 1) * N + v] * cy + f->gfce[(3 * q + 2) * N + v] * cz;
}

/* OpSclDomDivergence / OpSclBndDivergence face part for one vertex (rows p_v) */
static void div_faces(const orc_ns_geom* g, const ns_fields* f, int64_t v, trip_buf* tb) {
    const int64_t N = g->n, D = g->n_dir, P = 3 * N;
    for (int64_t i = g->np[v]; i < g->np[v + 1]; ++i) {
        const int64_t nb = g->ni[i];
        const double face = g->area[i];
        const double nn[3] = {g->norm[i], g->norm[D + i], g->norm[2 * D + i]};
        const double sx = g->skew[i], sy = g->skew[D + i], sz = g->skew[2 * D + i];
        const double den_f = face_den(g, v, i, f->den, f->gden);
        const double coeff = 0.5 * den_f * face;
        for (int c = 0; c < 3; ++c) {
            tpush(tb, P + v, c * N + nb, -coeff * nn[c]);
            tpush(tb, P + v, c * N + v, -coeff * nn[c]);
        }
        for (int64_t k = g->np[v]; k < g->np[v + 1]; ++k) {
            const double w_skew = g->gw[k] * sx + g->gw[D + k] * sy + g->gw[2 * D + k] * sz;
            for (int c = 0; c < 3; ++c) {
                const double val = -coeff * w_skew * nn[c];
                tpush(tb, P + v, c * N + g->ni[k], val);
                tpush(tb, P + v, c * N + v, -val);
            }
        }
        for (int64_t k = g->np[nb]; k < g->np[nb + 1]; ++k) {
            const double w_skew = g->gw[k] * sx + g->gw[D + k] * sy + g->gw[2 * D + k] * sz;
            for (int c = 0; c < 3; ++c) {
                const double val = -coeff * w_skew * nn[c];
                tpush(tb, P + v, c * N + g->ni[k], val);
                tpush(tb, P + v, c * N + nb, -val);
            }
        }
    }
}

/* OpSclDomPressureStabilizer / OpSclBndPressureStabilizer for one vertex (row p_v and b) */
static void pstab(const orc_ns_geom* g, const ns_fields* f, int64_t v, trip_buf* tb, double* b) {
    const int64_t N = g->n, D = g->n_dir, P = 3 * N, G = g->n_gc;
    double fv[3];
    force_centroid(g, f, v, fv);
    const double rc_v = f->rc[v], vol_v = g->cvol[v];
    for (int64_t i = g->np[v]; i < g->np[v + 1]; ++i) {
        const int64_t nb = g->ni[i];
        const double face = g->area[i], dist = g->dist[i];
        const double nx = g->norm[i], ny = g->norm[D + i], nz = g->norm[2 * D + i];
        double fn[3];
        force_centroid(g, f, nb, fn);
        const double rc_n = f->rc[nb], vol_n = g->cvol[nb];
        const double den_f = face_den(g, v, i, f->den, f->gden);
        const double coeff = den_f * 0.5 * (rc_v + rc_n) * face;
        tpush(tb, P + v, P + nb, coeff / dist);
        tpush(tb, P + v, P + v, -coeff / dist);
        const double coeff_v = den_f * 0.5 * rc_v / vol_v * face;
        for (int64_t k = g->gcp[v]; k < g->gcp[v + 1]; ++k)
            tpush(tb, P + v, P + g->gcv[k], -coeff_v * (g->gcc[k] * nx + g->gcc[G + k] * ny + g->gcc[2 * G + k] * nz));
        const double coeff_n = den_f * 0.5 * rc_n / vol_n * face;
        for (int64_t k = g->gcp[nb]; k < g->gcp[nb + 1]; ++k)
            tpush(tb, P + v, P + g->gcv[k], -coeff_n * (g->gcc[k] * nx + g->gcc[G + k] * ny + g->gcc[2 * G + k] * nz));
        double frc[3];
        for (int q = 0; q < 3; ++q)
            frc[q] = 0.5 * (rc_v + rc_n) * 0.5 * (f->fce[q * N + v] + f->fce[q * N + nb]) - 0.5 * (rc_v * fv[q] + rc_n * fn[q]);
        b[P + v] += den_f * (frc[0] * nx + frc[1] * ny + frc[2] * nz) * face;
    }
}

/* Triplets of SteadyFlow::assemble_matrix in push order (r/c/v may be NULL to count). b [4n] is
 * overwritten. node_bnd: boundary id per vertex (-1 for points); bnd_order: the velocity
 * boundaries in registration order; bc_vel [3][n] the boundary velocity at node vertices.
 * pref_vid: the vertex whose pressure row is replaced by p = pref. Returns the triplet count. */
int64_t orc_ns_triplets(const orc_ns_geom* g, const int32_t* node_bnd, int32_t n_bnd, const int32_t* bnd_order, const double* bc_vel,
                        int64_t pref_vid, double pref, const double* vel, const double* gvel, const double* den, const double* gden,
                        const double* visc, const double* gvisc, const double* fce, const double* gfce, const double* rc,
                        const double* flux, uint64_t* r, uint64_t* c, double* val, double* b) {
    const int64_t N = g->n, D = g->n_dir, B = g->n_bsub, P = 3 * N;
    const ns_fields F = {vel, gvel, den, gden, visc, gvisc, fce, gfce, rc, flux};
    trip_buf tb = {r, c, val, 0};
    double bdummy_one = 0.0;
    (void)bdummy_one;
    if (b) memset(b, 0, sizeof(double) * 4 * (size_t)N);
    double* bb = b ? b : (double*)calloc(4 * (size_t)N, sizeof(double));
    /* domain operators, each over the points (nodes are skipped) */
    for (int64_t v = 0; v < g->n_pts; ++v) /* advection */
        for (int64_t i = g->np[v]; i < g->np[v + 1]; ++i) {
            const int64_t nb = g->ni[i];
            const double visc_f = face_visc(g, v, i, visc, gvisc);
            const double cond = visc_f * g->area[i] / g->dist[i];
            const double fl = flux[i];
            const double pe = cond != 0.0 ? fl / cond : 0.0;
            double x = 1.0 - 0.1 * fabs(pe);
            x = x > 0.0 ? x : 0.0;
            const double coeff = cond * (pow5(x) - 1.0) + (-fl > 0.0 ? -fl : 0.0);
            for (int q = 0; q < 3; ++q) {
                tpush(&tb, q * N + v, q * N + nb, coeff);
                tpush(&tb, q * N + v, q * N + v, -coeff);
            }
        }
    for (int64_t v = 0; v < g->n_pts; ++v) /* pressure gradient */
        for (int64_t k = g->gcp[v]; k < g->gcp[v + 1]; ++k) {
            tpush(&tb, v, P + g->gcv[k], -g->gcc[k]);
            tpush(&tb, N + v, P + g->gcv[k], -g->gcc[g->n_gc + k]);
            tpush(&tb, 2 * N + v, P + g->gcv[k], -g->gcc[2 * g->n_gc + k]);
        }
    for (int64_t v = 0; v < g->n_pts; ++v) /* diffusion */
        for (int64_t i = g->np[v]; i < g->np[v + 1]; ++i) {
            const int64_t nb = g->ni[i];
            const double coeff = face_visc(g, v, i, visc, gvisc) * g->area[i] / g->dist[i];
            for (int q = 0; q < 3; ++q) {
                tpush(&tb, q * N + v, q * N + nb, coeff);
                tpush(&tb, q * N + v, q * N + v, -coeff);
            }
        }
    for (int64_t v = 0; v < g->n_pts; ++v) { /* transpose viscous term (explicit) */
        double s[3] = {0.0, 0.0, 0.0};
        for (int64_t i = g->np[v]; i < g->np[v + 1]; ++i) {
            const int64_t nb = g->ni[i];
            const double face = g->area[i];
            const double nx = g->norm[i], ny = g->norm[D + i], nz = g->norm[2 * D + i];
            const double visc_f = face_visc(g, v, i, visc, gvisc);
            double gf[9];
            for (int q = 0; q < 9; ++q) gf[q] = 0.5 * (gvel[q * N + v] + gvel[q * N + nb]);
            /* gf: u_x u_y u_z v_x v_y v_z w_x w_y w_z */
            s[0] += visc_f * (gf[0] * nx + gf[3] * ny + gf[6] * nz) * face;
            s[1] += visc_f * (gf[1] * nx + gf[4] * ny + gf[7] * nz) * face;
            s[2] += visc_f * (gf[2] * nx + gf[5] * ny + gf[8] * nz) * face;
        }
        for (int q = 0; q < 3; ++q) bb[q * N + v] += -s[q];
    }
    for (int64_t v = 0; v < g->n_pts; ++v) { /* dilatational viscous term (explicit) */
        const double div_v = gvel[v] + gvel[4 * N + v] + gvel[8 * N + v];
        double s[3] = {0.0, 0.0, 0.0};
        for (int64_t i = g->np[v]; i < g->np[v + 1]; ++i) {
            const int64_t nb = g->ni[i];
            const double face = g->area[i];
            const double nx = g->norm[i], ny = g->norm[D + i], nz = g->norm[2 * D + i];
            const double visc_f = face_visc(g, v, i, visc, gvisc);
            const double lam_f = (-2.0 / 3.0) * visc_f;
            const double div_n = gvel[nb] + gvel[4 * N + nb] + gvel[8 * N + nb];
            const double div_f = 0.5 * (div_v + div_n);
            const double coeff = lam_f * div_f * face;
            s[0] += coeff * nx;
            s[1] += coeff * ny;
            s[2] += coeff * nz;
        }
        for (int q = 0; q < 3; ++q) bb[q * N + v] += -s[q];
    }
    for (int64_t v = 0; v < g->n_pts; ++v) { /* body force */
        double fc[3];
        force_centroid(g, &F, v, fc);
        for (int q = 0; q < 3; ++q) bb[q * N + v] += -fc[q] * g->cvol[v];
    }
    for (int64_t v = 0; v < g->n_pts; ++v) div_faces(g, &F, v, &tb);
    for (int64_t v = 0; v < g->n_pts; ++v) pstab(g, &F, v, &tb, bb);
    /* velocity boundaries in registration order: Dirichlet, divergence, pressure stabilizer */
    for (int32_t q = 0; q < n_bnd; ++q) {
        const int32_t bid = bnd_order[q];
        for (int64_t v = g->n_pts; v < N; ++v)
            if (node_bnd[v] == bid)
                for (int c2 = 0; c2 < 3; ++c2) {
                    tpush(&tb, c2 * N + v, c2 * N + v, 1.0);
                    bb[c2 * N + v] += bc_vel[c2 * N + v];
                }
        for (int64_t v = g->n_pts; v < N; ++v) {
            if (node_bnd[v] != bid) continue;
            div_faces(g, &F, v, &tb);
            for (int64_t s = g->bp[v]; s < g->bp[v + 1]; ++s) {
                const double area = g->barea[s];
                const double nn[3] = {g->bnorm[s], g->bnorm[B + s], g->bnorm[2 * B + s]};
                const int64_t ms[3] = {v, g->bj[s], g->bk[s]};
                const double cs[3] = {g->bw[s] * den[v] * area, g->bw[B + s] * den[g->bj[s]] * area, g->bw[2 * B + s] * den[g->bk[s]] * area};
                for (int k = 0; k < 3; ++k)
                    for (int c2 = 0; c2 < 3; ++c2) tpush(&tb, P + v, c2 * N + ms[k], -cs[k] * nn[c2]);
            }
        }
        for (int64_t v = g->n_pts; v < N; ++v)
            if (node_bnd[v] == bid) pstab(g, &F, v, &tb, bb);
    }
    /* reference pressure: the row is replaced */
    const int64_t xid = P + pref_vid;
    if (r) {
        int64_t w = 0;
        for (int64_t t = 0; t < tb.t; ++t)
            if ((int64_t)r[t] != xid) {
                r[w] = r[t];
                c[w] = c[t];
                val[w] = val[t];
                ++w;
            }
        tb.t = w;
    }
    tpush(&tb, xid, xid, 1.0);
    bb[xid] = pref;
    if (!b) free(bb);
    return tb.t;
}
