/*
 * CPU oracle for the mesh stage — TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline's
 * input builder; never part of the product path).
 *
 * Restated independently of the product's C++ mesh code (csrc/host/mesh.cpp):
 *   orc_jitter_cube   the seeded jittered-cube point set (SplitMix64, Steele, Lea & Flood 2014),
 *                     coordinates rounded to multiples of 2^-18: the synthetic input contract;
 *   orc_delaunay      Bowyer-Watson insertion as src/base/delaunay.rs:6-170 performs it: a
 *                     super-tetrahedron 50 box sizes out, insertion in 10-bit Morton order (ties by
 *                     vid), a visibility walk whose first face rotates, a cavity of tetrahedra whose
 *                     circumsphere strictly contains the point, grown until star-shaped, new
 *                     tetrahedra appended (never reused) and matched across edges, super tetrahedra
 *                     dropped at the end. Predicates are exact: on the 2^-18 lattice the orientation
 *                     determinant fits 128-bit integers and the in-sphere determinant is summed in
 *                     192-bit integers, so every sign is the exact sign (the robust crate's role);
 *   orc_dual          the Voronoi dual of Tetrahedron::update_tet, src/base/geom_tet.rs:101-293:
 *                     boundary faces (faces of exactly one tetrahedron), face pieces per
 *                     (tetrahedron, edge, side) accumulated per edge in tetrahedron order, edges in
 *                     sorted (min, max) order, control volumes, boundary sub-faces and least-squares
 *                     gradient weights, in the reference's operation order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef __int128 i128;

/* ---------------------------------------------------------------- point set */
static uint64_t smx_next(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static double smx_uniform(uint64_t* s) { return (double)(smx_next(s) >> 11) * 0x1.0p-53; }
static double lattice(double x) { return nearbyint(ldexp(x, 18)) * ldexp(1.0, -18); }

/* n^3 grid on the unit cube, h = 1/(n-1): interior points jittered by (2u-1) jitter h per axis,
 * surface vertices only along the axes they are not fixed on; points first (grid order), then the
 * nodes of boundaries 0..5 (x=0, x=1, y=0, y=1, z=0, z=1; x faces before y before z), each in grid
 * order. pos[3 n^3], node_bnd[n^3] (-1 for points). Returns the number of points. */
int64_t orc_jitter_cube(int n, uint64_t seed, double jitter, double* pos, int32_t* node_bnd) {
    const double h = 1.0 / (double)(n - 1);
    const int64_t N = (int64_t)n * n * n;
    double* tmp = (double*)malloc(sizeof(double) * 3 * N);
    int32_t* bnd = (int32_t*)malloc(sizeof(int32_t) * N);
    uint64_t s = seed;
    int64_t g = 0;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i, ++g) {
                const double u0 = smx_uniform(&s), u1 = smx_uniform(&s), u2 = smx_uniform(&s);
                const int fx = (i == 0 || i == n - 1), fy = (j == 0 || j == n - 1), fz = (k == 0 || k == n - 1);
                double x = (double)i / (double)(n - 1), y = (double)j / (double)(n - 1), z = (double)k / (double)(n - 1);
                if (!fx) x += (2.0 * u0 - 1.0) * jitter * h;
                if (!fy) y += (2.0 * u1 - 1.0) * jitter * h;
                if (!fz) z += (2.0 * u2 - 1.0) * jitter * h;
                tmp[3 * g] = lattice(x);
                tmp[3 * g + 1] = lattice(y);
                tmp[3 * g + 2] = lattice(z);
                bnd[g] = !(fx || fy || fz) ? -1 : fx ? (i == 0 ? 0 : 1) : fy ? (j == 0 ? 2 : 3) : (k == 0 ? 4 : 5);
            }
    int64_t w = 0, npts = 0;
    for (int b = -1; b < 6; ++b)
        for (int64_t v = 0; v < N; ++v)
            if (bnd[v] == b) {
                memcpy(pos + 3 * w, tmp + 3 * v, 3 * sizeof(double));
                node_bnd[w] = b;
                ++w;
                if (b < 0) ++npts;
            }
    free(tmp);
    free(bnd);
    return npts;
}

/* ---------------------------------------------------------------- exact predicates */
typedef struct { int64_t x, y, z; } ip3;

/* det[a-d; b-d; c-d] (> 0: d below the counterclockwise plane a b c), the robust crate's orient3d sign */
static int orient(ip3 a, ip3 b, ip3 c, ip3 d) {
    const i128 ax = a.x - d.x, ay = a.y - d.y, az = a.z - d.z, bx = b.x - d.x, by = b.y - d.y, bz = b.z - d.z;
    const i128 cx = c.x - d.x, cy = c.y - d.y, cz = c.z - d.z;
    const i128 v = ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
    return (v > 0) - (v < 0);
}

/* 192-bit signed accumulator: three 64-bit limbs, two's complement */
typedef struct { uint64_t w[3]; } s192;
static void s192_add_prod(s192* acc, i128 a, int64_t b) {
    /* acc += a * b with |a| < 2^126, |b| < 2^62 */
    int neg = 0;
    unsigned __int128 ua, ub;
    if (a < 0) { ua = (unsigned __int128)(-a); neg ^= 1; } else ua = (unsigned __int128)a;
    if (b < 0) { ub = (unsigned __int128)(-(i128)b); neg ^= 1; } else ub = (unsigned __int128)b;
    const uint64_t a0 = (uint64_t)ua, a1 = (uint64_t)(ua >> 64), b0 = (uint64_t)ub;
    const unsigned __int128 p0 = (unsigned __int128)a0 * b0, p1 = (unsigned __int128)a1 * b0;
    uint64_t r[3];
    r[0] = (uint64_t)p0;
    const unsigned __int128 mid = (p0 >> 64) + (uint64_t)p1;
    r[1] = (uint64_t)mid;
    r[2] = (uint64_t)(mid >> 64) + (uint64_t)(p1 >> 64);
    if (neg) { /* two's complement negate */
        r[0] = ~r[0]; r[1] = ~r[1]; r[2] = ~r[2];
        if (++r[0] == 0 && ++r[1] == 0) ++r[2];
    }
    unsigned __int128 c = (unsigned __int128)acc->w[0] + r[0];
    acc->w[0] = (uint64_t)c;
    c = (c >> 64) + (unsigned __int128)acc->w[1] + r[1];
    acc->w[1] = (uint64_t)c;
    acc->w[2] = (uint64_t)((c >> 64) + acc->w[2] + r[2]);
}
static int s192_sign(const s192* a) {
    if ((int64_t)a->w[2] < 0) return -1;
    return (a->w[0] | a->w[1] | a->w[2]) ? 1 : 0;
}
static i128 det3(i128 ax, i128 ay, i128 az, i128 bx, i128 by, i128 bz, i128 cx, i128 cy, i128 cz) {
    return ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
}

/* > 0 when e lies strictly inside the sphere through a, b, c, d (orient(a, b, c, d) > 0): the
 * lifted 4x4 determinant with rows (p - e, |p - e|^2), expanded along the lifted column */
static int insphere(ip3 a, ip3 b, ip3 c, ip3 d, ip3 e) {
    const int64_t ax = a.x - e.x, ay = a.y - e.y, az = a.z - e.z, bx = b.x - e.x, by = b.y - e.y, bz = b.z - e.z;
    const int64_t cx = c.x - e.x, cy = c.y - e.y, cz = c.z - e.z, dx = d.x - e.x, dy = d.y - e.y, dz = d.z - e.z;
    const int64_t la = ax * ax + ay * ay + az * az, lb = bx * bx + by * by + bz * bz;
    const int64_t lc = cx * cx + cy * cy + cz * cz, ld = dx * dx + dy * dy + dz * dz;
    const i128 m_bcd = det3(bx, by, bz, cx, cy, cz, dx, dy, dz);
    const i128 m_acd = det3(ax, ay, az, cx, cy, cz, dx, dy, dz);
    const i128 m_abd = det3(ax, ay, az, bx, by, bz, dx, dy, dz);
    const i128 m_abc = det3(ax, ay, az, bx, by, bz, cx, cy, cz);
    /* det = -la m_bcd + lb m_acd - lc m_abd + ld m_abc (cofactor signs of the fourth column); with
     * orient(a, b, c, d) > 0 it is positive exactly when e is inside */
    s192 acc = {{0, 0, 0}};
    s192_add_prod(&acc, -m_bcd, la);
    s192_add_prod(&acc, m_acd, lb);
    s192_add_prod(&acc, -m_abd, lc);
    s192_add_prod(&acc, m_abc, ld);
    return s192_sign(&acc);
}

/* ---------------------------------------------------------------- Delaunay (Bowyer-Watson) */
typedef struct { int64_t key; int32_t t, m; } edge_slot;

static uint64_t hash64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    return k;
}

/* Tetrahedra of the convex hull of pos[3 N] into *tets (malloc'ed, 4 per tetrahedron, positively
 * oriented); returns their number, or -1 (duplicate point, no volume, location failure). */
int64_t orc_delaunay(int64_t N, const double* pos, int32_t** tets_out) {
    *tets_out = NULL;
    if (N < 4) return -1;
    ip3* P = (ip3*)malloc(sizeof(ip3) * (N + 4));
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t v = 0; v < N; ++v)
        for (int c = 0; c < 3; ++c) {
            lo[c] = fmin(lo[c], pos[3 * v + c]);
            hi[c] = fmax(hi[c], pos[3 * v + c]);
        }
    for (int64_t v = 0; v < N; ++v) {
        P[v].x = llround(ldexp(pos[3 * v], 18));
        P[v].y = llround(ldexp(pos[3 * v + 1], 18));
        P[v].z = llround(ldexp(pos[3 * v + 2], 18));
    }
    const double cen[3] = {0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1]), 0.5 * (lo[2] + hi[2])};
    double size = fmax(fmax(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]);
    if (!(size > 0.0)) size = 2.2250738585072014e-308;
    const double dirs[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
    for (int s = 0; s < 4; ++s) {
        P[N + s].x = llround(ldexp(cen[0] + 50.0 * size * dirs[s][0], 18));
        P[N + s].y = llround(ldexp(cen[1] + 50.0 * size * dirs[s][1], 18));
        P[N + s].z = llround(ldexp(cen[2] + 50.0 * size * dirs[s][2], 18));
    }
    int64_t cap = 8 * N + 64, nt = 1;
    int32_t (*tv)[4] = malloc(sizeof(int32_t[4]) * cap);
    int32_t (*ta)[4] = malloc(sizeof(int32_t[4]) * cap);
    uint8_t* dead = (uint8_t*)calloc(cap, 1);
    uint8_t* incav = (uint8_t*)calloc(cap, 1);
    tv[0][0] = (int32_t)N; tv[0][1] = (int32_t)N + 1; tv[0][2] = (int32_t)N + 2; tv[0][3] = (int32_t)N + 3;
    if (orient(P[N], P[N + 1], P[N + 2], P[N + 3]) < 0) { tv[0][0] = (int32_t)N + 1; tv[0][1] = (int32_t)N; }
    for (int k = 0; k < 4; ++k) ta[0][k] = -1;

    /* insertion order: 10-bit Morton code of the box-relative position, ties by vid */
    uint64_t* ord = (uint64_t*)malloc(sizeof(uint64_t) * N * 2);
    for (int64_t v = 0; v < N; ++v) {
        uint64_t q[3], code = 0;
        for (int c = 0; c < 3; ++c) {
            double t = (pos[3 * v + c] - lo[c]) / size * 1023.0;
            t = t < 0.0 ? 0.0 : (t > 1023.0 ? 1023.0 : t);
            q[c] = (uint64_t)t;
        }
        for (int b = 0; b < 10; ++b) code |= ((q[0] >> b) & 1) << (3 * b) | ((q[1] >> b) & 1) << (3 * b + 1) | ((q[2] >> b) & 1) << (3 * b + 2);
        ord[2 * v] = code;
        ord[2 * v + 1] = (uint64_t)v;
    }
    /* sort (code, vid) pairs: LSD radix over vid (already ascending) then a stable counting sort on code (30 bits) */
    {
        uint64_t* tmp = (uint64_t*)malloc(sizeof(uint64_t) * N * 2);
        for (int pass = 0; pass < 3; ++pass) {
            const int shift = 10 * pass;
            int64_t cnt[1025] = {0};
            for (int64_t v = 0; v < N; ++v) cnt[((ord[2 * v] >> shift) & 1023) + 1]++;
            for (int b = 0; b < 1024; ++b) cnt[b + 1] += cnt[b];
            for (int64_t v = 0; v < N; ++v) {
                const int64_t d = cnt[(ord[2 * v] >> shift) & 1023]++;
                tmp[2 * d] = ord[2 * v];
                tmp[2 * d + 1] = ord[2 * v + 1];
            }
            uint64_t* sw = ord; ord = tmp; tmp = sw;
        }
        free(tmp);
    }

    int64_t ecap = 1024;
    edge_slot* etab = (edge_slot*)malloc(sizeof(edge_slot) * ecap);
    int64_t* used = (int64_t*)malloc(sizeof(int64_t) * ecap);
    int64_t nused = 0;
    for (int64_t i = 0; i < ecap; ++i) etab[i].key = -1;
    int64_t cav_cap = 1024, ncav = 0;
    int32_t* cav = (int32_t*)malloc(sizeof(int32_t) * cav_cap);
    int64_t last = 0;
    unsigned turn = 0;
    int64_t result = 0;
    for (int64_t oi = 0; oi < N && result == 0; ++oi) {
        const int32_t vid = (int32_t)ord[2 * oi + 1];
        const ip3 p = P[vid];
        /* locate */
        int64_t t = last, steps = 0;
        for (;;) {
            if (++steps > 4 * nt) {
                t = -1;
                for (int64_t s = 0; s < nt && t < 0; ++s) {
                    if (dead[s]) continue;
                    int in = 1;
                    for (int k = 0; k < 4 && in; ++k) {
                        ip3 q[4] = {P[tv[s][0]], P[tv[s][1]], P[tv[s][2]], P[tv[s][3]]};
                        q[k] = p;
                        in = orient(q[0], q[1], q[2], q[3]) >= 0;
                    }
                    if (in) t = s;
                }
                break;
            }
            turn = (turn + 1) % 4;
            int moved = 0;
            for (int l = 0; l < 4; ++l) {
                const int k = (int)((l + turn) % 4);
                ip3 q[4] = {P[tv[t][0]], P[tv[t][1]], P[tv[t][2]], P[tv[t][3]]};
                q[k] = p;
                if (orient(q[0], q[1], q[2], q[3]) < 0) {
                    if (ta[t][k] < 0) { t = -1; break; }
                    t = ta[t][k];
                    moved = 1;
                    break;
                }
            }
            if (t < 0 || !moved) break;
        }
        if (t < 0) { result = -1; break; }
        for (int k = 0; k < 4; ++k) {
            const ip3 w = P[tv[t][k]];
            if (w.x == p.x && w.y == p.y && w.z == p.z) result = -1;
        }
        if (result) break;
        /* cavity */
        ncav = 0;
        cav[ncav++] = (int32_t)t;
        incav[t] = 1;
        for (int64_t i = 0; i < ncav; ++i) {
            const int32_t c = cav[i];
            for (int k = 0; k < 4; ++k) {
                const int32_t o = ta[c][k];
                if (o < 0 || incav[o]) continue;
                if (insphere(P[tv[o][0]], P[tv[o][1]], P[tv[o][2]], P[tv[o][3]], p) > 0) {
                    if (ncav == cav_cap) { cav_cap *= 2; cav = (int32_t*)realloc(cav, sizeof(int32_t) * cav_cap); }
                    incav[o] = 1;
                    cav[ncav++] = o;
                }
            }
        }
        /* grow until star-shaped */
        for (;;) {
            int star = 1;
            const int64_t n0 = ncav;  /* a pass visits the cavity as it was when the pass began */
            for (int64_t i = 0; i < n0 && result == 0; ++i) {
                const int32_t c = cav[i];
                for (int k = 0; k < 4; ++k) {
                    const int32_t o = ta[c][k];
                    if (o >= 0 && incav[o]) continue;
                    ip3 q[4] = {P[tv[c][0]], P[tv[c][1]], P[tv[c][2]], P[tv[c][3]]};
                    q[k] = p;
                    if (orient(q[0], q[1], q[2], q[3]) > 0) continue;
                    if (o < 0) { result = -1; break; }
                    if (ncav == cav_cap) { cav_cap *= 2; cav = (int32_t*)realloc(cav, sizeof(int32_t) * cav_cap); }
                    incav[o] = 1;
                    cav[ncav++] = o;
                    star = 0;
                }
            }
            if (result || star) break;
        }
        if (result) break;
        /* new tetrahedra: the face opposite p keeps the outside neighbour; faces through p are
         * matched by the edge they share with the cavity's boundary face */
        int64_t nb = 0;
        for (int64_t i = 0; i < ncav; ++i)
            for (int k = 0; k < 4; ++k) {
                const int32_t o = ta[cav[i]][k];
                if (!(o >= 0 && incav[o])) ++nb;
            }
        if (nt + nb > cap) {
            const int64_t nc = 2 * (nt + nb);
            tv = realloc(tv, sizeof(int32_t[4]) * nc);
            ta = realloc(ta, sizeof(int32_t[4]) * nc);
            dead = (uint8_t*)realloc(dead, nc);
            incav = (uint8_t*)realloc(incav, nc);
            memset(dead + cap, 0, nc - cap);
            memset(incav + cap, 0, nc - cap);
            cap = nc;
        }
        if (4 * nb > ecap) {
            for (int64_t u = 0; u < nused; ++u) etab[used[u]].key = -1;
            nused = 0;
            while (4 * nb > ecap) ecap *= 2;
            etab = (edge_slot*)realloc(etab, sizeof(edge_slot) * ecap);
            used = (int64_t*)realloc(used, sizeof(int64_t) * ecap);
            for (int64_t u = 0; u < ecap; ++u) etab[u].key = -1;
        }
        for (int64_t i = 0; i < ncav; ++i) {
            const int32_t c = cav[i];
            for (int k = 0; k < 4; ++k) {
                const int32_t o = ta[c][k];
                if (o >= 0 && incav[o]) continue;
                const int64_t tn = nt++;
                for (int l = 0; l < 4; ++l) {
                    tv[tn][l] = tv[c][l];
                    ta[tn][l] = -1;
                }
                tv[tn][k] = vid;
                dead[tn] = 0;
                incav[tn] = 0;
                ta[tn][k] = o;
                if (o >= 0)
                    for (int m = 0; m < 4; ++m)
                        if (ta[o][m] == c) { ta[o][m] = (int32_t)tn; break; }
                for (int m = 0; m < 4; ++m) {
                    if (m == k) continue;
                    int32_t e[2], ne = 0;
                    for (int l = 0; l < 4; ++l)
                        if (l != k && l != m) e[ne++] = tv[tn][l];
                    const int64_t a = e[0] < e[1] ? e[0] : e[1], b = e[0] < e[1] ? e[1] : e[0];
                    const int64_t key = a * (N + 4) + b;
                    uint64_t h = hash64((uint64_t)key) & (uint64_t)(ecap - 1);
                    while (etab[h].key != -1 && etab[h].key != key) h = (h + 1) & (uint64_t)(ecap - 1);
                    if (etab[h].key == key && etab[h].t >= 0) {
                        ta[tn][m] = etab[h].t;
                        ta[etab[h].t][etab[h].m] = (int32_t)tn;
                        etab[h].t = -1;
                    } else {
                        if (etab[h].key == -1) used[nused++] = (int64_t)h;
                        etab[h].key = key;
                        etab[h].t = (int32_t)tn;
                        etab[h].m = m;
                    }
                }
                last = tn;
            }
        }
        for (int64_t u = 0; u < nused; ++u) etab[used[u]].key = -1;
        nused = 0;
        for (int64_t i = 0; i < ncav; ++i) {
            dead[cav[i]] = 1;
            incav[cav[i]] = 0;
        }
    }
    if (result == 0) {
        int64_t keep = 0;
        for (int64_t t = 0; t < nt; ++t)
            if (!dead[t] && tv[t][0] < N && tv[t][1] < N && tv[t][2] < N && tv[t][3] < N) ++keep;
        int32_t* out = (int32_t*)malloc(sizeof(int32_t) * 4 * (keep > 0 ? keep : 1));
        int64_t w = 0;
        for (int64_t t = 0; t < nt; ++t)
            if (!dead[t] && tv[t][0] < N && tv[t][1] < N && tv[t][2] < N && tv[t][3] < N) {
                memcpy(out + 4 * w, tv[t], 4 * sizeof(int32_t));
                ++w;
            }
        *tets_out = out;
        result = keep > 0 ? keep : -1;
    }
    free(P); free(tv); free(ta); free(dead); free(incav); free(ord); free(etab); free(used); free(cav);
    return result;
}

void orc_free(void* p) { free(p); }

/* ---------------------------------------------------------------- Voronoi dual */
typedef struct { double x, y, z; } v3;
static v3 V(const double* p) { v3 r = {p[0], p[1], p[2]}; return r; }
static v3 add3(v3 a, v3 b) { v3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static v3 sub3(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static v3 scale3(double s, v3 a) { v3 r = {s * a.x, s * a.y, s * a.z}; return r; }
static double dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 cross3(v3 a, v3 b) { v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; return r; }
static double len3(v3 a) { return sqrt(dot3(a, a)); }
/* delaunay.rs:207-214 (centre only) */
static v3 circumcircle3(v3 a, v3 b, v3 c) {
    const v3 u = sub3(b, a), v = sub3(c, a);
    const v3 w = cross3(u, v);
    const v3 num = add3(scale3(dot3(u, u), cross3(v, w)), scale3(dot3(v, v), cross3(w, u)));
    return add3(a, scale3(0.5 / dot3(w, w), num));
}
/* delaunay.rs:216-221 */
static v3 circumsphere3(v3 a, v3 b, v3 c, v3 d) {
    const v3 u = sub3(b, a), v = sub3(c, a), w = sub3(d, a);
    const v3 num = add3(add3(scale3(dot3(u, u), cross3(v, w)), scale3(dot3(v, v), cross3(w, u))), scale3(dot3(w, w), cross3(u, v)));
    return add3(a, scale3(0.5 / dot3(u, cross3(v, w)), num));
}

/* LSD radix sort of 64-bit keys with 32-bit payloads (stable), `bits` significant bits */
static void radix_kv(int64_t n, uint64_t* key, int64_t* val, int bits) {
    uint64_t* k2 = (uint64_t*)malloc(sizeof(uint64_t) * n);
    int64_t* v2 = (int64_t*)malloc(sizeof(int64_t) * n);
    int64_t* cnt = (int64_t*)malloc(sizeof(int64_t) * 65537);
    for (int sh = 0; sh < bits; sh += 16) {
        memset(cnt, 0, sizeof(int64_t) * 65537);
        for (int64_t i = 0; i < n; ++i) cnt[((key[i] >> sh) & 0xFFFF) + 1]++;
        for (int b = 0; b < 65536; ++b) cnt[b + 1] += cnt[b];
        for (int64_t i = 0; i < n; ++i) {
            const int64_t d = cnt[(key[i] >> sh) & 0xFFFF]++;
            k2[d] = key[i];
            v2[d] = val[i];
        }
        memcpy(key, k2, sizeof(uint64_t) * n);
        memcpy(val, v2, sizeof(int64_t) * n);
    }
    free(k2);
    free(v2);
    free(cnt);
}

typedef struct {
    int64_t n, n_dir, n_bsub;
    int64_t* nbr_ptr;   /* [n+1] */
    int32_t* nbr_idx;   /* [n_dir] neighbours ascending */
    double* dist;       /* [n_dir] */
    double* area;       /* [n_dir] signed */
    double* norm;       /* [3][n_dir] outward */
    double* skew;       /* [3][n_dir] */
    double* grad_wgt;   /* [3][n_dir] */
    double* cvol;       /* [n] */
    double* cskew;      /* [3][n] */
    int64_t* bnd_ptr;   /* [n+1] */
    int32_t* bnd_j;     /* [n_bsub] */
    int32_t* bnd_k;
    double* bnd_area;
    double* bnd_norm;   /* [3][n_bsub] */
    double* bnd_wgt;    /* [3][n_bsub] */
} orc_dual_out;

/* The dual of a tetrahedralisation (all tetrahedra kept: the domain is their convex hull).
 * Returns 0, 1 (a boundary face joins an interior point), 2 (singular gradient), 3 (too many vertices). */
int orc_dual(int64_t N, int64_t n_pts, const double* pos, int64_t T, const int32_t* tet, orc_dual_out* out) {
    if (N <= 0 || N >= ((int64_t)1 << 21) || T <= 0) return 3;
    memset(out, 0, sizeof(*out));
    out->n = N;
    /* step 1: boundary faces, faces of exactly one tetrahedron (geom_tet.rs:101-116) */
    static const int FO[4][3] = {{1, 3, 2}, {0, 2, 3}, {0, 3, 1}, {0, 1, 2}};
    uint64_t* fk = (uint64_t*)malloc(sizeof(uint64_t) * 4 * T);
    int64_t* fi = (int64_t*)malloc(sizeof(int64_t) * 4 * T);
    for (int64_t t = 0; t < T; ++t)
        for (int k = 0; k < 4; ++k) {
            int64_t a = tet[4 * t + (k + 1) % 4], b = tet[4 * t + (k + 2) % 4], c = tet[4 * t + (k + 3) % 4], s;
            if (a > b) { s = a; a = b; b = s; }
            if (b > c) { s = b; b = c; c = s; }
            if (a > b) { s = a; a = b; b = s; }
            fk[4 * t + k] = ((uint64_t)a << 42) | ((uint64_t)b << 21) | (uint64_t)c;
            fi[4 * t + k] = 4 * t + k;
        }
    radix_kv(4 * T, fk, fi, 64);
    uint8_t* isb = (uint8_t*)calloc(4 * T, 1);
    for (int64_t i = 0; i < 4 * T;) {
        int64_t j = i + 1;
        while (j < 4 * T && fk[j] == fk[i]) ++j;
        if (j - i == 1) isb[fi[i]] = 1;
        i = j;
    }
    free(fk);
    free(fi);
    int64_t ns = 0;
    for (int64_t i = 0; i < 4 * T; ++i) ns += isb[i];
    int32_t* surf = (int32_t*)malloc(sizeof(int32_t) * 3 * (ns + 1));
    int64_t w = 0;
    int bad = 0;
    for (int64_t t = 0; t < T; ++t)
        for (int k = 0; k < 4; ++k)
            if (isb[4 * t + k]) {
                for (int q = 0; q < 3; ++q) {
                    surf[3 * w + q] = tet[4 * t + FO[k][q]];
                    if (surf[3 * w + q] < n_pts) bad = 1;
                }
                ++w;
            }
    free(isb);
    if (bad) { free(surf); return 1; }

    /* edges in sorted (min, max) order; upper neighbours per vertex as CSR for the lookup */
    uint64_t* ek = (uint64_t*)malloc(sizeof(uint64_t) * 6 * T);
    int64_t* ev = (int64_t*)malloc(sizeof(int64_t) * 6 * T);
    static const int EP[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    for (int64_t t = 0; t < T; ++t)
        for (int e = 0; e < 6; ++e) {
            int64_t a = tet[4 * t + EP[e][0]], b = tet[4 * t + EP[e][1]];
            if (a > b) { int64_t s = a; a = b; b = s; }
            ek[6 * t + e] = ((uint64_t)a << 21) | (uint64_t)b;
            ev[6 * t + e] = 0;
        }
    radix_kv(6 * T, ek, ev, 48);
    free(ev);
    int64_t E = 0;
    for (int64_t i = 0; i < 6 * T; ++i)
        if (i == 0 || ek[i] != ek[i - 1]) ek[E++] = ek[i];
    int64_t* up = (int64_t*)calloc(N + 1, sizeof(int64_t));
    int32_t* upn = (int32_t*)malloc(sizeof(int32_t) * E);
    for (int64_t e = 0; e < E; ++e) {
        up[(ek[e] >> 21) + 1]++;
        upn[e] = (int32_t)(ek[e] & 0x1FFFFF);
    }
    for (int64_t v = 0; v < N; ++v) up[v + 1] += up[v];
    free(ek);

    /* step 2: face pieces per (tetrahedron, edge, side), accumulated in that order (geom_tet.rs:122-171) */
    double* e_area = (double*)calloc(E, sizeof(double));
    v3* e_skew = (v3*)calloc(E, sizeof(v3));
    v3* cent_sum = (v3*)calloc(N, sizeof(v3));
    for (int64_t t = 0; t < T; ++t) {
        const int32_t* tv = tet + 4 * t;
        const v3 c_t = circumsphere3(V(pos + 3 * tv[0]), V(pos + 3 * tv[1]), V(pos + 3 * tv[2]), V(pos + 3 * tv[3]));
        for (int ed = 0; ed < 6; ++ed) {
            const int li = EP[ed][0], lj = EP[ed][1];
            int oth[2], no = 0;
            for (int l = 0; l < 4; ++l)
                if (l != li && l != lj) oth[no++] = l;
            const int32_t vi = tv[li], vj = tv[lj];
            const v3 pi = V(pos + 3 * vi), pj = V(pos + 3 * vj);
            const double dist = len3(sub3(pj, pi));
            const v3 e = scale3(1.0 / dist, sub3(pj, pi));
            const v3 m = scale3(0.5, add3(pi, pj));
            const int32_t lo = vi < vj ? vi : vj, hi = vi < vj ? vj : vi;
            int64_t id = up[lo];
            while (upn[id] != hi) ++id;
            for (int side = 0; side < 2; ++side) {
                const v3 pa = V(pos + 3 * tv[oth[side]]), pb = V(pos + 3 * tv[oth[1 - side]]);
                const v3 c_f = circumcircle3(pi, pj, pa);
                v3 u = sub3(sub3(pa, m), scale3(dot3(sub3(pa, m), e), e));
                u = scale3(1.0 / len3(u), u);
                v3 nn = cross3(e, u);
                if (dot3(sub3(pb, m), nn) < 0.0) nn = scale3(-1.0, nn);
                const double s1 = dot3(sub3(c_f, m), u);
                const double s2 = dot3(sub3(c_t, c_f), nn);
                const double area = 0.5 * s1 * s2;
                const v3 cent = scale3(1.0 / 3.0, add3(m, add3(c_f, c_t)));
                e_area[id] += area;
                e_skew[id] = add3(e_skew[id], scale3(area, sub3(cent, m)));
                const double vol = area * dist / 6.0;
                cent_sum[vi] = add3(cent_sum[vi], scale3(vol * 0.75, sub3(cent, pi)));
                cent_sum[vj] = add3(cent_sum[vj], scale3(vol * 0.75, sub3(cent, pj)));
            }
        }
    }

    /* step 3: neighbour, face and control-volume data, edges in sorted order (geom_tet.rs:173-206) */
    const int64_t D = 2 * E;
    out->n_dir = D;
    out->nbr_ptr = (int64_t*)calloc(N + 1, sizeof(int64_t));
    for (int64_t a = 0; a < N; ++a)
        for (int64_t id = up[a]; id < up[a + 1]; ++id) {
            out->nbr_ptr[a + 1]++;
            out->nbr_ptr[upn[id] + 1]++;
        }
    for (int64_t v = 0; v < N; ++v) out->nbr_ptr[v + 1] += out->nbr_ptr[v];
    out->nbr_idx = (int32_t*)malloc(sizeof(int32_t) * D);
    out->dist = (double*)malloc(sizeof(double) * D);
    out->area = (double*)malloc(sizeof(double) * D);
    out->norm = (double*)malloc(sizeof(double) * 3 * D);
    out->skew = (double*)malloc(sizeof(double) * 3 * D);
    out->grad_wgt = (double*)malloc(sizeof(double) * 3 * D);
    out->cvol = (double*)calloc(N, sizeof(double));
    out->cskew = (double*)malloc(sizeof(double) * 3 * N);
    int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * N);
    memcpy(cur, out->nbr_ptr, sizeof(int64_t) * N);
    for (int64_t a = 0; a < N; ++a)
        for (int64_t id = up[a]; id < up[a + 1]; ++id) {
            const int64_t b = upn[id];
            const v3 pa = V(pos + 3 * a), pb = V(pos + 3 * b);
            const double dist = len3(sub3(pb, pa));
            const v3 nrm = scale3(1.0 / dist, sub3(pb, pa));
            const double area = e_area[id];
            const v3 sk = fabs(area) > 1e-12 * dist * dist ? scale3(1.0 / area, e_skew[id]) : (v3){0.0, 0.0, 0.0};
            const v3 nrm_b = scale3(-1.0, nrm);
            const int64_t qa = cur[a]++, qb = cur[b]++;
            out->nbr_idx[qa] = (int32_t)b;
            out->nbr_idx[qb] = (int32_t)a;
            out->dist[qa] = out->dist[qb] = dist;
            out->area[qa] = out->area[qb] = area;
            out->norm[qa] = nrm.x; out->norm[D + qa] = nrm.y; out->norm[2 * D + qa] = nrm.z;
            out->norm[qb] = nrm_b.x; out->norm[D + qb] = nrm_b.y; out->norm[2 * D + qb] = nrm_b.z;
            out->skew[qa] = out->skew[qb] = sk.x;
            out->skew[D + qa] = out->skew[D + qb] = sk.y;
            out->skew[2 * D + qa] = out->skew[2 * D + qb] = sk.z;
            out->cvol[a] += area * dist / 6.0;
            out->cvol[b] += area * dist / 6.0;
        }
    free(cur);
    free(up);
    free(upn);
    free(e_area);
    free(e_skew);
    for (int64_t v = 0; v < N; ++v) {
        const v3 s = scale3(1.0 / out->cvol[v], cent_sum[v]);
        out->cskew[v] = s.x;
        out->cskew[N + v] = s.y;
        out->cskew[2 * N + v] = s.z;
    }
    free(cent_sum);

    /* step 4: boundary sub-faces, surface triangles in order (geom_tet.rs:208-259) */
    const int64_t B = 3 * ns;
    out->n_bsub = B;
    out->bnd_ptr = (int64_t*)calloc(N + 1, sizeof(int64_t));
    for (int64_t s = 0; s < ns; ++s)
        for (int q = 0; q < 3; ++q) out->bnd_ptr[surf[3 * s + q] + 1]++;
    for (int64_t v = 0; v < N; ++v) out->bnd_ptr[v + 1] += out->bnd_ptr[v];
    out->bnd_j = (int32_t*)malloc(sizeof(int32_t) * (B + 1));
    out->bnd_k = (int32_t*)malloc(sizeof(int32_t) * (B + 1));
    out->bnd_area = (double*)malloc(sizeof(double) * (B + 1));
    out->bnd_norm = (double*)malloc(sizeof(double) * 3 * (B + 1));
    out->bnd_wgt = (double*)malloc(sizeof(double) * 3 * (B + 1));
    cur = (int64_t*)malloc(sizeof(int64_t) * N);
    memcpy(cur, out->bnd_ptr, sizeof(int64_t) * N);
    for (int64_t s = 0; s < ns; ++s) {
        const int32_t* tr = surf + 3 * s;
        const v3 p0 = V(pos + 3 * tr[0]), p1 = V(pos + 3 * tr[1]), p2 = V(pos + 3 * tr[2]);
        v3 nrm = cross3(sub3(p1, p0), sub3(p2, p0));
        nrm = scale3(1.0 / len3(nrm), nrm);
        const v3 c = circumcircle3(p0, p1, p2);
        const double sq[3] = {dot3(sub3(p2, p1), sub3(p2, p1)), dot3(sub3(p0, p2), sub3(p0, p2)), dot3(sub3(p1, p0), sub3(p1, p0))};
        const double lr[3] = {sq[0] * (sq[1] + sq[2] - sq[0]), sq[1] * (sq[2] + sq[0] - sq[1]), sq[2] * (sq[0] + sq[1] - sq[2])};
        const double lsum = lr[0] + lr[1] + lr[2];
        const double lam[3] = {lr[0] / lsum, lr[1] / lsum, lr[2] / lsum};
        for (int loc = 0; loc < 3; ++loc) {
            const int32_t vi = tr[loc], vj = tr[(loc + 1) % 3], vk = tr[(loc + 2) % 3];
            const v3 pi = V(pos + 3 * vi), pj = V(pos + 3 * vj), pk = V(pos + 3 * vk);
            double area[2];
            for (int side = 0; side < 2; ++side) {
                const v3 pa = side == 0 ? pj : pk, pb = side == 0 ? pk : pj;
                const v3 m = scale3(0.5, add3(pi, pa));
                const v3 e = sub3(pa, pi);
                const double len = len3(e);
                const v3 u = sub3(sub3(pb, m), scale3(dot3(sub3(pb, m), e) / (len * len), e));
                area[side] = 0.25 * len * dot3(sub3(c, m), scale3(1.0 / len3(u), u));
            }
            const double area_sum = area[0] + area[1];
            const double l0 = lam[loc], l1 = lam[(loc + 1) % 3], l2 = lam[(loc + 2) % 3];
            const v3 cj = {(1.5 + l0) / 3.0, (0.5 + l1) / 3.0, l2 / 3.0};
            const v3 ck = {(1.5 + l0) / 3.0, l1 / 3.0, (0.5 + l2) / 3.0};
            const v3 wg = fabs(area_sum) > 1e-12 * len3(sub3(pj, pi)) * len3(sub3(pk, pi))
                              ? scale3(1.0 / area_sum, add3(scale3(area[0], cj), scale3(area[1], ck)))
                              : (v3){1.0, 0.0, 0.0};
            const int64_t q = cur[vi]++;
            out->bnd_j[q] = vj;
            out->bnd_k[q] = vk;
            out->bnd_area[q] = area_sum;
            out->bnd_norm[q] = nrm.x; out->bnd_norm[B + q] = nrm.y; out->bnd_norm[2 * B + q] = nrm.z;
            out->bnd_wgt[q] = wg.x; out->bnd_wgt[B + q] = wg.y; out->bnd_wgt[2 * B + q] = wg.z;
        }
    }
    free(cur);
    free(surf);

    /* step 5: least-squares gradient weights (geom_tet.rs:261-293) */
    int sing = 0;
    for (int64_t vc = 0; vc < N && !sing; ++vc) {
        const v3 pc = V(pos + 3 * vc);
        double mm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int64_t q = out->nbr_ptr[vc]; q < out->nbr_ptr[vc + 1]; ++q) {
            const v3 dv = sub3(V(pos + 3 * out->nbr_idx[q]), pc);
            const double d[3] = {dv.x, dv.y, dv.z};
            const double omega = 1.0 / (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            for (int r = 0; r < 3; ++r)
                for (int s = 0; s < 3; ++s) mm[r][s] += omega * d[r] * d[s];
        }
        const double ad[3][3] = {
            {mm[1][1] * mm[2][2] - mm[1][2] * mm[2][1], mm[0][2] * mm[2][1] - mm[0][1] * mm[2][2], mm[0][1] * mm[1][2] - mm[0][2] * mm[1][1]},
            {mm[1][2] * mm[2][0] - mm[1][0] * mm[2][2], mm[0][0] * mm[2][2] - mm[0][2] * mm[2][0], mm[0][2] * mm[1][0] - mm[0][0] * mm[1][2]},
            {mm[1][0] * mm[2][1] - mm[1][1] * mm[2][0], mm[0][1] * mm[2][0] - mm[0][0] * mm[2][1], mm[0][0] * mm[1][1] - mm[0][1] * mm[1][0]},
        };
        const double det = mm[0][0] * ad[0][0] + mm[0][1] * ad[1][0] + mm[0][2] * ad[2][0];
        const double tr = mm[0][0] + mm[1][1] + mm[2][2];
        if (!(det > 1e-12 * (tr * tr * tr))) {
            sing = 1;
            break;
        }
        for (int64_t q = out->nbr_ptr[vc]; q < out->nbr_ptr[vc + 1]; ++q) {
            const v3 d = sub3(V(pos + 3 * out->nbr_idx[q]), pc);
            const double omega = 1.0 / dot3(d, d);
            for (int r = 0; r < 3; ++r) out->grad_wgt[(int64_t)r * D + q] = omega * (ad[r][0] * d.x + ad[r][1] * d.y + ad[r][2] * d.z) / det;
        }
    }
    return sing ? 2 : 0;
}

void orc_dual_free(orc_dual_out* d) {
    free(d->nbr_ptr); free(d->nbr_idx); free(d->dist); free(d->area); free(d->norm); free(d->skew); free(d->grad_wgt);
    free(d->cvol); free(d->cskew); free(d->bnd_ptr); free(d->bnd_j); free(d->bnd_k); free(d->bnd_area); free(d->bnd_norm);
    free(d->bnd_wgt);
    memset(d, 0, sizeof(*d));
}
