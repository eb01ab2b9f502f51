// Symbolic setup of the coupled Navier-Stokes system; see ns_setup.hpp.
#include "ns_setup.hpp"

#include <algorithm>
#include <climits>

namespace vfv {

namespace {

struct GcEnt {
    int32_t vid;
    double c[3];
};

// Tetrahedron::update_tet step 6 (geom_tet.rs:295-347) for one vertex, in push order:
// per face the arithmetic-mean pair (v, n), then the skew terms of the LSQ gradients of v and of n
// ((m, +w) and (s, -w) per neighbour m of s), then the boundary sub-faces (v, j, k).
void gc_push_order(const Dual& d, int64_t v, std::vector<GcEnt>& e) {
    const int64_t D = d.n_dir, B = (int64_t)d.bnd_j.size();
    e.clear();
    for (int64_t i = d.nbr_ptr[v]; i < d.nbr_ptr[v + 1]; ++i) {
        const int32_t nb = d.nbr_idx[i];
        const double area = d.area[i];
        const double nx = d.norm[i], ny = d.norm[D + i], nz = d.norm[2 * D + i];
        const double sx = d.skew[i], sy = d.skew[D + i], sz = d.skew[2 * D + i];
        e.push_back({(int32_t)v, {0.5 * area * nx, 0.5 * area * ny, 0.5 * area * nz}});
        e.push_back({nb, {0.5 * area * nx, 0.5 * area * ny, 0.5 * area * nz}});
        const int64_t side[2] = {v, nb};
        for (int64_t s : side)
            for (int64_t k = d.nbr_ptr[s]; k < d.nbr_ptr[s + 1]; ++k) {
                const double w = 0.5 * (d.gw[k] * sx + d.gw[D + k] * sy + d.gw[2 * D + k] * sz) * area;
                e.push_back({d.nbr_idx[k], {w * nx, w * ny, w * nz}});
                e.push_back({(int32_t)s, {-w * nx, -w * ny, -w * nz}});
            }
    }
    for (int64_t b = d.bnd_ptr[v]; b < d.bnd_ptr[v + 1]; ++b) {
        const double area = d.bnd_area[b];
        const double nx = d.bnd_norm[b], ny = d.bnd_norm[B + b], nz = d.bnd_norm[2 * B + b];
        const double wv = d.bnd_wgt[b], wj = d.bnd_wgt[B + b], wk = d.bnd_wgt[2 * B + b];
        e.push_back({(int32_t)v, {wv * area * nx, wv * area * ny, wv * area * nz}});
        e.push_back({d.bnd_j[b], {wj * area * nx, wj * area * ny, wj * area * nz}});
        e.push_back({d.bnd_k[b], {wk * area * nx, wk * area * ny, wk * area * nz}});
    }
}

// The merge of slice::sort_by_key + dedup_by: a stable sort by vertex, then the entries of equal
// vertices summed in push order. Computed without sorting the entries: the first entry of a vertex
// keeps its place in `out` and the later ones are added to it in push order (the same sums), then
// the distinct vertices are sorted. stamp[u] == v marks vertex u as seen while merging vertex v's
// list; slot[u] is its place in `out`.
void gc_merge(const std::vector<GcEnt>& e, int32_t v, std::vector<int32_t>& stamp, std::vector<int32_t>& slot, std::vector<GcEnt>& out) {
    out.clear();
    for (const GcEnt& g : e) {
        if (stamp[g.vid] != v) {
            stamp[g.vid] = v;
            slot[g.vid] = (int32_t)out.size();
            out.push_back(g);
        } else {
            GcEnt& o = out[slot[g.vid]];
            for (int q = 0; q < 3; ++q) o.c[q] += g.c[q];
        }
    }
    std::sort(out.begin(), out.end(), [](const GcEnt& a, const GcEnt& b) { return a.vid < b.vid; });
}

int64_t deg(const Dual& d, int64_t v) { return d.nbr_ptr[v + 1] - d.nbr_ptr[v]; }

// Column sequence of row r in push order (appended to out).
void row_columns(const Dual& d, const NsLayout& L, int64_t r, std::vector<int32_t>& out) {
    const int64_t N = L.n, P = 3 * N;
    out.clear();
    if (r < P) {
        const int64_t q = r / N, v = r % N;
        if (v >= L.n_pts) {
            out.push_back((int32_t)r);
            return;
        }
        for (int64_t i = d.nbr_ptr[v]; i < d.nbr_ptr[v + 1]; ++i) {  // advection
            out.push_back((int32_t)(q * N + d.nbr_idx[i]));
            out.push_back((int32_t)r);
        }
        for (int32_t k = L.gcp[v]; k < L.gcp[v + 1]; ++k) out.push_back((int32_t)(P + L.gcv[k]));  // pressure gradient
        for (int64_t i = d.nbr_ptr[v]; i < d.nbr_ptr[v + 1]; ++i) {  // diffusion
            out.push_back((int32_t)(q * N + d.nbr_idx[i]));
            out.push_back((int32_t)r);
        }
        return;
    }
    const int64_t v = r - P;
    if (v == L.pref_vid) {
        out.push_back((int32_t)r);
        return;
    }
    for (int64_t i = d.nbr_ptr[v]; i < d.nbr_ptr[v + 1]; ++i) {  // divergence
        const int64_t nb = d.nbr_idx[i];
        for (int c = 0; c < 3; ++c) {
            out.push_back((int32_t)(c * N + nb));
            out.push_back((int32_t)(c * N + v));
        }
        for (int64_t k = d.nbr_ptr[v]; k < d.nbr_ptr[v + 1]; ++k)
            for (int c = 0; c < 3; ++c) {
                out.push_back((int32_t)(c * N + d.nbr_idx[k]));
                out.push_back((int32_t)(c * N + v));
            }
        for (int64_t k = d.nbr_ptr[nb]; k < d.nbr_ptr[nb + 1]; ++k)
            for (int c = 0; c < 3; ++c) {
                out.push_back((int32_t)(c * N + d.nbr_idx[k]));
                out.push_back((int32_t)(c * N + nb));
            }
    }
    if (v >= L.n_pts)
        for (int64_t b = d.bnd_ptr[v]; b < d.bnd_ptr[v + 1]; ++b) {  // boundary sub-faces of the divergence
            const int64_t ms[3] = {v, d.bnd_j[b], d.bnd_k[b]};
            for (int64_t m : ms)
                for (int c = 0; c < 3; ++c) out.push_back((int32_t)(c * N + m));
        }
    for (int64_t i = d.nbr_ptr[v]; i < d.nbr_ptr[v + 1]; ++i) {  // pressure stabiliser
        const int64_t nb = d.nbr_idx[i];
        out.push_back((int32_t)(P + nb));
        out.push_back((int32_t)r);
        for (int32_t k = L.gcp[v]; k < L.gcp[v + 1]; ++k) out.push_back((int32_t)(P + L.gcv[k]));
        for (int32_t k = L.gcp[nb]; k < L.gcp[nb + 1]; ++k) out.push_back((int32_t)(P + L.gcv[k]));
    }
}

}  // namespace

void build_grad_coeff(const Dual& d, NsLayout& L) {
    const int64_t n = d.n_tot;
    std::vector<std::vector<GcEnt>> per(n);
#pragma omp parallel
    {
        std::vector<GcEnt> e, m;
        std::vector<int32_t> stamp(n, -1), slot(n, 0);
#pragma omp for schedule(dynamic, 256)
        for (int64_t v = 0; v < n; ++v) {
            gc_push_order(d, v, e);
            gc_merge(e, (int32_t)v, stamp, slot, m);
            per[v] = m;
        }
    }
    L.gcp.assign(n + 1, 0);
    for (int64_t v = 0; v < n; ++v) L.gcp[v + 1] = L.gcp[v] + (int32_t)per[v].size();
    const int64_t ng = L.gcp[n];
    L.gcv.resize(ng);
    L.gcc.resize(3 * ng);
    for (int64_t v = 0; v < n; ++v)
        for (size_t k = 0; k < per[v].size(); ++k) {
            const int64_t t = L.gcp[v] + (int64_t)k;
            L.gcv[t] = per[v][k].vid;
            for (int q = 0; q < 3; ++q) L.gcc[q * ng + t] = per[v][k].c[q];
        }
}

std::string build_ns_layout(const Dual& d, int64_t pref_vid, NsLayout& L) {
    const int64_t n = d.n_tot, D = d.n_dir;
    if (4 * n >= (int64_t)INT_MAX) return "NS system too large for 32-bit row indices";
    if (pref_vid < 0 || pref_vid >= n) return "reference-pressure vertex out of range";
    L.n = n;
    L.n_pts = d.n_pts;
    L.pref_vid = pref_vid;
    build_grad_coeff(d, L);
    auto gcn = [&](int64_t v) -> int64_t { return L.gcp[v + 1] - L.gcp[v]; };
    // triplets per row and the per-face block offsets of the p rows
    const int64_t R = 4 * n, P = 3 * n;
    L.trip_ptr.assign(R + 1, 0);
    L.div_off.assign(D, 0);
    L.pst_off.assign(D, 0);
    L.sub_off.assign(n, 0);
    std::vector<int64_t> cnt(R, 0);
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < n; ++v) {
        const int64_t mom = v < d.n_pts ? 4 * deg(d, v) + gcn(v) : 1;
        for (int q = 0; q < 3; ++q) cnt[q * n + v] = mom;
        int64_t off = 0;
        for (int64_t i = d.nbr_ptr[v]; i < d.nbr_ptr[v + 1]; ++i) {
            L.div_off[i] = (int32_t)off;
            off += 6 + 6 * deg(d, v) + 6 * deg(d, d.nbr_idx[i]);
        }
        L.sub_off[v] = (int32_t)off;
        if (v >= d.n_pts) off += 9 * (d.bnd_ptr[v + 1] - d.bnd_ptr[v]);
        for (int64_t i = d.nbr_ptr[v]; i < d.nbr_ptr[v + 1]; ++i) {
            L.pst_off[i] = (int32_t)off;
            off += 2 + gcn(v) + gcn(d.nbr_idx[i]);
        }
        cnt[P + v] = v == pref_vid ? 1 : off;
    }
    for (int64_t r = 0; r < R; ++r) L.trip_ptr[r + 1] = L.trip_ptr[r] + cnt[r];
    // Distinct columns of a row are found with a per-thread stamp array over all R columns
    // (stamp[c] == r: column c already seen in row r); only those are sorted, and a per-thread
    // position table gives every triplet its slot. A row is handled by one thread, so the stamps
    // need no reset between rows.
    // pass 1: distinct columns per row
    std::vector<int64_t> nz(R, 0);
#pragma omp parallel
    {
        std::vector<int32_t> seq;
        std::vector<int32_t> stamp(R, -1);
#pragma omp for schedule(dynamic, 512)
        for (int64_t r = 0; r < R; ++r) {
            row_columns(d, L, r, seq);
            int64_t k = 0;
            for (int32_t c : seq)
                if (stamp[c] != (int32_t)r) {
                    stamp[c] = (int32_t)r;
                    ++k;
                }
            nz[r] = k;
        }
    }
    L.rp.assign(R + 1, 0);
    int64_t tot = 0;
    for (int64_t r = 0; r < R; ++r) {
        tot += nz[r];
        if (tot >= (int64_t)INT_MAX) return "NS pattern too large for 32-bit slot indices";
        L.rp[r + 1] = (int32_t)tot;
    }
    L.ci.resize(tot);  // ci, slot_ptr and slot_loc are written in full by pass 2
    L.slot_ptr.resize(tot + 1);
    L.slot_loc.resize(L.ntrip());
    L.slot_ptr[tot] = L.ntrip();
    // pass 2: columns, slots and the push-order triplet lists of every slot
    std::string err;
#pragma omp parallel
    {
        std::vector<int32_t> seq, cols, fill;
        std::vector<int32_t> stamp(R, -1), pos(R, 0);
#pragma omp for schedule(dynamic, 512)
        for (int64_t r = 0; r < R; ++r) {
            row_columns(d, L, r, seq);
            if ((int64_t)seq.size() != cnt[r]) {
#pragma omp critical
                err = "internal: triplet count mismatch";
                continue;
            }
            cols.clear();
            for (int32_t c : seq)
                if (stamp[c] != (int32_t)r) {
                    stamp[c] = (int32_t)r;
                    cols.push_back(c);
                }
            std::sort(cols.begin(), cols.end());
            const int64_t base = L.rp[r];
            std::copy(cols.begin(), cols.end(), L.ci.begin() + base);
            for (size_t s = 0; s < cols.size(); ++s) pos[cols[s]] = (int32_t)s;
            fill.assign(cols.size() + 1, 0);
            for (int32_t c : seq) fill[pos[c] + 1]++;
            for (size_t s = 0; s < cols.size(); ++s) fill[s + 1] += fill[s];
            const int64_t tb = L.trip_ptr[r];
            for (size_t s = 0; s < cols.size(); ++s) L.slot_ptr[base + s] = tb + fill[s];
            for (size_t t = 0; t < seq.size(); ++t) L.slot_loc[tb + fill[pos[seq[t]]]++] = (int32_t)t;
        }
    }
    return err;
}

}  // namespace vfv
