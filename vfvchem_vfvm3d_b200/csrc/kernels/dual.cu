// The Voronoi dual of a tetrahedralisation on the device (sm_100a): the data-parallel passes of
// the host build_dual (csrc/host/mesh.cpp) as kernels, giving the same dual bit for bit.
//
// Reference: Tetrahedron::update_tet, src/base/geom_tet.rs:122-293 — face pieces per
// (tetrahedron, edge, side), summed per edge in tetrahedron order; edges in sorted (min, max)
// order, which is each vertex's neighbours in ascending order; control volumes and their centroid
// offsets; least-squares gradient weights. Every sum runs in the order of the reference's serial
// loops, every product and quotient rounds like the host code (this file is compiled with
// -fmad=false; sqrt and division are IEEE), so the arrays equal the host dual's.
//
// Passes: vertex -> tetrahedra lists (count, scan, fill, per-vertex sort); neighbour lists
// (distinct vertices of the vertex's tetrahedra, sorted); reverse entries; face pieces per
// tetrahedron; per edge (a < b) the sums over the tetrahedra of the edge (the merge of a's and b's
// ascending tetrahedron lists) and the boundary-face test; per vertex the control volume, its
// centroid offset and the gradient weights. The boundary sub-faces (a surface-sized stage) use the
// host code on the flags the device found. Scans of the per-vertex counts run on the host.
#include "../internal.cuh"

#include <cmath>
#include <vector>

namespace vfv {
namespace {

constexpr int kMaxDeg = 96;  // neighbours (and incident tetrahedra) per vertex the passes handle

struct D3 { double x, y, z; };
__device__ __forceinline__ D3 P3(const double* pos, int64_t v) { return D3{pos[3 * v], pos[3 * v + 1], pos[3 * v + 2]}; }
__device__ __forceinline__ D3 add3(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 sub3(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 scale3(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot3(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross3(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ double len3(D3 a) { return sqrt(dot3(a, a)); }
__device__ __forceinline__ D3 circumcircle3(D3 a, D3 b, D3 c) {  // delaunay.rs:207-214
    const D3 u = sub3(b, a), v = sub3(c, a);
    const D3 w = cross3(u, v);
    const D3 num = add3(scale3(dot3(u, u), cross3(v, w)), scale3(dot3(v, v), cross3(w, u)));
    return add3(a, scale3(0.5 / dot3(w, w), num));
}
__device__ __forceinline__ D3 circumsphere3(D3 a, D3 b, D3 c, D3 d) {  // delaunay.rs:216-221
    const D3 u = sub3(b, a), v = sub3(c, a), w = sub3(d, a);
    const D3 num = add3(add3(scale3(dot3(u, u), cross3(v, w)), scale3(dot3(v, v), cross3(w, u))), scale3(dot3(w, w), cross3(u, v)));
    return add3(a, scale3(0.5 / dot3(u, cross3(v, w)), num));
}

__constant__ int kEE[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};

__global__ void k_vt_count(int64_t T, const int32_t* __restrict__ tet, int64_t* __restrict__ cnt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 4 * T) atomicAdd((unsigned long long*)&cnt[tet[i] + 1], 1ull);
}

__global__ void k_vt_fill(int64_t T, const int32_t* __restrict__ tet, unsigned long long* __restrict__ cur, int32_t* __restrict__ vt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 4 * T) vt[atomicAdd(&cur[tet[i]], 1ull)] = (int32_t)(i / 4);
}

// each vertex's tetrahedra ascending (insertion sort of a short list)
__global__ void k_vt_sort(int64_t N, const int64_t* __restrict__ ptr, int32_t* __restrict__ vt) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    int32_t* a = vt + ptr[v];
    const int64_t m = ptr[v + 1] - ptr[v];
    for (int64_t i = 1; i < m; ++i) {
        const int32_t x = a[i];
        int64_t j = i - 1;
        while (j >= 0 && a[j] > x) {
            a[j + 1] = a[j];
            --j;
        }
        a[j + 1] = x;
    }
}

// distinct vertices of v's tetrahedra other than v, ascending: count (out == null) or write
__global__ void k_nbr(int64_t N, const int32_t* __restrict__ tet, const int64_t* __restrict__ vtp, const int32_t* __restrict__ vt,
                      const int64_t* __restrict__ nptr, int32_t* __restrict__ nidx, int64_t* __restrict__ ncnt, int* __restrict__ err) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    int32_t buf[kMaxDeg];
    int m = 0;
    for (int64_t q = vtp[v]; q < vtp[v + 1]; ++q) {
        const int32_t* tv = tet + 4 * (int64_t)vt[q];
        for (int k = 0; k < 4; ++k) {
            const int32_t u = tv[k];
            if (u == v) continue;
            int pos = 0;
            while (pos < m && buf[pos] < u) ++pos;
            if (pos < m && buf[pos] == u) continue;
            if (m == kMaxDeg) {
                *err = 1;
                return;
            }
            for (int r = m; r > pos; --r) buf[r] = buf[r - 1];
            buf[pos] = u;
            ++m;
        }
    }
    if (!nidx) {
        ncnt[v + 1] = m;
        return;
    }
    int32_t* o = nidx + nptr[v];
    for (int r = 0; r < m; ++r) o[r] = buf[r];
}

// the two face pieces of each edge of each tetrahedron (the host's face_pieces)
__global__ void k_pieces(int64_t T, const int32_t* __restrict__ tet, const double* __restrict__ pos, double* __restrict__ pa,
                         double* __restrict__ pc) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const int32_t* tv = tet + 4 * t;
    const D3 c_t = circumsphere3(P3(pos, tv[0]), P3(pos, tv[1]), P3(pos, tv[2]), P3(pos, tv[3]));
    for (int e = 0; e < 6; ++e) {
        const int li = kEE[e][0], lj = kEE[e][1];
        int oth[2], no = 0;
        for (int l = 0; l < 4; ++l)
            if (l != li && l != lj) oth[no++] = l;
        const D3 pi = P3(pos, tv[li]), pj = P3(pos, tv[lj]);
        const double dist = len3(sub3(pj, pi));
        const D3 ee = scale3(1.0 / dist, sub3(pj, pi));
        const D3 m = scale3(0.5, add3(pi, pj));
        for (int side = 0; side < 2; ++side) {
            const D3 a = P3(pos, tv[oth[side]]), b = P3(pos, tv[oth[1 - side]]);
            const D3 c_f = circumcircle3(pi, pj, a);
            D3 u = sub3(sub3(a, m), scale3(dot3(sub3(a, m), ee), ee));
            u = scale3(1.0 / len3(u), u);
            D3 n = cross3(ee, u);
            if (dot3(sub3(b, m), n) < 0.0) n = scale3(-1.0, n);
            const double s1 = dot3(sub3(c_f, m), u);
            const double s2 = dot3(sub3(c_t, c_f), n);
            const int64_t q = 12 * t + 2 * e + side;
            pa[q] = 0.5 * s1 * s2;
            const D3 cen = scale3(1.0 / 3.0, add3(m, add3(c_f, c_t)));
            pc[3 * q] = cen.x;
            pc[3 * q + 1] = cen.y;
            pc[3 * q + 2] = cen.z;
        }
    }
}

// position of u in v's ascending neighbour list
__device__ __forceinline__ int64_t nbr_pos(const int64_t* nptr, const int32_t* nidx, int64_t v, int32_t u) {
    int64_t lo = nptr[v], hi = nptr[v + 1];
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (nidx[mid] < u) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Per edge (a, b), a < b (thread per directed entry ia of a with b > a): its tetrahedra are the
// common ones of a's and b's ascending lists; sum the pieces in that order, store the edge's data
// for both directed entries, and flag boundary faces (a, b, z), z > b, held by one tetrahedron.
__global__ void k_edges(int64_t N, const double* __restrict__ pos, const int32_t* __restrict__ tet, const int64_t* __restrict__ vtp,
                        const int32_t* __restrict__ vt, const int64_t* __restrict__ nptr, const int32_t* __restrict__ nidx,
                        const double* __restrict__ pa, const double* __restrict__ pc, int64_t D, int64_t* __restrict__ rev,
                        double* __restrict__ dist_o, double* __restrict__ area_o, double* __restrict__ norm_o, double* __restrict__ skew_o,
                        uint8_t* __restrict__ bface, const int32_t* __restrict__ owner) {
    const int64_t ia = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ia >= D) return;
    const int64_t a = owner[ia];
    const int32_t b = nidx[ia];
    if (b <= a) return;
    int32_t lst[kMaxDeg];
    int nl = 0;
    {
        int64_t p = vtp[a], q = vtp[b];
        const int64_t pe = vtp[a + 1], qe = vtp[b + 1];
        while (p < pe && q < qe && nl < kMaxDeg) {
            const int32_t x = vt[p], y = vt[q];
            if (x == y) {
                lst[nl++] = x;
                ++p;
                ++q;
            } else if (x < y) {
                ++p;
            } else {
                ++q;
            }
        }
    }
    double s_area = 0.0, s_x = 0.0, s_y = 0.0, s_z = 0.0;
    for (int j = 0; j < nl; ++j) {
        const int64_t t = lst[j];
        const int32_t* tv = tet + 4 * t;
        int e = 0;
        while (!((tv[kEE[e][0]] == a && tv[kEE[e][1]] == b) || (tv[kEE[e][0]] == b && tv[kEE[e][1]] == a))) ++e;
        const D3 m = scale3(0.5, add3(P3(pos, tv[kEE[e][0]]), P3(pos, tv[kEE[e][1]])));
        for (int side = 0; side < 2; ++side) {
            const int64_t q = 12 * t + 2 * e + side;
            const double area = pa[q];
            const D3 cent{pc[3 * q], pc[3 * q + 1], pc[3 * q + 2]};
            s_area += area;
            const D3 sk = scale3(area, sub3(cent, m));
            s_x += sk.x;
            s_y += sk.y;
            s_z += sk.z;
        }
        for (int l = 0; l < 4; ++l) {
            const int32_t z = tv[l];
            if (z <= b) continue;
            int holders = 0;
            for (int j2 = 0; j2 < nl && holders < 2; ++j2) {
                const int32_t* w = tet + 4 * (int64_t)lst[j2];
                holders += (w[0] == z) | (w[1] == z) | (w[2] == z) | (w[3] == z);
            }
            if (holders == 1) {
                int opp = 0;
                while (tv[opp] == a || tv[opp] == b || tv[opp] == z) ++opp;
                bface[4 * t + opp] = 1;
            }
        }
    }
    const D3 pa3 = P3(pos, a), pb3 = P3(pos, b);
    const double dist = len3(sub3(pb3, pa3));
    const D3 nrm = scale3(1.0 / dist, sub3(pb3, pa3));
    const D3 skew = (fabs(s_area) > 1e-12 * dist * dist) ? scale3(1.0 / s_area, D3{s_x, s_y, s_z}) : D3{0.0, 0.0, 0.0};
    const int64_t ib = nbr_pos(nptr, nidx, b, (int32_t)a);
    rev[ia] = ib;
    rev[ib] = ia;
    dist_o[ia] = dist_o[ib] = dist;
    area_o[ia] = area_o[ib] = s_area;
    const D3 mn = scale3(-1.0, nrm);
    norm_o[ia] = nrm.x;
    norm_o[D + ia] = nrm.y;
    norm_o[2 * D + ia] = nrm.z;
    norm_o[ib] = mn.x;
    norm_o[D + ib] = mn.y;
    norm_o[2 * D + ib] = mn.z;
    skew_o[ia] = skew_o[ib] = skew.x;
    skew_o[D + ia] = skew_o[D + ib] = skew.y;
    skew_o[2 * D + ia] = skew_o[2 * D + ib] = skew.z;
}

// per vertex: control volume (faces in neighbour order), centroid offset (pieces in tetrahedron,
// edge, side order) and least-squares gradient weights
__global__ void k_vertex(int64_t N, const double* __restrict__ pos, const int32_t* __restrict__ tet, const int64_t* __restrict__ vtp,
                         const int32_t* __restrict__ vt, const int64_t* __restrict__ nptr, const int32_t* __restrict__ nidx,
                         const double* __restrict__ pa, const double* __restrict__ pc, int64_t D, const double* __restrict__ dist_i,
                         const double* __restrict__ area_i, double* __restrict__ cvol, double* __restrict__ cskew, double* __restrict__ gw,
                         int64_t* __restrict__ bad) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    double vol = 0.0;
    for (int64_t i = nptr[v]; i < nptr[v + 1]; ++i) vol += area_i[i] * dist_i[i] / 6.0;
    cvol[v] = vol;
    double cx = 0.0, cy = 0.0, cz = 0.0;
    for (int64_t q = vtp[v]; q < vtp[v + 1]; ++q) {
        const int64_t t = vt[q];
        const int32_t* tv = tet + 4 * t;
        for (int e = 0; e < 6; ++e) {
            const int32_t vi = tv[kEE[e][0]], vj = tv[kEE[e][1]];
            if (vi != v && vj != v) continue;
            const D3 pi = P3(pos, vi), pj = P3(pos, vj);
            const double dist = len3(sub3(pj, pi));
            const D3 pv = vi == v ? pi : pj;
            for (int side = 0; side < 2; ++side) {
                const int64_t k = 12 * t + 2 * e + side;
                const double pvol = pa[k] * dist / 6.0;
                const D3 c = scale3(pvol * 0.75, sub3(D3{pc[3 * k], pc[3 * k + 1], pc[3 * k + 2]}, pv));
                cx += c.x;
                cy += c.y;
                cz += c.z;
            }
        }
    }
    const double s = 1.0 / vol;
    cskew[v] = s * cx;
    cskew[N + v] = s * cy;
    cskew[2 * N + v] = s * cz;
    const D3 p0 = P3(pos, v);
    double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int64_t i = nptr[v]; i < nptr[v + 1]; ++i) {
        const D3 dd = sub3(P3(pos, nidx[i]), p0);
        const double dv[3] = {dd.x, dd.y, dd.z};
        const double omega = 1.0 / (dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) m[r][c] += omega * dv[r] * dv[c];
    }
    const double adj[3][3] = {
        {m[1][1] * m[2][2] - m[1][2] * m[2][1], m[0][2] * m[2][1] - m[0][1] * m[2][2], m[0][1] * m[1][2] - m[0][2] * m[1][1]},
        {m[1][2] * m[2][0] - m[1][0] * m[2][2], m[0][0] * m[2][2] - m[0][2] * m[2][0], m[0][2] * m[1][0] - m[0][0] * m[1][2]},
        {m[1][0] * m[2][1] - m[1][1] * m[2][0], m[0][1] * m[2][0] - m[0][0] * m[2][1], m[0][0] * m[1][1] - m[0][1] * m[1][0]},
    };
    const double det = m[0][0] * adj[0][0] + m[0][1] * adj[1][0] + m[0][2] * adj[2][0];
    const double tr = m[0][0] + m[1][1] + m[2][2];
    if (!(det > 1e-12 * tr * tr * tr)) {
        atomicMin((unsigned long long*)bad, (unsigned long long)v);
        return;
    }
    for (int64_t i = nptr[v]; i < nptr[v + 1]; ++i) {
        const D3 dd = sub3(P3(pos, nidx[i]), p0);
        const double omega = 1.0 / dot3(dd, dd);
        for (int r = 0; r < 3; ++r) gw[r * D + i] = omega * (adj[r][0] * dd.x + adj[r][1] * dd.y + adj[r][2] * dd.z) / det;
    }
}

__global__ void k_owner(int64_t N, const int64_t* __restrict__ nptr, int32_t* __restrict__ owner) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    for (int64_t i = nptr[v]; i < nptr[v + 1]; ++i) owner[i] = (int32_t)v;
}

int blocks(int64_t n) { return (int)std::max<int64_t>(1, (n + 255) / 256); }

}  // namespace

// The dual of mesh (its tetrahedra set) computed on the device of ctx; d receives the same arrays
// as build_dual. Returns "" on success.
std::string build_dual_device(vfv_ctx* ctx, const Mesh& mesh, Dual& d) {
    const int64_t N = mesh.n_tot(), T = mesh.n_tet();
    if (N >= (int64_t)INT32_MAX || T >= (int64_t)INT32_MAX / 12) return "dual: mesh too large for 32-bit indices";
    cudaStream_t s = ctx->stream;
    auto ck = [](cudaError_t e) -> std::string { return e == cudaSuccess ? std::string() : std::string("dual on the device: ") + cudaGetErrorString(e); };
    std::string e;
#define DK(call)                    \
    do {                            \
        e = ck(call);               \
        if (!e.empty()) return e;   \
    } while (0)
    DBuf<double> pos, pa, pc;
    DBuf<int32_t> tet, vt, nidx, owner;
    DBuf<int64_t> vtp, nptr, scratch;
    DBuf<int> err;
    DK(pos.upload(mesh.pos.data(), mesh.pos.size(), s));
    DK(tet.upload(mesh.tets.data(), mesh.tets.size(), s));
    DK(err.alloc(1));
    DK(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    // vertex -> tetrahedra
    DK(vtp.alloc(N + 1));
    DK(cudaMemsetAsync(vtp.p, 0, (N + 1) * sizeof(int64_t), s));
    k_vt_count<<<blocks(4 * T), 256, 0, s>>>(T, tet.p, vtp.p);
    std::vector<int64_t> h(N + 1);
    DK(cudaMemcpyAsync(h.data(), vtp.p, (N + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    DK(cudaStreamSynchronize(s));
    for (int64_t v = 0; v < N; ++v) h[v + 1] += h[v];
    DK(cudaMemcpyAsync(vtp.p, h.data(), (N + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    DK(scratch.alloc(N + 1));
    DK(cudaMemcpyAsync(scratch.p, vtp.p, (N + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
    DK(vt.alloc(4 * T));
    k_vt_fill<<<blocks(4 * T), 256, 0, s>>>(T, tet.p, (unsigned long long*)scratch.p, vt.p);
    k_vt_sort<<<blocks(N), 256, 0, s>>>(N, vtp.p, vt.p);
    // neighbour lists
    DK(nptr.alloc(N + 1));
    DK(cudaMemsetAsync(nptr.p, 0, (N + 1) * sizeof(int64_t), s));
    k_nbr<<<blocks(N), 256, 0, s>>>(N, tet.p, vtp.p, vt.p, nullptr, nullptr, nptr.p, err.p);
    DK(cudaMemcpyAsync(h.data(), nptr.p, (N + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    int herr = 0;
    DK(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    DK(cudaStreamSynchronize(s));
    if (herr) return "dual on the device: a vertex has more than 96 neighbours";
    for (int64_t v = 0; v < N; ++v) h[v + 1] += h[v];
    const int64_t D = h[N];
    DK(cudaMemcpyAsync(nptr.p, h.data(), (N + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    DK(nidx.alloc(D));
    k_nbr<<<blocks(N), 256, 0, s>>>(N, tet.p, vtp.p, vt.p, nptr.p, nidx.p, nullptr, err.p);
    DK(owner.alloc(D));
    k_owner<<<blocks(N), 256, 0, s>>>(N, nptr.p, owner.p);
    // face pieces, edges, vertices
    DK(pa.alloc(12 * T));
    DK(pc.alloc(36 * T));
    k_pieces<<<blocks(T), 256, 0, s>>>(T, tet.p, pos.p, pa.p, pc.p);
    DBuf<int64_t> rev;
    DBuf<double> dist, area, norm, skew, cvol, cskew, gw;
    DBuf<uint8_t> bf;
    DBuf<int64_t> bad;
    DK(rev.alloc(D));
    DK(dist.alloc(D));
    DK(area.alloc(D));
    DK(norm.alloc(3 * D));
    DK(skew.alloc(3 * D));
    DK(bf.alloc(4 * T));
    DK(cudaMemsetAsync(bf.p, 0, 4 * T, s));
    k_edges<<<blocks(D), 256, 0, s>>>(N, pos.p, tet.p, vtp.p, vt.p, nptr.p, nidx.p, pa.p, pc.p, D, rev.p, dist.p, area.p, norm.p, skew.p,
                                      bf.p, owner.p);
    DK(cvol.alloc(N));
    DK(cskew.alloc(3 * N));
    DK(gw.alloc(3 * D));
    DK(bad.alloc(1));
    const int64_t none = INT64_MAX;
    DK(cudaMemcpyAsync(bad.p, &none, sizeof(int64_t), cudaMemcpyHostToDevice, s));
    k_vertex<<<blocks(N), 256, 0, s>>>(N, pos.p, tet.p, vtp.p, vt.p, nptr.p, nidx.p, pa.p, pc.p, D, dist.p, area.p, cvol.p, cskew.p, gw.p,
                                       bad.p);
    DK(cudaGetLastError());
    // results back into the host dual
    d = Dual();
    d.n_tot = N;
    d.n_pts = mesh.n_pts;
    d.n_dir = D;
    d.nbr_ptr = h;
    d.nbr_idx.resize(D);
    d.nbr_rev.resize(D);
    d.dist.resize(D);
    d.area.resize(D);
    d.norm.resize(3 * D);
    d.skew.resize(3 * D);
    d.gw.resize(3 * D);
    d.cvol.resize(N);
    d.cskew.resize(3 * N);
    std::vector<uint8_t> bface(4 * T);
    int64_t hbad = 0;
    DK(cudaMemcpyAsync(d.nbr_idx.data(), nidx.p, D * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    DK(cudaMemcpyAsync(d.nbr_rev.data(), rev.p, D * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    DK(cudaMemcpyAsync(d.dist.data(), dist.p, D * sizeof(double), cudaMemcpyDeviceToHost, s));
    DK(cudaMemcpyAsync(d.area.data(), area.p, D * sizeof(double), cudaMemcpyDeviceToHost, s));
    DK(cudaMemcpyAsync(d.norm.data(), norm.p, 3 * D * sizeof(double), cudaMemcpyDeviceToHost, s));
    DK(cudaMemcpyAsync(d.skew.data(), skew.p, 3 * D * sizeof(double), cudaMemcpyDeviceToHost, s));
    DK(cudaMemcpyAsync(d.gw.data(), gw.p, 3 * D * sizeof(double), cudaMemcpyDeviceToHost, s));
    DK(cudaMemcpyAsync(d.cvol.data(), cvol.p, N * sizeof(double), cudaMemcpyDeviceToHost, s));
    DK(cudaMemcpyAsync(d.cskew.data(), cskew.p, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
    DK(cudaMemcpyAsync(bface.data(), bf.p, 4 * T, cudaMemcpyDeviceToHost, s));
    DK(cudaMemcpyAsync(&hbad, bad.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    DK(cudaStreamSynchronize(s));
#undef DK
    if (hbad != INT64_MAX) return "dual: singular least-squares gradient at vid " + std::to_string(hbad);
    return boundary_subfaces(mesh, bface, d);
}

}  // namespace vfv
