// Host-side mesh and Voronoi-dual data model for the assemble-and-solve path.
//
// The reference builds its control volumes in src/base/geom_tet.rs (Tetrahedron::update_tet,
// :58-350) from a Bowyer-Watson Delaunay tetrahedralisation (src/base/delaunay.rs:6-170).
// This header holds the flattened, structure-of-arrays form of the same data, laid out the way
// the device kernels read it:
//   * vertices are ordered points first, then nodes (src/base/geom_dom.rs:41-54);
//   * neighbour lists are a CSR (nbr_ptr / nbr_idx) whose per-vertex order is the reference's
//     sorted-edge order (geom_tet.rs:173-206), which is ascending neighbour id;
//   * every per-face quantity is stored once per directed entry of that CSR, component-major
//     ([3][n_dir] for vectors) so a warp reading consecutive entries is coalesced.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace vfv {

// Boundary ids of the unit-cube meshes (names follow Nodes::new_from_bounds, src/base/nds.rs:48-88).
enum BoundaryId : int32_t { BND_L = 0, BND_R = 1, BND_F = 2, BND_K = 3, BND_B = 4, BND_T = 5, NUM_BND = 6 };

struct Mesh {
    int64_t n_pts = 0;              // interior points (vid < n_pts)
    int64_t n_nds = 0;              // boundary nodes (vid >= n_pts)
    std::vector<double> pos;        // [n_tot][3] vertex positions
    std::vector<int32_t> node_bnd;  // [n_nds] boundary id of every node (one boundary per node)
    std::vector<int32_t> tets;      // [n_tet][4] positively oriented tetrahedra (orient3d > 0)
    int64_t n_tot() const { return n_pts + n_nds; }
    int64_t n_tet() const { return (int64_t)tets.size() / 4; }
};

struct Dual {
    int64_t n_tot = 0, n_pts = 0, n_dir = 0;  // n_dir = 2 * number of Voronoi faces (Delaunay edges)
    // neighbour CSR (Tetrahedron::ngh_vid)
    std::vector<int64_t> nbr_ptr;   // [n_tot + 1]
    std::vector<int32_t> nbr_idx;   // [n_dir] neighbour vid, ascending per vertex
    std::vector<int64_t> nbr_rev;   // [n_dir] position of the reverse directed entry (n -> v)
    // per directed face (ngh_dist, face_area, face_norm, face_skew, grad_wgt)
    std::vector<double> dist;       // [n_dir]
    std::vector<double> area;       // [n_dir] signed Voronoi face area (shared by both directions)
    std::vector<double> norm;       // [3][n_dir] unit normal out of the owning control volume
    std::vector<double> skew;       // [3][n_dir] face centre minus edge midpoint (zero if |A| tiny)
    std::vector<double> gw;         // [3][n_dir] least-squares gradient weights
    // per vertex (cvol_vol, cvol_skew, bnd_sum)
    std::vector<double> cvol;       // [n_tot]
    std::vector<double> cskew;      // [3][n_tot]
    std::vector<double> bnd_sum;    // [n_tot]
    // boundary sub-faces (bnd_vid, bnd_area, bnd_norm, bnd_wgt) as a CSR over vertices
    std::vector<int64_t> bnd_ptr;   // [n_tot + 1]
    std::vector<int32_t> bnd_j, bnd_k;   // [n_bsub] the other two vertices of the surface triangle
    std::vector<double> bnd_area;   // [n_bsub]
    std::vector<double> bnd_norm;   // [3][n_bsub]
    std::vector<double> bnd_wgt;    // [3][n_bsub] (w_v, w_j, w_k)
};

// Seeded jittered-grid cube mesh: n^3 grid points on [0,1]^3 with spacing h = 1/(n-1).
// Interior grid points become points and are jittered uniformly by +-jitter*h on all three axes;
// surface grid points become nodes and are jittered only along the axes on which they are not
// pinned (face nodes in-plane, edge nodes along the edge, corners fixed), so the hull stays the
// exact unit cube. Each node belongs to one boundary: x faces win over y faces, y over z.
// Coordinates are rounded to multiples of 2^-18 so the Delaunay predicates are exact in
// 128-bit integer arithmetic. Random numbers come from SplitMix64(seed), three draws per grid
// point in (k, j, i) order with i fastest.
Mesh make_jitter_cube(int n, uint64_t seed, double jitter);

// Delaunay tetrahedralisation by Bowyer-Watson insertion with exact predicates: integer ones for
// vertices on the 2^-18 lattice within a box of 1.75 (the generated cubes), filtered double ones
// with an exact big-integer fallback for any other finite coordinates. Fills mesh.tets. Returns an
// empty string on success, else the error message.
std::string delaunay(Mesh& mesh);

// Voronoi dual of the tetrahedralisation (geom_tet.rs:122-293). Returns "" on success. The face
// pieces of all tetrahedra (384 bytes each) are kept while they fit piece_store_bytes, else
// recomputed where needed; the result is the same bit for bit either way and for any thread count.
constexpr double kDualPieceStoreBytes = 8.0 * 1024 * 1024 * 1024;
std::string build_dual(const Mesh& mesh, Dual& dual, double piece_store_bytes = kDualPieceStoreBytes);

// Boundary sub-faces of the faces flagged in bface (4 per tetrahedron); part of build_dual, shared
// with the device dual. Returns "" on success.
std::string boundary_subfaces(const Mesh& mesh, const std::vector<uint8_t>& bface, Dual& dual);

constexpr int kQuantBits = 18;  // coordinates are multiples of 2^-18

}  // namespace vfv
