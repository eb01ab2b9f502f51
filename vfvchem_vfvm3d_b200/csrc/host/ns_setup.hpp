// Symbolic setup of the coupled Navier-Stokes system (SteadyFlow, src/steady/core/steady_flow.rs)
// on the Voronoi dual: pressure-gradient coefficients, the triplet layout of every row in the
// reference's push order, and the CSR pattern with the per-slot lists of triplets that the device
// sums (in push order) into the matrix values.
//
// Unknowns are field-major, [u | v | w | p], n entries each (OperatorBase::add_vecvec_a and
// friends, src/operator/operator_base.rs:37-94). Every operator of SteadyFlow::assemble_matrix
// (steady_flow.rs:255-303) pushes only into the rows of the vertex it visits, so the push order
// restricted to one row is the operator order followed by the face order of that vertex:
//   u/v/w rows of a point:  advection (n, v per face), pressure gradient (grad_coeff of v),
//                           diffusion (n, v per face)
//   u/v/w rows of a node:   the Dirichlet diagonal
//   p row of a point:       divergence (per face: 6 + 6 deg v + 6 deg n), pressure stabiliser
//                           (per face: 2 + |gc v| + |gc n|)
//   p row of a node:        divergence faces, then 9 per boundary sub-face, then the stabiliser
//   p row of the reference vertex: the single diagonal (OpSclDomPressureReference drops the rest)
#pragma once
#include <cstdint>
#include <memory>
#include <new>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "mesh.hpp"

namespace vfv {

// Allocator whose value-less construct default-initialises, so resize() of the large layout
// arrays leaves their (trivial) elements unset instead of zeroing gigabytes that the setup then
// overwrites; the parallel pass that writes them touches the pages first.
template <typename T>
struct UninitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind { using other = UninitAlloc<U>; };
    UninitAlloc() = default;
    template <typename U>
    UninitAlloc(const UninitAlloc<U>&) noexcept {}
    template <typename U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) { ::new (static_cast<void*>(p)) U; }
    template <typename U, typename... A>
    void construct(U* p, A&&... a) { ::new (static_cast<void*>(p)) U(std::forward<A>(a)...); }
};
template <typename T>
using uninit_vector = std::vector<T, UninitAlloc<T>>;

struct NsLayout {
    int64_t n = 0, n_pts = 0, pref_vid = 0;
    // Tetrahedron::grad_coeff (geom_tet.rs:295-347) as a CSR over vertices, ascending vertex ids
    std::vector<int32_t> gcp;        // [n + 1]
    std::vector<int32_t> gcv;        // [n_gc]
    std::vector<double> gcc;         // [3][n_gc]
    // triplet layout
    std::vector<int64_t> trip_ptr;   // [4n + 1] first triplet of every row
    std::vector<int32_t> div_off;    // [n_dir] offset of face i's divergence block within the p row of its owner
    std::vector<int32_t> pst_off;    // [n_dir] offset of face i's stabiliser block within that row
    std::vector<int32_t> sub_off;    // [n] offset of the boundary sub-face block within the p row (nodes)
    // pattern and slot lists
    std::vector<int32_t> rp;         // CSR of the 4n x 4n matrix: row pointer [4n + 1]
    uninit_vector<int32_t> ci;       // [nnz] columns
    uninit_vector<int64_t> slot_ptr; // [nnz + 1] into slot_loc
    uninit_vector<int32_t> slot_loc; // [ntrip] triplet index within its row, push order per slot
    int64_t nnz() const { return (int64_t)ci.size(); }
    int64_t ntrip() const { return trip_ptr.empty() ? 0 : trip_ptr.back(); }
};

// Pressure-gradient coefficients: per vertex, the (vertex, c) pairs of the Green-Gauss gradient
// with skew-corrected face values, merged by vertex in push order (stable sort, then ordered sums).
void build_grad_coeff(const Dual& d, NsLayout& L);

// Full symbolic setup (grad_coeff included). Returns "" or an error message.
std::string build_ns_layout(const Dual& d, int64_t pref_vid, NsLayout& L);

}  // namespace vfv
