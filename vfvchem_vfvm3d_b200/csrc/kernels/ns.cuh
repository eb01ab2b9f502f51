// Device assembly of the coupled Navier-Stokes system (SteadyFlow::assemble_matrix,
// src/steady/core/steady_flow.rs:255-303) and the flow data it reads (flow_helper.rs:3-179).
// Compiled with -fmad=false: every value is formed with the reference's operation order and the
// matrix entries are sums of the row's triplets in push order, as the triplet build does.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace vfv {

struct NsDev {
    int64_t n, n_pts, n_dir, n_bsub, n_gc, pref_vid;
    double pref;
    // dual
    const int32_t *np, *ni;
    const double *dist, *area, *norm, *skew, *gw;  // norm, skew, gw: [3][n_dir]
    const double *cvol, *cskew;                    // cskew: [3][n]
    const int32_t *bp, *bj, *bk;
    const double *barea, *bnorm, *bw;              // [3][n_bsub]
    const int32_t *gcp, *gcv;                      // Tetrahedron::grad_coeff
    const double* gcc;                             // [3][n_gc]
    // fields (rho, mu, body force and boundary velocity are fixed; x is the Picard state)
    const double *den, *visc, *fce, *bc_vel;       // fce, bc_vel: [3][n]
    const double* x;                               // [u | v | w | p]
    const double *gvel, *gden, *gvisc, *gfce;      // [9][n], [3][n], [3][n], [9][n]
    double *rc, *mom, *flux;                       // [n], [3][n], [n_dir]
    // triplet layout and output
    const int64_t* trip_ptr;
    const int32_t *div_off, *pst_off, *sub_off;
    double* tv;
    double* b;                                     // [4n]
    const int32_t* rp;
    const int64_t* slot_ptr;
    const int32_t* slot_loc;
    double* val;
};

// rc, mom, flux (update_flow / update_flux), then triplet values, b, and the matrix values
void launch_ns_assemble(cudaStream_t s, const NsDev& D);

// 4x4 block-Jacobi with blocks {v, N+v, 2N+v, 3N+v} of a field-major 4-field system.
// Setup inverts every block (Gauss-Jordan, partial pivoting) into binv [16][nb]; a singular or
// non-finite block sets *bad.
void launch_bj4_setup(cudaStream_t s, int64_t nb, const int32_t* rp, const int32_t* ci, const double* val, double* binv, int* bad);

}  // namespace vfv
