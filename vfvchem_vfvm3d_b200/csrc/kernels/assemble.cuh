// Device data of the steady heat operator and the launchers of its kernels.
#pragma once
#include "../common.cuh"

namespace vfv {

enum RowKind : int32_t { ROW_POINT = 0, ROW_FLUX = 1, ROW_DIRICHLET = 2 };

// Device pointers read by k_assemble_heat. Geometry is structure-of-arrays, per directed face
// (n_dir entries, CSR order of the neighbour lists) and per vertex (n entries).
struct HeatDev {
    int64_t n, n_dir, n_bsub;
    const int32_t* np;      // [n+1] neighbour CSR
    const int32_t* ni;      // [n_dir]
    const double* area;     // [n_dir]
    const double* dist;     // [n_dir]
    const double* skew;     // [3][n_dir]
    const double* cvol;     // [n]
    const double* cskew;    // [3][n]
    const int32_t* kind;    // [n] RowKind
    const int32_t* node_bnd;  // [n] boundary id, -1 for points
    const int32_t* bp;      // [n+1] boundary sub-face CSR
    const int32_t* bj;      // [n_bsub]
    const int32_t* bk;      // [n_bsub]
    const double* barea;    // [n_bsub]
    const double* bw;       // [3][n_bsub]
    const int32_t* rp;      // [n+1] matrix CSR row pointer
    const int32_t* dloc;    // [n] number of neighbours below v (= diagonal offset in the row)
    // fields and their gradients ([3][n] each)
    const double* k;
    const double* q;
    const double* s;
    const double* T;
    const double* bcv;      // [n] Dirichlet value or Neumann flux on nodes
    const double* gk;
    const double* gq;
    const double* gs;
    const double* gT;
    // outputs
    double* val;            // [nnz]
    double* b;              // [n]
};

// Device data of the transient advection-diffusion operator (one species, implicit Euler):
// OpSclDomTimeUnity (opscl_dom_timeunity.rs:32-58), OpSclDomDiffusion (opscl_dom_diff.rs:40-91) and
// OpSclDomAdvection (opscl_dom_adv.rs:49-125) with their boundary twins on every node (zero-flux walls).
struct TransportDev {
    int64_t n, n_dir;
    const int32_t* np;
    const int32_t* ni;
    const double* area;
    const double* dist;
    const double* skew;     // [3][n_dir]
    const double* norm;     // [3][n_dir] unit normal out of the owning control volume
    const double* cvol;     // [n]
    const int32_t* rp;      // matrix CSR row pointer
    const int32_t* dloc;    // [n] diagonal offset in the row
    const double* D;        // [n] diffusivity
    const double* gD;       // [3][n] its gradient
    const double* vel;      // [3][n] velocity
    const double* gvel;     // [9][n] its gradient (du/dx, du/dy, du/dz, dv/dx, ...)
    double* flux;           // [n_dir] face mass flux (density 1)
    double dt;
    double* val;            // [nnz]
};

void launch_face_flux(cudaStream_t s, const TransportDev& T);
void launch_assemble_transport(cudaStream_t s, const TransportDev& T);
void launch_transport_rhs(cudaStream_t s, int64_t n, const double* cvol, double dt, const double* c_prev, double* b);

// part[blk] = sum over this block's rows v of lam_v sum_faces s_e (c_n - c_v), where
// s_e = d(cond + coeff)/dD for a uniform diffusivity D (transient adjoint of the transport batch)
void launch_transport_dAdD_dot(cudaStream_t s, const TransportDev& T, const double* lam, const double* c, double* part, unsigned* counter,
                               double* out);

void launch_grad(cudaStream_t s, int64_t n, const int32_t* np, const int32_t* ni, const double* gw, int64_t n_dir, int nf,
                 const double* const* f, double* out);
void launch_assemble_heat(cudaStream_t s, const HeatDev& H);
void launch_values_from_triplets(cudaStream_t s, int64_t nnz, const int64_t* sp, const int64_t* st, const double* tv, double* val);

}  // namespace vfv
