// Device data of the heat adjoint (see adjoint.cu).
#pragma once
#include "assemble.cuh"

namespace vfv {

struct AdjDev {
    int64_t n, n_dir;
    const int32_t* np;      // [n+1] neighbour CSR
    const int32_t* ni;      // [n_dir]
    const int32_t* rev;     // [n_dir] reverse directed face
    const int32_t* kind;    // [n] RowKind
    const double* area;
    const double* dist;
    const double* skew;     // [3][n_dir]
    const double* gw;       // [3][n_dir]
    const double* cvol;     // [n]
    const double* cskew;    // [3][n]
    const double* k;        // [n] conductivity
    const double* gk;       // [3][n] its gradient
    const double* T;        // [n] state
    const double* lambda;   // [n] adjoint state
    double* pv;             // [n_dir] work
    double* pn;             // [n_dir] work
    double* sk;             // [3][n_dir] work
    double* gkm;            // [n] work
    double* psi;            // [3][n] work
    double* dlogk;          // [n] out
    double* dq;             // [n] out
};

void launch_adjoint_partials(cudaStream_t s, const AdjDev& D);

}  // namespace vfv
