/*
 * vfv_gpu.h - C ABI of libvfvgpu, the B200 (sm_100a) assemble-and-solve path of vfvchem-vfvm3d.
 *
 * Plain C types only: opaque handles, pointers and sizes. Every entry point returns a status code
 * (VFV_OK = 0); the message of the last failure is vfv_last_error(ctx) (or vfv_last_error(NULL)
 * for failures before a context exists). No entry point falls back to a CPU implementation: when
 * no CUDA device is usable, vfv_ctx_create fails with VFV_CUDA_ERROR.
 *
 * Reference interfaces replaced (paths are within the vfvchem-vfvm3d project):
 *   trait LinearBase                      src/linear/linear_base.rs:5-10
 *     update_sparse  -> vfv_pattern_from_triplets
 *     build_matrix   -> vfv_values_from_triplets
 *     solve_matrix   -> vfv_solve / vfv_solve_device
 *   LinearGmres::new_with_options          src/linear/linear_gmres.rs:24-49  -> vfv_gmres_opts
 *   trait OperatorBase::apply (heat ops)    src/operator/operator_base.rs:5-7, driven by
 *   SteadyHeat::assemble_matrix             src/steady/core/steady_heat.rs:143-171 -> vfv_heat_assemble
 *   ScalarDomain::update_grad               src/base/scl_dom.rs:146-164 -> vfv_update_grad
 *   Tetrahedron::update_tet (geometry)      src/base/geom_tet.rs:58-350 -> vfv_mesh_* (host, once)
 *
 * Threading: a context owns one CUDA stream; calls on one context must not overlap (like the
 * reference's single-threaded `&mut dyn LinearBase`). Different contexts are independent.
 */
#ifndef VFV_GPU_H
#define VFV_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (a non-zero code maps onto VFVChemError::LinearGmresDidNotConverge or a
 *      new variant on the Rust side; src/base/error.rs:265-268) */
#define VFV_OK 0
#define VFV_NOT_CONVERGED 1 /* max_outer restart cycles without reaching tol */
#define VFV_NONFINITE 2     /* NaN/Inf in the residual or the Arnoldi process */
#define VFV_BAD_INPUT 3     /* invalid argument (sizes, indices, options) */
#define VFV_CUDA_ERROR 4    /* CUDA runtime failure or no device */
#define VFV_TIMEOUT 5       /* a bounded device wait gave up (see vfv_gmres_opts::wait_limit) */
#define VFV_IO_ERROR 6      /* an output file could not be written (the reference's WriteVtu / WriteCsv, error.rs:116-127) */

/* ---- preconditioners / precisions / orderings */
#define VFV_PRECOND_NONE 0
#define VFV_PRECOND_JACOBI 1 /* the reference's JacobiPreconLinOp (linear_gmres.rs:79) */
#define VFV_PRECOND_ILU0 2   /* added: ILU(0) on A's pattern */
#define VFV_PRECOND_BJ4 3    /* added: 4x4 block-Jacobi over rows {v, N+v, 2N+v, 3N+v} of a field-major
                                [u | v | w | p] system (n = 4N); graph engine only */
#define VFV_FP64 0           /* all Krylov vectors, SpMV and preconditioner in double */
#define VFV_MIXED 1          /* float inner GMRES cycles inside double iterative refinement */
#define VFV_ILU_MULTICOLOR 0 /* ILU(0) of the greedy-multicolour permutation (few levels) */
#define VFV_ILU_NATURAL 1    /* ILU(0) in the given order, level scheduled */
#define VFV_ORTHO_CGS2 0     /* classical Gram-Schmidt, two passes every step (default) */
#define VFV_ORTHO_DGKS 1     /* classical Gram-Schmidt, a second pass only when the first removed more than half of
                                ||w||^2 (Daniel, Gragg, Kaufman & Stewart 1976) */
#define VFV_ORTHO_CGS 2      /* classical Gram-Schmidt, one pass */
#define VFV_ENGINE_PERSISTENT 0 /* one cooperative kernel per restart cycle, grid barriers between phases */
#define VFV_ENGINE_GRAPH 1      /* a CUDA graph of one kernel per phase, replayed per restart cycle (default) */
#define VFV_ENGINE_OVERLAP 2    /* graph engine as flexible GMRES whose ILU(0) sweeps run on a second stream,
                                   overlapped with the orthogonalisation (ILU(0) only) */

/* ---- boundary-condition kinds of the heat operator (SteadyHeat::add_temp_bnd / add_hflx_bnd) */
#define VFV_BC_TEMP 0 /* Dirichlet: OpSclBndDirichlet */
#define VFV_BC_FLUX 1 /* flux: OpSclBndDiffusion + Production + Source + Neumann */

typedef struct vfv_ctx vfv_ctx;
typedef struct vfv_pattern vfv_pattern;
typedef struct vfv_mesh vfv_mesh;
typedef struct vfv_heat vfv_heat;
typedef struct vfv_transport vfv_transport;

/* Options of LinearGmres::new_with_options(num_thread, tol, restart, max_outer)
 * (linear_gmres.rs:24; defaults tol 1e-6, restart 50, max_outer 200 at :20-22).
 * Convergence: ||b - A x||_2 <= tol * ||b||_2, checked on the true double residual after every
 * restart cycle; right preconditioning, so the Arnoldi estimate is of the same residual. */
typedef struct {
    double tol;
    int32_t restart;   /* Krylov dimension m, 1 <= m <= 127 */
    int32_t max_outer; /* maximum number of restart cycles */
    int32_t precond;   /* VFV_PRECOND_* */
    int32_t precision; /* VFV_FP64 or VFV_MIXED */
    int32_t ilu_order; /* VFV_ILU_* (ILU(0) only) */
    int32_t engine;    /* VFV_ENGINE_*: how a restart cycle is launched */
    double inner_rtol; /* VFV_MIXED: an inner cycle also ends once its estimate drops by this factor (0 = full cycles) */
    int64_t wait_limit; /* polls before a bounded device wait gives up (0 = default 20,000,000; any wait also
                           ends after 2 s): the persistent engine's grid barriers, the single-launch
                           ILU(0) sweeps and the dataflow ILU(0) factorisation (orderings with many
                           levels: a warp per row waits for its pivot rows). A wait that gives up makes
                           the solve return VFV_TIMEOUT and leaves the context usable. */
    int32_t ilu_sweeps; /* ILU(0) only: 0 = exact triangular solves (level-scheduled sweeps); k in [1, 16] = k Jacobi
                           sweeps of each factor instead (u = y - N u and w = D^-1 (u - S w), k times each, for
                           L = I + N, U = D + S; Anzt, Chow & Dongarra 2015): a fixed linear preconditioner whose
                           sweeps are one bandwidth-bound launch each. With VFV_ILU_NATURAL they run in A's own
                           numbering. Graph and overlapped engines only. */
    int32_t ilu_sweeps_upper; /* with ilu_sweeps > 0: Jacobi sweeps of the upper factor, in [1, 16] (0 = ilu_sweeps) */
    int32_t ortho;      /* VFV_ORTHO_*: Gram-Schmidt of each Arnoldi step (graph and overlapped engines; batches of
                           meshes and the persistent engine use CGS2) */
    int32_t ilu_sweep_half; /* VFV_MIXED with ilu_sweeps > 0: nonzero stores the swept factors' values in half
                               precision, each row divided by its largest magnitude (kept in float beside it), so
                               every stored value lies in [-1, 1]; the sweeps still compute in float */
} vfv_gmres_opts;

typedef struct {
    int32_t status;   /* VFV_OK / VFV_NOT_CONVERGED / VFV_NONFINITE */
    int32_t iters;    /* total Arnoldi steps */
    int32_t cycles;   /* restart (refinement) cycles */
    int32_t levels;   /* ILU(0) levels of the chosen ordering (0 without ILU) */
    double relres;    /* final ||b - A x|| / ||b|| (double) */
    double bnorm;     /* ||b|| */
} vfv_solve_info;

/* Fills opts with the reference defaults: tol 1e-6, restart 50, max_outer 200, Jacobi, FP64 (graph engine). */
void vfv_gmres_default_opts(vfv_gmres_opts* opts);

/* ---- context */
int vfv_ctx_create(int device, vfv_ctx** out);
void vfv_ctx_destroy(vfv_ctx* ctx);
const char* vfv_last_error(const vfv_ctx* ctx);
int vfv_ctx_synchronize(vfv_ctx* ctx);
/* the context's CUDA stream (cudaStream_t) for callers that enqueue work around the library */
void* vfv_ctx_stream(vfv_ctx* ctx);
/* number of kernels this context has launched so far (every node of a replayed CUDA graph counts) */
int64_t vfv_ctx_launch_count(const vfv_ctx* ctx);

/* ---- sparse pattern: LinearBase::update_sparse (linear_gmres.rs:53-64).
 * rows/cols[ntrip] are the (row, col) pairs of the triplet list in push order. The pattern is
 * the sorted, de-duplicated set (explicit zeros kept); a slot map remembers which triplets fall
 * into each slot so build_matrix sums them in push order. */
int vfv_pattern_from_triplets(vfv_ctx* ctx, int64_t n, int64_t ntrip, const uint64_t* rows, const uint64_t* cols, vfv_pattern** out);
/* a pattern given directly as CSR (rowptr[n+1], colind[nnz] ascending per row); no slot map */
int vfv_pattern_from_csr(vfv_ctx* ctx, int64_t n, const int32_t* rowptr, const int32_t* colind, vfv_pattern** out);
void vfv_pattern_destroy(vfv_pattern* p);
int vfv_pattern_info(const vfv_pattern* p, int64_t* n, int64_t* nnz, int64_t* ntrip);

/* ---- values: LinearBase::build_matrix (linear_gmres.rs:66-74); vals[ntrip] in push order (host) */
int vfv_values_from_triplets(vfv_ctx* ctx, vfv_pattern* p, const double* vals);
/* values given per CSR slot (host or device pointer) */
int vfv_values_set(vfv_ctx* ctx, vfv_pattern* p, const double* vals, int on_device);
/* copy the matrix out (any pointer may be NULL) */
int vfv_csr_export(vfv_ctx* ctx, const vfv_pattern* p, int32_t* rowptr, int32_t* colind, double* vals);

/* ---- solve: LinearBase::solve_matrix (linear_gmres.rs:76-84). b, x0, x are HOST arrays of
 * length n; x0 is the warm start (the previous Picard iterate). x may alias x0. */
int vfv_solve(vfv_ctx* ctx, vfv_pattern* p, const double* b, const double* x0, double* x, const vfv_gmres_opts* opts,
              vfv_solve_info* info);
/* same with DEVICE arrays on the context's device */
int vfv_solve_device(vfv_ctx* ctx, vfv_pattern* p, const double* b, const double* x0, double* x, const vfv_gmres_opts* opts,
                     vfv_solve_info* info);
/* y = A x (device arrays); SpMV of the solver, exposed for measurement */
int vfv_spmv_device(vfv_ctx* ctx, const vfv_pattern* p, const double* x, double* y);
/* y = A x with float values/vectors (the mixed-precision inner SpMV); the float copy of the
 * values is made on first use and refreshed by every vfv_values_* call */
int vfv_spmv_device_f32(vfv_ctx* ctx, vfv_pattern* p, const float* x, float* y);
/* Autotuner: measures the pattern's SpMV in each of its shapes (2 to 32 lanes per row, 1 to 8 strides
 * of indices and values loaded per lane before the gathers; double and float values) and keeps the
 * fastest for every later SpMV and solver of this pattern; call before its first solve. Returns the
 * chosen lanes (either pointer may be NULL). */
int vfv_pattern_autotune(vfv_ctx* ctx, vfv_pattern* p, int32_t* lanes64, int32_t* lanes32);
/* the SpMV shape in use: lanes per row and strides per lane, double and float (pointers may be NULL) */
int vfv_pattern_spmv_shape(const vfv_pattern* p, int32_t* lanes64, int32_t* strides64, int32_t* lanes32, int32_t* strides32);
/* Sets the SpMV lanes per row by hand (2, 4, 8, 16 or 32 each, 4 strides per lane); VFV_BAD_INPUT otherwise. */
int vfv_pattern_set_spmv_lanes(vfv_ctx* ctx, vfv_pattern* p, int32_t lanes64, int32_t lanes32);
/* z = M^-1 r for the ILU(0) preconditioner of the pattern's current values (device arrays, double) */
int vfv_ilu0_apply_device(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, const double* r, double* z, int32_t* levels);
/* z = M^-1 r with the float copy of the factor (the mixed-precision inner preconditioner), exposed
 * for measurement: enqueued on the context's stream without synchronising; t is a work vector of n
 * floats that must not alias r or z (r and z may alias). */
int vfv_ilu0_apply_device_f32(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, const float* r, float* t, float* z, int32_t* levels);
/* z = M^-1 r with `sweeps` (1..16) Jacobi sweeps of each ILU(0) factor (vfv_gmres_opts::ilu_sweeps),
 * in double or with the float copy of the factor; enqueued on the context's stream without
 * synchronisation (calls after the first for a pattern, ordering and precision allocate nothing).
 * r and z may alias. */
int vfv_ilu0_sweep_apply_device(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, int sweeps, const double* r, double* z);
int vfv_ilu0_sweep_apply_device_f32(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, int sweeps, const float* r, float* z);
/* the same with the row-scaled half-precision values of vfv_gmres_opts::ilu_sweep_half */
int vfv_ilu0_sweep_apply_device_f16(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, int sweeps, const float* r, float* z);
/* Storage of the swept factors once built: bytes per column index (2: 16-bit offsets from the row,
 * when the factor's bandwidth allows; 4: absolute). */
int vfv_ilu0_sweep_layout(const vfv_pattern* p, int ilu_order, int32_t* col_bytes);
/* Same result as vfv_ilu0_apply_device, allocating nothing. No counterpart in the reference: for
 * callers that may not allocate device memory while they run (a time-step loop under a fixed
 * memory budget, a host framework whose allocator owns the device memory, code that must not
 * take the device-wide synchronisation of cudaMalloc/cudaFree mid-step). The work vector comes
 * from a fixed 2 MiB device array inside the library, so n is limited to 262,144 rows (larger
 * patterns are rejected with VFV_BAD_INPUT). The pattern's ILU(0) storage must already exist:
 * call vfv_ilu0_apply_device (or an ILU(0) solve) on it once first. The first call on each device
 * looks up the array's device address. Every call synchronises the context's stream before it
 * returns. All calls in the process share the one array on a device: calls that overlap on the GPU
 * race. */
int vfv_ilu0_apply_device_noalloc(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, const double* r, double* z, int32_t* levels);
/* the symmetric permutation the ILU(0) factor lives on: perm[n] (new -> old) and the row ranges of
 * its levels lev_ptr[nlev+1] (any pointer may be NULL; call once with NULLs to learn nlev) */
int vfv_ilu0_ordering(vfv_ctx* ctx, vfv_pattern* p, int ilu_order, int32_t* perm, int32_t* lev_ptr, int32_t* nlev);

/* ---- mesh (host, once per mesh): jittered unit cube, Delaunay, Voronoi dual */
int vfv_mesh_jitter_cube(int n, uint64_t seed, double jitter, vfv_mesh** out);
/* a mesh from given vertices (points first, then nodes with a boundary id each; the vertices' hull
 * must be their bounding box). The Delaunay predicates give exact signs for any finite coordinates
 * (the reference's robust orient3d / insphere, delaunay.rs:1,10): integer arithmetic for vertices
 * on the 2^-18 lattice within a box of 1.75, else filtered double arithmetic with an exact
 * big-integer fallback. Coordinates must be finite and at most 1e50 in magnitude (VFV_BAD_INPUT). */
int vfv_mesh_from_vertices(int64_t n_pts, int64_t n_nds, const double* pos, const int32_t* node_bnd, vfv_mesh** out);
void vfv_mesh_destroy(vfv_mesh* m);

/* ---- output (host): the reference's VTU and CSV files, byte for byte (numbers as Rust's {:.9}).
 * path is the whole file name (the reference forms "<name>_<ts:04>.<type>", scl_dom.rs:60-62 and
 * write_vtu.rs:7). VFV_IO_ERROR when the file cannot be written, VFV_BAD_INPUT for bad arguments. */
/* A field over the mesh's vertices (points, then nodes) with its tetrahedra: write_scldom_vtu
 * (ncomp 1) and write_vecdom_vtu (ncomp 3), src/base/write_vtu.rs:5,192. values: [n_tot][ncomp]. */
int vfv_mesh_write_vtu(const vfv_mesh* m, const double* values, int ncomp, const char* path);
/* The same field as CSV lines: write_scldom_csv / write_vecdom_csv, src/base/write_csv.rs:5,68. */
int vfv_mesh_write_csv(const vfv_mesh* m, const double* values, int ncomp, const char* path);
/* A field on n vertices at pos[n][3] (a boundary's or interface's nodes), one vertex cell each:
 * write_sclbnd_vtu / write_vecbnd_vtu / write_vecitf_vtu (write_vtu.rs:71,259,322); values NULL writes
 * the empty value array of write_sclitf_vtu (write_vtu.rs:133). */
int vfv_points_write_vtu(int64_t n, const double* pos, const double* values, int ncomp, const char* path);
/* The same as CSV lines: write_sclbnd_csv, write_sclitf_csv, write_vecbnd_csv, write_vecitf_csv
 * (write_csv.rs:30,49,93,112). */
int vfv_points_write_csv(int64_t n, const double* pos, const double* values, int ncomp, const char* path);
/* Recomputes the mesh's Voronoi dual from its tetrahedra on the device of ctx (Tetrahedron::update_tet,
 * src/base/geom_tet.rs:122-293: face pieces, sorted-edge sums, control volumes, boundary sub-faces,
 * least-squares weights); the result equals the host dual bit for bit and replaces it. */
int vfv_mesh_dual_device(vfv_ctx* ctx, vfv_mesh* m);
/* vfv_mesh_jitter_cubes with the duals built on the device (Delaunay on the host, meshes in parallel) */
int vfv_mesh_jitter_cubes_device_dual(vfv_ctx* ctx, int count, const int32_t* n, const uint64_t* seeds, double jitter, vfv_mesh** out);
/* count meshes at once (built in parallel on the host): out[i] = jitter cube of n[i]^3 points, seeds[i] */
int vfv_mesh_jitter_cubes(int count, const int32_t* n, const uint64_t* seeds, double jitter, vfv_mesh** out);
/* counts: vertices split, tetrahedra, directed faces (2 x Voronoi faces), boundary sub-faces */
int vfv_mesh_info(const vfv_mesh* m, int64_t* n_pts, int64_t* n_nds, int64_t* n_tet, int64_t* n_dir, int64_t* n_bsub);
/* copy arrays out; any pointer may be NULL. Vector quantities are component-major [3][count]. */
int vfv_mesh_export(const vfv_mesh* m, double* pos, int32_t* node_bnd, int32_t* tets);
int vfv_mesh_export_dual(const vfv_mesh* m, int64_t* nbr_ptr, int32_t* nbr_idx, double* dist, double* area, double* norm,
                         double* skew, double* grad_wgt, double* cvol, double* cskew, int64_t* bnd_ptr, int32_t* bnd_j,
                         int32_t* bnd_k, double* bnd_area, double* bnd_norm, double* bnd_wgt);

/* ---- steady heat operator on the device (SteadyHeat with one domain, steady_heat.rs:80-171).
 * bnd_kind[b] is VFV_BC_TEMP or VFV_BC_FLUX for every boundary id used by the mesh nodes. The
 * matrix pattern is fixed at creation; vfv_heat_pattern returns it (owned by the heat handle). */
int vfv_heat_create(vfv_ctx* ctx, const vfv_mesh* m, int32_t n_bnd, const int32_t* bnd_kind, vfv_heat** out);
void vfv_heat_destroy(vfv_heat* h);
vfv_pattern* vfv_heat_pattern(vfv_heat* h);
/* Gradients of k (conductivity), q (source), s (production) and T (unknown), then the matrix
 * values and b. k, q, s, T, bc_val are arrays of n_tot doubles (bc_val: Dirichlet value or outward
 * flux on nodes, ignored on points); on_device selects device (1) or host (0) pointers. b_out may
 * be NULL (b stays on the device, see vfv_heat_rhs_device). */
int vfv_heat_assemble(vfv_ctx* ctx, vfv_heat* h, const double* k, const double* q, const double* s, const double* T,
                      const double* bc_val, int on_device, double* b_out);
/* device pointer of the assembled right-hand side (n_tot doubles, owned by h) */
const double* vfv_heat_rhs_device(vfv_heat* h);
/* Adjoint gradient of an objective J(T) of the heat solution (zero production, s = 0), the
 * backward() of the assembly + solve: solves A^T lambda = dJ/dT with GMRES (opts) and returns
 * dJ/d(log k) and dJ/dq per vertex, for the k, q of the last vfv_heat_assemble. Host arrays of
 * n_tot doubles; lambda, dJdlogk, dJdq may be NULL. No reference counterpart (the reference has no
 * adjoint); its operators are the ones of SteadyHeat::assemble_matrix, steady_heat.rs:143-171. */
int vfv_heat_adjoint(vfv_ctx* ctx, vfv_heat* h, const double* T, const double* dJdT, const vfv_gmres_opts* opts, double* lambda,
                     double* dJdlogk, double* dJdq, vfv_solve_info* info);
/* gradient of one field on the heat mesh: grad[3][n_tot] (host arrays) */
int vfv_update_grad(vfv_ctx* ctx, vfv_heat* h, const double* f, double* grad);

/* ---- batched transient transport: one species, implicit Euler, zero-flux walls.
 * The meshes are concatenated into one block-diagonal system; every kernel runs over all of them.
 * Per row, in push order: OpSclDomTimeUnity (opscl_dom_timeunity.rs:32-58), OpSclDomDiffusion
 * (opscl_dom_diff.rs:40-91), OpSclDomAdvection (power law, opscl_dom_adv.rs:49-125) with the face mass
 * flux of flow_helper::update_flux (flow_helper.rs:72-179) at zero pressure and body force; density
 * and species weight 1. The reference has no solver that wires this composition (TransientMass has
 * no advection). */
int vfv_transport_create(vfv_ctx* ctx, int nmesh, vfv_mesh* const* meshes, double dt, vfv_transport** out);
void vfv_transport_destroy(vfv_transport* t);
vfv_pattern* vfv_transport_pattern(vfv_transport* t);
/* row_ptr[nmesh+1] (may be NULL): row offsets of the meshes in the concatenated system */
int vfv_transport_info(const vfv_transport* t, int64_t* n_tot, int64_t* nnz, int32_t* nmesh, int64_t* row_ptr);
/* matrix from the diffusivity D[n_tot] and velocity vel[3][n_tot] (host or device arrays) */
int vfv_transport_assemble(vfv_ctx* ctx, vfv_transport* t, const double* D, const double* vel, int on_device);
/* nsteps implicit-Euler steps from c0 (host, n_tot) to c_out (host). Per step one batched GMRES in
 * which every mesh has its own Krylov recurrence (its own dot products, Hessenberg matrix, Givens
 * rotations and stopping test, as if it were solved alone: TransientBase::solve solves each system
 * by itself, src/transient/transient_base.rs:83-109), converged when every mesh meets
 * ||b_i - A_i c_i|| <= tol ||b_i||; a mesh that has converged is masked out of the orthogonalisation.
 * The graph engine is used whatever opts->engine says. iters[nsteps] (may be NULL): Arnoldi steps of
 * the batch per time step (a step counts while any mesh is active). */
int vfv_transport_run(vfv_ctx* ctx, vfv_transport* t, const double* c0, int nsteps, const vfv_gmres_opts* opts, double* c_out,
                      int32_t* iters);
/* Arnoldi steps of every mesh summed over the time steps of the last vfv_transport_run (steps[nmesh]) */
int vfv_transport_mesh_steps(const vfv_transport* t, int64_t* steps);
/* Transient adjoint (no reference counterpart): J = 0.5 ||c_nsteps - target||^2 and dJ/dD for the
 * uniform diffusivity D of the last vfv_transport_assemble. Forward states are checkpointed every
 * `every` steps and recomputed segment by segment during the backward sweep of transposed solves.
 * adj_iters (may be NULL): nsteps entries, [k] = GMRES iterations of the transposed solve giving
 * lambda_{k+1}. */
int vfv_transport_adjoint_D(vfv_ctx* ctx, vfv_transport* t, const double* c0, int nsteps, int every, const double* target,
                            const vfv_gmres_opts* opts, double* J, double* dJdD, int32_t* adj_iters);

/* ---------------------------------------------------------------- coupled Navier-Stokes (SteadyFlow)
 * The field-major [u | v | w | p] system (n = 4 N unknowns) of SteadyFlow::assemble_matrix
 * (src/steady/core/steady_flow.rs:255-303) for one domain whose six faces are velocity boundaries
 * (OpVecBndDirichlet + OpSclBndDivergence + OpSclBndPressureStabilizer per boundary) and whose
 * pressure is fixed at one vertex (OpSclDomPressureReference, opscl_dom_pref.rs:40-64), with the
 * Rhie-Chow flow data of flow_helper::update_flow (src/operator/core/flow_helper.rs:3-179). Pattern:
 * bit-exact to the reference's triplet build; values: the row's triplets summed in push order. */
typedef struct vfv_flow vfv_flow;

/* Symbolic setup only, on the host (no device): nnz and triplet count of the system, and its CSR
 * pattern when rowptr [4N+1] / colind [nnz] are given. Replaces update_sparse for this system. */
int vfv_flow_pattern_host(const vfv_mesh* mesh, int64_t pref_vid, int64_t* nnz, int64_t* ntrip, int32_t* rowptr, int32_t* colind);
/* rho, mu [N]; fce, bc_vel [3][N] (body force rho g; boundary velocity at node vertices);
 * pref_vid: vertex whose pressure row becomes p = pref. Every node must lie on a boundary. */
int vfv_flow_create(vfv_ctx* ctx, const vfv_mesh* mesh, const double* rho, const double* mu, const double* fce, const double* bc_vel,
                    int64_t pref_vid, double pref, vfv_flow** out);
void vfv_flow_destroy(vfv_flow* f);
vfv_pattern* vfv_flow_pattern(vfv_flow* f); /* owned by the flow handle */
int vfv_flow_info(const vfv_flow* f, int64_t* n_unknowns, int64_t* nnz, int64_t* ntrip);
/* A(x), b(x) at the state x = [u | v | w | p] (update_grad, update_flow, assemble_matrix,
 * build_matrix of steady_base.rs:60-66 / :86-91); b may be NULL. Host or device pointers. */
int vfv_flow_assemble(vfv_ctx* ctx, vfv_flow* f, const double* x, double* b);
int vfv_flow_assemble_device(vfv_ctx* ctx, vfv_flow* f, const double* x_dev, double* b_dev);
/* Damped Picard iteration of SteadyBase::solve (src/steady/steady_base.rs:70-112): per iteration
 * assemble at x, solve A x_u = b with x as the initial guess, x = (1 - damp) x + damp x_u, and the
 * scaled change of scaled_residual (src/base/scaling.rs:113-136); stops below tol. x (host, [4N])
 * holds the initial state (boundary velocities loaded) and receives the result. res, lin_iters
 * (max_iter entries) may be NULL. solve_seconds: device time of the linear solves. Errors as the
 * reference: SolverNonPositiveMaxIter / SolverNonPositiveTolerance / SolverInvalidDamping ->
 * VFV_BAD_INPUT, SteadyNonFiniteResidual -> VFV_NONFINITE, SteadyDidNotConverge -> VFV_NOT_CONVERGED. */
int vfv_flow_picard(vfv_ctx* ctx, vfv_flow* f, double* x, int max_iter, double tol, double damp, const vfv_gmres_opts* opts,
                    double* res, int32_t* lin_iters, int32_t* iters_done, double* solve_seconds);

#ifdef __cplusplus
}
#endif

#endif /* VFV_GPU_H */
