/*
 * C ABI of libfpb200.so: the B200 (sm_100a) composite-geometry FFT / domain-decomposition Poisson
 * solve of Focalors_Poisson's 2D path.
 *
 * Conventions
 *   - Fields are row-major nx x ny float64 (or float32) arrays, value(i, j) = f[i*ny + j], exactly the
 *     reference's field2 layout (base/field/field2.cpp:304-314).
 *   - Boundary codes are the reference's PDEBoundaryType values (base/location_boundary.h:62-69):
 *     0 Dirichlet, 1 Neumann, 2 Periodic, 3 Adjacented; faces are its LocationType order
 *     (base/location_boundary.h:8-16): 0 XNegative, 1 XPositive, 2 YNegative, 3 YPositive.
 *   - Every entry point returns an fp_status; no C++ exception crosses the ABI. fp_last_error()
 *     describes the last failure on the calling thread.
 *   - Pointers are host memory unless FP_DEVICE is set in `flags`, in which case they are device
 *     memory and the work is queued on `stream` (a cudaStream_t, NULL = legacy default stream) without
 *     a host synchronisation unless FP_SYNC is also set. Host-pointer calls are synchronous.
 *   - There is no CPU fallback: without a usable CUDA device every compute call fails with
 *     FP_ERR_CUDA.
 */
#ifndef FP_CAPI_H
#define FP_CAPI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fp_status
{
    FP_OK                = 0,
    FP_ERR_INVALID       = 1, /* bad argument, unsupported boundary combination, bad geometry */
    FP_ERR_CUDA          = 2, /* CUDA runtime error (no device, launch failure, ...) */
    FP_ERR_UNSUPPORTED   = 3, /* size beyond what this build supports */
    FP_ERR_NOT_CONVERGED = 4, /* GMRES stopped at max_iter above tol (result still written) */
    FP_ERR_NAN           = 5, /* non-finite value met */
    FP_ERR_NOMEM         = 6  /* device allocation failed */
} fp_status;

#define FP_DEVICE 1 /* pointers are device memory, work queued on `stream` */
#define FP_SYNC 2   /* synchronise `stream` before returning */

#define FP_F64 0
#define FP_F32 1

/* Message for the last failing call on this thread ("" if none). */
const char* fp_last_error(void);

/* Number of CUDA kernels this library has launched in the process so far (all threads). */
long long fp_launch_count(void);

/* ---------------------------------------------------------------------------------------------
 * y-direction transforms: PoissonFFT2D_{DD,NN,ND,DN,PP}::transform / transform_transpose
 * (reference pe/poisson/poisson_fft2d.h:8-136, pe/poisson/poisson_fft2d.cpp:19-465). The family is
 * chosen from the y boundary pair like PoissonSolver2DBase::create_fft
 * (pe/poisson/poisson_solver2d_base.cpp:64-91). `in` and `out` may alias.
 * ------------------------------------------------------------------------------------------- */
int fp_transform_f64(int bc_yneg, int bc_ypos, int nx, int ny, int inverse, const double* in, double* out,
                     int flags, void* stream);
int fp_transform_f32(int bc_yneg, int bc_ypos, int nx, int ny, int inverse, const float* in, float* out,
                     int flags, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Single rectangle: PoissonSolver2D(nx, ny, hx, hy, bc_xneg, bc_xpos, bc_yneg, bc_ypos) and its
 * solve(field2&) (reference pe/poisson/poisson_solver2d.h:10-34, pe/poisson/poisson_solver2d.cpp:3-90):
 * forward y-transform, one tridiagonal "chasing" solve per wavenumber along x, inverse transform.
 * bc[4] in face order. `batch` fields are stored back to back (batch * nx * ny values), solved in
 * place.
 * ------------------------------------------------------------------------------------------- */
typedef struct fp_rect fp_rect;

int fp_rect_create(int nx, int ny, double hx, double hy, const int* bc, int precision, fp_rect** out);
int fp_rect_solve_f64(fp_rect* r, double* f, long long batch, int flags, void* stream);
int fp_rect_solve_f32(fp_rect* r, float* f, long long batch, int flags, void* stream);
/* The chasing step of PoissonSolver2D::solve alone (ChasingMethod2D::chasing, reference
 * pe/poisson/chasing_method2d.cpp:3-89): every wavenumber's tridiagonal system along x solved in place on
 * fields that are already in the y-transformed space, FP_F64 solvers. Same pointer and stream semantics as
 * fp_rect_solve_f64. */
int fp_rect_chase_f64(fp_rect* r, double* f, long long batch, int flags, void* stream);
int fp_rect_destroy(fp_rect* r);

/* fp_rect_solve_f64 for callers that cannot allocate device memory when they solve: code whose device
 * memory belongs to another allocator (a framework's caching allocator, a fixed memory budget), where a
 * library cudaMalloc would fail or synchronise the device behind that allocator. No counterpart in the
 * reference (its solve is host-only). Same result as fp_rect_solve_f64 with FP_DEVICE: `f` is device memory, the work is queued on `stream`, nothing is
 * allocated or freed. Its scratch is one fixed device array of 2^21 doubles (16 MiB) that every GPU
 * loading the library holds until exit; solves needing more (4 * batch * (nx/32) * ny doubles when nx
 * is a multiple of 32, none otherwise) are rejected with FP_ERR_UNSUPPORTED. The first call on a
 * device looks the array's address up (do it before any stream capture); calls that overlap on the GPU
 * share the array and race. `r` must be an FP_F64 solver. */
int fp_rect_solve_f64_noalloc(fp_rect* r, double* f, long long batch, void* stream);

/* ---------------------------------------------------------------------------------------------
 * 3D rectangle: PoissonSolver3D(nx, ny, nz, hx, hy, hz, 6 x PDEBoundaryType) and its solve(field3&)
 * (reference pe/poisson/poisson_solver3d.h:10-37, pe/poisson/poisson_solver3d.cpp:3-123): z-transform,
 * y-transform, one tridiagonal solve per (z, y) mode pair along x, inverse transforms. Fields are field3
 * arrays, value(i, j, k) = f[(i*ny + j)*nz + k] (base/field/field3.cpp:378-388); bc[6] in the order x-, x+,
 * y-, y+, z-, z+. `batch` fields back to back, solved in place; pointer and stream semantics as
 * fp_rect_solve_f64.
 * ------------------------------------------------------------------------------------------- */
typedef struct fp_rect3d fp_rect3d;

int fp_rect3d_create(int nx, int ny, int nz, double hx, double hy, double hz, const int* bc, fp_rect3d** out);
int fp_rect3d_solve_f64(fp_rect3d* r, double* f, long long batch, int flags, void* stream);
int fp_rect3d_destroy(fp_rect3d* r);

/* ---------------------------------------------------------------------------------------------
 * Composite geometry: Geometry2D + Variable2D + ConcatPoissonSolver2D (reference
 * base/domain/geometry2d.h:15-59, pe/concat/concat_solver2d.h:18-56): a tree of rectangles coupled
 * through shared faces, solved by block elimination with a Schur-complement GMRES at every internal
 * node (pe/concat/gmres_solver2d.cpp:123-252). The Schur matrices (pe/concat/schur_mat2d.cpp:5-106)
 * are built at creation by batched unit-impulse solves on the device.
 * ------------------------------------------------------------------------------------------- */
typedef struct fp_composite fp_composite;

typedef struct fp_geometry
{
    int           n_domains;
    const int*    nx;          /* cells per domain along x */
    const int*    ny;          /* cells per domain along y */
    const double* hx;          /* grid spacing per domain */
    const double* hy;
    const int*    bc;          /* 4 per domain, face order; faces named by a connection become Adjacented */
    int           n_connections;
    const int*    connections; /* 3 per connection (a, face of a, b): Geometry2D::connect(a, face, b) */
    int           root;        /* -1: tree centre as TreeUtils::findOptimalRoot (ties -> lower index) */
} fp_geometry;

typedef struct fp_solve_info
{
    int    gmres_iterations; /* Arnoldi steps of the root GMRES in this solve */
    int    gmres_restarts;   /* restart cycles of the root GMRES */
    double gmres_residual;   /* last residual norm / estimate of the root GMRES */
    int    converged;        /* 1 if every GMRES met its tolerance */
    int    refinements;      /* fp_composite_solve_f32ir: refinement steps taken */
    double rel_change;       /* fp_composite_solve_f32ir: last |correction| / |solution| (L2 over all cells) */
} fp_solve_info;

#define FP_GMRES_FULLFIELD 4 /* create flag: Krylov vectors are full fields, as the reference */
#define FP_CHECK_CONVERGENCE 8 /* solve flag: return FP_ERR_NOT_CONVERGED when GMRES missed tol */
/* create flag: do not build the interface inverse. By default every internal node with at most 16384
 * interface cells gets the inverse of its dense interface operator I - P A^-1 S (batched rectangle
 * solves + Newton-Schulz on the device at creation); a solve then starts from y = X g and refines while
 * the reference's full-field residual test fails, falling back to plain GMRES. */
#define FP_NO_INTERFACE_INVERSE 16
/* create flag: never use the spectral direct path. By default a geometry inside that path's scope (see
 * fp_batch_create: a Dirichlet root with leaves on full faces, nx of every subdomain a multiple of 32 and
 * >= 64) is solved by the exact spectral interface solve of the batched solver, one transform pass per
 * subdomain each way, instead of the Schur GMRES; the answer is the converged solution of the reference's
 * GMRES, so its GMRES parameters do not apply (fp_solve_info reports 0 iterations). */
#define FP_NO_SPECTRAL 512

/* Creation builds the tree, the per-domain rectangle plans and every Schur matrix. Defaults of the
 * reference: m = 20, tol = 1e-8, max_iter = 100 (concat_solver2d.h:48-50). */
int fp_composite_create(const fp_geometry* g, int m, double tol, int max_iter, int flags, fp_composite** out);
/* ConcatPoissonSolver2D::set_parameter (concat_solver2d.cpp:7-17). */
int fp_composite_set_parameter(fp_composite* c, int m, double tol, int max_iter);
/* ConcatPoissonSolver2D::solve: fields[d] (RHS in, solution out, in place); ghosts[4*d + face] are the
 * Variable2D ghost buffers (NULL = zero), length ny for x faces and nx for y faces. */
int fp_composite_solve_f64(fp_composite* c, double* const* fields, const double* const* ghosts, int flags,
                           void* stream, fp_solve_info* info);
/* The same problem by mixed-precision iterative refinement (no counterpart in the reference, which is
 * FP64 only): inner solves with FP32 transforms (FP64 rows, FP64 chase, FP64 interface operations),
 * the FP64 residual of the composite 5-point operator, until |correction| <= rel_tol |solution| (or
 * the observed contraction predicts the error left after the last correction is below rel_tol) or
 * max_refine steps (FP_ERR_NOT_CONVERGED with FP_CHECK_CONVERGENCE if the target was missed).
 * With FP_IR_INNER_F64 the inner solves are the FP64 ones (refinement then only removes the single
 * FP64 solve's round-off, about eps * cond(A)). Device-resident fields hold the iterate while the
 * refinement runs (their right-hand sides are kept in an assembled copy), so after an error they hold
 * neither the right-hand side nor a finished solution. */
#define FP_IR_INNER_F64 32
/* With FP32 inner solves: make the first inner solve the FP64 one (its answer already carries only FP64
 * round-off, eps * cond(A)), so that one or two FP32 corrections finish the refinement. Spectral path only;
 * ignored on the Schur GMRES path. */
#define FP_IR_FIRST_F64 1024
int fp_composite_solve_f32ir(fp_composite* c, double* const* fields, const double* const* ghosts, int flags,
                             void* stream, double rel_tol, int max_refine, fp_solve_info* info);
/* Adjoint (transposed) solve of the map rhs -> solution with the ghost buffers held fixed: the gradient
 * of a loss L(u) with respect to the right-hand side is fp_composite_adjoint_*(dL/du). In place:
 * fields <- H A^-1 fields, H = diag(hx_d^2) per domain, A the composite 5-point operator that
 * ConcatPoissonSolver2D::solve inverts (pe/concat/concat_solver2d.cpp:101-157), which is symmetric, so
 * the transposed solve runs through the same kernels as the forward one. No counterpart in the reference
 * (it has no gradients). Geometries without a Dirichlet face (singular A) give FP_ERR_UNSUPPORTED.
 * _f32ir: by iterative refinement, same rel_tol / max_refine / FP_IR_INNER_F64 meaning as
 * fp_composite_solve_f32ir. Same host/device field semantics as the solves. */
int fp_composite_adjoint_f64(fp_composite* c, double* const* fields, int flags, void* stream, fp_solve_info* info);
int fp_composite_adjoint_f32ir(fp_composite* c, double* const* fields, int flags, void* stream, double rel_tol,
                               int max_refine, fp_solve_info* info);
/* Pipelined solves of a stream of independent problems with HOST buffers (no counterpart in the reference,
 * whose ConcatPoissonSolver2D::solve is synchronous): the call queues the host-to-device copy of rhs (and of
 * the ghost buffers), the solve in the given form and the device-to-host copy of the solution into out, and
 * returns without waiting; fp_composite_wait waits for every queued call. Consecutive calls overlap: while
 * one problem is solved, the next one's right-hand sides are copied in and the previous one's solution is
 * copied out (two device slots, one copy stream each way; the solve runs on `stream`). rhs[d], out[d]: host
 * arrays of nx*ny doubles per subdomain, out may equal rhs; page-locked host memory lets the copies overlap
 * the solves (pageable memory gives the same results without the overlap). The host arrays of a queued call
 * must not be modified or read before fp_composite_wait returns. A call whose rhs or ghost pointer is the out
 * pointer of a queued call reads it after that call's copy out; other overlaps between calls' host arrays are
 * the caller's to avoid. Forms:
 *   FP_FORM_F64      one FP64 solve (fp_composite_solve_f64)
 *   FP_FORM_F64IR    refinement with FP64 inner solves (fp_composite_solve_f32ir with FP_IR_INNER_F64)
 *   FP_FORM_F32IR    refinement with FP32 inner solves (fp_composite_solve_f32ir)
 *   FP_FORM_MIXEDIR  the FP64 solve, then FP32 corrections (fp_composite_solve_f32ir with FP_IR_FIRST_F64)
 * rel_tol and max_refine as for fp_composite_solve_f32ir (ignored by FP_FORM_F64). On the spectral path
 * nothing in the call waits for the device (with max_refine > 1 the refinement's loop runs inside a CUDA
 * graph); on the Schur GMRES path the solve synchronises the stream, so only the copies overlap. Every
 * other call on this solver first waits for the queued ones. */
#define FP_FORM_F64 0
#define FP_FORM_F64IR 1
#define FP_FORM_F32IR 2
#define FP_FORM_MIXEDIR 3
int fp_composite_solve_async(fp_composite* c, const double* const* rhs, double* const* out,
                             const double* const* ghosts, int form, double rel_tol, int max_refine, void* stream);
/* Waits for the calls queued by fp_composite_solve_async. info: the last queued call's refinement steps and
 * change (and GMRES figures on the Schur path). FP_CHECK_CONVERGENCE in flags as for the solves; FP_ERR_NAN if
 * any queued refinement met a non-finite value. Returns FP_OK at once when nothing is queued. */
int fp_composite_wait(fp_composite* c, int flags, fp_solve_info* info);
/* Subtree decomposition over GPUs (one process per GPU; the analogue of the reference's MPI decomposition of
 * the composite solve, pe/concat/concat_solver2d_slab_x.cpp, for a tree): the root domain is one part, and each
 * subtree under a child of the root is a part of its own, solved by the same algorithm as
 * ConcatPoissonSolver2D::solve (concat_solver2d.cpp:101-157) split at the root's faces. Per solve every subtree
 * part sends the root one interface vector (its solved copy along the shared face) and receives one back (the
 * root's solution along that face); the root part's GMRES needs the children's Schur matrices only, which the
 * subtree parts compute once (fp_composite_part_schur) and the root part receives at set-up. The results are
 * those of the undivided Schur GMRES solve (FP_NO_SPECTRAL). Device pointers only; all parts use the same
 * m, tol, max_iter.
 *   fp_composite_part_create: a subtree part is the subtree's geometry with its root's face toward the root
 *     domain marked Adjacented (3) and n_ext = 0; the root part is the root domain alone (root = 0) with its
 *     n_ext children in other parts given by the root's faces, in increasing face order. */
int fp_composite_part_create(const fp_geometry* g, int m, double tol, int max_iter, int flags, int n_ext,
                             const int* ext_faces, fp_composite** out);
/* Subtree part: S (cn x cn device doubles, cn = the face's length) = the Schur matrix of the part's root toward
 * the root domain across `face` (SchurMat2D_*::construct, schur_mat2d.cpp:5-106). */
int fp_composite_part_schur(fp_composite* c, int face, double* S, void* stream);
/* Root part: the Schur matrix of external child k (index in face order). */
int fp_composite_set_external_schur(fp_composite* c, int k, const double* S);
/* Subtree part, first half of a solve: boundary assembly, hx^2 scaling, the upward pass including the part's
 * root; edge_out (cn doubles) = the part root's solved copy along `face`. */
int fp_composite_part_upward(fp_composite* c, double* const* fields, const double* const* ghosts, int face,
                             double* edge_out, void* stream, fp_solve_info* info);
/* Subtree part, second half: the part root's field loses parent_edge (the root domain's solution along the
 * shared face) along `face`, then the part root's solve and the downward pass. */
int fp_composite_part_downward(fp_composite* c, double* const* fields, int face, const double* parent_edge,
                               void* stream, fp_solve_info* info);
/* Root part: assembly, scaling, child_edges[k] subtracted along external child k's face, the root's GMRES solve;
 * edges_out[k] = the root's solution along child k's face (for that child's part_downward). */
int fp_composite_root_solve(fp_composite* c, double* const* fields, const double* const* ghosts,
                            const double* const* child_edges, double* const* edges_out, void* stream,
                            fp_solve_info* info);
/* Relative residual |fs - A u| / |fs| of a candidate solution u of the composite problem with right-hand
 * side `rhs` and ghost buffers `ghosts` (fs = their assembled, hx^2-scaled form, the right-hand side
 * ConcatPoissonSolver2D::solve works on; A = its composite 5-point operator). No counterpart in the
 * reference; used to check solutions. Device pointers only (FP_DEVICE semantics); nothing is modified. */
int fp_composite_residual(fp_composite* c, const double* const* u, const double* const* rhs,
                          const double* const* ghosts, void* stream, double* rel_residual);
/* Tree actually used: root index and BFS level of every domain (root = 0). */
int fp_composite_tree(const fp_composite* c, int* root, int* level_of);
int fp_composite_destroy(fp_composite* c);

/* ---------------------------------------------------------------------------------------------------
 * 3D composite solve: ConcatPoissonSolver3D (reference pe/concat/concat_solver3d.cpp:5-247) over a tree of
 * boxes connected on whole faces (Geometry3D::connect, base/domain/geometry3d.cpp:27-60), each box solved by
 * PoissonSolver3D and every box with children by GMRESSolver3D (pe/concat/gmres_solver3d.cpp:155-306) with the
 * Schur matrices of SchurMat3D_* (pe/concat/schur_mat3d.cpp), built on the device at creation.
 * A field holds nx*ny*nz doubles, value(i, j, k) = f[(i*ny + j)*nz + k] (base/field/field3.cpp:378-388).
 * Faces (LocationType order): 0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+. */
typedef struct fp_geometry3
{
    int           n_domains;
    const int*    nx;          /* per domain */
    const int*    ny;
    const int*    nz;
    const double* hx;          /* per domain (lx / nx) */
    const double* hy;
    const double* hz;
    const int*    bc;          /* 6 per domain (PDEBoundaryType), ignored on connected faces */
    int           n_connections;
    const int*    connections; /* 3 per connection: a, face of a, b (Geometry3D::connect(a, face, b));
                                  the connected faces must have the same cell counts */
    int           root;        /* -1: the reference's rule (TreeUtils::findOptimalRoot) */
} fp_geometry3;
typedef struct fp_composite3d fp_composite3d;

/* Builds the tree, the per-box 3D rectangle plans and every Schur matrix (ConcatPoissonSolver3D constructor
 * with set_parameter(m, tol, max_iter); the reference's defaults are m = 20, tol = 1e-8, max_iter = 100). */
int fp_composite3d_create(const fp_geometry3* g, int m, double tol, int max_iter, fp_composite3d** out);
/* ConcatPoissonSolver3D::set_parameter (concat_solver3d.cpp:5-18): the Schur matrices are built again. */
int fp_composite3d_set_parameter(fp_composite3d* c, int m, double tol, int max_iter);
/* ConcatPoissonSolver3D::solve: fields[d] (RHS in, solution out, in place); ghosts[6*d + face]: the Variable3D
 * ghost planes (NULL = zero), row-major (ny, nz) on x faces, (nx, nz) on y faces, (nx, ny) on z faces. Host
 * pointers, or device pointers with FP_DEVICE (FP_SYNC, FP_CHECK_CONVERGENCE as for the 2D solves); info: the
 * root GMRES's iterations, restarts, last residual and convergence. */
int fp_composite3d_solve_f64(fp_composite3d* c, double* const* fields, const double* const* ghosts, int flags,
                             void* stream, fp_solve_info* info);
/* Tree actually used: root index and BFS level of every domain (root = 0). */
int fp_composite3d_tree(const fp_composite3d* c, int* root, int* level_of);
int fp_composite3d_destroy(fp_composite3d* c);

/* ---------------------------------------------------------------------------------------------------
 * Batched composite solves: many independent ConcatPoissonSolver2D problems of uneven sizes solved
 * together (pe/concat/concat_solver2d.cpp:101-157 per problem), every stage one launch over all problems.
 * No counterpart in the reference, which solves one geometry per solver object; each problem is what a
 * ConcatPoissonSolver2D over that geometry computes (the converged solution of its Schur GMRES).
 * Supported problems: a root rectangle with Dirichlet faces and leaf rectangles attached on full faces
 * (depth-1 tree: L, T, cross), each leaf's sides along its interface Dirichlet and its far face Dirichlet
 * or Neumann, nx of every subdomain a multiple of 32 and >= 64; others give FP_ERR_UNSUPPORTED. The interface system is solved exactly in the DST bases (closed-form responses,
 * one dense reduced system per problem whose inverse is built at creation).
 * ------------------------------------------------------------------------------------------------- */
typedef struct fp_batch fp_batch;
#define FP_BATCH_F32 64          /* create flag: FP32 storage and arithmetic in the inner solves */
#define FP_BATCH_NO_AUTOTUNE 128 /* create flag: keep the default launch shapes (no timing at creation) */
#define FP_BATCH_GRAPH 256       /* solve flag: capture the launch sequence into a CUDA graph once per
                                    (field pointers, steps) and replay it on later calls */
/* problems[p].root is ignored (the reference's rule picks the root). */
int fp_batch_create(const fp_geometry* problems, int n_problems, int flags, fp_batch** out);
/* fields: device pointers (FP_DEVICE required), one per subdomain, problems back to back in creation
 * order; solved in place. ghosts: 4 device pointers per subdomain (or null entries / null). steps == 0:
 * one solve in the storage precision; steps >= 1: that many inner solves in FP64 iterative refinement
 * (FP64 residual of the composite operator). Queued on `stream`; FP_SYNC waits. */
int fp_batch_solve(fp_batch* b, double* const* fields, const double* const* ghosts, int flags, void* stream,
                   int steps);
/* Per-problem |fs - A u| / |fs| (as fp_composite_residual); rel_residuals: host array of n_problems. */
int fp_batch_residuals(fp_batch* b, const double* const* u, const double* const* rhs, const double* const* ghosts,
                       void* stream, double* rel_residuals);
/* Counts, the autotuned launch shape (DST threads per CTA, DST CTAs per SM of a persistent grid or 1 << 20 for
 * one CTA per work item, chase threads per CTA) and the number of kernels in the captured graph (0 before the
 * first FP_BATCH_GRAPH solve). */
int fp_batch_info(const fp_batch* b, int* n_problems, int* n_domains, int* launch_shape, long long* graph_kernels);
int fp_batch_destroy(fp_batch* b);

/* ---------------------------------------------------------------------------------------------------
 * Device-side field set-up: Variable2D::set_value and Variable2D::set_buffer_value (reference
 * base/domain/variable2d.cpp:345-416, 467-511) for analytic functions, evaluated on the device so that a
 * right-hand side or ghost buffer need not be filled on the host and copied. The function is a sum of up to
 * 48 separable terms  a * X(x) * Y(y), each factor one of
 *   FP_FACTOR_ONE        1
 *   FP_FACTOR_SIN        sin(p0 t + p1)
 *   FP_FACTOR_COS        cos(p0 t + p1)
 *   FP_FACTOR_GAUSS      exp(-((t - p0) / p1)^2)
 *   FP_FACTOR_QUADRATIC  p0 + p1 t + p2 t^2
 * Positions follow the reference's variable positions: value (i, j) sits at (ox + (i + sx) hx,
 * oy + (j + sy) hy) with (sx, sy) = (0.5, 0.5) for FP_POS_CENTER, (0, 0.5) XFACE, (0.5, 0) YFACE, (0, 0)
 * CORNER. Pointers are device memory; the work is queued on `stream` (NULL = legacy default stream).
 * ------------------------------------------------------------------------------------------------- */
#define FP_FACTOR_ONE 0
#define FP_FACTOR_SIN 1
#define FP_FACTOR_COS 2
#define FP_FACTOR_GAUSS 3
#define FP_FACTOR_QUADRATIC 4
#define FP_POS_CENTER 0
#define FP_POS_XFACE 1
#define FP_POS_YFACE 2
#define FP_POS_CORNER 3

typedef struct fp_term
{
    double a;               /* coefficient */
    int    kind_x, kind_y;  /* FP_FACTOR_* of the x and y factors */
    double px[3], py[3];    /* their parameters */
} fp_term;

/* f (nx x ny, row-major) = (or += with accumulate) the sum of the terms at the value positions: the
 * values Variable2D::set_value(func) stores for domain offset (ox, oy) and steps hx, hy. */
int fp_field_fill(double* f, int nx, int ny, double hx, double hy, double ox, double oy, int position,
                  const fp_term* terms, int nterms, int accumulate, void* stream);
/* The ghost buffer of `face` (LocationType order; ny values for x faces, nx for y faces, one more for
 * FP_POS_CORNER): the sum of the terms one cell outside the face, as Variable2D::set_buffer_value. */
int fp_buffer_fill(double* buf, int face, int nx, int ny, double hx, double hy, double ox, double oy, int position,
                   const fp_term* terms, int nterms, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FP_CAPI_H */
