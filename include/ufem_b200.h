/* ufem_b200.h -- C ABI of the B200-native UFEM Navier-Stokes hot path.
 *
 * Replaces, for P1 triangles and tetrahedra, the per-time-step pipeline of the
 * reference's UFEM NavierStokes solver action and its Trilinos LSS fill:
 *
 *   ZeroLSS -> LinearizeU -> Assembly -> BoundaryConditions -> SolveLSS -> Update
 *   (plugins/UFEM/src/UFEM/ns_implementation/NavierStokes.cpp:100-122,172-179)
 *
 * Conventions (identical to the reference):
 *   - navier_stokes_solution field: N x neq doubles per node (u, v, [w], p),
 *     neq = dim + 1 (Solver.cpp:358-464 creates it by tag; u before p).
 *   - linearized_velocity field: N x 4*dim doubles per node (u_adv, u1, u2, u3).
 *   - global dof = node*neq + comp; CSR row r = node*neq + eq holds the columns
 *     adj(node)*neq + c for the sorted node neighbourhood adj(node) (self
 *     included): the point form of the default FEVbr block matrix
 *     (SparsityBuilder.cpp:157-189, TrilinosDetail.cpp:251-311).
 *   - every function returns 0 on success and a negative UFEM_ERR_* code on
 *     failure; ufem_last_error() gives a message (thread-local).  No C++
 *     exception crosses this boundary.  There is no CPU fallback: if no
 *     sm_100 device is present, ufem_ns_create fails with UFEM_ERR_CUDA.
 *   - a handle owns all of its device memory; the caller owns host buffers.
 *     One handle may be driven by one host thread at a time; distinct handles
 *     are independent.  `stream` arguments are cudaStream_t values (NULL = the
 *     legacy default stream).
 */
#ifndef UFEM_B200_H
#define UFEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UFEM_OK 0
#define UFEM_ERR_ARG (-1)     /* invalid argument (cf3 BadValue / SetupError)   */
#define UFEM_ERR_CUDA (-2)    /* CUDA runtime error or no usable device          */
#define UFEM_ERR_MESH (-3)    /* invalid mesh: node id out of range, det J == 0  */
#define UFEM_ERR_STATE (-4)   /* call out of order (e.g. assemble before state)  */
#define UFEM_ERR_NOMEM (-5)   /* device allocation failed                         */
#define UFEM_ERR_LIMIT (-6)   /* a node has more than 63 neighbours               */
#define UFEM_ERR_SOLVE (-7)   /* Krylov solve failed (see ufem_krylov_status)     */
#define UFEM_ERR_IO (-8)      /* restart file unreadable or malformed (cf3 FileFormatError) */

/* Mesh: coords N x dim (row-major), conn E x (dim+1), host memory. */
typedef struct ufem_mesh {
  int32_t dim;          /* 2: Triag2D (LagrangeP1), 3: Tetra3D (LagrangeP1) */
  int32_t reserved;
  int64_t nb_nodes;
  int64_t nb_elems;
  const double* coords;
  const uint32_t* conn;
} ufem_mesh;

/* Options of the NavierStokes action and its ComputeTauImpl
 * (NavierStokes.cpp:74-98, SUPG.hpp:94-104, NavierStokesPhysics.cpp:24-91). */
typedef struct ufem_ns_options {
  double theta;                 /* theta-method coefficient, default 1      */
  double dt;                    /* time step (LSSActionUnsteady::dt)       */
  double rho;                   /* density; nu_eff is given per node        */
  int32_t supg_type;            /* 0 tezduyar, 1 metric (default), 2 cf2    */
  int32_t use_specializations;  /* 1 (reference default): closed-form P1    */
  double c1, c2;                /* metric constants, default 1 and 16       */
  double alpha_ps, alpha_su, alpha_bu;  /* tau scaling, default 1          */
  double u_ref;                 /* cf2 reference velocity, default 1        */
  int32_t precision;            /* 0: FP64 element arithmetic (plain drop-in)
                                   1: FP32 element arithmetic, FP64 scatter */
  int32_t reserved;
} ufem_ns_options;

/* Krylov options (SolveLSS / Belos GMRES replacement). */
typedef struct ufem_krylov_opts {
  int32_t method;      /* 0: GMRES(restart)  1: BiCGStab (default)  2: CG (SPD)   */
  int32_t restart;     /* GMRES restart length, default 30                         */
  int32_t max_iters;   /* total Krylov iterations (per refinement pass), 3000    */
  int32_t precond;     /* 0 none, 1 point Jacobi (default), 2 node-block Jacobi,
                          3 two-level (CG, semi-implicit pressure only),
                          4 two-level for the coupled system (BiCGStab, GMRES):
                            point Jacobi + a coarse correction on box aggregates
                            of the pressure rows, coarse matrix = Galerkin
                            product of the pressure block, summed on the device
                            at every solve; from a handle's second solve on, a
                            solve uses the previous solve's coarse inverse while
                            its own is inverted on a host thread              */
  double tol;          /* ||b - A x|| / ||b|| target, default 1e-10                */
  int32_t mixed;       /* 0: all FP64; 1: FP32 inner Krylov + FP64 refinement
                          whose residual is b - A x of the stored system; 2: the
                          same with the residual of the FP64 system evaluated
                          element by element (no FP64 matrix: the FP32-element
                          system of precision 1 becomes the inner operator and
                          the answer is the FP64 system's); single handles only,
                          no periodic links                                       */
  int32_t max_refine;  /* outer refinement passes when mixed, default 20          */
  double inner_tol;    /* relative tolerance of each inner FP32 solve, 1e-3       */
} ufem_krylov_opts;

typedef struct ufem_krylov_status {
  int32_t converged;   /* 1 if ||b - A x|| / ||b|| <= tol (checked in FP64)       */
  int32_t status;      /* 0 ok, 1 max iterations, 2 breakdown, 3 non-finite      */
  int32_t iterations;  /* total Krylov iterations                                 */
  int32_t refinements; /* outer FP64 refinement passes (mixed only)               */
  double rel_residual; /* final FP64 ||b - A x|| / ||b||                          */
} ufem_krylov_status;

typedef struct ufem_ns_handle ufem_ns_handle;

/* Phase timings of the last calls, milliseconds, from CUDA events recorded on
 * the call's stream when timing is enabled (component timers of the
 * reference, common/AllocatedComponent.cpp:24-80). */
typedef struct ufem_ns_timings {
  double linearize_ms;
  double assembly_ms;     /* the row-owner assembly kernel alone */
  double dirichlet_ms;
  double solve_ms;
  double update_ms;
} ufem_ns_timings;

/* Device pointers of the assembled system, for in-process consumers. */
typedef struct ufem_ns_device_view {
  const int64_t* rowptr;   /* nb_rows + 1 */
  const int32_t* colidx;   /* nnz          */
  const double* vals;      /* nnz          */
  const double* rhs;       /* nb_rows      */
  const double* solution;  /* nb_rows      */
  int64_t nb_rows;
  int64_t nnz;
} ufem_ns_device_view;

const char* ufem_last_error(void);
const char* ufem_version(void);

/* Fixture mesh generators (cf3/Tools/MeshGeneration/MeshGeneration.cpp:209-253
 * for triangles; Kuhn 6-tet split for the cube).  Interior nodes are jittered by
 * U(-jitter*h, +jitter*h) per coordinate from a counter-based hash of `seed`.
 * coords: (nx+1)(ny+1) x 2 / (n+1)^3 x 3; conn: 2*nx*ny x 3 / 6n^3 x 4. */
int ufem_mesh_rectangle_tris(int32_t nx, int32_t ny, double jitter, uint64_t seed, double* coords,
                             uint32_t* conn);
int ufem_mesh_cube_tets(int32_t n, double jitter, uint64_t seed, double* coords, uint32_t* conn);

void ufem_ns_default_options(ufem_ns_options* opts);
void ufem_krylov_default_opts(ufem_krylov_opts* opts);

/* LSSAction::create_lss (LSSAction.cpp:137-153) + LSS::System::create
 * (System.cpp:82-110): copies the mesh to the device, builds the node graph,
 * the point CSR pattern and the row-owner assembly plan. */
int ufem_ns_create(const ufem_mesh* mesh, const ufem_ns_options* opts, ufem_ns_handle** out);
/* Periodic links (the mesh dictionary's periodic_links_nodes / periodic_links_active,
 * LSSAction.cpp:245-269, made by PeriodicMeshPartitioner::create_link_periodic_nodes):
 * node slaves[i] is the same unknown as masters[i].  As in the reference's map,
 * element contributions at a slave are assembled into its master's rows and
 * columns (chains of links resolve to the final master); the slave keeps rows of
 * its own that tie it to the master (x_slave - x_master = 0, rhs 0), so the
 * solve and the update give it the master's values and dof numbering stays
 * node*neq + comp.  Boundary conditions on a slave act on its master's row.
 * UFEM_ERR_ARG for a node linked twice, a cycle or an id out of range;
 * UFEM_ERR_MESH when an element holds a node and its partner. */
int ufem_ns_create_periodic(const ufem_mesh* mesh, const ufem_ns_options* opts, const uint32_t* slaves,
                            const uint32_t* masters, int64_t nlinks, ufem_ns_handle** out);
/* NavierStokes option triggers (trigger_assembly, NavierStokes.cpp:130-192). */
int ufem_ns_set_options(ufem_ns_handle* h, const ufem_ns_options* opts);
/* Device memory held by the handle (bytes, approximate to a few percent): its
 * mesh, graph, system and field arrays, and the solver workspace allocated so
 * far (none for the vectors of a batch member, which live in its batch). */
int ufem_ns_device_bytes(const ufem_ns_handle* h, int64_t* bytes);
int ufem_ns_sizes(const ufem_ns_handle* h, int64_t* nb_rows, int64_t* nnz, int64_t* block_nnz);
/* Host copies of the CSR pattern (rowptr nb_rows+1, colidx nnz). */
int ufem_ns_csr(ufem_ns_handle* h, int64_t* rowptr, int32_t* colidx);
/* Node graph (starting indices N+1, node connectivity block_nnz). */
int ufem_ns_graph(ufem_ns_handle* h, int64_t* start, uint32_t* adj);

/* Fields: up N x neq, lin N x 4*dim (u_adv, u1, u2, u3), nu N, force N x dim
 * (NULL: zero body force).  Copies host -> device. */
int ufem_ns_set_state(ufem_ns_handle* h, const double* up, const double* lin, const double* nu,
                      const double* force);
int ufem_ns_get_state(ufem_ns_handle* h, double* up, double* lin);
/* Stream-ordered forms of the two calls above: the host buffers must stay valid
 * (and, for an overlapping copy, be pinned) until `stream` reaches the copy. */
int ufem_ns_upload_state(ufem_ns_handle* h, const double* up, const double* lin, const double* nu,
                         const double* force, void* stream);
int ufem_ns_download_state(ufem_ns_handle* h, double* up, double* lin, void* stream);
/* The LSS solution vector (the increment; kept across steps like ZeroLSS
 * with reset_solution=false). */
int ufem_ns_set_solution(ufem_ns_handle* h, const double* sol);
int ufem_ns_get_solution(ufem_ns_handle* h, double* sol);

/* Constant Dirichlet conditions, applied in call order (BoundaryConditions
 * node loops -> System::dirichlet(node, comp, new - old, symmetric),
 * Proto/DirichletBC.hpp:34-51, TrilinosFEVbrMatrix.cpp:482-553). */
int ufem_ns_clear_dirichlet(ufem_ns_handle* h);
int ufem_ns_add_dirichlet(ufem_ns_handle* h, const uint32_t* nodes, int64_t n, int32_t comp,
                          const double* values);
/* Same, with a component per entry: lets a vector condition be listed node by
 * node (u, v, [w] of each node in turn), the order DirichletBCSetter uses
 * (Proto/DirichletBC.hpp:42-48). */
int ufem_ns_add_dirichlet_dofs(ufem_ns_handle* h, const uint32_t* nodes, const int32_t* comps,
                               const double* values, int64_t n);

/* Dirichlet values from a function of the node coordinates and time:
 * BCDirichletFunction (plugins/UFEM/src/UFEM/BCDirichletFunction.cpp:61-92 with
 * solving_for_difference, i.e. dirichlet(var) = f: the component ends at f).
 * `expr` is a formula in x, y, z (node coordinates; z = 0 in 2D) and t (the
 * handle's time): numbers, + - * / ^ (right-associative, above unary minus),
 * parentheses, pi and sin cos tan asin acos atan sinh cosh tanh exp log sqrt
 * abs.  It is compiled here (UFEM_ERR_ARG with the position of a syntax error)
 * and evaluated on the device, in FP64 with CUDA's math functions, at every
 * ufem_ns_apply_dirichlet; the entries join the ordered Dirichlet list exactly
 * as constant ones (first application moves the columns, last sets the row). */
int ufem_ns_add_dirichlet_function(ufem_ns_handle* h, const uint32_t* nodes, int64_t n, int32_t comp,
                                   const char* expr);
/* The time that function conditions see (Time::current_time).  It starts at 0
 * and advances by dt at every ufem_ns_update (the reference's AdvanceTime). */
int ufem_ns_set_time(ufem_ns_handle* h, double t);
int ufem_ns_get_time(const ufem_ns_handle* h, double* t);

/* Constant Neumann condition: BCNeumannConstant
 * (plugins/UFEM/src/UFEM/BCNeumannConstant.cpp:54-60), defined there on Line2D
 * faces only, so 2D meshes only here (UFEM_ERR_ARG otherwise).  faces: nfaces
 * x 2 node ids; each face adds integral<1>(N^T flux |normal|) to the RHS rows of
 * component `comp` of its two nodes, evaluated as the reference does
 * (one Gauss point of weight 2 times the face's jacobian determinant |dx|/2,
 * N = 1/2, |normal| = |dx|/2: flux |dx|^2 / 4 per node).  The contributions are
 * added before the Dirichlet conditions, face by face in the order given. */
int ufem_ns_add_neumann(ufem_ns_handle* h, const uint32_t* faces, int64_t nfaces, int32_t comp, double flux);
int ufem_ns_clear_neumann(ufem_ns_handle* h);

/* ZeroLSS + LinearizeU + Assembly (NavierStokesAssembly.hpp:27-75 or
 * NavierStokesSpecializations.hpp:26-303).  Asynchronous on `stream`. */
int ufem_ns_assemble(ufem_ns_handle* h, void* stream);
/* BoundaryConditions: symmetric Dirichlet on the assembled system. */
int ufem_ns_apply_dirichlet(ufem_ns_handle* h, void* stream);
/* SolveLSS (SolveLSS.cpp:44-55): Krylov solve for the increment. */
int ufem_ns_solve(ufem_ns_handle* h, const ufem_krylov_opts* kopts, ufem_krylov_status* status,
                  void* stream);
/* Optional: allocate the Krylov workspace and build the static structure of the
 * preconditioner that solves with `kopts` will use (the coarse space of precond
 * 4), ahead of the first solve -- e.g. on the host thread that created the
 * handle, while the GPU steps other handles.  batched = 1 prepares a future
 * batch member (no one-handle vectors; the batch's aggregate caps).  For one
 * handle (batched = 0) whose system has been assembled and conditioned
 * (ufem_ns_assemble, then ufem_ns_apply_dirichlet), precond 4 also gets the
 * coarse inverse of that system, which the next solve uses as its lagged
 * inverse, so that the first solve does not wait for a host inversion; the
 * call returns when it is done.  No counterpart in the reference. */
int ufem_ns_prepare_solve(ufem_ns_handle* h, const ufem_krylov_opts* kopts, int32_t batched);
/* Allocation-free variant of ufem_ns_solve.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc: applications that hand all device
 * memory to their own pool or enforce a fixed device-memory budget, and loops
 * that must not take the implicit device synchronisation of a first-use
 * allocation.  ufem_ns_solve allocates its Krylov workspace on first use; this
 * entry point instead uses a fixed scratch area inside the library (about 9.5 MB
 * of device memory, held on every GPU that loads the library until the process
 * exits) and calls no cudaMalloc, cudaFree or allocating library routine.
 *  - Solves the system the handle holds: BiCGStab (method 1) with point Jacobi or
 *    no preconditioner, FP64 (mixed = 0), restarted from its iterate after a
 *    breakdown as ufem_ns_solve restarts it; other options give UFEM_ERR_ARG.
 *  - At most UFEM_NOALLOC_MAX_ROWS rows; larger systems give UFEM_ERR_LIMIT.
 *  - The first call on a device looks up the scratch area's device address; make
 *    that first call before any stream capture.
 *  - Every call shares the one scratch area (it keeps the last call's contents,
 *    and each call initialises what it reads): calls that overlap on the GPU,
 *    from any handle or stream, race.  Serialise them. */
#define UFEM_NOALLOC_MAX_ROWS 131072
int ufem_ns_solve_noalloc(ufem_ns_handle* h, const ufem_krylov_opts* kopts, ufem_krylov_status* status,
                          void* stream);
/* Residual of the FP64 system for the current solution vector x, evaluated
 * element by element in FP64 without a matrix (NavierStokesAssembly.hpp:69-71:
 * b = a - A u over the elements, M = invdt T + theta A): r = b - M x with the
 * symmetric Dirichlet conditions as ufem_ns_apply_dirichlet sets them
 * (constrained columns at their first application's value, constrained rows
 * r = 0) and the Neumann contributions in b.  It is the refinement residual of
 * mixed = 2 solves.  Call after ufem_ns_assemble and ufem_ns_apply_dirichlet of
 * the step; r: host buffer of nb_rows doubles.  Not for periodic links. */
int ufem_ns_fp64_residual(ufem_ns_handle* h, double* r, void* stream);
/* UpdateActions (NavierStokes.cpp:172-179). */
int ufem_ns_update(ufem_ns_handle* h, void* stream);
/* nsteps full time steps; status of the last solve. */
int ufem_ns_step(ufem_ns_handle* h, int32_t nsteps, const ufem_krylov_opts* kopts,
                 ufem_krylov_status* status, void* stream);

/* Restart files of the device-resident state.
 * ufem_ns_write_restart replaces WriteRestartFile::execute
 * (solver/actions/WriteRestartFile.cpp:62-90): `path` receives the XML restart
 * node (version 1, nb_procs 1, current_time, time_step, iteration, one <field>
 * node per table) and `path`.bin the tables as raw FP64 rows with a checksum
 * each -- navier_stokes_solution, linearized_velocity, navier_stokes_viscosity
 * and body_force when set, in the layouts of ufem_ns_set_state, and the linear
 * system's solution vector (the next solve's initial guess).
 * ufem_ns_read_restart replaces ReadRestartFile::execute (ReadRestartFile.cpp:67-110):
 * it checks version, process count, node count and dimension and every table's
 * shape and checksum (UFEM_ERR_IO otherwise), restores the state, sets the
 * handle's time (ufem_ns_set_time) to the file's current_time and returns the
 * time, time step and iteration (each output may be NULL).  Stepping a handle
 * read from a restart gives bitwise the same states as stepping the handle that
 * wrote it. */
int ufem_ns_write_restart(ufem_ns_handle* h, const char* path, double current_time, double time_step,
                          int64_t iteration);
int ufem_ns_read_restart(ufem_ns_handle* h, const char* path, double* current_time, double* time_step,
                         int64_t* iteration);

/* Overlapped host transfers.  No counterpart in the reference (its fields are
 * host tables its CPU assembly reads in place).  For callers that keep each
 * step's fields in host memory and want each step's RHS back: the copies of
 * one step overlap the assembly of another.
 *  - ufem_ns_stage_state copies up, lin, nu (the ufem_ns_set_state layouts; the
 *    body force is left as set) into one of two device staging buffers on
 *    `copy_stream` and returns; UFEM_ERR_STATE if two staged states are still
 *    uncommitted.
 *  - ufem_ns_commit_state makes `stream` wait for the oldest staged copy and
 *    unpacks it into the handle's fields (the values ufem_ns_upload_state writes);
 *    UFEM_ERR_STATE if nothing is staged.
 *  - ufem_ns_fetch_rhs copies the RHS into one of two device output buffers on
 *    `stream` (after the work queued there) and reads it into `rhs` (nb_rows
 *    doubles) on `copy_stream`; it is complete when `copy_stream` is.
 * Host buffers should be pinned for the copies to overlap.  Giving
 * ufem_ns_fetch_rhs a copy stream of its own (not the one ufem_ns_stage_state
 * uses) lets the read-backs run concurrently with the uploads (the host link
 * carries both directions at once).  A staged buffer is
 * reused only after its commit has read it and an output buffer only after its
 * read-back, so each host buffer may be reused once the copy stream has passed
 * its copy.  The buffers (2 x N x (neq + 4 dim + 1) + 2 x nb_rows doubles) are
 * allocated on the first call. */
int ufem_ns_stage_state(ufem_ns_handle* h, const double* up, const double* lin, const double* nu,
                        void* copy_stream);
int ufem_ns_commit_state(ufem_ns_handle* h, void* stream);
int ufem_ns_fetch_rhs(ufem_ns_handle* h, double* rhs, void* stream, void* copy_stream);

/* Host copies of the assembled system (vals nnz, rhs nb_rows); either may be NULL. */
int ufem_ns_get_system(ufem_ns_handle* h, double* vals, double* rhs);
int ufem_ns_download_system(ufem_ns_handle* h, double* vals, double* rhs, void* stream);
int ufem_ns_device_view_get(const ufem_ns_handle* h, ufem_ns_device_view* view);
/* y = A x (FP64, host buffers) -- LSS::Matrix::apply with alpha=1, beta=0. */
int ufem_ns_apply(ufem_ns_handle* h, const double* x, double* y);
/* y = A x with device buffers of nb_rows doubles on `stream` (the SpMV of the
 * solvers) -- LSS::Matrix::apply (math/LSS/Matrix.hpp) for device-resident
 * callers such as the distributed solve of a decomposed mesh. */
int ufem_ns_apply_device(ufem_ns_handle* h, const double* d_x, double* d_y, void* stream);

/* Assembly kernel selection.  No counterpart in the reference (one code path
 * there).  variant 0: warp per group of consecutive rows holding at most 32
 * incident elements (rows with more use the chunk kernel); variant 1: chunk
 * kernel (one CTA per range of whole rows) for every row.  warps_per_cta:
 * 2, 4 or 8 (variant 0 only).  All variants sum every CSR value in element
 * order; they agree to rounding level (the compiler may contract multiply-adds
 * of the element expression differently in each kernel), and each one is
 * deterministic. */
int ufem_ns_set_assembly_kernel(ufem_ns_handle* h, int32_t variant, int32_t warps_per_cta);
int ufem_ns_get_assembly_kernel(ufem_ns_handle* h, int32_t* variant, int32_t* warps_per_cta);
/* Autotuner: times every (variant, warps_per_cta) candidate on this handle's
 * mesh and state (`reps` launches each after one warm-up, CUDA events on
 * `stream`), keeps the fastest and reports it.  Requires ufem_ns_set_state.
 * Overwrites the assembled system (assemble again afterwards). */
int ufem_ns_tune_assembly(ufem_ns_handle* h, void* stream, int32_t reps, int32_t* variant,
                          int32_t* warps_per_cta, float* ms_per_launch);

/* ---- batches: many meshes per launch (no counterpart in the reference) ----
 * A batch steps several handles of the same dim, precision and element form
 * together: every phase of a time step is one launch over all members (the
 * assembly one persistent launch), and the solve is BiCGStab with point Jacobi
 * (or none) and per-member scalars, so each member converges on its own and
 * its results are bitwise the same alone and in any batch.  The iteration
 * blocks are replayed from captured CUDA graphs.  Members stay owned by the
 * caller and must outlive the batch; a member's BC list may change between
 * steps, its mesh may not.  mixed = 1 iterates with an FP32 copy of each
 * member's operator (allocated on first use, then written by every assembly),
 * FP64 vectors and dot products, and replaces the recursive residual by the
 * FP64 residual of the assembled FP64 system every 32 iterations and before
 * accepting convergence (status.refinements counts the replacements). */
typedef struct ufem_batch ufem_batch;
int ufem_batch_create(ufem_ns_handle* const* members, int32_t n, ufem_batch** out);
/* Holds or resumes members (active[m] = 0: held) without rebuilding the batch.
 * No counterpart in the reference.  A held member is not solved and not updated
 * (its state and time stay as they are; its status reads converged with 0
 * iterations); assembly and the Dirichlet passes still run over it.  The handle
 * of a held member must stay alive until the batch is destroyed.  Lets a
 * serving loop retire finished requests without stalling the others. */
int ufem_batch_set_active(ufem_batch* b, const int32_t* active);
int ufem_batch_size(const ufem_batch* b, int32_t* n, int64_t* rows);
int ufem_batch_set_graphs(ufem_batch* b, int32_t enable);
int ufem_batch_set_assembly_warps(ufem_batch* b, int32_t warps_per_cta);
/* Batch autotuner (project-written, no counterpart in the reference): times the
 * batched warp assembly with 2, 4 and 8 warps per CTA on the members' own meshes
 * and states (warm-up + `reps` launches, CUDA events on `stream`), keeps the
 * fastest for this batch and returns it with its time per launch (outputs may be
 * NULL).  The members' systems are overwritten: assemble before solving. */
int ufem_batch_tune_assembly(ufem_batch* b, void* stream, int32_t reps, int32_t* warps_per_cta,
                             float* ms_per_launch);
/* LinearizeU + assembly + symmetric Dirichlet of every member. */
int ufem_batch_assemble(ufem_batch* b, void* stream);
/* statuses: one per member, or NULL.  BiCGStab (method 1) with precond 0, 1 or
 * 4 (the coupled two-level preconditioner, each member with its own coarse
 * space on at most 16 x 16 (2D) or 5^3 (3D) aggregates, coarse matrices
 * refreshed at every solve).  mixed 0: FP64 operator; 1: FP32 copy of the
 * operator with FP64 residual replacement; 2: FP32-operator inner solves refined
 * against each member's matrix-free FP64 residual (as ufem_ns_solve with mixed 2:
 * for members with FP32 element matrices, whose answers are then the FP64
 * systems'; members without periodic links; inner_tol and max_refine apply). */
int ufem_batch_solve(ufem_batch* b, const ufem_krylov_opts* kopts, ufem_krylov_status* statuses, void* stream);
int ufem_batch_update(ufem_batch* b, void* stream);
int ufem_batch_step(ufem_batch* b, const ufem_krylov_opts* kopts, ufem_krylov_status* statuses, void* stream);
void ufem_batch_destroy(ufem_batch* b);

int ufem_ns_enable_timing(ufem_ns_handle* h, int32_t enable);
int ufem_ns_get_timings(ufem_ns_handle* h, ufem_ns_timings* t);

void ufem_ns_destroy(ufem_ns_handle* h);

/* ---------------------------------------------------------------------------
 * Semi-implicit (pressure-correction) scheme: NavierStokesSemiImplicit
 * (plugins/UFEM/src/UFEM/ns_semi_implicit/implementation/NavierStokesSemiImplicit.cpp).
 * Two systems over the node graph -- velocity (dim equations per node, matrix
 * T + theta dt M reassembled every step, MatrixAssembly.hpp:52-149) and pressure
 * (one equation, theta (tau_ps + dt) grad N^T grad N assembled once,
 * PressureSystem.cpp:110-140) -- and nb_iterations predictor/corrector passes
 * per step (InnerLoop::execute, NavierStokesSemiImplicit.cpp:104-191).  Element
 * expressions in FP64 (opts->precision is ignored); both systems are solved by
 * Jacobi-preconditioned CG unless ufem_nssi_set_krylov says otherwise.
 * Fields use the coupled handle's layouts (up N x (dim+1), lin N x 4 dim, nu N,
 * force N x dim or NULL: enable_body_force off). */
typedef struct ufem_nssi_handle ufem_nssi_handle;
/* NavierStokesSemiImplicit constructor + regions (on_regions_set, :418-497);
 * nb_iterations is the "nb_iterations" option (default 2); periodic links as in
 * ufem_ns_create_periodic (nlinks 0: none). */
int ufem_nssi_create(const ufem_mesh* mesh, const ufem_ns_options* opts, int32_t nb_iterations,
                     const uint32_t* slaves, const uint32_t* masters, int64_t nlinks, ufem_nssi_handle** out);
/* Krylov options of the velocity and pressure solves (SolveUSystem /
 * SolvePSystem, :99-100); NULL keeps the current one.  Defaults: CG with point
 * Jacobi for the velocity, CG with the two-level preconditioner (precond 3:
 * point Jacobi plus a Galerkin coarse correction on geometric aggregates,
 * built from the pressure matrix once its conditions are applied; point Jacobi
 * if that coarse matrix is singular) for the pressure, both to 1e-10. */
int ufem_nssi_set_krylov(ufem_nssi_handle* h, const ufem_krylov_opts* velocity, const ufem_krylov_opts* pressure);
int ufem_nssi_set_state(ufem_nssi_handle* h, const double* up, const double* lin, const double* nu,
                        const double* force);
int ufem_nssi_get_state(ufem_nssi_handle* h, double* up, double* lin);
/* VelocityLSS.BC / PressureLSS.BC constant conditions, in call order. */
int ufem_nssi_add_velocity_dirichlet(ufem_nssi_handle* h, const uint32_t* nodes, int64_t n, int32_t comp,
                                     const double* values);
int ufem_nssi_add_pressure_dirichlet(ufem_nssi_handle* h, const uint32_t* nodes, int64_t n, const double* values);
/* BCDirichletFunction values (formula in x, y, z, t, as ufem_ns_add_dirichlet_function),
 * evaluated at the step's start time; the time advances by dt per step. */
int ufem_nssi_add_velocity_dirichlet_function(ufem_nssi_handle* h, const uint32_t* nodes, int64_t n, int32_t comp,
                                              const char* expr);
int ufem_nssi_add_pressure_dirichlet_function(ufem_nssi_handle* h, const uint32_t* nodes, int64_t n,
                                              const char* expr);
int ufem_nssi_set_time(ufem_nssi_handle* h, double t);
int ufem_nssi_clear_dirichlet(ufem_nssi_handle* h);
/* WriteRestartFile / ReadRestartFile of the solver's restart fields (u, p,
 * linearized velocity, viscosity, force).  After a read, call
 * ufem_nssi_initialize(h, 0, stream): the pressure matrix follows the read
 * velocity, as the reference's initial conditions after Restarts do. */
int ufem_nssi_write_restart(ufem_nssi_handle* h, const char* path, double current_time, double time_step,
                            int64_t iteration);
int ufem_nssi_read_restart(ufem_nssi_handle* h, const char* path, double* current_time, double* time_step,
                           int64_t* iteration);
/* The solver's initial conditions (trigger_initial_conditions, :400-455):
 * nu_eff into the element records, with reset_history u_adv = u1 = u2 = u3 = u,
 * the pressure matrix (tau from the current u) and the lumped velocity mass. */
int ufem_nssi_initialize(ufem_nssi_handle* h, int32_t reset_history, void* stream);
/* nsteps time steps: LinearizeU, velocity assembly, SetSolution, InnerLoop,
 * Update (:329-375).  Statuses fold all solves of the call (iterations summed,
 * worst status, largest residual); may be NULL. */
int ufem_nssi_step(ufem_nssi_handle* h, int32_t nsteps, ufem_krylov_status* velocity, ufem_krylov_status* pressure,
                   void* stream);
int ufem_nssi_get_time(const ufem_nssi_handle* h, double* t);
int ufem_nssi_sizes(const ufem_nssi_handle* h, int64_t* velocity_nnz, int64_t* pressure_nnz);
/* Inspection (no counterpart; parity tests): host copies of one system
 * (which 0: velocity, 1: pressure; any pointer may be NULL), the velocity
 * matrix of the current state without conditions, the lumped-mass reciprocal. */
int ufem_nssi_get_system(ufem_nssi_handle* h, int32_t which, int64_t* rowptr, int32_t* colidx, double* vals,
                         double* rhs, double* sol);
int ufem_nssi_assemble_velocity_matrix(ufem_nssi_handle* h, void* stream);
int ufem_nssi_get_lumped_inverse(ufem_nssi_handle* h, double* minv);
int64_t ufem_nssi_device_bytes(const ufem_nssi_handle* h);
void ufem_nssi_destroy(ufem_nssi_handle* h);

#ifdef __cplusplus
}
#endif

#endif /* UFEM_B200_H */
