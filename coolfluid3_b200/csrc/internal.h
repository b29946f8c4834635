// internal.h -- shared declarations of the B200 UFEM library (not part of the ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ufem_b200.h"

namespace ufem {

// ---------------------------------------------------------------------------
// Error reporting across the C ABI: a thread-local message plus a code.
// ---------------------------------------------------------------------------
int set_error(int code, const std::string& msg);
// Host helper threads (see host.cu): takes up to `want` of the process-wide
// spare threads (possibly none) and gives them back; the caller's own thread
// is never counted.
int acquire_spare_threads(int want);
void release_spare_threads(int n);

// Serialises device-lifecycle calls (allocation, free, device-wide
// synchronisation) with CUDA-graph capture: a capture in one host thread must
// not overlap an implicit device synchronisation issued by another.
std::recursive_mutex& device_mutex();
using DeviceLock = std::lock_guard<std::recursive_mutex>;

#define UFEM_CUDA_TRY(expr)                                                              \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess)                                                               \
      return ::ufem::set_error(UFEM_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

// Scalar parameters of the element expression, passed to kernels by value.
struct NSParams {
  double theta, inv_theta, dt, invdt, rho, inv_rho;
  double tau_c1, tau_std, two_dt;
  double c2, a_ps, a_su, a_bu, u_ref;
  int supg_type;
  int has_force;
};

// Row-owner assembly plans.  Incidences (row node, element) are sorted by
// (row node, element id), so each CSR entry is summed in element order.
//  - chunk plan: ranges of whole rows whose incidences fit one CTA of `cap`
//    threads (one thread per incidence);
//  - warp plan: ranges of consecutive rows with at most 32 incidences in total,
//    one warp each (one lane per incidence).  Rows with more than 32 incidences
//    are left to a chunk plan that lists only those rows.
struct AssemblyPlan {
  int cap = 0;                 // incidences per chunk (== CTA threads)
  int nchunks = 0;
  int2* chunks = nullptr;      // [first row, end row) per chunk (device)
};
struct WarpPlan {
  int cap = 32;                // incidences per group (lanes per warp that evaluate elements)
  int ngroups = 0;
  int4* groups = nullptr;      // first row, end row, first incidence, incidences (device)
  AssemblyPlan big64, big32;   // rows with more than 32 incidences
};

// Everything the warp assembly kernel reads or writes for one mesh.  A launch
// takes an array of these plus a prefix of their group counts, so one
// persistent launch assembles one mesh (a handle) or many (a batch).
struct AsmDesc {
  const double* coords;
  const double* uadv;
  const double* state;
  const float* node32;
  const double* force;
  const int64_t* start;
  const int32_t* row_inc;
  const int32_t* inc_elem;
  const uint32_t* inc_info;
  const int4* conn;
  const int4* groups;
  double* vals;
  float* vals32;  // null: no FP32 copy of the values
  double* rhs;
  NSParams p;
};

// Assembly kernel variants (selected per handle, see ufem_ns_set_assembly_kernel).
enum AssemblyVariant { kAsmWarp = 0, kAsmChunk = 1, kAsmWarp24 = 2 };

// Symmetric-Dirichlet plan (sequential semantics of TrilinosFEVbrMatrix::
// symmetric_dirichlet reduced to an order-preserving parallel form).
struct DirichletPlan {
  int64_t nbc = 0;             // unique (node, comp) dofs
  int64_t nfix_rows = 0;       // non-BC rows holding BC columns
  int64_t nfix = 0;            // entries moved to the RHS
  int64_t* bc_dof = nullptr;   // nbc
  double* bc_first = nullptr;  // value of the first application (moves columns)
  double* bc_last = nullptr;   // value of the last application (sets row/rhs/sol)
  int64_t* bc_diag = nullptr;  // CSR position of the diagonal of each BC row
  int64_t* fix_row = nullptr;  // nfix_rows
  int64_t* fix_ptr = nullptr;  // nfix_rows + 1
  int64_t* fix_pos = nullptr;  // nfix CSR positions, per row in first-application order
  int32_t* fix_bc = nullptr;   // nfix index into bc arrays
  double* vfirst = nullptr;    // per step: bc_first - old
  // constant Neumann faces: per RHS dof (neu_dof), its face contributions in
  // face order (neu_val[neu_ptr[i] .. neu_ptr[i+1]))
  // function values (BCDirichletFunction): expression of the first / last
  // application of each dof (-1: constant), byte code of all expressions
  int32_t* fn_first = nullptr;
  int32_t* fn_last = nullptr;
  int32_t* fn_code = nullptr;
  int32_t* fn_off = nullptr;   // expression e: fn_code[fn_off[e] .. fn_off[e+1])
  double* fn_const = nullptr;
  int64_t nneu = 0;
  int64_t* neu_dof = nullptr;
  int64_t* neu_ptr = nullptr;
  double* neu_val = nullptr;
  bool dirty = true;
  int64_t version = 0;         // incremented at every rebuild of the plan
};

struct KrylovWork;

// Double-buffered host transfers of pipeline.cu (staged inputs, RHS outputs).
struct StagePipe {
  double* buf[2] = {nullptr, nullptr};  // N x (neq + 4 dim + 1): up | lin | nu
  double* out[2] = {nullptr, nullptr};  // nrows: RHS copies being read back
  cudaEvent_t staged[2] = {}, consumed[2] = {}, out_ready[2] = {}, out_free[2] = {};
  bool consumed_rec[2] = {false, false}, out_free_rec[2] = {false, false};
  int pending[2] = {0, 0};
  int npending = 0, next = 0, out_next = 0;
};

}  // namespace ufem

struct ufem_ns_handle {
  int dim = 0, nn = 0, neq = 0;
  int64_t N = 0, E = 0;
  int64_t nrows = 0, nnz = 0, bnnz = 0;
  ufem_ns_options opt{};
  bool state_set = false;
  bool view = false;  // a system over another handle's graph and fields (semi-implicit scheme)

  // host copies used by planning
  std::vector<int64_t> start_h;   // N+1
  std::vector<int32_t> adj_h;     // bnnz
  std::vector<double> coords_h;   // N x dim (constant Neumann faces, coarse-preconditioner aggregates)
  std::vector<uint32_t> p2m_h;    // periodic links: row node of each node (empty: no links)
  struct BCEntry { uint32_t node; int comp; double value; int32_t fn = -1; };  // fn: expression id or -1
  std::vector<std::vector<int32_t>> fn_code;   // compiled Dirichlet function expressions
  std::vector<std::vector<double>> fn_const;
  double time = 0.0;                            // current time (function BCs); advanced by dt at each update
  std::vector<BCEntry> bcs;
  int64_t bc_list_version = 0;  // incremented whenever the condition lists change
  struct NeumannFace { uint32_t a, b; int comp; double flux; };
  std::vector<NeumannFace> neumann;  // constant Neumann conditions on Line2D faces

  // device mesh and fields (node records padded to 4 doubles)
  double* d_coords = nullptr;   // N x 4 (x, y, [z], 0)
  int32_t* d_conn = nullptr;    // E x 4 (triangles padded with node 0)
  double* d_state = nullptr;    // N x 4 (u, v, [w], p) : p at index dim
  double* d_hist = nullptr;     // 3 x N x 4 (u1, u2, u3)
  double* d_uadv = nullptr;     // N x 4 (u_adv xyz, nu at index 3)
  double* d_nu = nullptr;       // N
  double* d_force = nullptr;    // N x 4 or null
  float* d_node32 = nullptr;    // N x 8: FP32 (u_adv, nu, u, p) for the FP32 element path

  // graph + CSR
  int64_t* d_start = nullptr;   // N+1
  int32_t* d_adj = nullptr;     // bnnz
  int64_t* d_rowptr = nullptr;  // nrows+1
  int32_t* d_colidx = nullptr;  // nnz
  double* d_vals = nullptr;     // nnz
  float* d_vals32 = nullptr;    // nnz (allocated when a mixed solve first runs)
  double* d_rhs = nullptr;
  double* d_sol = nullptr;
  int64_t* d_diagpos = nullptr; // nrows

  int64_t ntie = 0;               // linked (slave) nodes: tie rows x_slave - x_master = 0
  int32_t* d_tie = nullptr;       // ntie x 2: slave, master

  // row-owner incidences
  int32_t* d_row_inc = nullptr;   // N+1
  int32_t* d_inc_elem = nullptr;  // E*nn
  uint32_t* d_inc_info = nullptr; // E*nn : 6-bit slots + local index << 24

  ufem::AssemblyPlan plan64;       // chunks sized for the FP64-element chunk kernel (all rows)
  ufem::AssemblyPlan plan32;       // chunks sized for the FP32-element chunk kernel (all rows)
  ufem::WarpPlan wplan;            // warp-per-row-group kernel, groups of <= 32 incidences
  ufem::WarpPlan wplan24;          // tetrahedra: groups of <= 24 incidences (smaller staging, more warps)
  int asm_variant = ufem::kAsmWarp;
  int asm_warps = 4;               // warps per CTA of the warp kernel
  ufem::DirichletPlan bcp;
  ufem::StagePipe pipe;
  ufem::KrylovWork* kw = nullptr;
  bool vals32_valid = false;            // d_vals32 holds the current system (written by the assembly)
  bool conditioned = false;             // the Dirichlet conditions ran after the latest assembly

  // transfer staging (reference field layouts <-> padded node records)
  double* d_stage = nullptr;      // N x 4*dim doubles
  double* d_x = nullptr;          // apply() operands
  double* d_y = nullptr;

  // timing: event pairs (start, stop) for linearize, assembly, dirichlet, solve, update
  bool timing = false;
  cudaEvent_t ev[10] = {};
  bool ev_rec[5] = {};
};

namespace ufem {

// kernels (assembly.cu)
int launch_build_csr(ufem_ns_handle* h, cudaStream_t s);
int launch_linearize(ufem_ns_handle* h, cudaStream_t s);
int launch_assembly(ufem_ns_handle* h, cudaStream_t s, bool write32);
void fill_params(const ufem_ns_handle* h, NSParams& p);
void fill_desc(const ufem_ns_handle* h, bool write32, AsmDesc& d, const WarpPlan* plan = nullptr);
// Warp assembly of many meshes in one persistent launch (same dim and precision;
// rows with more than 32 incidences go through each mesh's chunk plan).
int launch_assembly_batch(int dim, int precision, bool spec, int warps, int ngroups, int nmesh,
                          const AsmDesc* d_descs, const int* d_gprefix, cudaStream_t s);
int launch_dirichlet(ufem_ns_handle* h, cudaStream_t s);
// Adds the constant Neumann contributions to the RHS (before the Dirichlet passes).
int launch_neumann(ufem_ns_handle* h, cudaStream_t s);
// r = b - M dx of the FP64 system (FP64 element pass, no matrix), dx = h->d_sol;
// dx_work: nrows scratch doubles (assembly.cu).
int launch_mf_residual(ufem_ns_handle* h, double* dx_work, double* res, cudaStream_t s);

// bcfunction.cu: Dirichlet values from expressions of (x, y, z, t)
constexpr int kExprMaxDepth = 32;
constexpr int32_t kExprPushConst = 0;  // byte-code word: op | operand << 8
int compile_expression(const std::string& src, std::vector<int32_t>& code, std::vector<double>& consts,
                       std::string& err);
// Evaluates the function values of the first / last applications at h->time.
int launch_dirichlet_functions(ufem_ns_handle* h, cudaStream_t s);
int launch_update(ufem_ns_handle* h, cudaStream_t s);
int assembly_chunk_capacity(int dim, int precision);
int configure_kernels();

int launch_assembly_big_rows(ufem_ns_handle* h, cudaStream_t s, bool write32);
// Tie rows of periodic (slave) nodes: identity at the slave, minus identity at its master, rhs 0.
int launch_tie_rows(ufem_ns_handle* h, cudaStream_t s, bool write32);

// host.cu
int build_bc_plan(ufem_ns_handle* h);
// A handle with the mesh, fields, node graph and incidences but no coupled
// system (the semi-implicit scheme keeps its systems in views).
int create_base(const ufem_mesh* mesh, const ufem_ns_options* opts, const uint32_t* slaves, const uint32_t* masters,
                int64_t nlinks, ufem_ns_handle** out);
// A system of `neq` equations per node over the base handle's node graph; its
// Dirichlet kernels read the field component at `state_offset` of the base's
// node records.
int make_system_view(ufem_ns_handle* base, int neq, int state_offset, ufem_ns_handle** out);
void destroy_handle(ufem_ns_handle* h);

// Krylov (krylov.cu)
int krylov_solve(ufem_ns_handle* h, const ufem_krylov_opts* ko, ufem_krylov_status* st, cudaStream_t s);
int krylov_apply(ufem_ns_handle* h, const double* d_x, double* d_y, cudaStream_t s);
int krylov_fp64_residual(ufem_ns_handle* h, double* r_host, cudaStream_t s);
// Coarse space of the coupled two-level preconditioner of one handle, rebuilt
// when its Dirichlet plan or the aggregate caps change (rebuilt = true) and its
// coarse matrix refreshed from the current system (krylov.cu).  lag: from the
// handle's second refresh on, the inverse is the previous refresh's matrix's,
// and this refresh's matrix is inverted on a host thread for the next one.
// nc = 0: no usable coarse space (point Jacobi).
struct CoarseView {
  int nc = 0;
  const int32_t* agg = nullptr;
  const int32_t* agg_ptr = nullptr;
  const int32_t* agg_rows = nullptr;
  const double* ainv = nullptr;
};
int krylov_coupled_coarse(ufem_ns_handle* h, cudaStream_t s, int max_side_2d, int max_side_3d, bool* rebuilt,
                          CoarseView* view, bool lag);
// The same for the active members of a batch, not lagged: every member's
// coarse matrix summed and copied on `s`, one synchronisation, the inversions
// on host threads in parallel (each the one-handle inversion, bitwise), the
// inverses uploaded on `s`.
int krylov_coupled_coarse_members(ufem_ns_handle* const* hs, const int32_t* active, int n, cudaStream_t s,
                                  int max_side_2d, int max_side_3d, bool* rebuilt, CoarseView* views);
// Aggregate caps (boxes a side) of the coupled two-level preconditioner: one
// handle (its coarse inverse is computed on a host thread while the previous
// one is used), and batch members (every member's inverse before the batch solve).
constexpr int kCoarseSide2D = 20, kCoarseSide3D = 8;
constexpr int kBatchCoarseSide2D = 16, kBatchCoarseSide3D = 5;
// Allocations and static preconditioner structure of the solves `ko` describes,
// ahead of the first solve (batched: for a batch member).
int krylov_prepare(ufem_ns_handle* h, const ufem_krylov_opts* ko, int batched);
void krylov_free(ufem_ns_handle* h);
// Device bytes the handle's solver workspace holds (vectors allocated so far,
// coarse-space data); 0 without one.
int64_t krylov_device_bytes(const ufem_ns_handle* h);
// Aggregates of the two-level CG preconditioner (precond 3) of a one-equation
// system: agg[row] in [0, nc) or -1; builds and inverts the Galerkin coarse
// matrix from the system's current values.  If that matrix is not positive
// definite the coarse space is left empty (krylov_coarse_size returns 0).
int krylov_set_coarse(ufem_ns_handle* h, const std::vector<int32_t>& agg, int nc, cudaStream_t s);
int krylov_coarse_size(const ufem_ns_handle* h);
// Allocates the FP32 copy of the values (converted from the current FP64
// values); later assemblies write both.
int ensure_vals32(ufem_ns_handle* h, cudaStream_t s);
// pipeline.cu: frees the staging and output buffers and their events.
void free_stage_pipe(ufem_ns_handle* h);

}  // namespace ufem
