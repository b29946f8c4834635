// host.cu -- C ABI of the B200 UFEM library: handle lifetime, mesh preprocessing
// (node graph, point CSR pattern, row-owner incidence plan), field transfer,
// Dirichlet planning and the time-step driver.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace ufem {

std::recursive_mutex& device_mutex() {
  static std::recursive_mutex m;
  return m;
}

static thread_local std::string g_err;

int set_error(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

namespace {
// Helper threads the library's host loops may run at once, over all callers:
// one less than the machine's hardware threads, shared, so that handles built
// or coarse spaces inverted concurrently (a serving loop's creator and worker
// threads) do not each start a thread per core beside the threads that drive
// the GPU.  -1 until first use.
std::atomic<int> g_spare_threads{-1};
}  // namespace

int acquire_spare_threads(int want) {
  int unset = -1;
  g_spare_threads.compare_exchange_strong(
      unset, int(std::max<unsigned>(1u, std::thread::hardware_concurrency())) - 1);
  int cur = g_spare_threads.load();
  while (want > 0 && cur > 0) {
    const int take = std::min(want, cur);
    if (g_spare_threads.compare_exchange_weak(cur, cur - take)) return take;
  }
  return 0;
}

void release_spare_threads(int n) {
  if (n > 0) g_spare_threads.fetch_add(n);
}

namespace {

// f(a, b) over [0, n) in contiguous ranges, on the calling thread and as many
// spare helper threads as the loop can use (one per 8192 items); every range
// writes its own outputs, so results do not depend on the split.
template <typename F>
void parallel_for(int64_t n, F&& f) {
  const int hw = int(std::max<unsigned>(1u, std::thread::hardware_concurrency()));
  const int got = acquire_spare_threads(int(std::max<int64_t>(0, std::min<int64_t>(hw, (n + 8191) / 8192) - 1)));
  const int64_t nt = 1 + got;
  if (nt <= 1) {
    f(int64_t(0), n);
    return;
  }
  std::vector<std::thread> th;
  for (int64_t t = 1; t < nt; ++t) {
    const int64_t a = n * t / nt, b = n * (t + 1) / nt;
    th.emplace_back([&f, a, b] { f(a, b); });
  }
  f(int64_t(0), n / nt);  // the first range on the calling thread
  for (auto& x : th) x.join();
  release_spare_threads(got);
}

inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
inline double uniform01(uint64_t seed, uint64_t idx) {
  const uint64_t z = mix64(seed + (idx + 1) * 0x9E3779B97F4A7C15ULL);
  return static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);
}

template <typename T>
int dmalloc(T** p, size_t count, const char* what) {
  DeviceLock lk(device_mutex());
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(UFEM_ERR_NOMEM, std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(e));
  }
  return UFEM_OK;
}

template <typename T>
void dfree(T*& p) {
  DeviceLock lk(device_mutex());
  if (p) cudaFree(p);
  p = nullptr;
}

int validate_options(const ufem_ns_options* o) {
  if (!o) return set_error(UFEM_ERR_ARG, "options pointer is NULL");
  if (!(o->theta > 0.0 && o->theta <= 1.0))
    return set_error(UFEM_ERR_ARG, "theta must lie in (0, 1] (NavierStokesAssembly.hpp:38-40 rejects values outside [0, 1]; 0 divides the pressure rows by zero)");
  if (!(o->dt > 0.0) || !std::isfinite(o->dt)) return set_error(UFEM_ERR_ARG, "dt must be positive and finite");
  if (!(o->rho > 0.0) || !std::isfinite(o->rho)) return set_error(UFEM_ERR_ARG, "rho must be positive and finite");
  if (o->supg_type < 0 || o->supg_type > 2) return set_error(UFEM_ERR_ARG, "supg_type must be 0, 1 or 2");
  if (o->precision < 0 || o->precision > 1) return set_error(UFEM_ERR_ARG, "precision must be 0 or 1");
  return UFEM_OK;
}

// Reference field layouts <-> padded 4-double node records.
__global__ void unpack_kernel(int64_t N, int src_stride, int src_off, int count, const double* __restrict__ src,
                              double* __restrict__ dst) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int k = 0; k < 4; ++k) dst[4 * i + k] = (k < count) ? src[i * src_stride + src_off + k] : 0.0;
}

__global__ void pack_kernel(int64_t N, int dst_stride, int dst_off, int count, const double* __restrict__ src,
                            double* __restrict__ dst) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int k = 0; k < count; ++k) dst[i * dst_stride + dst_off + k] = src[4 * i + k];
}

inline unsigned blocks(int64_t n, int t) { return unsigned((n + t - 1) / t); }

int check_device() {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return set_error(UFEM_ERR_CUDA, std::string("no CUDA device: ") + (e == cudaSuccess ? "count 0" : cudaGetErrorString(e)));
  int dev = 0;
  UFEM_CUDA_TRY(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  UFEM_CUDA_TRY(cudaGetDeviceProperties(&prop, dev));
  if (prop.major != 10)
    return set_error(UFEM_ERR_CUDA, std::string("device ") + prop.name + " is not sm_100 (this library is built for sm_100a only)");
  return UFEM_OK;
}

void free_bc_plan(DirichletPlan& b) {
  dfree(b.bc_dof); dfree(b.bc_first); dfree(b.bc_last); dfree(b.bc_diag);
  dfree(b.fix_row); dfree(b.fix_ptr); dfree(b.fix_pos); dfree(b.fix_bc); dfree(b.vfirst);
  dfree(b.neu_dof); dfree(b.neu_ptr); dfree(b.neu_val);
  dfree(b.fn_first); dfree(b.fn_last); dfree(b.fn_code); dfree(b.fn_off); dfree(b.fn_const);
  b.nbc = b.nfix_rows = b.nfix = b.nneu = 0;
}

// Slot of node `b` in the sorted neighbourhood of node `a`, or -1.
inline int64_t slot_of(const ufem_ns_handle* h, int64_t a, int64_t b) {
  const int32_t* first = h->adj_h.data() + h->start_h[a];
  const int32_t* last = h->adj_h.data() + h->start_h[a + 1];
  const int32_t* it = std::lower_bound(first, last, int32_t(b));
  return (it != last && *it == b) ? int64_t(it - first) : -1;
}

inline int64_t row_start(const ufem_ns_handle* h, int64_t node, int r) {
  const int64_t S = h->start_h[node + 1] - h->start_h[node];
  return int64_t(h->neq) * h->neq * h->start_h[node] + int64_t(r) * S * h->neq;
}

}  // namespace

// Turn the ordered BC list into the parallel plan.  Final state of the
// sequential reference (TrilinosFEVbrMatrix.cpp:482-553 applied in order):
//  - a constrained row is an identity row with rhs = sol = value_last - old;
//  - in every other row, each constrained column is moved to the RHS with the
//    value of that dof's FIRST application (later applications find a zero),
//    in first-application order, then zeroed.
// Constant Neumann faces (BCNeumannConstant.cpp:54-60 on Line2D): each face
// adds (weight * detJ) * ((N_i * flux) * |normal|) to the RHS dof of both of
// its nodes -- one Gauss point (weight 2), detJ = |x1 - x0| / 2
// (Line2D.cpp:109-114), N_i = 1/2, normal = (dy, -dx) / 2 (Line2D.cpp:83-87).
// The contributions are static (fixed mesh and flux): they are evaluated here
// once, in FP64, and kept per dof in face order so that the device adds them
// in the reference's order.
int build_neumann_plan(ufem_ns_handle* h) {
  DirichletPlan& bp = h->bcp;
  if (h->neumann.empty()) return UFEM_OK;
  const int neq = h->neq;
  std::vector<std::pair<int64_t, double>> c;  // (dof, contribution) in face order
  c.reserve(h->neumann.size() * 2);
  for (const auto& f : h->neumann) {
    const double* xa = &h->coords_h[size_t(f.a) * 2];
    const double* xb = &h->coords_h[size_t(f.b) * 2];
    const double dxdxi = 0.5 * (xb[0] - xa[0]), dydxi = 0.5 * (xb[1] - xa[1]);
    const double detj = std::sqrt(dxdxi * dxdxi + dydxi * dydxi);
    const double nx = 0.5 * (xb[1] - xa[1]), ny = 0.5 * (-xb[0] + xa[0]);
    const double nrm = std::sqrt(nx * nx + ny * ny);
    const double w = 2.0 * detj;
    const double v = w * ((0.5 * f.flux) * nrm);
    const int64_t ra = h->p2m_h.empty() ? f.a : h->p2m_h[f.a], rb = h->p2m_h.empty() ? f.b : h->p2m_h[f.b];
    c.push_back({ra * neq + f.comp, v});
    c.push_back({rb * neq + f.comp, v});
  }
  std::stable_sort(c.begin(), c.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
  std::vector<int64_t> dof, ptr(1, 0);
  std::vector<double> val;
  for (size_t i = 0; i < c.size(); ++i) {
    if (dof.empty() || dof.back() != c[i].first) {
      if (!dof.empty()) ptr.push_back(int64_t(val.size()));
      dof.push_back(c[i].first);
    }
    val.push_back(c[i].second);
  }
  ptr.push_back(int64_t(val.size()));
  int rc;
  if ((rc = dmalloc(&bp.neu_dof, dof.size(), "neumann dofs")) || (rc = dmalloc(&bp.neu_ptr, ptr.size(), "neumann")) ||
      (rc = dmalloc(&bp.neu_val, val.size(), "neumann values")))
    return rc;
  UFEM_CUDA_TRY(cudaMemcpy(bp.neu_dof, dof.data(), dof.size() * 8, cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemcpy(bp.neu_ptr, ptr.data(), ptr.size() * 8, cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemcpy(bp.neu_val, val.data(), val.size() * 8, cudaMemcpyHostToDevice));
  bp.nneu = int64_t(dof.size());
  return UFEM_OK;
}

int build_bc_plan(ufem_ns_handle* h) {
  DirichletPlan& bp = h->bcp;
  free_bc_plan(bp);
  bp.dirty = false;
  ++bp.version;
  int rc;
  if ((rc = build_neumann_plan(h))) return rc;
  if (h->bcs.empty()) return UFEM_OK;
  const int neq = h->neq;
  std::vector<int32_t> uid(size_t(h->nrows), -1);
  std::vector<int64_t> dofs;
  std::vector<double> first, last;
  std::vector<int32_t> ffirst, flast;  // expression of the first / last application, -1: constant
  for (const auto& e : h->bcs) {  // a linked node's condition acts on its master's row
    const int64_t dof = int64_t(h->p2m_h.empty() ? e.node : h->p2m_h[e.node]) * neq + e.comp;
    int32_t& u = uid[dof];
    if (u < 0) {
      u = int32_t(dofs.size());
      dofs.push_back(dof);
      first.push_back(e.value);
      last.push_back(e.value);
      ffirst.push_back(e.fn);
      flast.push_back(e.fn);
    } else {
      last[u] = e.value;
      flast[u] = e.fn;
    }
  }
  struct Fix {
    int64_t row, pos;
    int32_t bc;
  };
  std::vector<Fix> fixes;
  std::vector<int64_t> diag(dofs.size());
  for (size_t u = 0; u < dofs.size(); ++u) {
    const int64_t b = dofs[u] / neq;
    const int c = int(dofs[u] % neq);
    diag[u] = row_start(h, b, c) + slot_of(h, b, b) * neq + c;
    for (int64_t k = h->start_h[b]; k < h->start_h[b + 1]; ++k) {
      const int64_t col = h->adj_h[k];
      const int64_t sb = slot_of(h, col, b);
      if (sb < 0) continue;  // row does not hold the node (never for P1 graphs)
      for (int j = 0; j < neq; ++j) {
        const int64_t row = col * neq + j;
        if (uid[row] >= 0) continue;
        fixes.push_back(Fix{row, row_start(h, col, j) + sb * neq + c, int32_t(u)});
      }
    }
  }
  std::stable_sort(fixes.begin(), fixes.end(), [](const Fix& a, const Fix& b) { return a.row < b.row; });
  std::vector<int64_t> frow, fptr, fpos;
  std::vector<int32_t> fbc;
  for (size_t i = 0; i < fixes.size(); ++i) {
    if (i == 0 || fixes[i].row != fixes[i - 1].row) {
      frow.push_back(fixes[i].row);
      fptr.push_back(int64_t(i));
    }
    fpos.push_back(fixes[i].pos);
    fbc.push_back(fixes[i].bc);
  }
  fptr.push_back(int64_t(fixes.size()));
  bp.nbc = int64_t(dofs.size());
  bp.nfix_rows = int64_t(frow.size());
  bp.nfix = int64_t(fixes.size());
  if ((rc = dmalloc(&bp.bc_dof, dofs.size(), "bc_dof")) || (rc = dmalloc(&bp.bc_first, dofs.size(), "bc_first")) ||
      (rc = dmalloc(&bp.bc_last, dofs.size(), "bc_last")) || (rc = dmalloc(&bp.bc_diag, dofs.size(), "bc_diag")) ||
      (rc = dmalloc(&bp.vfirst, dofs.size(), "vfirst")) || (rc = dmalloc(&bp.fix_row, frow.size(), "fix_row")) ||
      (rc = dmalloc(&bp.fix_ptr, fptr.size(), "fix_ptr")) || (rc = dmalloc(&bp.fix_pos, fpos.size(), "fix_pos")) ||
      (rc = dmalloc(&bp.fix_bc, fbc.size(), "fix_bc")))
    return rc;
  UFEM_CUDA_TRY(cudaMemcpy(bp.bc_dof, dofs.data(), dofs.size() * 8, cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemcpy(bp.bc_first, first.data(), first.size() * 8, cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemcpy(bp.bc_last, last.data(), last.size() * 8, cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemcpy(bp.bc_diag, diag.data(), diag.size() * 8, cudaMemcpyHostToDevice));
  if (!h->fn_code.empty()) {  // function values: per-dof expression ids and the concatenated byte code
    std::vector<int32_t> code, off(1, 0);
    std::vector<double> k;
    for (size_t e = 0; e < h->fn_code.size(); ++e) {
      const int32_t base = int32_t(k.size());
      for (int32_t w : h->fn_code[e])  // constant operands are rebased onto the concatenated table
        code.push_back((w & 255) == kExprPushConst ? (kExprPushConst | (((w >> 8) + base) << 8)) : w);
      k.insert(k.end(), h->fn_const[e].begin(), h->fn_const[e].end());
      off.push_back(int32_t(code.size()));
    }
    if ((rc = dmalloc(&bp.fn_first, dofs.size(), "fn_first")) || (rc = dmalloc(&bp.fn_last, dofs.size(), "fn_last")) ||
        (rc = dmalloc(&bp.fn_code, code.size(), "fn_code")) || (rc = dmalloc(&bp.fn_off, off.size(), "fn_off")) ||
        (rc = dmalloc(&bp.fn_const, std::max<size_t>(k.size(), 1), "fn_const")))
      return rc;
    UFEM_CUDA_TRY(cudaMemcpy(bp.fn_first, ffirst.data(), ffirst.size() * 4, cudaMemcpyHostToDevice));
    UFEM_CUDA_TRY(cudaMemcpy(bp.fn_last, flast.data(), flast.size() * 4, cudaMemcpyHostToDevice));
    UFEM_CUDA_TRY(cudaMemcpy(bp.fn_code, code.data(), code.size() * 4, cudaMemcpyHostToDevice));
    UFEM_CUDA_TRY(cudaMemcpy(bp.fn_off, off.data(), off.size() * 4, cudaMemcpyHostToDevice));
    if (!k.empty()) UFEM_CUDA_TRY(cudaMemcpy(bp.fn_const, k.data(), k.size() * 8, cudaMemcpyHostToDevice));
  }
  if (!frow.empty()) {
    UFEM_CUDA_TRY(cudaMemcpy(bp.fix_row, frow.data(), frow.size() * 8, cudaMemcpyHostToDevice));
    UFEM_CUDA_TRY(cudaMemcpy(bp.fix_ptr, fptr.data(), fptr.size() * 8, cudaMemcpyHostToDevice));
    UFEM_CUDA_TRY(cudaMemcpy(bp.fix_pos, fpos.data(), fpos.size() * 8, cudaMemcpyHostToDevice));
    UFEM_CUDA_TRY(cudaMemcpy(bp.fix_bc, fbc.data(), fbc.size() * 4, cudaMemcpyHostToDevice));
  }
  return UFEM_OK;
}

namespace {

void record(ufem_ns_handle* h, int phase, bool stop, cudaStream_t s) {
  if (!h->timing) return;
  cudaEventRecord(h->ev[2 * phase + (stop ? 1 : 0)], s);
  if (stop) h->ev_rec[phase] = true;
}

void destroy_impl(ufem_ns_handle* h) {
  DeviceLock lk(device_mutex());
  if (h->view) {  // a system view borrows the graph, fields and tie list of its base handle
    h->d_start = nullptr;
    h->d_adj = nullptr;
    h->d_state = nullptr;
    h->d_tie = nullptr;
    h->d_coords = nullptr;
  }
  krylov_free(h);
  free_stage_pipe(h);
  free_bc_plan(h->bcp);
  dfree(h->d_coords); dfree(h->d_conn); dfree(h->d_state); dfree(h->d_hist); dfree(h->d_uadv);
  dfree(h->d_nu); dfree(h->d_force); dfree(h->d_node32); dfree(h->d_start); dfree(h->d_adj); dfree(h->d_rowptr);
  dfree(h->d_colidx); dfree(h->d_vals); dfree(h->d_vals32); dfree(h->d_rhs); dfree(h->d_sol);
  dfree(h->d_diagpos); dfree(h->d_row_inc); dfree(h->d_inc_elem); dfree(h->d_inc_info);
  dfree(h->plan64.chunks); dfree(h->plan32.chunks); dfree(h->d_tie);
  for (WarpPlan* wp : {&h->wplan, &h->wplan24}) {
    dfree(wp->groups);
    dfree(wp->big64.chunks);
    dfree(wp->big32.chunks);
  } dfree(h->d_stage); dfree(h->d_x); dfree(h->d_y);
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  delete h;
}

}  // namespace
}  // namespace ufem

using namespace ufem;

namespace ufem {
namespace {

// Periodic links -> node-to-row map (the reference's periodic_links_nodes /
// periodic_links_active, LSSAction.cpp:245-269): a linked (slave) node's row
// is its master's; chains resolve to the final master.  Empty map: no links.
int periodic_map(int64_t N, const uint32_t* slaves, const uint32_t* masters, int64_t nlinks,
                 std::vector<uint32_t>& p2m) {
  p2m.clear();
  if (nlinks == 0) return UFEM_OK;
  if (nlinks < 0 || !slaves || !masters) return set_error(UFEM_ERR_ARG, "invalid periodic link arrays");
  std::vector<int64_t> link(size_t(N), -1);
  for (int64_t i = 0; i < nlinks; ++i) {
    if (int64_t(slaves[i]) >= N || int64_t(masters[i]) >= N)
      return set_error(UFEM_ERR_ARG, "periodic link node id out of range");
    if (slaves[i] == masters[i]) return set_error(UFEM_ERR_ARG, "a node cannot be linked to itself");
    if (link[slaves[i]] >= 0)
      return set_error(UFEM_ERR_ARG, "node " + std::to_string(slaves[i]) + " is linked twice");
    link[slaves[i]] = masters[i];
  }
  p2m.resize(size_t(N));
  for (int64_t i = 0; i < N; ++i) {
    int64_t cur = i, steps = 0;
    while (link[cur] >= 0) {
      cur = link[cur];
      if (++steps > nlinks) return set_error(UFEM_ERR_ARG, "periodic links form a cycle");
    }
    p2m[i] = uint32_t(cur);
  }
  return UFEM_OK;
}

}  // namespace
}  // namespace ufem

namespace {
int create_impl(const ufem_mesh* mesh, const ufem_ns_options* opts, const uint32_t* slaves,
                const uint32_t* masters, int64_t nlinks, ufem_ns_handle** out, bool coupled = true) {
  if (!out) return set_error(UFEM_ERR_ARG, "out handle pointer is NULL");
  *out = nullptr;
  if (!mesh || !mesh->coords || !mesh->conn) return set_error(UFEM_ERR_ARG, "mesh or its arrays are NULL");
  if (mesh->dim != 2 && mesh->dim != 3) return set_error(UFEM_ERR_ARG, "dim must be 2 (Triag2D) or 3 (Tetra3D)");
  if (mesh->nb_nodes <= 0 || mesh->nb_elems <= 0) return set_error(UFEM_ERR_ARG, "empty mesh");
  int rc;
  if ((rc = validate_options(opts))) return rc;
  const int dim = mesh->dim, nn = dim + 1, neq = dim + 1;
  const int64_t N = mesh->nb_nodes, E = mesh->nb_elems;
  if (E * nn >= (int64_t(1) << 31) || N >= (int64_t(1) << 31) / neq)
    return set_error(UFEM_ERR_LIMIT, "mesh too large for 32-bit incidence/column indices");
  // --- validate connectivity and element Jacobians (non-invertible J is
  //     rejected, as cf3_assert(is_invertible) does in ElementData.hpp:311-313)
  {
    std::atomic<int64_t> bad_elem{-1}, bad_node{-1};
    parallel_for(E, [&](int64_t a, int64_t b) {
      for (int64_t e = a; e < b; ++e) {
        const uint32_t* c = mesh->conn + e * nn;
        bool ok = true;
        for (int k = 0; k < nn; ++k)
          if (int64_t(c[k]) >= N) ok = false;
        if (!ok) {
          bad_node = e;
          continue;
        }
        double J[3][3] = {{0}};
        for (int r = 0; r < dim; ++r)
          for (int q = 0; q < dim; ++q) J[r][q] = mesh->coords[int64_t(c[r + 1]) * dim + q] - mesh->coords[int64_t(c[0]) * dim + q];
        const double det = dim == 2 ? J[0][0] * J[1][1] - J[1][0] * J[0][1]
                                    : J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                                          J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                                          J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        if (!(det != 0.0) || !std::isfinite(det)) bad_elem = e;
      }
    });
    if (bad_node >= 0)
      return set_error(UFEM_ERR_MESH, "element " + std::to_string(int64_t(bad_node)) + " references a node id >= nb_nodes");
    if (bad_elem >= 0)
      return set_error(UFEM_ERR_MESH, "element " + std::to_string(int64_t(bad_elem)) + " has a non-invertible Jacobian");
    // every node must belong to an element: its LSS row would otherwise be empty
    // (the reference keeps such nodes out of the system via used_node_map)
    std::vector<uint8_t> used(size_t(N), 0);
    for (int64_t k = 0; k < E * nn; ++k) used[mesh->conn[k]] = 1;
    for (int64_t i = 0; i < N; ++i)
      if (!used[i]) return set_error(UFEM_ERR_MESH, "node " + std::to_string(i) + " is not referenced by any element");
  }
  std::vector<uint32_t> p2m;  // row of each node (periodic links); empty: the identity
  if ((rc = periodic_map(N, slaves, masters, nlinks, p2m))) return rc;
  auto row_of = [&](uint32_t node) { return p2m.empty() ? node : p2m[node]; };
  if (!p2m.empty())
    for (int64_t e = 0; e < E; ++e)
      for (int a = 0; a < nn; ++a)
        for (int b = a + 1; b < nn; ++b)
          if (row_of(mesh->conn[e * nn + a]) == row_of(mesh->conn[e * nn + b]))
            return set_error(UFEM_ERR_MESH, "element " + std::to_string(e) +
                                                " holds a node and its periodic partner (the mesh is too thin)");
  if ((rc = check_device())) return rc;
  if ((rc = configure_kernels())) return rc;

  ufem_ns_handle* h = new ufem_ns_handle();
  h->dim = dim;
  h->nn = nn;
  h->neq = neq;
  h->N = N;
  h->E = E;
  h->opt = *opts;
  h->p2m_h = p2m;
  auto fail = [&](int code) {
    destroy_impl(h);
    return code;
  };

  // --- node -> incident elements, ascending element id (counting sort)
  std::vector<int32_t> row_inc(N + 1, 0);
  for (int64_t e = 0; e < E; ++e)
    for (int a = 0; a < nn; ++a) row_inc[row_of(mesh->conn[e * nn + a]) + 1]++;
  for (int64_t i = 0; i < N; ++i) row_inc[i + 1] += row_inc[i];
  std::vector<int32_t> inc_elem(size_t(E) * nn);
  std::vector<uint8_t> inc_local(size_t(E) * nn);
  {
    std::vector<int32_t> fill(row_inc.begin(), row_inc.end() - 1);
    for (int64_t e = 0; e < E; ++e)
      for (int a = 0; a < nn; ++a) {
        const int32_t p = fill[row_of(mesh->conn[e * nn + a])]++;
        inc_elem[p] = int32_t(e);
        inc_local[p] = uint8_t(a);
      }
  }
  // --- node graph: sorted unique neighbours incl. self (SparsityBuilder.cpp:157-189)
  h->start_h.assign(N + 1, 0);
  {
    std::vector<int64_t> cnt(N, 0);
    parallel_for(N, [&](int64_t a, int64_t b) {
      std::vector<int32_t> tmp;
      for (int64_t i = a; i < b; ++i) {
        tmp.clear();
        for (int32_t p = row_inc[i]; p < row_inc[i + 1]; ++p) {
          const uint32_t* c = mesh->conn + int64_t(inc_elem[p]) * nn;
          for (int k = 0; k < nn; ++k) tmp.push_back(int32_t(row_of(c[k])));
        }
        if (!p2m.empty() && p2m[i] != uint32_t(i)) {  // linked node: tie row over itself and its master
          tmp.push_back(int32_t(i));
          tmp.push_back(int32_t(p2m[i]));
        }
        std::sort(tmp.begin(), tmp.end());
        cnt[i] = std::unique(tmp.begin(), tmp.end()) - tmp.begin();
      }
    });
    for (int64_t i = 0; i < N; ++i) {
      if (cnt[i] > 63)
        return fail(set_error(UFEM_ERR_LIMIT, "node " + std::to_string(i) + " has " + std::to_string(cnt[i]) +
                                                  " graph neighbours; the row-owner plan encodes at most 63"));
      h->start_h[i + 1] = h->start_h[i] + cnt[i];
    }
    h->adj_h.resize(h->start_h[N]);
    parallel_for(N, [&](int64_t a, int64_t b) {
      std::vector<int32_t> tmp;
      for (int64_t i = a; i < b; ++i) {
        tmp.clear();
        for (int32_t p = row_inc[i]; p < row_inc[i + 1]; ++p) {
          const uint32_t* c = mesh->conn + int64_t(inc_elem[p]) * nn;
          for (int k = 0; k < nn; ++k) tmp.push_back(int32_t(row_of(c[k])));
        }
        if (!p2m.empty() && p2m[i] != uint32_t(i)) {  // linked node: tie row over itself and its master
          tmp.push_back(int32_t(i));
          tmp.push_back(int32_t(p2m[i]));
        }
        std::sort(tmp.begin(), tmp.end());
        tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
        std::copy(tmp.begin(), tmp.end(), h->adj_h.begin() + h->start_h[i]);
      }
    });
  }
  h->bnnz = h->start_h[N];
  h->nrows = N * neq;
  h->nnz = h->bnnz * neq * neq;
  if (N < 1 || h->nnz >= (int64_t(1) << 40)) return fail(set_error(UFEM_ERR_LIMIT, "system too large"));
  // --- incidence info: 6-bit slot of each element node in the row's neighbourhood, local index << 24
  std::vector<uint32_t> inc_info(size_t(E) * nn);
  parallel_for(N, [&](int64_t a, int64_t b) {
    for (int64_t i = a; i < b; ++i)
      for (int32_t p = row_inc[i]; p < row_inc[i + 1]; ++p) {
        const uint32_t* c = mesh->conn + int64_t(inc_elem[p]) * nn;
        uint32_t info = uint32_t(inc_local[p]) << 24;
        for (int k = 0; k < nn; ++k) info |= uint32_t(slot_of(h, i, row_of(c[k]))) << (6 * k);
        if (nn == 3) info |= 63u << 18;  // no 4th node
        inc_info[p] = info;
      }
  });
  // --- chunks of whole rows with at most `cap` incidences (and slots), one plan
  // per kernel width; `only_big` restricts a plan to the rows the warp kernel
  // leaves out (more than 32 incidences).
  auto inc_of = [&](int64_t i) { return int64_t(row_inc[i + 1] - row_inc[i]); };
  auto slots_of = [&](int64_t i) { return h->start_h[i + 1] - h->start_h[i]; };
  auto make_chunks = [&](int cap, int big_above, std::vector<int2>& chunks) -> bool {
    const bool only_big = big_above > 0;
    int64_t i = 0;
    while (i < N) {
      // rows without incidences (tie rows of linked nodes) are written by the tie kernel
      if ((only_big && inc_of(i) <= big_above) || inc_of(i) == 0) { ++i; continue; }
      const int64_t first = i;
      int64_t k = 0, sl = 0;  // incidences and neighbourhood slots of the chunk, each <= cap
      while (i < N && (!only_big || inc_of(i) > big_above) && inc_of(i) > 0 && k + inc_of(i) <= cap &&
             sl + slots_of(i) <= cap) {
        k += inc_of(i);
        sl += slots_of(i);
        ++i;
      }
      if (i == first) return false;
      chunks.push_back(make_int2(int(first), int(i)));
    }
    return true;
  };
  std::vector<int2> chunks64, chunks32;
  if (!make_chunks(assembly_chunk_capacity(dim, 0), 0, chunks64) ||
      !make_chunks(assembly_chunk_capacity(dim, 1), 0, chunks32))
    return fail(set_error(UFEM_ERR_LIMIT, "a node has more incident elements than one assembly chunk holds"));
  h->plan64.cap = assembly_chunk_capacity(dim, 0);
  h->plan64.nchunks = int(chunks64.size());
  h->plan32.cap = assembly_chunk_capacity(dim, 1);
  h->plan32.nchunks = int(chunks32.size());
  // --- warp groups: consecutive rows with at most `cap` incidences in total;
  // rows with more go to a chunk plan that lists only them
  struct WarpPlanHost {
    std::vector<int4> groups;
    std::vector<int2> big64, big32;
  };
  auto make_warp_plan = [&](int cap, WarpPlan& wp, WarpPlanHost& hp) -> bool {
    for (int64_t i = 0; i < N;) {
      if (inc_of(i) > cap || inc_of(i) == 0) { ++i; continue; }
      const int64_t first = i;
      int64_t k = 0;
      while (i < N && inc_of(i) <= cap && inc_of(i) > 0 && k + inc_of(i) <= cap) k += inc_of(i++);
      hp.groups.push_back(make_int4(int(first), int(i), row_inc[first], int(k)));
    }
    if (!make_chunks(assembly_chunk_capacity(dim, 0), cap, hp.big64) ||
        !make_chunks(assembly_chunk_capacity(dim, 1), cap, hp.big32))
      return false;
    wp.cap = cap;
    wp.ngroups = int(hp.groups.size());
    wp.big64.cap = h->plan64.cap;
    wp.big64.nchunks = int(hp.big64.size());
    wp.big32.cap = h->plan32.cap;
    wp.big32.nchunks = int(hp.big32.size());
    return true;
  };
  WarpPlanHost wh32, wh24;
  if (!make_warp_plan(32, h->wplan, wh32) || (dim == 3 && !make_warp_plan(24, h->wplan24, wh24)))
    return fail(set_error(UFEM_ERR_LIMIT, "a node has more incident elements than one assembly chunk holds"));

  // --- device allocations and uploads.  Allocations take the library's device
  // mutex one by one (dmalloc); the uploads, the zeroing and the CSR build run on
  // a private stream that this call waits for alone, so building a handle does
  // not wait for (or hold up) the work other host threads have on the device.
  cudaStream_t cs = nullptr;
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess)
    return fail(set_error(UFEM_ERR_CUDA, "cudaStreamCreate failed"));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } stream_guard{cs};
  h->coords_h.assign(mesh->coords, mesh->coords + size_t(N) * dim);
  std::vector<double> c4(size_t(N) * 4, 0.0);
  for (int64_t i = 0; i < N; ++i)
    for (int k = 0; k < dim; ++k) c4[i * 4 + k] = mesh->coords[i * dim + k];
  std::vector<int32_t> conn4(size_t(E) * 4);
  for (int64_t e = 0; e < E; ++e)
    for (int k = 0; k < 4; ++k) conn4[e * 4 + k] = int32_t(mesh->conn[e * nn + (k < nn ? k : 0)]);
  if ((rc = dmalloc(&h->d_coords, c4.size(), "coords")) || (rc = dmalloc(&h->d_conn, conn4.size(), "conn")) ||
      (rc = dmalloc(&h->d_state, size_t(N) * 4, "state")) || (rc = dmalloc(&h->d_hist, size_t(N) * 12, "history")) ||
      (rc = dmalloc(&h->d_uadv, size_t(N) * 4, "u_adv")) || (rc = dmalloc(&h->d_nu, size_t(N), "nu")) ||
      (rc = dmalloc(&h->d_start, size_t(N) + 1, "start")) || (rc = dmalloc(&h->d_adj, size_t(h->bnnz), "adj")) ||
      (coupled && ((rc = dmalloc(&h->d_rowptr, size_t(h->nrows) + 1, "rowptr")) ||
                   (rc = dmalloc(&h->d_colidx, size_t(h->nnz), "colidx")) ||
                   (rc = dmalloc(&h->d_vals, size_t(h->nnz), "vals")) ||
                   (rc = dmalloc(&h->d_rhs, size_t(h->nrows), "rhs")) ||
                   (rc = dmalloc(&h->d_sol, size_t(h->nrows), "sol")) ||
                   (rc = dmalloc(&h->d_diagpos, size_t(h->nrows), "diagpos")))) ||
      (rc = dmalloc(&h->d_row_inc, size_t(N) + 1, "row_inc")) ||
      (rc = dmalloc(&h->d_inc_elem, inc_elem.size(), "inc_elem")) ||
      (rc = dmalloc(&h->d_inc_info, inc_info.size(), "inc_info")) ||
      (rc = dmalloc(&h->plan64.chunks, chunks64.size(), "chunks64")) ||
      (rc = dmalloc(&h->plan32.chunks, chunks32.size(), "chunks32")) ||
      (rc = dmalloc(&h->d_stage, size_t(N) * 4 * dim, "stage")))
    return fail(rc);
  if (coupled && opts->precision == 1 && ((rc = dmalloc(&h->d_vals32, size_t(h->nnz), "vals32")) ||
                               (rc = dmalloc(&h->d_node32, size_t(h->N) * 8, "node32"))))
    return fail(rc);
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, cs);  // pageable source: staged before return
  };
  cudaError_t ce = cudaSuccess;
  if ((ce = up(h->d_coords, c4.data(), c4.size() * 8)) || (ce = up(h->d_conn, conn4.data(), conn4.size() * 4)) ||
      (ce = up(h->d_start, h->start_h.data(), h->start_h.size() * 8)) ||
      (ce = up(h->d_adj, h->adj_h.data(), h->adj_h.size() * 4)) ||
      (ce = up(h->d_row_inc, row_inc.data(), row_inc.size() * 4)) ||
      (ce = up(h->d_inc_elem, inc_elem.data(), inc_elem.size() * 4)) ||
      (ce = up(h->d_inc_info, inc_info.data(), inc_info.size() * 4)) ||
      (ce = up(h->plan64.chunks, chunks64.data(), chunks64.size() * sizeof(int2))) ||
      (ce = up(h->plan32.chunks, chunks32.data(), chunks32.size() * sizeof(int2))))
    return fail(set_error(UFEM_ERR_CUDA, std::string("upload: ") + cudaGetErrorString(ce)));
  auto upload_warp_plan = [&](WarpPlan& wp, const WarpPlanHost& hp) -> int {
    int r;
    if ((r = dmalloc(&wp.groups, std::max<size_t>(hp.groups.size(), 1), "groups")) ||
        (r = dmalloc(&wp.big64.chunks, std::max<size_t>(hp.big64.size(), 1), "big rows")) ||
        (r = dmalloc(&wp.big32.chunks, std::max<size_t>(hp.big32.size(), 1), "big rows")))
      return r;
    cudaError_t e;
    if ((e = up(wp.groups, hp.groups.data(), hp.groups.size() * sizeof(int4))) ||
        (e = up(wp.big64.chunks, hp.big64.data(), hp.big64.size() * sizeof(int2))) ||
        (e = up(wp.big32.chunks, hp.big32.data(), hp.big32.size() * sizeof(int2))))
      return set_error(UFEM_ERR_CUDA, std::string("upload: ") + cudaGetErrorString(e));
    return UFEM_OK;
  };
  if ((rc = upload_warp_plan(h->wplan, wh32)) || (dim == 3 && (rc = upload_warp_plan(h->wplan24, wh24))))
    return fail(rc);
  if (!p2m.empty()) {  // tie rows of the linked nodes
    std::vector<int32_t> tie;
    for (int64_t i = 0; i < N; ++i)
      if (p2m[i] != uint32_t(i)) {
        tie.push_back(int32_t(i));
        tie.push_back(int32_t(p2m[i]));
      }
    h->ntie = int64_t(tie.size() / 2);
    if ((rc = dmalloc(&h->d_tie, std::max<size_t>(tie.size(), 1), "tie rows"))) return fail(rc);
    if ((ce = up(h->d_tie, tie.data(), tie.size() * 4)))
      return fail(set_error(UFEM_ERR_CUDA, std::string("upload: ") + cudaGetErrorString(ce)));
  }
  if ((coupled && ((ce = cudaMemsetAsync(h->d_sol, 0, size_t(h->nrows) * 8, cs)) ||
                   (ce = cudaMemsetAsync(h->d_rhs, 0, size_t(h->nrows) * 8, cs)))) ||
      (ce = cudaMemsetAsync(h->d_state, 0, size_t(N) * 32, cs)) ||
      (ce = cudaMemsetAsync(h->d_hist, 0, size_t(N) * 96, cs)) ||
      (ce = cudaMemsetAsync(h->d_uadv, 0, size_t(N) * 32, cs)) || (ce = cudaMemsetAsync(h->d_nu, 0, size_t(N) * 8, cs)))
    return fail(set_error(UFEM_ERR_CUDA, std::string("memset: ") + cudaGetErrorString(ce)));
  if (coupled && (rc = launch_build_csr(h, cs))) return fail(rc);
  if ((ce = cudaStreamSynchronize(cs)) != cudaSuccess)
    return fail(set_error(UFEM_ERR_CUDA, std::string("CSR build: ") + cudaGetErrorString(ce)));
  for (auto& e : h->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return fail(set_error(UFEM_ERR_CUDA, "cudaEventCreate failed"));
  *out = h;
  return UFEM_OK;
}
}  // namespace

namespace ufem {

int create_base(const ufem_mesh* mesh, const ufem_ns_options* opts, const uint32_t* slaves, const uint32_t* masters,
                int64_t nlinks, ufem_ns_handle** out) {
  return create_impl(mesh, opts, slaves, masters, nlinks, out, false);
}

int make_system_view(ufem_ns_handle* base, int neq, int state_offset, ufem_ns_handle** out) {
  *out = nullptr;
  ufem_ns_handle* v = new ufem_ns_handle();
  v->view = true;
  v->dim = base->dim;
  v->nn = base->nn;
  v->neq = neq;
  v->N = base->N;
  v->E = base->E;
  v->opt = base->opt;
  v->start_h = base->start_h;
  v->adj_h = base->adj_h;
  v->p2m_h = base->p2m_h;
  v->bnnz = base->bnnz;
  v->nrows = base->N * neq;
  v->nnz = base->bnnz * neq * neq;
  v->d_start = base->d_start;
  v->d_adj = base->d_adj;
  v->d_state = base->d_state + state_offset;
  v->d_coords = base->d_coords;  // function Dirichlet values
  v->ntie = base->ntie;
  v->d_tie = base->d_tie;
  int rc;
  {
    DeviceLock device_lock(device_mutex());
    if ((rc = dmalloc(&v->d_rowptr, size_t(v->nrows) + 1, "rowptr")) ||
        (rc = dmalloc(&v->d_colidx, size_t(v->nnz), "colidx")) || (rc = dmalloc(&v->d_vals, size_t(v->nnz), "vals")) ||
        (rc = dmalloc(&v->d_rhs, size_t(v->nrows), "rhs")) || (rc = dmalloc(&v->d_sol, size_t(v->nrows), "sol")) ||
        (rc = dmalloc(&v->d_diagpos, size_t(v->nrows), "diagpos"))) {
      destroy_impl(v);
      return rc;
    }
    cudaError_t ce;
    if ((ce = cudaMemset(v->d_sol, 0, size_t(v->nrows) * 8)) || (ce = cudaMemset(v->d_rhs, 0, size_t(v->nrows) * 8)) ||
        (ce = cudaMemset(v->d_vals, 0, size_t(v->nnz) * 8))) {
      destroy_impl(v);
      return set_error(UFEM_ERR_CUDA, std::string("memset: ") + cudaGetErrorString(ce));
    }
  }
  if ((rc = launch_build_csr(v, 0))) {
    destroy_impl(v);
    return rc;
  }
  cudaError_t ce = cudaDeviceSynchronize();
  if (ce != cudaSuccess) {
    destroy_impl(v);
    return set_error(UFEM_ERR_CUDA, std::string("CSR build: ") + cudaGetErrorString(ce));
  }
  *out = v;
  return UFEM_OK;
}

void destroy_handle(ufem_ns_handle* h) {
  if (h) destroy_impl(h);
}

}  // namespace ufem

extern "C" {

const char* ufem_last_error(void) { return ufem::g_err.c_str(); }
const char* ufem_version(void) { return "coolfluid3_b200 0.1 (UFEM PSPG/SUPG Navier-Stokes, sm_100a)"; }

void ufem_ns_default_options(ufem_ns_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->theta = 1.0;
  o->dt = 0.01;
  o->rho = 1.0;
  o->supg_type = 1;
  o->use_specializations = 1;
  o->c1 = 1.0;
  o->c2 = 16.0;
  o->alpha_ps = o->alpha_su = o->alpha_bu = 1.0;
  o->u_ref = 1.0;
  o->precision = 0;
}

void ufem_krylov_default_opts(ufem_krylov_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->method = 1;  // BiCGStab: on the PSPG/SUPG systems it needs ~2-8x fewer SpMVs than GMRES(30..200) with Jacobi
  o->restart = 30;
  o->max_iters = 3000;
  o->precond = 1;
  o->tol = 1e-10;
  o->mixed = 0;
  o->max_refine = 20;
  o->inner_tol = 1e-3;
}

int ufem_mesh_rectangle_tris(int32_t nx, int32_t ny, double jitter, uint64_t seed, double* coords, uint32_t* conn) {
  if (nx <= 0 || ny <= 0 || !coords || !conn) return set_error(UFEM_ERR_ARG, "invalid rectangle mesh arguments");
  const double xs = 1.0 / nx, ys = 1.0 / ny;
  for (int j = 0; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i) {
      const int64_t node = int64_t(j) * (nx + 1) + i;
      double x = static_cast<double>(i) * xs, y = static_cast<double>(j) * ys;
      if (i > 0 && i < nx && j > 0 && j < ny) {
        x += (2.0 * uniform01(seed, node * 4 + 0) - 1.0) * jitter * xs;
        y += (2.0 * uniform01(seed, node * 4 + 1) - 1.0) * jitter * ys;
      }
      coords[node * 2] = x;
      coords[node * 2 + 1] = y;
    }
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const uint32_t n0 = uint32_t(j * (nx + 1) + i), n1 = n0 + 1, n3 = uint32_t((j + 1) * (nx + 1) + i), n2 = n3 + 1;
      uint32_t* c = conn + 6 * (int64_t(j) * nx + i);
      c[0] = n0; c[1] = n2; c[2] = n3;
      c[3] = n0; c[4] = n1; c[5] = n2;
    }
  return UFEM_OK;
}

int ufem_mesh_cube_tets(int32_t n, double jitter, uint64_t seed, double* coords, uint32_t* conn) {
  if (n <= 0 || !coords || !conn) return set_error(UFEM_ERR_ARG, "invalid cube mesh arguments");
  const double h = 1.0 / n;
  const int64_t s = n + 1;
  parallel_for(s, [&](int64_t k0, int64_t k1) {
    for (int64_t k = k0; k < k1; ++k)
      for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
          const int64_t node = (k * s + j) * s + i;
          double p[3] = {i * h, j * h, double(k) * h};
          if (i > 0 && i < n && j > 0 && j < n && k > 0 && k < n)
            for (int c = 0; c < 3; ++c) p[c] += (2.0 * uniform01(seed, node * 4 + c) - 1.0) * jitter * h;
          for (int c = 0; c < 3; ++c) coords[node * 3 + c] = p[c];
        }
  });
  static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  static const int odd[6] = {0, 1, 1, 0, 0, 1};
  parallel_for(n, [&](int64_t k0, int64_t k1) {
    for (int64_t k = k0; k < k1; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          const int64_t cell = (k * n + j) * n + i;
          for (int t = 0; t < 6; ++t) {
            int64_t v[3] = {i, j, k};
            uint32_t ids[4];
            ids[0] = uint32_t((v[2] * s + v[1]) * s + v[0]);
            for (int m = 0; m < 3; ++m) {
              v[perm[t][m]] += 1;
              ids[m + 1] = uint32_t((v[2] * s + v[1]) * s + v[0]);
            }
            if (odd[t]) std::swap(ids[2], ids[3]);
            for (int m = 0; m < 4; ++m) conn[(cell * 6 + t) * 4 + m] = ids[m];
          }
        }
  });
  return UFEM_OK;
}

int ufem_ns_create(const ufem_mesh* mesh, const ufem_ns_options* opts, ufem_ns_handle** out) {
  return create_impl(mesh, opts, nullptr, nullptr, 0, out);
}

int ufem_ns_create_periodic(const ufem_mesh* mesh, const ufem_ns_options* opts, const uint32_t* slaves,
                            const uint32_t* masters, int64_t nlinks, ufem_ns_handle** out) {
  if (nlinks < 0 || (nlinks > 0 && (!slaves || !masters)))
    return set_error(UFEM_ERR_ARG, "invalid periodic link arrays");
  return create_impl(mesh, opts, slaves, masters, nlinks, out);
}

int ufem_ns_set_options(ufem_ns_handle* h, const ufem_ns_options* opts) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  int rc;
  if ((rc = validate_options(opts))) return rc;
  h->opt = *opts;
  if (opts->precision == 1 && !h->d_vals32 && (rc = dmalloc(&h->d_vals32, size_t(h->nnz), "vals32"))) return rc;
  if (opts->precision == 1 && !h->d_node32 && (rc = dmalloc(&h->d_node32, size_t(h->N) * 8, "node32"))) return rc;
  h->vals32_valid = false;
  return UFEM_OK;
}

int ufem_ns_device_bytes(const ufem_ns_handle* h, int64_t* bytes) {
  if (!h || !bytes) return set_error(UFEM_ERR_ARG, "NULL argument");
  const int64_t N = h->N, E = h->E, R = h->nrows, Z = h->nnz;
  int64_t b = N * (32 + 32 + 96 + 32 + 8) + E * 16 + (N + 1) * 12 + h->bnnz * 4 + (R + 1) * 8 + Z * 12 +
              R * (8 + 8 + 8) + E * h->nn * 8 + N * 16 + N * 4 * h->dim * 8;
  if (h->d_force) b += N * 32;
  if (h->d_vals32) b += Z * 4;
  if (h->d_node32) b += N * 32;
  b += krylov_device_bytes(h);  // solver workspace allocated so far (none for a batch member's vectors)
  if (h->pipe.buf[0]) b += 2 * (N * (h->neq + 4 * h->dim + 1) + R) * 8;  // overlapped-transfer buffers, once used
  if (h->d_tie) b += h->ntie * 8;
  b += h->bcp.nbc * 40 + h->bcp.nfix_rows * 16 + h->bcp.nfix * 12;
  *bytes = b;
  return UFEM_OK;
}

int ufem_ns_sizes(const ufem_ns_handle* h, int64_t* nb_rows, int64_t* nnz, int64_t* block_nnz) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (nb_rows) *nb_rows = h->nrows;
  if (nnz) *nnz = h->nnz;
  if (block_nnz) *block_nnz = h->bnnz;
  return UFEM_OK;
}

int ufem_ns_csr(ufem_ns_handle* h, int64_t* rowptr, int32_t* colidx) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (rowptr) UFEM_CUDA_TRY(cudaMemcpy(rowptr, h->d_rowptr, size_t(h->nrows + 1) * 8, cudaMemcpyDeviceToHost));
  if (colidx) UFEM_CUDA_TRY(cudaMemcpy(colidx, h->d_colidx, size_t(h->nnz) * 4, cudaMemcpyDeviceToHost));
  return UFEM_OK;
}

int ufem_ns_graph(ufem_ns_handle* h, int64_t* start, uint32_t* adj) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (start) std::copy(h->start_h.begin(), h->start_h.end(), start);
  if (adj)
    for (size_t k = 0; k < h->adj_h.size(); ++k) adj[k] = uint32_t(h->adj_h[k]);
  return UFEM_OK;
}

int ufem_ns_upload_state(ufem_ns_handle* h, const double* up, const double* lin, const double* nu, const double* force,
                         void* stream) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (!up || !lin || !nu) return set_error(UFEM_ERR_ARG, "up, lin and nu are required");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t N = h->N;
  const int d = h->dim, neq = h->neq;
  const unsigned g = blocks(N, 256);
  // solution field (u, v, [w], p) -> padded record, p at index dim
  UFEM_CUDA_TRY(cudaMemcpyAsync(h->d_stage, up, size_t(N) * neq * 8, cudaMemcpyHostToDevice, s));
  unpack_kernel<<<g, 256, 0, s>>>(N, neq, 0, neq, h->d_stage, h->d_state);
  UFEM_CUDA_TRY(cudaGetLastError());
  // linearized_velocity (u_adv, u1, u2, u3); the stage buffer is reused, so wait
  UFEM_CUDA_TRY(cudaStreamSynchronize(s));
  UFEM_CUDA_TRY(cudaMemcpyAsync(h->d_stage, lin, size_t(N) * 4 * d * 8, cudaMemcpyHostToDevice, s));
  unpack_kernel<<<g, 256, 0, s>>>(N, 4 * d, 0, d, h->d_stage, h->d_uadv);
  unpack_kernel<<<g, 256, 0, s>>>(N, 4 * d, d, d, h->d_stage, h->d_hist);
  unpack_kernel<<<g, 256, 0, s>>>(N, 4 * d, 2 * d, d, h->d_stage, h->d_hist + 4 * N);
  unpack_kernel<<<g, 256, 0, s>>>(N, 4 * d, 3 * d, d, h->d_stage, h->d_hist + 8 * N);
  UFEM_CUDA_TRY(cudaGetLastError());
  UFEM_CUDA_TRY(cudaMemcpyAsync(h->d_nu, nu, size_t(N) * 8, cudaMemcpyHostToDevice, s));
  if (force) {
    int rc;
    if (!h->d_force && (rc = dmalloc(&h->d_force, size_t(N) * 4, "force"))) return rc;
    UFEM_CUDA_TRY(cudaStreamSynchronize(s));
    UFEM_CUDA_TRY(cudaMemcpyAsync(h->d_stage, force, size_t(N) * d * 8, cudaMemcpyHostToDevice, s));
    unpack_kernel<<<g, 256, 0, s>>>(N, d, 0, d, h->d_stage, h->d_force);
    UFEM_CUDA_TRY(cudaGetLastError());
  } else if (h->d_force) {
    UFEM_CUDA_TRY(cudaStreamSynchronize(s));
    dfree(h->d_force);
  }
  h->state_set = true;
  return UFEM_OK;
}

int ufem_ns_set_state(ufem_ns_handle* h, const double* up, const double* lin, const double* nu, const double* force) {
  int rc = ufem_ns_upload_state(h, up, lin, nu, force, nullptr);
  if (rc) return rc;
  UFEM_CUDA_TRY(cudaStreamSynchronize(nullptr));
  return UFEM_OK;
}

int ufem_ns_download_state(ufem_ns_handle* h, double* up, double* lin, void* stream) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t N = h->N;
  const int d = h->dim, neq = h->neq;
  const unsigned g = blocks(N, 256);
  if (up) {
    pack_kernel<<<g, 256, 0, s>>>(N, neq, 0, neq, h->d_state, h->d_stage);
    UFEM_CUDA_TRY(cudaGetLastError());
    UFEM_CUDA_TRY(cudaMemcpyAsync(up, h->d_stage, size_t(N) * neq * 8, cudaMemcpyDeviceToHost, s));
  }
  if (lin) {
    if (up) UFEM_CUDA_TRY(cudaStreamSynchronize(s));
    pack_kernel<<<g, 256, 0, s>>>(N, 4 * d, 0, d, h->d_uadv, h->d_stage);
    pack_kernel<<<g, 256, 0, s>>>(N, 4 * d, d, d, h->d_hist, h->d_stage);
    pack_kernel<<<g, 256, 0, s>>>(N, 4 * d, 2 * d, d, h->d_hist + 4 * N, h->d_stage);
    pack_kernel<<<g, 256, 0, s>>>(N, 4 * d, 3 * d, d, h->d_hist + 8 * N, h->d_stage);
    UFEM_CUDA_TRY(cudaGetLastError());
    UFEM_CUDA_TRY(cudaMemcpyAsync(lin, h->d_stage, size_t(N) * 4 * d * 8, cudaMemcpyDeviceToHost, s));
  }
  return UFEM_OK;
}

int ufem_ns_get_state(ufem_ns_handle* h, double* up, double* lin) {
  int rc = ufem_ns_download_state(h, up, lin, nullptr);
  if (rc) return rc;
  UFEM_CUDA_TRY(cudaStreamSynchronize(nullptr));
  return UFEM_OK;
}

int ufem_ns_set_solution(ufem_ns_handle* h, const double* sol) {
  if (!h || !sol) return set_error(UFEM_ERR_ARG, "NULL argument");
  UFEM_CUDA_TRY(cudaMemcpy(h->d_sol, sol, size_t(h->nrows) * 8, cudaMemcpyHostToDevice));
  return UFEM_OK;
}

int ufem_ns_get_solution(ufem_ns_handle* h, double* sol) {
  if (!h || !sol) return set_error(UFEM_ERR_ARG, "NULL argument");
  UFEM_CUDA_TRY(cudaMemcpy(sol, h->d_sol, size_t(h->nrows) * 8, cudaMemcpyDeviceToHost));
  return UFEM_OK;
}

int ufem_ns_add_neumann(ufem_ns_handle* h, const uint32_t* faces, int64_t nfaces, int32_t comp, double flux) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (h->dim != 2)
    return set_error(UFEM_ERR_ARG, "constant Neumann conditions are defined on Line2D faces (2D meshes)");
  if (nfaces < 0 || (nfaces > 0 && !faces)) return set_error(UFEM_ERR_ARG, "invalid face array");
  if (comp < 0 || comp >= h->neq) return set_error(UFEM_ERR_ARG, "component out of range");
  if (!std::isfinite(flux)) return set_error(UFEM_ERR_ARG, "flux must be finite");
  for (int64_t i = 0; i < 2 * nfaces; ++i)
    if (int64_t(faces[i]) >= h->N) return set_error(UFEM_ERR_ARG, "Neumann face node id out of range");
  for (int64_t i = 0; i < nfaces; ++i) h->neumann.push_back({faces[2 * i], faces[2 * i + 1], comp, flux});
  h->bcp.dirty = true;
  ++h->bc_list_version;
  return UFEM_OK;
}

int ufem_ns_clear_neumann(ufem_ns_handle* h) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  h->neumann.clear();
  h->bcp.dirty = true;
  ++h->bc_list_version;
  return UFEM_OK;
}

int ufem_ns_add_dirichlet_function(ufem_ns_handle* h, const uint32_t* nodes, int64_t n, int32_t comp,
                                    const char* expr) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (!expr) return set_error(UFEM_ERR_ARG, "NULL expression");
  if (n < 0 || (n > 0 && !nodes)) return set_error(UFEM_ERR_ARG, "invalid node array");
  if (comp < 0 || comp >= h->neq) return set_error(UFEM_ERR_ARG, "component out of range");
  for (int64_t i = 0; i < n; ++i)
    if (int64_t(nodes[i]) >= h->N) return set_error(UFEM_ERR_ARG, "Dirichlet node id out of range");
  std::vector<int32_t> code;
  std::vector<double> k;
  std::string err;
  if (compile_expression(expr, code, k, err) != UFEM_OK) return set_error(UFEM_ERR_ARG, "Dirichlet function: " + err);
  const int32_t id = int32_t(h->fn_code.size());
  h->fn_code.push_back(std::move(code));
  h->fn_const.push_back(std::move(k));
  for (int64_t i = 0; i < n; ++i) h->bcs.push_back({nodes[i], comp, 0.0, id});
  h->bcp.dirty = true;
  ++h->bc_list_version;
  return UFEM_OK;
}

int ufem_ns_set_time(ufem_ns_handle* h, double t) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (!std::isfinite(t)) return set_error(UFEM_ERR_ARG, "time must be finite");
  h->time = t;
  return UFEM_OK;
}

int ufem_ns_get_time(const ufem_ns_handle* h, double* t) {
  if (!h || !t) return set_error(UFEM_ERR_ARG, "NULL argument");
  *t = h->time;
  return UFEM_OK;
}

int ufem_ns_clear_dirichlet(ufem_ns_handle* h) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  h->bcs.clear();
  h->fn_code.clear();
  h->fn_const.clear();
  h->bcp.dirty = true;
  ++h->bc_list_version;
  return UFEM_OK;
}

int ufem_ns_add_dirichlet(ufem_ns_handle* h, const uint32_t* nodes, int64_t n, int32_t comp, const double* values) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (n < 0 || (n > 0 && (!nodes || !values))) return set_error(UFEM_ERR_ARG, "invalid node/value arrays");
  if (comp < 0 || comp >= h->neq) return set_error(UFEM_ERR_ARG, "component out of range");
  for (int64_t i = 0; i < n; ++i)
    if (int64_t(nodes[i]) >= h->N) return set_error(UFEM_ERR_ARG, "Dirichlet node id out of range");
  for (int64_t i = 0; i < n; ++i) h->bcs.push_back({nodes[i], comp, values[i]});
  h->bcp.dirty = true;
  ++h->bc_list_version;
  return UFEM_OK;
}

int ufem_ns_add_dirichlet_dofs(ufem_ns_handle* h, const uint32_t* nodes, const int32_t* comps, const double* values,
                               int64_t n) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (n < 0 || (n > 0 && (!nodes || !comps || !values))) return set_error(UFEM_ERR_ARG, "invalid dof arrays");
  for (int64_t i = 0; i < n; ++i) {
    if (int64_t(nodes[i]) >= h->N) return set_error(UFEM_ERR_ARG, "Dirichlet node id out of range");
    if (comps[i] < 0 || comps[i] >= h->neq) return set_error(UFEM_ERR_ARG, "component out of range");
  }
  for (int64_t i = 0; i < n; ++i) h->bcs.push_back({nodes[i], comps[i], values[i]});
  h->bcp.dirty = true;
  ++h->bc_list_version;
  return UFEM_OK;
}

int ufem_ns_assemble(ufem_ns_handle* h, void* stream) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (!h->state_set) return set_error(UFEM_ERR_STATE, "ufem_ns_set_state must be called before assembly");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc;
  record(h, 0, false, s);
  if ((rc = launch_linearize(h, s))) return rc;
  record(h, 0, true, s);
  record(h, 1, false, s);
  const bool w32 = h->d_vals32 != nullptr;
  if ((rc = launch_assembly(h, s, w32))) return rc;
  if ((rc = launch_tie_rows(h, s, w32))) return rc;
  record(h, 1, true, s);
  h->vals32_valid = w32;
  h->conditioned = false;
  return UFEM_OK;
}

int ufem_ns_set_assembly_kernel(ufem_ns_handle* h, int32_t variant, int32_t warps_per_cta) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (variant != kAsmWarp && variant != kAsmChunk && variant != kAsmWarp24)
    return set_error(UFEM_ERR_ARG, "assembly variant must be 0, 1 or 2");
  if (variant == kAsmWarp24 && h->dim != 3)
    return set_error(UFEM_ERR_ARG, "assembly variant 2 (24-incidence groups) is for tetrahedra");
  if (warps_per_cta != 2 && warps_per_cta != 4 && warps_per_cta != 8)
    return set_error(UFEM_ERR_ARG, "warps_per_cta must be 2, 4 or 8");
  h->asm_variant = variant;
  h->asm_warps = warps_per_cta;
  return UFEM_OK;
}

int ufem_ns_get_assembly_kernel(ufem_ns_handle* h, int32_t* variant, int32_t* warps_per_cta) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (variant) *variant = h->asm_variant;
  if (warps_per_cta) *warps_per_cta = h->asm_warps;
  return UFEM_OK;
}

int ufem_ns_tune_assembly(ufem_ns_handle* h, void* stream, int32_t reps, int32_t* variant, int32_t* warps_per_cta,
                          float* ms_per_launch) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (!h->state_set) return set_error(UFEM_ERR_STATE, "ufem_ns_set_state must be called before tuning");
  if (reps < 1) reps = 5;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool w32 = h->d_vals32 != nullptr;
  struct Cand { int variant, warps; };
  std::vector<Cand> cands = {{kAsmWarp, 2}, {kAsmWarp, 4}, {kAsmWarp, 8}, {kAsmChunk, 4}};
  if (h->dim == 3) {
    cands.push_back({kAsmWarp24, 2});
    cands.push_back({kAsmWarp24, 4});
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  UFEM_CUDA_TRY(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return set_error(UFEM_ERR_CUDA, "cudaEventCreate failed");
  }
  int rc = UFEM_OK;
  float best = -1.0f;
  Cand pick = cands[0];
  const int saved_v = h->asm_variant, saved_w = h->asm_warps;
  if ((rc = launch_linearize(h, s)) == UFEM_OK) {
    for (const Cand& c : cands) {
      h->asm_variant = c.variant;
      h->asm_warps = c.warps;
      if ((rc = launch_assembly(h, s, w32))) break;  // warm-up
      cudaEventRecord(e0, s);
      for (int r = 0; r < reps && rc == UFEM_OK; ++r) rc = launch_assembly(h, s, w32);
      if (rc) break;
      cudaEventRecord(e1, s);
      cudaError_t ce = cudaEventSynchronize(e1);
      float ms = 0.0f;
      if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
      if (ce != cudaSuccess) {
        rc = set_error(UFEM_ERR_CUDA, std::string("assembly tuning: ") + cudaGetErrorString(ce));
        break;
      }
      ms /= float(reps);
      if (best < 0.0f || ms < best) {
        best = ms;
        pick = c;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {
    h->asm_variant = saved_v;
    h->asm_warps = saved_w;
    return rc;
  }
  h->asm_variant = pick.variant;
  h->asm_warps = pick.warps;
  h->vals32_valid = w32;
  if (variant) *variant = pick.variant;
  if (warps_per_cta) *warps_per_cta = pick.warps;
  if (ms_per_launch) *ms_per_launch = best;
  return UFEM_OK;
}

int ufem_ns_apply_dirichlet(ufem_ns_handle* h, void* stream) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc;
  if (h->bcp.dirty) {
    UFEM_CUDA_TRY(cudaStreamSynchronize(s));
    if ((rc = build_bc_plan(h))) return rc;
  }
  record(h, 2, false, s);
  if ((rc = launch_dirichlet_functions(h, s))) return rc;
  if ((rc = launch_neumann(h, s))) return rc;
  if ((rc = launch_dirichlet(h, s))) return rc;
  record(h, 2, true, s);
  h->conditioned = true;
  return UFEM_OK;
}

int ufem_ns_solve(ufem_ns_handle* h, const ufem_krylov_opts* kopts, ufem_krylov_status* status, void* stream) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  ufem_krylov_opts o;
  ufem_krylov_default_opts(&o);
  if (kopts) o = *kopts;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  record(h, 3, false, s);
  ufem_krylov_status st{};
  int rc = krylov_solve(h, &o, &st, s);
  if (rc) return rc;
  record(h, 3, true, s);
  if (status) *status = st;
  if (!st.converged) {
    static const char* why[] = {"ok", "maximum iterations reached", "breakdown", "non-finite values"};
    return set_error(UFEM_ERR_SOLVE, std::string("Krylov solve did not converge: ") + why[st.status & 3] +
                                         ", relative residual " + std::to_string(st.rel_residual));
  }
  return UFEM_OK;
}

int ufem_ns_prepare_solve(ufem_ns_handle* h, const ufem_krylov_opts* kopts, int32_t batched) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  ufem_krylov_opts o;
  ufem_krylov_default_opts(&o);
  if (kopts) o = *kopts;
  return krylov_prepare(h, &o, batched);
}

int ufem_ns_fp64_residual(ufem_ns_handle* h, double* r, void* stream) {
  if (!h || !r) return set_error(UFEM_ERR_ARG, "NULL argument");
  if (!h->state_set) return set_error(UFEM_ERR_STATE, "set the state before asking for the residual");
  return krylov_fp64_residual(h, r, static_cast<cudaStream_t>(stream));
}

int ufem_ns_update(ufem_ns_handle* h, void* stream) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  record(h, 4, false, s);
  int rc = launch_update(h, s);
  record(h, 4, true, s);
  if (rc == UFEM_OK) h->time += h->opt.dt;  // AdvanceTime after the step (function BCs read the time)
  return rc;
}

int ufem_ns_step(ufem_ns_handle* h, int32_t nsteps, const ufem_krylov_opts* kopts, ufem_krylov_status* status,
                 void* stream) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (nsteps < 0) return set_error(UFEM_ERR_ARG, "nsteps < 0");
  int rc;
  for (int32_t k = 0; k < nsteps; ++k) {
    if ((rc = ufem_ns_assemble(h, stream))) return rc;
    if ((rc = ufem_ns_apply_dirichlet(h, stream))) return rc;
    if ((rc = ufem_ns_solve(h, kopts, status, stream))) return rc;
    if ((rc = ufem_ns_update(h, stream))) return rc;
  }
  return UFEM_OK;
}

int ufem_ns_download_system(ufem_ns_handle* h, double* vals, double* rhs, void* stream) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (vals) UFEM_CUDA_TRY(cudaMemcpyAsync(vals, h->d_vals, size_t(h->nnz) * 8, cudaMemcpyDeviceToHost, s));
  if (rhs) UFEM_CUDA_TRY(cudaMemcpyAsync(rhs, h->d_rhs, size_t(h->nrows) * 8, cudaMemcpyDeviceToHost, s));
  return UFEM_OK;
}

int ufem_ns_get_system(ufem_ns_handle* h, double* vals, double* rhs) {
  int rc = ufem_ns_download_system(h, vals, rhs, nullptr);
  if (rc) return rc;
  {
    DeviceLock lk(device_mutex());
    UFEM_CUDA_TRY(cudaDeviceSynchronize());
  }
  return UFEM_OK;
}

int ufem_ns_device_view_get(const ufem_ns_handle* h, ufem_ns_device_view* v) {
  if (!h || !v) return set_error(UFEM_ERR_ARG, "NULL argument");
  v->rowptr = h->d_rowptr;
  v->colidx = h->d_colidx;
  v->vals = h->d_vals;
  v->rhs = h->d_rhs;
  v->solution = h->d_sol;
  v->nb_rows = h->nrows;
  v->nnz = h->nnz;
  return UFEM_OK;
}

int ufem_ns_apply(ufem_ns_handle* h, const double* x, double* y) {
  if (!h || !x || !y) return set_error(UFEM_ERR_ARG, "NULL argument");
  int rc;
  if (!h->d_x && ((rc = dmalloc(&h->d_x, size_t(h->nrows), "apply x")) || (rc = dmalloc(&h->d_y, size_t(h->nrows), "apply y"))))
    return rc;
  UFEM_CUDA_TRY(cudaMemcpy(h->d_x, x, size_t(h->nrows) * 8, cudaMemcpyHostToDevice));
  if ((rc = krylov_apply(h, h->d_x, h->d_y, nullptr))) return rc;
  UFEM_CUDA_TRY(cudaMemcpy(y, h->d_y, size_t(h->nrows) * 8, cudaMemcpyDeviceToHost));
  return UFEM_OK;
}

int ufem_ns_apply_device(ufem_ns_handle* h, const double* d_x, double* d_y, void* stream) {
  if (!h || !d_x || !d_y) return set_error(UFEM_ERR_ARG, "NULL argument");
  return krylov_apply(h, d_x, d_y, static_cast<cudaStream_t>(stream));
}

int ufem_ns_enable_timing(ufem_ns_handle* h, int32_t enable) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  h->timing = enable != 0;
  for (auto& r : h->ev_rec) r = false;
  return UFEM_OK;
}

int ufem_ns_get_timings(ufem_ns_handle* h, ufem_ns_timings* t) {
  if (!h || !t) return set_error(UFEM_ERR_ARG, "NULL argument");
  double out[5] = {0, 0, 0, 0, 0};
  for (int p = 0; p < 5; ++p) {
    if (!h->ev_rec[p]) continue;
    UFEM_CUDA_TRY(cudaEventSynchronize(h->ev[2 * p + 1]));
    float ms = 0.f;
    UFEM_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev[2 * p], h->ev[2 * p + 1]));
    out[p] = ms;
  }
  t->linearize_ms = out[0];
  t->assembly_ms = out[1];
  t->dirichlet_ms = out[2];
  t->solve_ms = out[3];
  t->update_ms = out[4];
  return UFEM_OK;
}

void ufem_ns_destroy(ufem_ns_handle* h) {
  if (!h) return;
  {
    DeviceLock lk(device_mutex());
    cudaDeviceSynchronize();
  }
  destroy_impl(h);
}

}  // extern "C"
