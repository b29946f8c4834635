// batch.cu -- many independent meshes stepped together (no counterpart in the
// reference, which runs one UFEM solver per process).
//
// A batch holds handles of the same dimension, element precision and element
// form.  Every phase of a time step is one launch over all members:
//  - linearisation, the symmetric Dirichlet passes and the update run over the
//    concatenated node / boundary-condition index spaces (a thread finds its
//    mesh by binary search over a prefix of the member sizes);
//  - the assembly is the persistent warp kernel over all members' row groups;
//  - the solve is BiCGStab with point Jacobi and PER-MESH scalars: each member
//    is split into fixed chunks of kChunkNodes nodes, vector kernels produce
//    one partial per chunk, and the last CTA of each mesh to finish (an atomic
//    counter per mesh) folds that mesh's partials in a fixed order and updates
//    its scalars, so an iteration is seven launches.  A member's arithmetic therefore depends only on its own
//    data: its results are bitwise the same alone (a batch of one) and in any
//    mix.  Converged members drop out (their kernels return at once) while the
//    others continue.  The mixed-precision solve iterates with an FP32 copy of
//    each operator and replaces the residual by the FP64 one every few blocks.
// The iteration block (8 BiCGStab iterations) is captured once into a CUDA
// graph and replayed; the host reads the members' done flags between blocks.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "internal.h"
#include "spmv_node.cuh"

namespace ufem {
namespace {

constexpr int kChunkNodes = 512;  // nodes per solver chunk (one CTA, one partial): 2048 rows for tets
constexpr int kThreads = 256;
constexpr int kBlockIters = 8;    // BiCGStab iterations per host check / graph replay
constexpr int kDc = 16;           // per-mesh double scalars
constexpr int kIc = 12;           // per-mesh int flags
constexpr int kMaxRestarts = 10;  // BiCGStab restarts after breakdowns in one solve

// per-mesh scalar slots (dctl[m * kDc + ...])
constexpr int sBnorm = 0, sBeta = 1, sEst = 2, sRho = 5, sRhoOld = 6, sAlpha = 7, sOmega = 8, sTrue = 9,
              sTol = 10, sTS = 11, sTT = 12, sLastTrue = 13, sRnorm = 14;
// per-mesh flags (ictl[m * kIc + ...])
constexpr int fDone = 0, fStatus = 2, fIters = 3, fMaxit = 4, fOuter = 5, fFinal = 6, fRepl = 7, fLastRepl = 8,
              fSkipRepl = 9;
// Mixed solve: a member's residual is replaced by the FP64 one when it claims
// convergence and every kReplaceIters of its own iterations (a per-member
// schedule, so its arithmetic does not depend on the other members).  Every
// replacement perturbs the BiCGStab recurrences; on the lid-driven systems a
// period of 32 cost 1.9x the FP64 iterations, 128 1.57x, 512 1.49x.
constexpr int kReplaceIters = 512;
// Matrix-free refinement (mixed = 2): iterations of one FP32-operator inner
// solve, as the one-handle refinement caps them (FP32 recurrences stagnate
// near the FP32-attainable accuracy; a fresh FP64 residual does better).
constexpr int kInnerIterCap = 400;
// graph slots of the captured iteration blocks: FP64, FP32 operator, and the
// matrix-free refinement's inner solve (its operands are the batch's own
// correction and scaled-residual vectors)
constexpr int kSlotMf = 2;

struct BatchMesh {
  int64_t N, nrows, row_off;  // row_off: first row in the concatenated solver vectors
  int dim, neq;
  double* state;
  double* hist;  // u1, u2, u3 (3 x N x 4)
  const double* nu;
  double* uadv;
  float* node32;
  const int64_t* start;
  const int32_t* adj;
  const int64_t* diagpos;
  const int64_t* rowptr;
  double* vals;
  float* vals32;
  double* rhs;
  double* sol;
  int64_t nbc, nfix_rows;
  const int64_t* bc_dof;
  const double* bc_first;
  const double* bc_last;
  const int64_t* bc_diag;
  double* vfirst;
  const int64_t* fix_row;
  const int64_t* fix_ptr;
  const int64_t* fix_pos;
  const int32_t* fix_bc;
  int active;  // 0: held (ufem_batch_set_active): no solve, no update
  // coarse space of the coupled two-level preconditioner (nc = 0: none)
  int nc;
  int64_t c_off;  // first coarse dof in the concatenated coarse vectors
  const int32_t* agg;
  const int32_t* agg_ptr;
  const int32_t* agg_rows;
  const double* ainv;
};

struct Chunk {
  int mesh, lo, hi, pad;  // local rows [lo, hi) of `mesh`
};

__device__ __forceinline__ int find_mesh(const int64_t* __restrict__ prefix, int nmesh, int64_t i) {
  int lo = 0, hi = nmesh - 1;
  while (lo < hi) {  // last m with prefix[m] <= i
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(prefix + mid) <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ double block_sum(double v, double* sm) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sm[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < int(blockDim.x >> 5); ++k) s += sm[k];
  __syncthreads();
  return s;
}

// ---- node-parallel phases ------------------------------------------------------

// LinearizeU + FP32 node copy, as linearize_kernel, over all members' nodes.
__global__ void linearize_batch_kernel(int64_t total, int nmesh, const int64_t* __restrict__ node_prefix,
                                       const BatchMesh* __restrict__ bm) {
  const int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int m = find_mesh(node_prefix, nmesh, g);
  const BatchMesh& M = bm[m];
  const int64_t i = g - node_prefix[m];
  const int dim = M.dim;
  const double* u1 = M.hist;
  const double* u2 = M.hist + 4 * M.N;
  const double* u3 = M.hist + 8 * M.N;
  double out[4] = {0, 0, 0, 0};
  for (int k = 0; k < dim; ++k) {
    const int64_t o = 4 * i + k;
    double v = __dsub_rn(__dmul_rn(2.1875, M.state[o]), __dmul_rn(2.1875, u1[o]));
    v = __dadd_rn(v, __dmul_rn(1.3125, u2[o]));
    v = __dsub_rn(v, __dmul_rn(0.3125, u3[o]));
    out[k] = v;
  }
  out[3] = M.nu[i];
  reinterpret_cast<double2*>(M.uadv + 4 * i)[0] = make_double2(out[0], out[1]);
  reinterpret_cast<double2*>(M.uadv + 4 * i)[1] = make_double2(out[2], out[3]);
  if (M.node32 != nullptr) {
    float4* q = reinterpret_cast<float4*>(M.node32) + 2 * i;
    q[0] = make_float4(float(out[0]), float(out[1]), float(out[2]), float(out[3]));
    const double* x = M.state + 4 * i;
    q[1] = make_float4(float(x[0]), float(x[1]), dim == 3 ? float(x[2]) : 0.0f, float(x[dim]));
  }
}

// u3 = u2, u2 = u1, u1 = u, u += du, p += dp
__global__ void update_batch_kernel(int64_t total, int nmesh, const int64_t* __restrict__ node_prefix,
                                    const BatchMesh* __restrict__ bm) {
  const int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int m = find_mesh(node_prefix, nmesh, g);
  const BatchMesh& M = bm[m];
  if (!M.active) return;
  const int64_t i = g - node_prefix[m];
  const int dim = M.dim, neq = M.neq;
  double* u1 = M.hist;
  double* u2 = M.hist + 4 * M.N;
  double* u3 = M.hist + 8 * M.N;
  for (int k = 0; k < dim; ++k) {
    const int64_t o = 4 * i + k;
    u3[o] = u2[o];
    u2[o] = u1[o];
    const double u = M.state[o];
    u1[o] = u;
    M.state[o] = __dadd_rn(u, M.sol[i * neq + k]);
  }
  M.state[4 * i + dim] = __dadd_rn(M.state[4 * i + dim], M.sol[i * neq + dim]);
}

// Symmetric Dirichlet over all members, the three passes of the one-mesh form.
__global__ void dirichlet_values_batch_kernel(int64_t total, int nmesh, const int64_t* __restrict__ bc_prefix,
                                              const BatchMesh* __restrict__ bm) {
  const int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int m = find_mesh(bc_prefix, nmesh, g);
  const BatchMesh& M = bm[m];
  const int64_t u = g - bc_prefix[m];
  const int64_t dof = M.bc_dof[u];
  const int64_t node = dof / M.neq;
  const int comp = int(dof - node * M.neq);
  M.vfirst[u] = __dsub_rn(M.bc_first[u], M.state[4 * node + comp]);
}

__global__ void dirichlet_columns_batch_kernel(int64_t total, int nmesh, const int64_t* __restrict__ fix_prefix,
                                               const BatchMesh* __restrict__ bm) {
  constexpr unsigned FULL = 0xffffffffu;
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;  // 8 lanes per row, as the one-mesh kernel
  if ((t >> 5) * 4 >= total) return;  // whole warp
  const int64_t g = t >> 3;
  const int sub = int(t & 7), gbase = int(threadIdx.x & 31) & ~7;
  const bool valid = g < total;
  const int m = valid ? find_mesh(fix_prefix, nmesh, g) : 0;
  const BatchMesh& M = bm[m];
  int64_t row = 0, k0 = 0;
  int len = 0;
  double r = 0.0;
  if (valid) {
    const int64_t q = g - fix_prefix[m];
    row = M.fix_row[q];
    k0 = M.fix_ptr[q];
    len = int(M.fix_ptr[q + 1] - k0);
    r = M.rhs[row];
  }
  int maxlen = len;
  maxlen = max(maxlen, __shfl_xor_sync(FULL, maxlen, 8));
  maxlen = max(maxlen, __shfl_xor_sync(FULL, maxlen, 16));
  for (int kb = 0; kb < maxlen; kb += 8) {
    const int n = len - kb;
    double term = 0.0;
    int64_t pos = -1;
    if (sub < n) {
      pos = M.fix_pos[k0 + kb + sub];
      term = __dmul_rn(-M.vals[pos], M.vfirst[M.fix_bc[k0 + kb + sub]]);
    }
    for (int j = 0; j < 8; ++j) {  // first-application order
      const double tj = __shfl_sync(FULL, term, gbase + j);
      if (j < n) r = __dadd_rn(r, tj);
    }
    if (sub < n) {
      M.vals[pos] = 0.0;
      if (M.vals32) M.vals32[pos] = 0.0f;
    }
  }
  if (valid && sub == 0) M.rhs[row] = r;
}

__global__ void dirichlet_rows_batch_kernel(int64_t total, int nmesh, const int64_t* __restrict__ bc_prefix,
                                            const BatchMesh* __restrict__ bm) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t g = t >> 3;  // eight lanes per constrained dof
  const int sub = int(t & 7);
  if (g >= total) return;
  const int m = find_mesh(bc_prefix, nmesh, g);
  const BatchMesh& M = bm[m];
  const int64_t u = g - bc_prefix[m];
  const int64_t dof = M.bc_dof[u];
  const int64_t diag = M.bc_diag[u];
  for (int64_t p = M.rowptr[dof] + sub; p < M.rowptr[dof + 1]; p += 8) {
    const double v = (p == diag) ? 1.0 : 0.0;
    M.vals[p] = v;
    if (M.vals32) M.vals32[p] = float(v);
  }
  if (sub == 0) {
    const int64_t node = dof / M.neq;
    const int comp = int(dof - node * M.neq);
    const double v = __dsub_rn(M.bc_last[u], M.state[4 * node + comp]);
    M.rhs[dof] = v;
    M.sol[dof] = v;
  }
}

// ---- solver kernels --------------------------------------------------------------
// Vector locations: a BiCGStab operand is either one of the batch's
// concatenated work vectors (offset by the mesh's row_off) or a member's own
// rhs / sol array.
enum Loc { kWork = 0, kRhs = 1, kSol = 2 };

template <int L>
__device__ __forceinline__ double* vec(const BatchMesh& M, double* work) {
  if constexpr (L == kRhs) return M.rhs;
  else if constexpr (L == kSol) return M.sol;
  else return work + M.row_off;
}

// y = A x over the solver chunks (one CTA per chunk of at most kChunkNodes
// nodes of one member; each warp walks its nodes with spmv4_walk, and for
// triangles 8-lane groups with spmv_group_walk, 4 nodes per warp at a time,
// each with the next node's loads in flight): a finished member's chunks return
// after one flag read, so an iteration costs what the members still iterating
// need, not a launch over every node of the batch.
template <int NEQ, typename MT, int XL>
__global__ void __launch_bounds__(256) spmv_chunk_kernel(const Chunk* __restrict__ chunks,
                                                         const BatchMesh* __restrict__ bm, double* xwork,
                                                         double* __restrict__ ywork, const int* __restrict__ ictl,
                                                         int skip_flag) {
  const Chunk c = chunks[blockIdx.x];
  if (ictl[c.mesh * kIc + skip_flag]) return;
  const BatchMesh& M = bm[c.mesh];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double* x = vec<XL>(M, xwork);
  double* y = ywork + M.row_off;
  const MT* vals;
  if constexpr (std::is_same<MT, float>::value) vals = M.vals32; else vals = M.vals;
  static_assert(NEQ == 4, "the tetrahedron chunks; triangles use spmv3_chunk_kernel");
  // the warp's nodes of the chunk, with the next node's loads in flight
  spmv4_walk<MT, double, double>(c.lo / NEQ + warp, c.hi / NEQ, int(blockDim.x >> 5), M.start, M.adj, vals, x, y,
                                 lane);
}

template <typename MT, int XL>
__global__ void __launch_bounds__(256) spmv3_chunk_kernel(const Chunk* __restrict__ chunks,
                                                          const BatchMesh* __restrict__ bm, double* xwork,
                                                          double* __restrict__ ywork, const int* __restrict__ ictl,
                                                          int skip_flag) {
  const Chunk c = chunks[blockIdx.x];
  if (ictl[c.mesh * kIc + skip_flag]) return;
  const BatchMesh& M = bm[c.mesh];
  const int grp = threadIdx.x >> 3, sub = threadIdx.x & 7;  // 4 nodes per warp, 8 lanes each
  const MT* vals;
  if constexpr (std::is_same<MT, float>::value) vals = M.vals32; else vals = M.vals;
  // the chunk's nodes, 32 at a time (the same trip count for every lane), with
  // each group's next node's loads in flight
  spmv_group_walk<3, MT, double, double>(c.lo / 3, c.hi / 3, int(blockDim.x >> 3), grp, sub, M.start, M.adj, vals,
                                         vec<XL>(M, xwork), ywork + M.row_off);
}

// dinv = 1 / diag (point Jacobi) of the operator the solve uses.
template <typename MT>
__global__ void jacobi_batch_kernel(const Chunk* __restrict__ chunks, const BatchMesh* __restrict__ bm,
                                    double* __restrict__ dinv, const int* __restrict__ ictl) {
  const Chunk c = chunks[blockIdx.x];
  if (ictl[c.mesh * kIc + fDone]) return;
  const BatchMesh& M = bm[c.mesh];
  const MT* vals;
  if constexpr (std::is_same<MT, float>::value) vals = M.vals32; else vals = M.vals;
#pragma unroll 4
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    const double d = double(vals[M.diagpos[i]]);
    dinv[M.row_off + i] = d != 0.0 ? 1.0 / d : 1.0;
  }
}

// r = b - w (w = A x), partials of r.r and b.b; rh = r when `init`.
template <int BL>
__global__ void residual_batch_kernel(const Chunk* __restrict__ chunks, const BatchMesh* __restrict__ bm,
                                      double* bwork, const double* __restrict__ w, double* __restrict__ r,
                                      double* __restrict__ rh, double* __restrict__ part, int nchunks,
                                      const int* __restrict__ ictl, int skip_done) {
  __shared__ double sm[32];
  const Chunk c = chunks[blockIdx.x];
  if (skip_done && ictl[c.mesh * kIc + fDone]) return;  // uniform per CTA
  const BatchMesh& M = bm[c.mesh];
  const double* b = vec<BL>(M, bwork);
  const int64_t off = M.row_off;
  double s2 = 0.0, b2 = 0.0;
#pragma unroll 4
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    const double bi = b[i];
    const double ri = bi - w[off + i];
    r[off + i] = ri;
    if (rh) rh[off + i] = ri;
    s2 += ri * ri;
    b2 += bi * bi;
  }
  s2 = block_sum(s2, sm);
  b2 = block_sum(b2, sm);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s2;
    part[nchunks + blockIdx.x] = b2;
  }
}

// Per-mesh fold of chunk partials: one warp per mesh, fixed order.
__device__ __forceinline__ void fold2(const double* part, int nchunks, int c0, int c1, double& a,
                                      double& b) {
  const int lane = threadIdx.x & 31;
  a = 0.0;
  b = 0.0;
  for (int k = c0 + lane; k < c1; k += 32) {  // L2 reads: partials written by other CTAs of this launch
    a += __ldcg(part + k);
    b += __ldcg(part + nchunks + k);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
}

// ---- fused iteration kernels ------------------------------------------------
// A chunk CTA writes its partial(s), and the last CTA of the mesh to finish
// (per-mesh counter, reset by that CTA) folds all of the mesh's partials in
// chunk order and applies the scalar update: deterministic, no waiting.
__device__ __forceinline__ bool last_chunk_of_mesh(int* counter, int nchunks_mesh, int* s_flag) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) *s_flag = (atomicAdd(counter, 1) == nchunks_mesh - 1) ? 1 : 0;
  __syncthreads();
  if (*s_flag == 0) return false;
  __threadfence();
  if (threadIdx.x == 0) *counter = 0;  // ready for the next launch
  return true;
}

// Dot partials over a vector chunk, MODE 1: rh.v (-> alpha), MODE 2: t.s and
// t.t (-> omega); the mesh's last CTA folds the partials in chunk order and
// updates the scalar.
template <int MODE>
__global__ void dot_fold_batch_kernel(const Chunk* __restrict__ chunks, const BatchMesh* __restrict__ bm,
                                      const int* __restrict__ cprefix, const double* __restrict__ a,
                                      const double* __restrict__ bv, double* __restrict__ part, int nchunks,
                                      double* __restrict__ dctl, int* __restrict__ ictl,
                                      int* __restrict__ counters) {
  __shared__ double sm[32];
  __shared__ int s_flag;
  const Chunk c = chunks[blockIdx.x];
  const int m = c.mesh;
  if (ictl[m * kIc + fDone]) return;  // uniform per CTA
  const int64_t off = bm[m].row_off;
  double pa = 0.0, pb = 0.0;
#pragma unroll 4
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    const int64_t k = off + i;
    const double ai = a[k];
    pa += ai * bv[k];              // MODE 1: rh . v ; MODE 2: t . s
    if (MODE == 2) pb += ai * ai;  // t . t
  }
  pa = block_sum(pa, sm);
  if (MODE == 2) pb = block_sum(pb, sm);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = pa;
    part[nchunks + blockIdx.x] = pb;
  }
  const int c0 = cprefix[m], c1 = cprefix[m + 1];
  if (!last_chunk_of_mesh(counters + m * 4 + MODE - 1, c1 - c0, &s_flag)) return;
  if (threadIdx.x >= 32) return;
  double fa, fb;
  fold2(part, nchunks, c0, c1, fa, fb);
  if (threadIdx.x != 0) return;
  double* d = dctl + m * kDc;
  int* f = ictl + m * kIc;
  if (MODE == 1) {  // alpha = rho / (rh . v)
    if (fa == 0.0 || !isfinite(fa)) {
      f[fDone] = 1;
      f[fStatus] = isfinite(fa) ? 2 : 3;
      return;
    }
    const double al = d[sRho] / fa;
    if (!(fabs(al) < 1e150)) {
      f[fDone] = 1;
      f[fStatus] = 2;
      return;
    }
    d[sAlpha] = al;
  } else {  // omega = (t . s) / (t . t)
    const double om = (fb != 0.0) ? fa / fb : 0.0;
    d[sTS] = fa;
    d[sTT] = fb;
    d[sOmega] = om;
    if (!isfinite(om)) {
      f[fDone] = 1;
      f[fStatus] = 3;
    } else if (om == 0.0 && fb != 0.0) {
      f[fStatus] = 2;  // breakdown: x still advances by alpha ph, then the solve stops
    }
  }
}

// x += alpha ph + omega sh ; r = s - omega t ; partials of r.r and rh.r; the
// mesh's last CTA computes rho_new, the residual estimate and convergence.
template <int XL>
__global__ void bicg_xr_end_batch_kernel(const Chunk* __restrict__ chunks, const BatchMesh* __restrict__ bm,
                                         const int* __restrict__ cprefix, const double* __restrict__ ph,
                                         const double* __restrict__ sh, const double* __restrict__ s,
                                         const double* __restrict__ t, const double* __restrict__ rh,
                                         double* xwork, double* __restrict__ r, double* __restrict__ dctl,
                                         int* __restrict__ ictl, double* __restrict__ part, int nchunks,
                                         int* __restrict__ counters) {
  __shared__ double sm[32];
  __shared__ int s_flag;
  const Chunk c = chunks[blockIdx.x];
  const int m = c.mesh;
  if (ictl[m * kIc + fDone]) return;
  const BatchMesh& M = bm[m];
  const double al = dctl[m * kDc + sAlpha], om = dctl[m * kDc + sOmega];
  const int64_t off = M.row_off;
  double* x = vec<XL>(M, xwork);
  double rr = 0.0, hr = 0.0;
#pragma unroll 4
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    const int64_t k = off + i;
    x[i] = x[i] + al * ph[k] + om * sh[k];
    const double ri = s[k] - om * t[k];
    r[k] = ri;
    rr += ri * ri;
    hr += rh[k] * ri;
  }
  rr = block_sum(rr, sm);
  hr = block_sum(hr, sm);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = rr;
    part[nchunks + blockIdx.x] = hr;
  }
  const int c0 = cprefix[m], c1 = cprefix[m + 1];
  if (!last_chunk_of_mesh(counters + m * 4 + 2, c1 - c0, &s_flag)) return;
  if (threadIdx.x >= 32) return;
  double nn, rho_new;
  fold2(part, nchunks, c0, c1, nn, rho_new);
  if (threadIdx.x != 0) return;
  double* d = dctl + m * kDc;
  int* f = ictl + m * kIc;
  const double rn = sqrt(nn);
  d[sEst] = rn;
  d[sRhoOld] = d[sRho];
  d[sRho] = rho_new;
  f[fIters] += 1;
  if (f[fStatus] == 2) {
    f[fDone] = 1;
  } else if (!isfinite(rn) || !isfinite(rho_new)) {
    f[fDone] = 1;
    f[fStatus] = 3;
  } else if (rn <= d[sTol] * d[sBnorm]) {
    f[fDone] = 1;
  } else if (rho_new == 0.0) {
    f[fDone] = 1;
    f[fStatus] = 2;
  } else if (f[fIters] >= f[fMaxit]) {
    f[fDone] = 1;
    f[fStatus] = 1;
  }
}

// Start of a solve: ||r0||, ||b||, BiCGStab scalars, per-mesh tol / maxit.
// `outer_done` meshes (already converged in the refinement loop) stay done.
__global__ void bicg_init_batch_kernel(int nmesh, const int* __restrict__ cprefix, const double* __restrict__ part,
                                       int nchunks, double* __restrict__ dctl, int* __restrict__ ictl, double tol,
                                       int maxit, int use_outer) {
  const int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (m >= nmesh) return;
  double rr, bb;
  fold2(part, nchunks, cprefix[m], cprefix[m + 1], rr, bb);
  if ((threadIdx.x & 31) != 0) return;
  double* d = dctl + m * kDc;
  int* f = ictl + m * kIc;
  const double beta = sqrt(rr), bnorm = sqrt(bb);
  d[sBeta] = beta;
  d[sBnorm] = bnorm;
  d[sEst] = beta;
  d[sRho] = rr;
  d[sRhoOld] = 1.0;
  d[sAlpha] = 1.0;
  d[sOmega] = 1.0;
  d[sTol] = tol;
  d[sLastTrue] = beta;
  f[fMaxit] = maxit;
  f[fIters] = 0;
  f[fStatus] = isfinite(beta) ? 0 : 3;
  f[fDone] = (f[fStatus] != 0 || beta <= tol * bnorm || bnorm == 0.0 || (use_outer && f[fOuter])) ? 1 : 0;
  f[fFinal] = f[fDone];  // (residual replacement only visits meshes that are not final)
  f[fRepl] = 0;
  f[fLastRepl] = 0;
}

// p = r + beta (p - omega v), ph = D^-1 p
__global__ void bicg_p_batch_kernel(const Chunk* __restrict__ chunks, const BatchMesh* __restrict__ bm, int pkind,
                                    const double* __restrict__ dinv, const double* __restrict__ r,
                                    const double* __restrict__ v, double* __restrict__ p, double* __restrict__ ph,
                                    const double* __restrict__ dctl, const int* __restrict__ ictl) {
  const Chunk c = chunks[blockIdx.x];
  if (ictl[c.mesh * kIc + fDone]) return;
  const double* d = dctl + c.mesh * kDc;
  const double beta = (d[sRho] / d[sRhoOld]) * (d[sAlpha] / d[sOmega]);
  const double om = d[sOmega];
  const int64_t off = bm[c.mesh].row_off;
#pragma unroll 4
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    const int64_t k = off + i;
    const double pi = r[k] + beta * (p[k] - om * v[k]);
    p[k] = pi;
    ph[k] = (pkind == 1 || pkind == 4) ? dinv[k] * pi : pi;
  }
}



// Coupled two-level preconditioner over the batch (z += R Ac^-1 R^T v per
// member).  Restriction: one warp per coarse dof of all members, the sum over
// its aggregate's rows (ascending) in a fixed lane partition and shuffle tree.
__global__ void restrict_batch_kernel(int64_t total_c, int nmesh, const int64_t* __restrict__ cprefix,
                                      const BatchMesh* __restrict__ bm, const double* __restrict__ v,
                                      double* __restrict__ c, const int* __restrict__ ictl) {
  const int64_t q = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (q >= total_c) return;  // whole warps
  const int m = find_mesh(cprefix, nmesh, q);
  if (ictl[m * kIc + fDone]) return;
  const BatchMesh& M = bm[m];
  const int I = int(q - cprefix[m]);
  double s = 0.0;
  for (int k = M.agg_ptr[I] + lane; k < M.agg_ptr[I + 1]; k += 32) s += v[M.row_off + M.agg_rows[k]];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) c[q] = s;
}

// y = Ac^-1 c per member, one warp per coarse row.
__global__ void coarse_batch_kernel(int64_t total_c, int nmesh, const int64_t* __restrict__ cprefix,
                                    const BatchMesh* __restrict__ bm, const double* __restrict__ c,
                                    double* __restrict__ y, const int* __restrict__ ictl) {
  const int64_t q = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (q >= total_c) return;
  const int m = find_mesh(cprefix, nmesh, q);
  if (ictl[m * kIc + fDone]) return;
  const BatchMesh& M = bm[m];
  const int I = int(q - cprefix[m]);
  const double* row = M.ainv + int64_t(I) * M.nc;
  const double* cm = c + M.c_off;
  double s = 0.0;
  for (int J = lane; J < M.nc; J += 32) s += row[J] * cm[J];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) y[q] = s;
}

// z += y[agg] on the coarse rows of each chunk's member.
__global__ void prolong_add_batch_kernel(const Chunk* __restrict__ chunks, const BatchMesh* __restrict__ bm,
                                         const double* __restrict__ y, double* __restrict__ z,
                                         const int* __restrict__ ictl) {
  const Chunk c = chunks[blockIdx.x];
  if (ictl[c.mesh * kIc + fDone]) return;
  const BatchMesh& M = bm[c.mesh];
  if (M.nc == 0) return;
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    const int a = M.agg[i];
    if (a >= 0) z[M.row_off + i] += y[M.c_off + a];
  }
}

// s = r - alpha v, sh = D^-1 s
__global__ void bicg_s_batch_kernel(const Chunk* __restrict__ chunks, const BatchMesh* __restrict__ bm, int pkind,
                                    const double* __restrict__ dinv, const double* __restrict__ r,
                                    const double* __restrict__ v, double* __restrict__ s, double* __restrict__ sh,
                                    const double* __restrict__ dctl, const int* __restrict__ ictl) {
  const Chunk c = chunks[blockIdx.x];
  if (ictl[c.mesh * kIc + fDone]) return;
  const double al = dctl[c.mesh * kDc + sAlpha];
  const int64_t off = bm[c.mesh].row_off;
#pragma unroll 4
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    const int64_t k = off + i;
    const double si = r[k] - al * v[k];
    s[k] = si;
    sh[k] = (pkind == 1 || pkind == 4) ? dinv[k] * si : si;
  }
}




// True residual of the finished solve: relres = ||b - A x|| / ||b|| into dctl[sTrue].
__global__ void true_res_batch_kernel(int nmesh, const int* __restrict__ cprefix, const double* __restrict__ part,
                                      int nchunks, double* __restrict__ dctl) {
  const int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (m >= nmesh) return;
  double rr, bb;
  fold2(part, nchunks, cprefix[m], cprefix[m + 1], rr, bb);
  if ((threadIdx.x & 31) != 0) return;
  const double bn = sqrt(bb);
  dctl[m * kDc + sTrue] = bn > 0.0 ? sqrt(rr) / bn : (isfinite(rr) ? 0.0 : NAN);
  dctl[m * kDc + sBnorm] = bn;
}

// Mixed solve, FP64 residual replacement ("reliable update"): the iterations
// apply the FP32 copy of the operator, whose rounding makes the recursive
// residual drift from the true one; every few blocks r is replaced by the FP64
// residual b - A x of the assembled FP64 system (x is kept in FP64), and rho =
// rh . r is recomputed.  The Krylov directions are kept, so the iteration
// count stays close to that of the FP64 solve while the answer is FP64's.
template <int BL>
__global__ void replace_batch_kernel(const Chunk* __restrict__ chunks, const BatchMesh* __restrict__ bm,
                                     double* bwork, const double* __restrict__ w, double* __restrict__ r,
                                     const double* __restrict__ rh, double* __restrict__ part, int nchunks,
                                     const int* __restrict__ ictl) {
  __shared__ double sm[32];
  const Chunk c = chunks[blockIdx.x];
  if (ictl[c.mesh * kIc + fSkipRepl]) return;
  const BatchMesh& M = bm[c.mesh];
  const double* b = vec<BL>(M, bwork);
  const int64_t off = M.row_off;
  double rr = 0.0, hr = 0.0;
#pragma unroll 4
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    const double ri = b[i] - w[off + i];
    r[off + i] = ri;
    rr += ri * ri;
    hr += rh[off + i] * ri;
  }
  rr = block_sum(rr, sm);
  hr = block_sum(hr, sm);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = rr;
    part[nchunks + blockIdx.x] = hr;
  }
}

// After a replacement: converged on the TRUE residual -> final; iteration
// limit, breakdown or non-finite -> final with that status; otherwise go on
// (also when the recursive residual had already claimed convergence).
__global__ void replace_end_batch_kernel(int nmesh, const int* __restrict__ cprefix,
                                         const double* __restrict__ part, int nchunks, double* __restrict__ dctl,
                                         int* __restrict__ ictl) {
  const int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (m >= nmesh || ictl[m * kIc + fSkipRepl]) return;
  double rr, hr;
  fold2(part, nchunks, cprefix[m], cprefix[m + 1], rr, hr);
  if ((threadIdx.x & 31) != 0) return;
  double* d = dctl + m * kDc;
  int* f = ictl + m * kIc;
  const double rn = sqrt(rr);
  d[sEst] = rn;
  if (!isfinite(rn) || !isfinite(hr)) {
    f[fStatus] = 3;
    f[fDone] = f[fFinal] = 1;
  } else if (rn <= d[sTol] * d[sBnorm]) {
    f[fStatus] = 0;
    f[fDone] = f[fFinal] = 1;
  } else if (f[fDone] && f[fStatus] != 0) {  // iteration limit or breakdown
    f[fFinal] = 1;
  } else if (rn > 10.0 * d[sLastTrue]) {
    // the true residual grew since the last replacement: treat as a breakdown,
    // the solve restarts from this iterate
    f[fStatus] = 2;
    f[fDone] = f[fFinal] = 1;
  } else {
    d[sRho] = hr;
    f[fDone] = 0;
  }
  d[sLastTrue] = rn;
  f[fRepl] += 1;
  f[fLastRepl] = f[fIters];
}

// x = 0 where b = 0 (the solution of A x = 0), as the one-mesh solver does.
template <int XL>
__global__ void zero_x_if_b0_kernel(const Chunk* __restrict__ chunks, const BatchMesh* __restrict__ bm,
                                    double* xwork, const double* __restrict__ dctl, const int* __restrict__ ictl,
                                    int use_outer) {
  const Chunk c = chunks[blockIdx.x];
  if (dctl[c.mesh * kDc + sBnorm] != 0.0 || (use_outer && ictl[c.mesh * kIc + fOuter])) return;
  double* x = vec<XL>(bm[c.mesh], xwork);
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) x[i] = 0.0;
}

__global__ void zero_batch_kernel(const Chunk* __restrict__ chunks, const BatchMesh* __restrict__ bm,
                                  double* __restrict__ a, double* __restrict__ b) {
  const Chunk c = chunks[blockIdx.x];
  const int64_t off = bm[c.mesh].row_off;
#pragma unroll 4
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    a[off + i] = 0.0;
    if (b) b[off + i] = 0.0;
  }
}

// ---- matrix-free refinement (mixed = 2) --------------------------------------
// The refinement of the one-handle solve, for every member at once: r = b - M x
// of each member's FP64 system from the element pass (launch_mf_residual, one
// launch per member), the members' norms, the FP32-operator inner solve of
// A32 z = r / ||r|| (batched BiCGStab), x += ||r|| z.  Members outside the pass
// (converged, stopped or held) carry fOuter.

// chunk partials of r.r and b.b (b: the member's assembled RHS); members outside
// the pass write zeros
__global__ void mf_norm_batch_kernel(const Chunk* __restrict__ chunks, const BatchMesh* __restrict__ bm,
                                     const double* __restrict__ r, double* __restrict__ part, int nchunks,
                                     const int* __restrict__ ictl) {
  __shared__ double sm[32];
  const Chunk c = chunks[blockIdx.x];
  const BatchMesh& M = bm[c.mesh];
  double s2 = 0.0, b2 = 0.0;
  if (!ictl[c.mesh * kIc + fOuter]) {  // uniform per CTA
    const int64_t off = M.row_off;
    for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
      const double ri = r[off + i], bi = M.rhs[i];
      s2 += ri * ri;
      b2 += bi * bi;
    }
  }
  s2 = block_sum(s2, sm);
  b2 = block_sum(b2, sm);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s2;
    part[nchunks + blockIdx.x] = b2;
  }
}

// per member, one warp, chunk order: ||r||, ||b|| and ||r|| / ||b||
__global__ void mf_fold_batch_kernel(int nmesh, const int* __restrict__ cprefix, const double* __restrict__ part,
                                     int nchunks, double* __restrict__ dctl) {
  const int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (m >= nmesh) return;
  double rr, bb;
  fold2(part, nchunks, cprefix[m], cprefix[m + 1], rr, bb);
  if ((threadIdx.x & 31) != 0) return;
  const double rn = sqrt(rr), bn = sqrt(bb);
  dctl[m * kDc + sRnorm] = rn;
  dctl[m * kDc + sBnorm] = bn;
  dctl[m * kDc + sTrue] = bn > 0.0 ? rn / bn : (isfinite(rr) ? 0.0 : NAN);
}

// inner right-hand side r / ||r|| and a zero correction, members in the pass
__global__ void mf_scale_batch_kernel(const Chunk* __restrict__ chunks, const BatchMesh* __restrict__ bm,
                                      const double* __restrict__ r, double* __restrict__ bin,
                                      double* __restrict__ z, const double* __restrict__ dctl,
                                      const int* __restrict__ ictl) {
  const Chunk c = chunks[blockIdx.x];
  if (ictl[c.mesh * kIc + fOuter]) return;
  const int64_t off = bm[c.mesh].row_off;
  const double inv = 1.0 / dctl[c.mesh * kDc + sRnorm];
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    bin[off + i] = r[off + i] * inv;
    z[off + i] = 0.0;
  }
}

// x += ||r|| z, members in the pass
__global__ void mf_update_batch_kernel(const Chunk* __restrict__ chunks, const BatchMesh* __restrict__ bm,
                                       const double* __restrict__ z, const double* __restrict__ dctl,
                                       const int* __restrict__ ictl) {
  const Chunk c = chunks[blockIdx.x];
  if (ictl[c.mesh * kIc + fOuter]) return;
  const BatchMesh& M = bm[c.mesh];
  const double sc = dctl[c.mesh * kDc + sRnorm];
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) M.sol[i] += sc * z[M.row_off + i];
}

template <typename T>
int dmal(T** p, size_t n) {
  DeviceLock lk(device_mutex());
  const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(UFEM_ERR_NOMEM, std::string("batch cudaMalloc: ") + cudaGetErrorString(e));
  }
  return UFEM_OK;
}
template <typename T>
void dfr(T*& p) {
  DeviceLock lk(device_mutex());
  if (p) cudaFree(p);
  p = nullptr;
}

}  // namespace
}  // namespace ufem

using namespace ufem;

struct ufem_batch {
  std::vector<ufem_ns_handle*> members;
  std::vector<int32_t> active;  // per member: 1 stepped, 0 held
  bool active_dirty = false;
  std::vector<CoarseView> coarse;  // per member (two-level preconditioner); nc = 0: none
  int64_t total_c = 0;             // coarse dofs of all members
  int64_t* d_coarse_prefix = nullptr;
  double* cvec = nullptr;          // total_c: R^T v of every member
  double* yvec = nullptr;          // total_c: Ac^-1 R^T v
  int64_t c_cap = 0;
  int dim = 0, neq = 0, precision = 0, spec = 0, warps = 4;
  int nmesh = 0;
  int64_t total_nodes = 0, total_rows = 0, total_bc = 0, total_fix = 0;
  int ngroups = 0, nchunks = 0;
  bool graphs = true;
  // device
  AsmDesc* d_asm = nullptr;
  int* d_gprefix = nullptr;
  BatchMesh* d_mesh = nullptr;
  int64_t* d_node_prefix = nullptr;
  int64_t* d_bc_prefix = nullptr;
  int64_t* d_fix_prefix = nullptr;
  Chunk* d_chunks = nullptr;
  int* d_cprefix = nullptr;
  double *r = nullptr, *rh = nullptr, *p = nullptr, *v = nullptr, *s = nullptr, *t = nullptr, *ph = nullptr,
         *sh = nullptr, *dinv = nullptr, *w = nullptr;
  double* part = nullptr;
  int* counters = nullptr;  // per mesh: last-CTA counters of the fused kernels (4 ints)
  double* dctl = nullptr;
  int* ictl = nullptr;
  double* h_dctl = nullptr;
  int* h_ictl = nullptr;
  // captured iteration blocks: [FP64, FP32 operator, matrix-free inner solve]
  cudaGraphExec_t block_exec[3] = {nullptr, nullptr, nullptr};
  cudaStream_t capture_stream = nullptr;
  int block_pkind[3] = {-1, -1, -1};
  // matrix-free refinement (mixed = 2): the members' FP64 residuals, the inner
  // solve's right-hand sides (residual / its norm) and corrections
  double *mfr = nullptr, *mfb = nullptr, *mfz = nullptr;
};

namespace {

void batch_free(ufem_batch* b) {
  DeviceLock lk(device_mutex());
  for (auto& g : b->block_exec)
    if (g) cudaGraphExecDestroy(g);
  if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
  dfr(b->d_asm); dfr(b->d_gprefix); dfr(b->d_mesh); dfr(b->d_node_prefix); dfr(b->d_bc_prefix);
  dfr(b->d_fix_prefix); dfr(b->d_chunks); dfr(b->d_cprefix);
  dfr(b->r); dfr(b->rh); dfr(b->p); dfr(b->v); dfr(b->s); dfr(b->t); dfr(b->ph); dfr(b->sh); dfr(b->dinv);
  dfr(b->w); dfr(b->part); dfr(b->counters); dfr(b->dctl); dfr(b->ictl);
  dfr(b->d_coarse_prefix); dfr(b->cvec); dfr(b->yvec);
  dfr(b->mfr); dfr(b->mfb); dfr(b->mfz);
  if (b->h_dctl) cudaFreeHost(b->h_dctl);
  if (b->h_ictl) cudaFreeHost(b->h_ictl);
  delete b;
}

// (Re)build the member descriptors: Dirichlet plans and pointers may change
// between steps (new BC lists, FP32 buffers allocated on option changes).
int batch_refresh(ufem_batch* b) {
  int rc;
  std::vector<AsmDesc> ad(b->nmesh);
  std::vector<BatchMesh> bm(b->nmesh);
  std::vector<int64_t> bcp(b->nmesh + 1, 0), fxp(b->nmesh + 1, 0);
  for (int m = 0; m < b->nmesh; ++m) {
    ufem_ns_handle* h = b->members[m];
    if (h->bcp.dirty && (rc = build_bc_plan(h))) return rc;
    fill_desc(h, h->d_vals32 != nullptr, ad[m]);
    BatchMesh& M = bm[m];
    M.N = h->N;
    M.nrows = h->nrows;
    M.dim = h->dim;
    M.neq = h->neq;
    M.state = h->d_state;
    M.hist = h->d_hist;
    M.nu = h->d_nu;
    M.uadv = h->d_uadv;
    M.node32 = h->opt.precision == 1 ? h->d_node32 : nullptr;
    M.start = h->d_start;
    M.adj = h->d_adj;
    M.diagpos = h->d_diagpos;
    M.rowptr = h->d_rowptr;
    M.vals = h->d_vals;
    M.vals32 = h->d_vals32;
    M.rhs = h->d_rhs;
    M.sol = h->d_sol;
    const DirichletPlan& P = h->bcp;
    M.nbc = P.nbc;
    M.nfix_rows = P.nfix_rows;
    M.bc_dof = P.bc_dof;
    M.bc_first = P.bc_first;
    M.bc_last = P.bc_last;
    M.bc_diag = P.bc_diag;
    M.vfirst = P.vfirst;
    M.fix_row = P.fix_row;
    M.fix_ptr = P.fix_ptr;
    M.fix_pos = P.fix_pos;
    M.fix_bc = P.fix_bc;
    M.active = b->active[m];
    const CoarseView cv = m < int(b->coarse.size()) ? b->coarse[m] : CoarseView{};
    M.nc = cv.nc;
    M.agg = cv.agg;
    M.agg_ptr = cv.agg_ptr;
    M.agg_rows = cv.agg_rows;
    M.ainv = cv.ainv;
    bcp[m + 1] = bcp[m] + P.nbc;
    fxp[m + 1] = fxp[m] + P.nfix_rows;
  }
  int64_t off = 0;
  std::vector<int64_t> cpre(size_t(b->nmesh) + 1, 0);
  for (int m = 0; m < b->nmesh; ++m) {
    bm[m].row_off = off;
    off += bm[m].nrows;
    bm[m].c_off = cpre[size_t(m)];
    cpre[size_t(m) + 1] = cpre[size_t(m)] + bm[m].nc;
  }
  if (cpre[size_t(b->nmesh)] != b->total_c) {  // the coarse kernels' grids change: recapture the iteration graphs
    DeviceLock lk(device_mutex());
    for (int k = 0; k < 3; ++k)
      if (b->block_exec[k]) {
        cudaGraphExecDestroy(b->block_exec[k]);
        b->block_exec[k] = nullptr;
      }
  }
  b->total_c = cpre[size_t(b->nmesh)];
  if (b->total_c > b->c_cap) {
    dfr(b->cvec);
    dfr(b->yvec);
    if ((rc = dmal(&b->cvec, size_t(b->total_c))) || (rc = dmal(&b->yvec, size_t(b->total_c)))) return rc;
    b->c_cap = b->total_c;
  }
  if (!b->d_coarse_prefix && (rc = dmal(&b->d_coarse_prefix, size_t(b->nmesh) + 1))) return rc;
  UFEM_CUDA_TRY(cudaMemcpy(b->d_coarse_prefix, cpre.data(), cpre.size() * 8, cudaMemcpyHostToDevice));
  b->total_bc = bcp[b->nmesh];
  b->total_fix = fxp[b->nmesh];
  UFEM_CUDA_TRY(cudaMemcpy(b->d_asm, ad.data(), ad.size() * sizeof(AsmDesc), cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemcpy(b->d_mesh, bm.data(), bm.size() * sizeof(BatchMesh), cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemcpy(b->d_bc_prefix, bcp.data(), bcp.size() * 8, cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemcpy(b->d_fix_prefix, fxp.data(), fxp.size() * 8, cudaMemcpyHostToDevice));
  b->active_dirty = false;
  return UFEM_OK;
}

bool batch_dirty(const ufem_batch* b) {
  if (b->active_dirty) return true;
  for (const ufem_ns_handle* h : b->members)
    if (h->bcp.dirty) return true;
  return false;
}

inline unsigned blocks_for(int64_t n, int threads) { return unsigned((n + threads - 1) / threads); }

template <typename MT, int XL>
int spmv_b(ufem_batch* b, double* x, double* y, cudaStream_t st, int skip_flag = fDone) {
  const unsigned nc = unsigned(b->nchunks);
  if (b->neq == 4)
    spmv_chunk_kernel<4, MT, XL><<<nc, 256, 0, st>>>(b->d_chunks, b->d_mesh, x, y, b->ictl, skip_flag);
  else
    spmv3_chunk_kernel<MT, XL><<<nc, 256, 0, st>>>(b->d_chunks, b->d_mesh, x, y, b->ictl, skip_flag);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

// z += R Ac^-1 R^T v for every member with a coarse space (two-level form).
int coarse_correct_b(ufem_batch* b, const double* v, double* z, cudaStream_t st) {
  if (b->total_c == 0) return UFEM_OK;
  const unsigned gw = unsigned((b->total_c * 32 + 255) / 256);
  restrict_batch_kernel<<<gw, 256, 0, st>>>(b->total_c, b->nmesh, b->d_coarse_prefix, b->d_mesh, v, b->cvec, b->ictl);
  coarse_batch_kernel<<<gw, 256, 0, st>>>(b->total_c, b->nmesh, b->d_coarse_prefix, b->d_mesh, b->cvec, b->yvec,
                                          b->ictl);
  prolong_add_batch_kernel<<<unsigned(b->nchunks), kThreads, 0, st>>>(b->d_chunks, b->d_mesh, b->yvec, z, b->ictl);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

// One BiCGStab iteration for every member that is not done: seven launches
// (p update; SpMV; rh.v + alpha; s update; SpMV; t.s, t.t + omega; x, r update
// + rho and convergence), the scalars computed by each mesh's last CTA.
template <typename MT, int XL>
int bicg_iteration(ufem_batch* b, int pkind, double* xwork, cudaStream_t st) {
  const unsigned nc = unsigned(b->nchunks);
  int rc;
  bicg_p_batch_kernel<<<nc, kThreads, 0, st>>>(b->d_chunks, b->d_mesh, pkind, b->dinv, b->r, b->v, b->p, b->ph,
                                                b->dctl, b->ictl);
  if (pkind == 4 && (rc = coarse_correct_b(b, b->p, b->ph, st))) return rc;
  if ((rc = spmv_b<MT, kWork>(b, b->ph, b->v, st))) return rc;
  dot_fold_batch_kernel<1><<<nc, kThreads, 0, st>>>(b->d_chunks, b->d_mesh, b->d_cprefix, b->rh, b->v, b->part,
                                                     b->nchunks, b->dctl, b->ictl, b->counters);
  bicg_s_batch_kernel<<<nc, kThreads, 0, st>>>(b->d_chunks, b->d_mesh, pkind, b->dinv, b->r, b->v, b->s, b->sh,
                                                b->dctl, b->ictl);
  if (pkind == 4 && (rc = coarse_correct_b(b, b->s, b->sh, st))) return rc;
  if ((rc = spmv_b<MT, kWork>(b, b->sh, b->t, st))) return rc;
  dot_fold_batch_kernel<2><<<nc, kThreads, 0, st>>>(b->d_chunks, b->d_mesh, b->d_cprefix, b->t, b->s, b->part,
                                                     b->nchunks, b->dctl, b->ictl, b->counters);
  bicg_xr_end_batch_kernel<XL><<<nc, kThreads, 0, st>>>(b->d_chunks, b->d_mesh, b->d_cprefix, b->ph, b->sh, b->s,
                                                         b->t, b->rh, xwork, b->r, b->dctl, b->ictl, b->part,
                                                         b->nchunks, b->counters);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

// r = b - A x with partials; XL / BL: where x and b live.
template <typename MT, int XL, int BL>
int residual_b(ufem_batch* b, double* x, double* bw, bool init_rh, bool skip_done, cudaStream_t st) {
  int rc;
  if ((rc = spmv_b<MT, XL>(b, x, b->w, st))) return rc;
  residual_batch_kernel<BL><<<unsigned(b->nchunks), kThreads, 0, st>>>(
      b->d_chunks, b->d_mesh, bw, b->w, b->r, init_rh ? b->rh : nullptr, b->part, b->nchunks, b->ictl,
      skip_done ? 1 : 0);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

// BiCGStab over the batch.  MT: operator values; XL/BL: solution and RHS
// locations; `use_outer`: skip meshes already converged in refinement.
template <typename MT, int XL, int BL>
int bicgstab_b(ufem_batch* b, int pkind, double tol, int maxit, bool use_outer, int slot, cudaStream_t st,
               bool reliable = false, double* xw = nullptr, double* bw = nullptr) {
  // xw / bw: the solution and RHS when they are batch work vectors (kWork);
  // for kSol / kRhs they are the members' own arrays and these stay null
  const unsigned nc = unsigned(b->nchunks);
  const unsigned gm = blocks_for(int64_t(b->nmesh) * 32, 256);
  int rc;
  // every mesh takes part in the set-up (flags are reset by the init kernel)
  if (use_outer)  // flags prepared by the caller in the host mirror: fOuter set, the rest zero
    UFEM_CUDA_TRY(cudaMemcpyAsync(b->ictl, b->h_ictl, sizeof(int) * kIc * b->nmesh, cudaMemcpyHostToDevice, st));
  else
    UFEM_CUDA_TRY(cudaMemsetAsync(b->ictl, 0, sizeof(int) * kIc * b->nmesh, st));
  if (pkind == 1 || pkind == 4)
    jacobi_batch_kernel<MT><<<nc, kThreads, 0, st>>>(b->d_chunks, b->d_mesh, b->dinv, b->ictl);
  // the initial residual is FP64 in a mixed solve (residual replacement)
  if ((rc = reliable ? residual_b<double, XL, BL>(b, xw, bw, true, false, st)
                     : residual_b<MT, XL, BL>(b, xw, bw, true, false, st)))
    return rc;
  zero_batch_kernel<<<nc, kThreads, 0, st>>>(b->d_chunks, b->d_mesh, b->p, b->v);
  bicg_init_batch_kernel<<<gm, 256, 0, st>>>(b->nmesh, b->d_cprefix, b->part, b->nchunks, b->dctl, b->ictl, tol,
                                             maxit, use_outer ? 1 : 0);
  zero_x_if_b0_kernel<XL><<<nc, kThreads, 0, st>>>(b->d_chunks, b->d_mesh, xw, b->dctl, b->ictl, use_outer ? 1 : 0);
  UFEM_CUDA_TRY(cudaGetLastError());
  const bool use_graph = b->graphs;
  if (use_graph && (b->block_exec[slot] == nullptr || b->block_pkind[slot] != pkind)) {
    DeviceLock lk(device_mutex());  // no implicit device synchronisation from other threads during capture
    if (b->block_exec[slot]) {
      cudaGraphExecDestroy(b->block_exec[slot]);
      b->block_exec[slot] = nullptr;
    }
    cudaGraph_t g = nullptr;
    UFEM_CUDA_TRY(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
    int crc = UFEM_OK;
    for (int k = 0; k < kBlockIters && crc == UFEM_OK; ++k) crc = bicg_iteration<MT, XL>(b, pkind, xw, b->capture_stream);
    const cudaError_t ce = cudaStreamEndCapture(b->capture_stream, &g);
    if (crc) {
      if (g) cudaGraphDestroy(g);
      return crc;
    }
    if (ce != cudaSuccess) return set_error(UFEM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    const cudaError_t ie = cudaGraphInstantiate(&b->block_exec[slot], g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return set_error(UFEM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    b->block_pkind[slot] = pkind;
  }
  // The host reads the members' flags after 1, then 2, 4 and at most 8 replays
  // of the 8-iteration block: few synchronisations on long solves, little
  // overshoot on short ones (finished members' kernels return at once).  The
  // schedule depends on the iteration count only, so a member's arithmetic
  // (replacements included) is the same alone and in any batch.
  int blocks = 0;
  for (int it = 0, reps = 1; it < maxit + kBlockIters; it += reps * kBlockIters, reps = std::min(2 * reps, 8)) {
    for (int r = 0; r < reps; ++r) {
      if (use_graph) {
        UFEM_CUDA_TRY(cudaGraphLaunch(b->block_exec[slot], st));
      } else {
        for (int k = 0; k < kBlockIters; ++k)
          if ((rc = bicg_iteration<MT, XL>(b, pkind, xw, st))) return rc;
      }
    }
    ++blocks;
    UFEM_CUDA_TRY(cudaMemcpyAsync(b->h_ictl, b->ictl, sizeof(int) * kIc * b->nmesh, cudaMemcpyDeviceToHost, st));
    UFEM_CUDA_TRY(cudaStreamSynchronize(st));
    bool all = true;
    for (int m = 0; m < b->nmesh && all; ++m) all = b->h_ictl[m * kIc + fDone] != 0;
    if (!reliable) {
      if (all) break;
      continue;
    }
    // members due for a replacement: not final, and either claiming
    // convergence (or stopped) or kReplaceIters past their last replacement
    bool any_due = false;
    for (int m = 0; m < b->nmesh; ++m) {
      int* f = b->h_ictl + m * kIc;
      const bool due = !f[fFinal] && (f[fDone] || f[fIters] - f[fLastRepl] >= kReplaceIters);
      f[fSkipRepl] = due ? 0 : 1;
      any_due = any_due || due;
    }
    (void)blocks;
    if (any_due) {
      UFEM_CUDA_TRY(cudaMemcpyAsync(b->ictl, b->h_ictl, sizeof(int) * kIc * b->nmesh, cudaMemcpyHostToDevice, st));
      if ((rc = spmv_b<double, XL>(b, xw, b->w, st, fSkipRepl))) return rc;
      replace_batch_kernel<BL><<<nc, kThreads, 0, st>>>(b->d_chunks, b->d_mesh, bw, b->w, b->r, b->rh, b->part,
                                                       b->nchunks, b->ictl);
      replace_end_batch_kernel<<<gm, 256, 0, st>>>(b->nmesh, b->d_cprefix, b->part, b->nchunks, b->dctl, b->ictl);
      UFEM_CUDA_TRY(cudaGetLastError());
      UFEM_CUDA_TRY(cudaMemcpyAsync(b->h_ictl, b->ictl, sizeof(int) * kIc * b->nmesh, cudaMemcpyDeviceToHost, st));
      UFEM_CUDA_TRY(cudaStreamSynchronize(st));
      bool fin = true;
      for (int m = 0; m < b->nmesh && fin; ++m) fin = b->h_ictl[m * kIc + fFinal] != 0;
      if (fin) break;
    }
  }
  return UFEM_OK;
}

// FP64 true residual of every member's current solution into dctl[sTrue].
int true_residual_b(ufem_batch* b, cudaStream_t st) {
  int rc;
  UFEM_CUDA_TRY(cudaMemsetAsync(b->ictl, 0, sizeof(int) * kIc * b->nmesh, st));
  if ((rc = residual_b<double, kSol, kRhs>(b, nullptr, nullptr, false, false, st))) return rc;
  true_res_batch_kernel<<<blocks_for(int64_t(b->nmesh) * 32, 256), 256, 0, st>>>(b->nmesh, b->d_cprefix, b->part,
                                                                                 b->nchunks, b->dctl);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

// mixed = 2: FP32-operator inner solves refined against each member's FP64
// residual from the element pass (the one-handle refinement of krylov.cu, for
// every member at once).  The pass count and every member's arithmetic depend
// only on that member's own residuals, so a member's result is the same alone
// and in any batch.
int batch_mf_solve(ufem_batch* b, const ufem_krylov_opts& o, ufem_krylov_status* statuses, cudaStream_t st) {
  const int n = b->nmesh;
  const unsigned nc = unsigned(b->nchunks);
  const unsigned gm = blocks_for(int64_t(n) * 32, 256);
  const size_t R = size_t(b->total_rows);
  int rc;
  if (!b->mfr && ((rc = dmal(&b->mfr, R)) || (rc = dmal(&b->mfb, R)) || (rc = dmal(&b->mfz, R)))) return rc;
  std::vector<int64_t> off(size_t(n) + 1, 0);
  for (int m = 0; m < n; ++m) off[size_t(m) + 1] = off[size_t(m)] + b->members[m]->nrows;
  std::vector<int> done(n, 0), conv(n, 0), iters(n, 0), refs(n, 0), status(n, 0);
  std::vector<double> relres(n, NAN);
  for (int m = 0; m < n; ++m)
    if (!b->active[m]) done[m] = 1;  // held: nothing to solve
  auto put_outer = [&]() -> int {
    for (int m = 0; m < n; ++m) {
      for (int q = 0; q < kIc; ++q) b->h_ictl[m * kIc + q] = 0;
      b->h_ictl[m * kIc + fOuter] = done[m];
    }
    UFEM_CUDA_TRY(cudaMemcpyAsync(b->ictl, b->h_ictl, sizeof(int) * kIc * n, cudaMemcpyHostToDevice, st));
    return UFEM_OK;
  };
  const int inner_iters = std::min(o.max_iters, kInnerIterCap);
  for (int ref = 0; ref <= o.max_refine; ++ref) {
    // FP64 residuals of the members still refining, then their norms
    for (int m = 0; m < n; ++m)
      if (!done[m] && (rc = launch_mf_residual(b->members[m], b->w + off[size_t(m)], b->mfr + off[size_t(m)], st)))
        return rc;
    if ((rc = put_outer())) return rc;
    mf_norm_batch_kernel<<<nc, kThreads, 0, st>>>(b->d_chunks, b->d_mesh, b->mfr, b->part, b->nchunks, b->ictl);
    mf_fold_batch_kernel<<<gm, 256, 0, st>>>(n, b->d_cprefix, b->part, b->nchunks, b->dctl);
    UFEM_CUDA_TRY(cudaGetLastError());
    UFEM_CUDA_TRY(cudaMemcpyAsync(b->h_dctl, b->dctl, sizeof(double) * kDc * n, cudaMemcpyDeviceToHost, st));
    UFEM_CUDA_TRY(cudaStreamSynchronize(st));
    bool any = false;
    for (int m = 0; m < n; ++m) {
      if (done[m]) continue;
      const double rr = b->h_dctl[m * kDc + sTrue], bn = b->h_dctl[m * kDc + sBnorm];
      if (!std::isfinite(rr)) {
        status[m] = 3;
        done[m] = 1;
        continue;
      }
      relres[m] = rr;
      if (bn == 0.0) {  // zero right-hand side: the increment is zero
        UFEM_CUDA_TRY(cudaMemsetAsync(b->members[m]->d_sol, 0, size_t(b->members[m]->nrows) * 8, st));
        relres[m] = 0.0;
        conv[m] = 1;
        done[m] = 1;
        continue;
      }
      if (rr <= o.tol) {
        conv[m] = 1;
        done[m] = 1;
        continue;
      }
      if (ref == o.max_refine || iters[m] >= o.max_iters * (o.max_refine + 1)) {
        status[m] = 1;
        done[m] = 1;
        continue;
      }
      any = true;
    }
    if (!any) break;
    // inner: A32 z = r / ||r|| for the members in this pass, then x += ||r|| z
    if ((rc = put_outer())) return rc;
    mf_scale_batch_kernel<<<nc, kThreads, 0, st>>>(b->d_chunks, b->d_mesh, b->mfr, b->mfb, b->mfz, b->dctl, b->ictl);
    UFEM_CUDA_TRY(cudaGetLastError());
    if ((rc = bicgstab_b<float, kWork, kWork>(b, o.precond, o.inner_tol, inner_iters, true, kSlotMf, st, false,
                                              b->mfz, b->mfb)))
      return rc;
    UFEM_CUDA_TRY(cudaMemcpyAsync(b->h_ictl, b->ictl, sizeof(int) * kIc * n, cudaMemcpyDeviceToHost, st));
    UFEM_CUDA_TRY(cudaStreamSynchronize(st));
    for (int m = 0; m < n; ++m) {
      if (done[m]) continue;
      iters[m] += b->h_ictl[m * kIc + fIters];
      ++refs[m];
      // a breakdown leaves a finite partial correction, applied; a non-finite
      // inner iterate is never applied
      if (b->h_ictl[m * kIc + fStatus] == 3) {
        status[m] = 3;
        relres[m] = NAN;
        done[m] = 1;
      }
    }
    if ((rc = put_outer())) return rc;
    mf_update_batch_kernel<<<nc, kThreads, 0, st>>>(b->d_chunks, b->d_mesh, b->mfz, b->dctl, b->ictl);
    UFEM_CUDA_TRY(cudaGetLastError());
  }
  UFEM_CUDA_TRY(cudaStreamSynchronize(st));
  if (statuses) {
    for (int m = 0; m < n; ++m) {
      ufem_krylov_status& sm = statuses[m];
      sm = ufem_krylov_status{};
      if (!b->active[m]) {  // held: nothing was solved
        sm.converged = 1;
        continue;
      }
      sm.iterations = iters[m];
      sm.refinements = refs[m];
      sm.rel_residual = relres[m];
      sm.converged = conv[m];
      sm.status = conv[m] ? 0 : (status[m] ? status[m] : 1);
    }
  }
  return UFEM_OK;
}

}  // namespace

extern "C" {

int ufem_batch_create(ufem_ns_handle* const* members, int32_t n, ufem_batch** out) {
  if (!members || !out || n < 1) return set_error(UFEM_ERR_ARG, "ufem_batch_create: members, n >= 1 and out required");
  *out = nullptr;
  for (int32_t m = 0; m < n; ++m) {
    const ufem_ns_handle* h = members[m];
    if (!h) return set_error(UFEM_ERR_ARG, "ufem_batch_create: NULL member");
    if (!h->state_set) return set_error(UFEM_ERR_STATE, "ufem_batch_create: every member needs its state set");
    if (h->dim != members[0]->dim || h->opt.precision != members[0]->opt.precision ||
        h->opt.use_specializations != members[0]->opt.use_specializations)
      return set_error(UFEM_ERR_ARG, "ufem_batch_create: members must share dim, precision and element form");
    for (int32_t q = 0; q < m; ++q)
      if (members[q] == h) return set_error(UFEM_ERR_ARG, "ufem_batch_create: a handle appears twice");
  }
  ufem_batch* b = new ufem_batch();
  b->members.assign(members, members + n);
  b->active.assign(size_t(n), 1);
  b->nmesh = n;
  b->dim = members[0]->dim;
  b->neq = members[0]->neq;
  b->precision = members[0]->opt.precision;
  b->spec = members[0]->opt.use_specializations;
  b->warps = members[0]->asm_warps;
  std::vector<int> gprefix(n + 1, 0);
  std::vector<int64_t> nprefix(n + 1, 0);
  std::vector<Chunk> chunks;
  std::vector<int> cprefix(n + 1, 0);
  for (int m = 0; m < n; ++m) {
    const ufem_ns_handle* h = members[m];
    gprefix[m + 1] = gprefix[m] + h->wplan.ngroups;
    nprefix[m + 1] = nprefix[m] + h->N;
    for (int64_t n0 = 0; n0 < h->N; n0 += kChunkNodes)
      chunks.push_back(Chunk{m, int(n0 * h->neq), int(std::min<int64_t>(h->N, n0 + kChunkNodes) * h->neq), 0});
    cprefix[m + 1] = int(chunks.size());
    b->total_rows += h->nrows;
  }
  b->total_nodes = nprefix[n];
  b->ngroups = gprefix[n];
  b->nchunks = int(chunks.size());
  const size_t R = size_t(b->total_rows);
  int rc;
  if ((rc = dmal(&b->d_asm, n)) || (rc = dmal(&b->d_gprefix, n + 1)) || (rc = dmal(&b->d_mesh, n)) ||
      (rc = dmal(&b->d_node_prefix, n + 1)) || (rc = dmal(&b->d_bc_prefix, n + 1)) ||
      (rc = dmal(&b->d_fix_prefix, n + 1)) || (rc = dmal(&b->d_chunks, chunks.size())) ||
      (rc = dmal(&b->d_cprefix, n + 1)) || (rc = dmal(&b->r, R)) || (rc = dmal(&b->rh, R)) ||
      (rc = dmal(&b->p, R)) || (rc = dmal(&b->v, R)) || (rc = dmal(&b->s, R)) || (rc = dmal(&b->t, R)) ||
      (rc = dmal(&b->ph, R)) || (rc = dmal(&b->sh, R)) || (rc = dmal(&b->dinv, R)) || (rc = dmal(&b->w, R)) ||
      (rc = dmal(&b->part, 2 * chunks.size())) || (rc = dmal(&b->dctl, size_t(kDc) * n)) ||
      (rc = dmal(&b->counters, size_t(4) * n)) ||
      (rc = dmal(&b->ictl, size_t(kIc) * n))) {
    batch_free(b);
    return rc;
  }
  cudaError_t ce;
  DeviceLock device_lock(device_mutex());
  if ((ce = cudaMallocHost(reinterpret_cast<void**>(&b->h_dctl), sizeof(double) * kDc * n)) != cudaSuccess ||
      (ce = cudaMallocHost(reinterpret_cast<void**>(&b->h_ictl), sizeof(int) * kIc * n)) != cudaSuccess ||
      (ce = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (ce = cudaMemcpy(b->d_gprefix, gprefix.data(), gprefix.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (ce = cudaMemcpy(b->d_node_prefix, nprefix.data(), nprefix.size() * 8, cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (ce = cudaMemcpy(b->d_chunks, chunks.data(), chunks.size() * sizeof(Chunk), cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (ce = cudaMemcpy(b->d_cprefix, cprefix.data(), cprefix.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (ce = cudaMemset(b->counters, 0, sizeof(int) * 4 * n)) != cudaSuccess) {
    batch_free(b);
    return set_error(UFEM_ERR_CUDA, std::string("ufem_batch_create: ") + cudaGetErrorString(ce));
  }
  if ((rc = batch_refresh(b))) {
    batch_free(b);
    return rc;
  }
  *out = b;
  return UFEM_OK;
}

int ufem_batch_set_active(ufem_batch* b, const int32_t* active) {
  if (!b || !active) return set_error(UFEM_ERR_ARG, "NULL argument");
  for (int m = 0; m < b->nmesh; ++m) {
    const int32_t a = active[m] ? 1 : 0;
    if (a != b->active[m]) {
      b->active[m] = a;
      b->active_dirty = true;
    }
  }
  return UFEM_OK;
}

int ufem_batch_size(const ufem_batch* b, int32_t* n, int64_t* rows) {
  if (!b) return set_error(UFEM_ERR_ARG, "NULL batch");
  if (n) *n = b->nmesh;
  if (rows) *rows = b->total_rows;
  return UFEM_OK;
}

int ufem_batch_set_graphs(ufem_batch* b, int32_t enable) {
  if (!b) return set_error(UFEM_ERR_ARG, "NULL batch");
  b->graphs = enable != 0;
  return UFEM_OK;
}

int ufem_batch_set_assembly_warps(ufem_batch* b, int32_t warps_per_cta) {
  if (!b) return set_error(UFEM_ERR_ARG, "NULL batch");
  if (warps_per_cta != 2 && warps_per_cta != 4 && warps_per_cta != 8)
    return set_error(UFEM_ERR_ARG, "warps_per_cta must be 2, 4 or 8");
  b->warps = warps_per_cta;
  return UFEM_OK;
}

int ufem_batch_tune_assembly(ufem_batch* b, void* stream, int32_t reps, int32_t* warps_per_cta,
                              float* ms_per_launch) {
  if (!b) return set_error(UFEM_ERR_ARG, "NULL batch");
  for (const ufem_ns_handle* h : b->members)
    if (!h->state_set) return set_error(UFEM_ERR_STATE, "every member's state must be set before tuning");
  if (reps < 1) reps = 5;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc;
  if (batch_dirty(b)) {
    UFEM_CUDA_TRY(cudaStreamSynchronize(st));
    if ((rc = batch_refresh(b))) return rc;
  }
  linearize_batch_kernel<<<blocks_for(b->total_nodes, 256), 256, 0, st>>>(b->total_nodes, b->nmesh,
                                                                          b->d_node_prefix, b->d_mesh);
  UFEM_CUDA_TRY(cudaGetLastError());
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  UFEM_CUDA_TRY(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return set_error(UFEM_ERR_CUDA, "cudaEventCreate failed");
  }
  float best = -1.0f;
  int pick = b->warps;
  rc = UFEM_OK;
  for (int w : {2, 4, 8}) {
    auto launch = [&] {
      return launch_assembly_batch(b->dim, b->precision, b->spec != 0, w, b->ngroups, b->nmesh, b->d_asm,
                                   b->d_gprefix, st);
    };
    if ((rc = launch())) break;  // warm-up
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps && rc == UFEM_OK; ++r) rc = launch();
    if (rc) break;
    cudaEventRecord(e1, st);
    cudaError_t ce = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
    if (ce != cudaSuccess) {
      rc = set_error(UFEM_ERR_CUDA, std::string("batch assembly tuning: ") + cudaGetErrorString(ce));
      break;
    }
    ms /= float(reps);
    if (best < 0.0f || ms < best) {
      best = ms;
      pick = w;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  b->warps = pick;
  if (warps_per_cta) *warps_per_cta = pick;
  if (ms_per_launch) *ms_per_launch = best;
  return UFEM_OK;  // the members' systems are overwritten: assemble before solving
}

int ufem_batch_assemble(ufem_batch* b, void* stream) {
  if (!b) return set_error(UFEM_ERR_ARG, "NULL batch");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc;
  if (batch_dirty(b)) {
    UFEM_CUDA_TRY(cudaStreamSynchronize(st));
    if ((rc = batch_refresh(b))) return rc;
  }
  linearize_batch_kernel<<<blocks_for(b->total_nodes, 256), 256, 0, st>>>(b->total_nodes, b->nmesh,
                                                                          b->d_node_prefix, b->d_mesh);
  UFEM_CUDA_TRY(cudaGetLastError());
  if ((rc = launch_assembly_batch(b->dim, b->precision, b->spec != 0, b->warps, b->ngroups, b->nmesh, b->d_asm,
                                  b->d_gprefix, st)))
    return rc;
  for (ufem_ns_handle* h : b->members) {  // rows with more than 32 elements (none on most meshes)
    h->vals32_valid = h->d_vals32 != nullptr;
    const AssemblyPlan& big = h->opt.precision == 1 ? h->wplan.big32 : h->wplan.big64;
    if (big.nchunks > 0 && (rc = launch_assembly_big_rows(h, st, h->d_vals32 != nullptr))) return rc;
    if ((rc = launch_tie_rows(h, st, h->d_vals32 != nullptr))) return rc;
  }
  for (ufem_ns_handle* h : b->members) {  // function values and constant Neumann faces, before the Dirichlet passes
    if ((rc = launch_dirichlet_functions(h, st))) return rc;
    if (h->bcp.nneu > 0 && (rc = launch_neumann(h, st))) return rc;
  }
  if (b->total_bc > 0) {
    dirichlet_values_batch_kernel<<<blocks_for(b->total_bc, 256), 256, 0, st>>>(b->total_bc, b->nmesh,
                                                                                 b->d_bc_prefix, b->d_mesh);
    if (b->total_fix > 0)
      dirichlet_columns_batch_kernel<<<blocks_for(b->total_fix * 8, 256), 256, 0, st>>>(b->total_fix, b->nmesh,
                                                                                         b->d_fix_prefix, b->d_mesh);
    dirichlet_rows_batch_kernel<<<blocks_for(b->total_bc * 8, 256), 256, 0, st>>>(b->total_bc, b->nmesh,
                                                                                   b->d_bc_prefix, b->d_mesh);
    UFEM_CUDA_TRY(cudaGetLastError());
  }
  return UFEM_OK;
}

int ufem_batch_solve(ufem_batch* b, const ufem_krylov_opts* kopts, ufem_krylov_status* statuses, void* stream) {
  if (!b) return set_error(UFEM_ERR_ARG, "NULL batch");
  ufem_krylov_opts o;
  ufem_krylov_default_opts(&o);
  if (kopts) o = *kopts;
  if (o.method != 1) return set_error(UFEM_ERR_ARG, "the batched solve is BiCGStab (method 1)");
  if (o.precond != 0 && o.precond != 1 && o.precond != 4)
    return set_error(UFEM_ERR_ARG, "the batched solve supports precond 0, 1 or 4");
  if (o.max_iters <= 0) o.max_iters = 3000;
  if (o.tol <= 0) o.tol = 1e-10;
  if (o.max_refine <= 0) o.max_refine = 20;
  if (o.inner_tol <= 0) o.inner_tol = 1e-3;
  if (o.mixed < 0 || o.mixed > 2) return set_error(UFEM_ERR_ARG, "mixed must be 0, 1 or 2");
  const bool mixed = o.mixed != 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc;
  if (mixed) {  // FP32 operator copies: allocated once, written by every later assembly
    bool added = false;
    for (ufem_ns_handle* h : b->members)
      if (h->d_vals32 == nullptr) {
        if ((rc = ensure_vals32(h, st))) return rc;
        added = true;
      }
    if (added) {
      UFEM_CUDA_TRY(cudaStreamSynchronize(st));
      if ((rc = batch_refresh(b))) return rc;
    }
  }
  if (o.precond == 4) {
    // every member's coarse space and coarse matrix (of its current system);
    // aggregates capped at kBatchCoarseSide2D^2 (2D) and kBatchCoarseSide3D^3
    // (3D) boxes, so that the host inversions of all members stay short
    if (b->coarse.size() != size_t(b->nmesh)) b->coarse.assign(size_t(b->nmesh), CoarseView{});
    bool any_new = false;
    std::vector<CoarseView> cv(size_t(b->nmesh));
    std::unique_ptr<bool[]> rebuilt(new bool[size_t(b->nmesh)]);
    // not lagged: each member's inverse is of its current matrix (with the
    // previous step's, the hardest cfg4-like members converged less often)
    if ((rc = krylov_coupled_coarse_members(b->members.data(), b->active.data(), b->nmesh, st, kBatchCoarseSide2D,
                                            kBatchCoarseSide3D, rebuilt.get(), cv.data())))
      return rc;
    for (int m = 0; m < b->nmesh; ++m) {
      if (!b->active[m]) continue;
      const CoarseView& old = b->coarse[m];
      if (rebuilt[m] || cv[m].nc != old.nc || cv[m].ainv != old.ainv || cv[m].agg != old.agg) any_new = true;
      b->coarse[m] = cv[m];
    }
    if (any_new) {
      UFEM_CUDA_TRY(cudaStreamSynchronize(st));
      if ((rc = batch_refresh(b))) return rc;
    }
  } else if (!b->coarse.empty()) {  // back to point Jacobi: no coarse spaces in the descriptors
    b->coarse.clear();
    UFEM_CUDA_TRY(cudaStreamSynchronize(st));
    if ((rc = batch_refresh(b))) return rc;
  }
  if (o.mixed == 2) return batch_mf_solve(b, o, statuses, st);
  std::vector<int> iters(b->nmesh, 0), status(b->nmesh, 0), refines(b->nmesh, 0);  // refines: FP64 replacements
  // Plain: FP64 operator.  Mixed: FP32 copy of the operator in the
  // iterations, FP64 vectors, dot products and residual replacement.
  auto run = [&](int maxit, bool outer) -> int {
    return mixed ? bicgstab_b<float, kSol, kRhs>(b, o.precond, o.tol, maxit, outer, 1, st, true)
                 : bicgstab_b<double, kSol, kRhs>(b, o.precond, o.tol, maxit, outer, 0, st, false);
  };
  bool all_active = true;
  for (int m = 0; m < b->nmesh; ++m) all_active = all_active && b->active[m];
  if (all_active) {
    if ((rc = run(o.max_iters, false))) return rc;
  } else {  // held members keep their outer flag set: their kernels return at once
    for (int m = 0; m < b->nmesh; ++m) {
      for (int q = 0; q < kIc; ++q) b->h_ictl[m * kIc + q] = 0;
      b->h_ictl[m * kIc + fOuter] = b->active[m] ? 0 : 1;
    }
    if ((rc = run(o.max_iters, true))) return rc;
  }
  UFEM_CUDA_TRY(cudaMemcpyAsync(b->h_ictl, b->ictl, sizeof(int) * kIc * b->nmesh, cudaMemcpyDeviceToHost, st));
  UFEM_CUDA_TRY(cudaStreamSynchronize(st));
  for (int m = 0; m < b->nmesh; ++m) {
    iters[m] = b->h_ictl[m * kIc + fIters];
    status[m] = b->h_ictl[m * kIc + fStatus];
    refines[m] = b->h_ictl[m * kIc + fRepl];
  }
  // members that broke down (rho or omega ~ 0) restart from their iterate;
  // the others are held by their outer flag
  for (int restart = 0; restart < kMaxRestarts; ++restart) {
    int used = 0;
    bool any = false;
    for (int m = 0; m < b->nmesh; ++m)
      if (b->active[m] && status[m] == 2 && iters[m] < o.max_iters) {
        any = true;
        used = std::max(used, iters[m]);
      }
    if (!any) break;
    for (int m = 0; m < b->nmesh; ++m) {
      for (int q = 0; q < kIc; ++q) b->h_ictl[m * kIc + q] = 0;
      b->h_ictl[m * kIc + fOuter] = (b->active[m] && status[m] == 2 && iters[m] < o.max_iters) ? 0 : 1;
    }
    if ((rc = run(o.max_iters - used, true))) return rc;
    UFEM_CUDA_TRY(cudaMemcpyAsync(b->h_ictl, b->ictl, sizeof(int) * kIc * b->nmesh, cudaMemcpyDeviceToHost, st));
    UFEM_CUDA_TRY(cudaStreamSynchronize(st));
    for (int m = 0; m < b->nmesh; ++m) {
      if (b->h_ictl[m * kIc + fOuter]) continue;
      iters[m] += b->h_ictl[m * kIc + fIters];
      status[m] = b->h_ictl[m * kIc + fStatus];
      refines[m] += b->h_ictl[m * kIc + fRepl];
    }
  }
  {
    // Members whose iteration ended above the FP64 tolerance finish with the
    // FP64 operator from their current iterate: every such member of the mixed
    // form (its FP32-operator stage), and a plain FP64 member that stopped
    // before its iteration limit because its recursive residual met the
    // tolerance while the true one had drifted above it (a fresh start
    // recomputes r = b - A x).  The finish has max_iters of its own for every
    // member, so no member's arithmetic depends on the others in its batch.
    if ((rc = true_residual_b(b, st))) return rc;
    UFEM_CUDA_TRY(cudaMemcpyAsync(b->h_dctl, b->dctl, sizeof(double) * kDc * b->nmesh, cudaMemcpyDeviceToHost, st));
    UFEM_CUDA_TRY(cudaStreamSynchronize(st));
    bool any = false;
    std::vector<int> redo(b->nmesh, 0);
    for (int m = 0; m < b->nmesh; ++m) {
      const double rr = b->h_dctl[m * kDc + sTrue];
      redo[m] = b->active[m] && !(std::isfinite(rr) && rr <= o.tol) && std::isfinite(rr) &&
                        (mixed || iters[m] < o.max_iters) ? 1 : 0;
      any = any || redo[m];
    }
    if (any) {
      for (int m = 0; m < b->nmesh; ++m) {
        for (int q = 0; q < kIc; ++q) b->h_ictl[m * kIc + q] = 0;
        b->h_ictl[m * kIc + fOuter] = redo[m] ? 0 : 1;
      }
      if ((rc = bicgstab_b<double, kSol, kRhs>(b, o.precond, o.tol, o.max_iters, true, 0, st, false))) return rc;
      UFEM_CUDA_TRY(cudaMemcpyAsync(b->h_ictl, b->ictl, sizeof(int) * kIc * b->nmesh, cudaMemcpyDeviceToHost, st));
      UFEM_CUDA_TRY(cudaStreamSynchronize(st));
      for (int m = 0; m < b->nmesh; ++m) {
        if (!redo[m]) continue;
        iters[m] += b->h_ictl[m * kIc + fIters];
        status[m] = b->h_ictl[m * kIc + fStatus];
      }
    }
  }
  // final FP64 residuals
  if ((rc = true_residual_b(b, st))) return rc;
  UFEM_CUDA_TRY(cudaMemcpyAsync(b->h_dctl, b->dctl, sizeof(double) * kDc * b->nmesh, cudaMemcpyDeviceToHost, st));
  UFEM_CUDA_TRY(cudaStreamSynchronize(st));
  if (statuses) {
    for (int m = 0; m < b->nmesh; ++m) {
      const double rr = b->h_dctl[m * kDc + sTrue];
      ufem_krylov_status& s = statuses[m];
      if (!b->active[m]) {  // held: nothing was solved
        s = ufem_krylov_status{};
        s.converged = 1;
        continue;
      }
      s.iterations = iters[m];
      s.refinements = refines[m];
      s.rel_residual = rr;
      s.converged = std::isfinite(rr) && rr <= o.tol;
      s.status = s.converged ? 0 : (status[m] ? status[m] : (std::isfinite(rr) ? 1 : 3));
    }
  }
  return UFEM_OK;
}

int ufem_batch_update(ufem_batch* b, void* stream) {
  if (!b) return set_error(UFEM_ERR_ARG, "NULL batch");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  update_batch_kernel<<<blocks_for(b->total_nodes, 256), 256, 0, st>>>(b->total_nodes, b->nmesh, b->d_node_prefix,
                                                                       b->d_mesh);
  UFEM_CUDA_TRY(cudaGetLastError());
  for (int m = 0; m < b->nmesh; ++m)
    if (b->active[m]) b->members[m]->time += b->members[m]->opt.dt;  // as ufem_ns_update
  return UFEM_OK;
}

int ufem_batch_step(ufem_batch* b, const ufem_krylov_opts* kopts, ufem_krylov_status* statuses, void* stream) {
  int rc;
  if ((rc = ufem_batch_assemble(b, stream))) return rc;
  if ((rc = ufem_batch_solve(b, kopts, statuses, stream))) return rc;
  return ufem_batch_update(b, stream);
}

void ufem_batch_destroy(ufem_batch* b) {
  if (b) batch_free(b);
}

}  // extern "C"
