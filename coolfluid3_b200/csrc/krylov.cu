// krylov.cu -- SolveLSS replacement: restarted GMRES and BiCGStab with a Jacobi
// preconditioner on the assembled point CSR, plus FP64 iterative refinement
// around an FP32 inner solve.
//
// The reference solves with Belos block GMRES + Ifpack ILU through Stratimikos
// (TrilinosStratimikosStrategy.cpp:135-177, BelosGMRESParameters.cpp:28-41).
// Here the SpMV walks the node graph (one warp per block row), dot products and
// norms are reduced in FP64 in a fixed order (deterministic, no atomics), and the
// Krylov scalars (Hessenberg, Givens rotations, BiCGStab alpha/omega, the
// convergence test) live on the device, so whole stretches of iterations are
// enqueued without a host round trip.  Kernels read a device "done" flag and
// return at once after convergence.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <type_traits>
#include <vector>

#include "internal.h"
#include "spmv_node.cuh"

namespace ufem {

struct KrylovWork {
  int64_t n = 0;
  int m = 0;
  int nblk = 0;
  // FP64 vectors
  double *V = nullptr, *w = nullptr, *z = nullptr, *t = nullptr, *r = nullptr, *dinv = nullptr;
  // FP32 vectors for the inner GMRES solve of the mixed path
  float *V32 = nullptr, *w32 = nullptr, *z32 = nullptr, *t32 = nullptr, *r32 = nullptr, *x32 = nullptr,
        *q32 = nullptr, *dinv32 = nullptr;
  // BiCGStab vectors
  double *bp = nullptr, *bv = nullptr, *bs = nullptr, *bt = nullptr, *brh = nullptr, *bph = nullptr, *bsh = nullptr;
  // reductions and solver scalars (device)
  double* part = nullptr;  // (m+2) x nblk
  double* hbuf = nullptr;  // 2 x (m+2)
  double* H = nullptr;     // (m+1) x m
  double *cs = nullptr, *sn = nullptr, *g = nullptr, *y = nullptr;
  double* dctl = nullptr;  // scalars, see kD* below
  int* ictl = nullptr;     // [0]=done [1]=jcount [2]=status [3]=iterations (BiCGStab)
  double* h_dctl = nullptr;  // pinned mirrors
  int* h_ictl = nullptr;
  // CUDA graph of an 8-iteration CG block per operator type (FP64, FP32),
  // captured for one set of operands and replayed between host checks.
  struct CGGraph {
    cudaGraphExec_t exec = nullptr;
    const void* key[16] = {};
    int pkind = -1, maxit = 0;
    double tol = 0.0;
  };
  CGGraph cg_graph[2];
  CGGraph bicg_graph[2];   // the same for BiCGStab
  // Iterations of the previous BiCGStab solve per operator type: the host's
  // first look at the done flag comes after that many (rounded down to a
  // graph block), so a solve like the last one launches few iterations past
  // its convergence.
  int bicg_expect[2] = {0, 0};
  int cg_expect[2] = {0, 0};   // the same for CG
  bool use_graph = true;   // false for the allocation-free solve (instantiation allocates)
  cudaStream_t capture_stream = nullptr;
  int cg_nblk = 0;             // blocks of the fused CG kernels (more than nblk: they are latency-bound)
  int* cg_counter = nullptr;   // last-block ticket of the fused CG folds
  // Two-level preconditioner (precond 3; CG on one-equation systems): point
  // Jacobi plus a piecewise-constant correction on aggregates of rows,
  // z = D^-1 r + R Ac^-1 R^T r with the Galerkin coarse matrix Ac = R^T A R.
  int nc = 0;                  // aggregates (0: not set up)
  int coarse_version = 0;
  int32_t* agg = nullptr;      // nrows: aggregate of each row, -1 for none
  int32_t* agg_ptr = nullptr;  // nc + 1
  int32_t* agg_rows = nullptr; // the members of each aggregate, ascending
  double* ainv = nullptr;      // nc x nc, row-major
  double* cvec = nullptr;      // nc: R^T r
  double* yvec = nullptr;      // nc: Ac^-1 R^T r
  // Two-level preconditioner of the coupled system (precond 4): point Jacobi
  // plus the same piecewise-constant correction on aggregates of pressure rows
  // (agg .. yvec above, built for the coupled rows).  Its coarse matrix, the
  // Galerkin product of the pressure-pressure block, is rebuilt at every solve
  // on the device: the block's CSR positions are sorted once by (aggregate of
  // the row, aggregate of the column) and each segment is summed by one warp.
  int64_t* cp_pos = nullptr;   // sorted CSR positions of the coarse pressure-pressure entries
  int32_t* cp_seg = nullptr;   // cp_nseg + 1 segment starts
  int32_t* cp_dst = nullptr;   // dense index I * nc + J of each segment
  int cp_nseg = 0;
  double* acd = nullptr;       // nc x nc coarse matrix on the device
  double* h_ac = nullptr;      // pinned host copy (nc x nc)
  int64_t cp_bc_version = -1;  // condition lists the structure was built for (bc_list_version)
  int cp_caps = -1;            // aggregate caps it was built with (2D side * 1000 + 3D side)
  bool cp_spd = false;         // the coarse inverse on the device is valid
  // Lagged refresh: the coarse matrix of solve k is inverted on a host thread
  // while solve k runs with the inverse from solve k-1 (the first solve after a
  // (re)build inverts its own matrix before it starts).
  std::thread cp_thread;
  bool cp_pending = false;     // cp_thread holds the next inverse in h_ac2
  bool cp_lag_ready = false;   // the device inverse is the latest solve's: the next lagged solve keeps it
  bool cp_next_spd = false;
  double* h_ac2 = nullptr;     // pinned: the inverse the thread produces
  cudaEvent_t cp_event = nullptr;
};

namespace {

// dctl slots
constexpr int kBnorm = 0, kBeta = 1, kEst = 2, kHnext = 3, kTrue = 4;
constexpr int kRho = 5, kRhoOld = 6, kAlpha = 7, kOmega = 8, kRhV = 9, kTS = 10, kTT = 11, kR2 = 12, kScale = 13;
constexpr int kRedThreads = 256;
// Blocks of the vector kernels and their reductions for n rows: one per 1024
// rows, at most 4 a B200 SM (enough loads in flight to stream the vectors).
// The allocating and the allocation-free solves use the same count, so their
// reductions add in the same order.
constexpr int kRedBlocksMax = 4 * 148;
inline int red_blocks(int64_t n) {
  return int(std::min<int64_t>(kRedBlocksMax, std::max<int64_t>(1, (n + 1023) / 1024)));
}
constexpr int kInnerIterCap = 400;  // iterations of one FP32 inner solve of the mixed path
constexpr int kMaxRestarts = 10;    // BiCGStab restarts after breakdowns in one solve
constexpr int kCGMaxBlocks = 8 * 148;  // blocks of the fused CG kernels

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum (fixed shuffle tree + fixed smem order); valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* sm) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sm[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < int(blockDim.x >> 5); ++k) s += sm[k];
  __syncthreads();
  return s;
}

// Runs fn(lo, hi) on nt threads over [n0, n) cut into ranges of equal work
// (cost(u): the work of unit u); each unit's arithmetic is the same whatever
// the cut.
template <typename F, typename C>
void parallel_ranges(int nt, int n0, int n, C&& cost, F&& fn) {
  const int extra = (nt <= 1 || n - n0 < 2) ? 0 : acquire_spare_threads(nt - 1);
  nt = 1 + extra;
  if (nt <= 1) {
    fn(n0, n);
    return;
  }
  double total = 0.0;
  for (int u = n0; u < n; ++u) total += cost(u);
  std::vector<std::thread> th;
  int lo = n0;
  double acc = 0.0;
  for (int t = 0; t < nt && lo < n; ++t) {
    int hi = lo;
    const double goal = total * (t + 1) / nt;
    while (hi < n && (t + 1 == nt || acc + 0.5 * cost(hi) < goal)) acc += cost(hi++);
    if (hi == lo) continue;
    if (hi == n) fn(lo, hi);  // the last range on the calling thread
    else th.emplace_back(fn, lo, hi);
    lo = hi;
  }
  for (auto& x : th) x.join();
  release_spare_threads(extra);
}

// In-place inverse of an SPD matrix (row-major, n x n): A = L L^T, X = L^-1,
// A^-1 = X^T X (the LAPACK potrf / trtri / lauum sequence, n^3 / 2
// multiply-adds), every inner loop a contiguous multiply-add over rows that
// stay in cache (the Cholesky in panels of 32 columns, L^-1 in groups of 8
// columns, the product in groups of 8 rows).  From n = 256 the last two
// phases are split over `threads` host threads (default: up to 4, since several
// handles may refresh their coarse spaces at once), in ranges of equal work;
// every element's arithmetic is the same whatever the split.  False if a pivot
// is not positive (a coarse matrix of a system without conditions that fix its
// constant mode is singular).
bool spd_invert(double* A, int n, int threads = 0) {
  const int nt = n < 256 ? 1
                         : (threads > 0 ? threads
                                        : int(std::max(1u, std::min(4u, std::thread::hardware_concurrency()))));
  // Cholesky A = L L^T, right-looking in panels of kPanel columns: every
  // element receives its updates L[i][k] L[j][k] in ascending k (the order of
  // the column-by-column algorithm).  The panel is factored in a contiguous
  // copy P (row i: its kPanel columns); Lt row k holds column k of L.
  constexpr int kPanel = 32;
  std::vector<double> W(A, A + size_t(n) * n), Lt(size_t(n) * n, 0.0), P(size_t(n) * kPanel);
  for (int p0 = 0; p0 < n; p0 += kPanel) {
    const int p1 = std::min(n, p0 + kPanel), b = p1 - p0;
    for (int i = p0; i < n; ++i)
      for (int q = 0; q < b; ++q) P[size_t(i) * kPanel + q] = W[size_t(i) * n + p0 + q];
    for (int k = p0; k < p1; ++k) {
      const int kq = k - p0;
      const double d = P[size_t(k) * kPanel + kq];
      if (!(d > 0.0) || !std::isfinite(d)) return false;
      const double lkk = std::sqrt(d);
      P[size_t(k) * kPanel + kq] = lkk;
      for (int i = k + 1; i < n; ++i) P[size_t(i) * kPanel + kq] /= lkk;
      for (int i = k + 1; i < n; ++i) {  // the panel's remaining columns
        double* __restrict__ pi = &P[size_t(i) * kPanel];
        const double lik = pi[kq];
        const int je = std::min(i, p1 - 1) - p0;
        for (int j = kq + 1; j <= je; ++j) pi[j] -= lik * P[size_t(p0 + j) * kPanel + kq];
      }
    }
    for (int q = 0; q < b; ++q)
      for (int i = p0 + q; i < n; ++i) Lt[size_t(p0 + q) * n + i] = P[size_t(i) * kPanel + q];
    if (p1 < n)  // the trailing rows and columns: the panel's rank-b update, on this thread (a
                 // fork per panel costs more than it saves beside a serving loop's threads)
      parallel_ranges(1, p1, n, [p1](int i) { return double(i - p1 + 1); }, [&, p0, p1](int r0, int r1) {
        for (int i = r0; i < r1; ++i) {
          double* __restrict__ wi = &W[size_t(i) * n];
          for (int k = p0; k < p1; ++k) {
            const double* __restrict__ lk = &Lt[size_t(k) * n];
            const double lik = lk[i];
            for (int j = p1; j <= i; ++j) wi[j] -= lik * lk[j];
          }
        }
      });
  }
  // X = L^-1 by forward substitution, kCols columns at a time (X^T rows of
  // kCols values: every L column is read once per group of columns).
  constexpr int kCols = 8;
  std::vector<double> X(size_t(n) * n, 0.0);  // X[i][c]
  parallel_ranges(nt, 0, (n + kCols - 1) / kCols,
                  [n](int g) { const double r = n - g * kCols; return r * r; },
                  [&](int g0, int g1) {
    std::vector<double> x(size_t(n) * kCols);
    for (int g = g0; g < g1; ++g) {
      const int c0 = g * kCols, w = std::min(kCols, n - c0);
      std::fill(x.begin(), x.end(), 0.0);
      for (int q = 0; q < w; ++q) x[size_t(c0 + q) * kCols + q] = 1.0;
      for (int k = c0; k < n; ++k) {  // row k of x is final once columns < k of L are applied
        const double* __restrict__ lk = &Lt[size_t(k) * n];
        double v[kCols];
        for (int q = 0; q < kCols; ++q) v[q] = x[size_t(k) * kCols + q] / lk[k];
        for (int q = 0; q < kCols; ++q) x[size_t(k) * kCols + q] = v[q];
        for (int i = k + 1; i < n; ++i) {
          const double lik = lk[i];
          double* __restrict__ xi = &x[size_t(i) * kCols];
          for (int q = 0; q < kCols; ++q) xi[q] -= lik * v[q];
        }
      }
      for (int i = c0; i < n; ++i)
        for (int q = 0; q < w; ++q) X[size_t(i) * n + c0 + q] = x[size_t(i) * kCols + q];
    }
  });
  // A^-1 = X^T X: row i = sum over k >= i of X[k][i] X[k][0..k], kRows rows at
  // a time (each X row is read once per group of rows).
  constexpr int kRows = 8;
  parallel_ranges(nt, 0, (n + kRows - 1) / kRows,
                  [n](int g) { const double r0 = g * kRows; return double(n) * n - r0 * r0; },
                  [&](int g0, int g1) {
    for (int g = g0; g < g1; ++g) {
      const int i0 = g * kRows, h = std::min(kRows, n - i0);
      for (int r = 0; r < h; ++r) std::fill(A + size_t(i0 + r) * n, A + size_t(i0 + r + 1) * n, 0.0);
      for (int k = i0; k < n; ++k) {
        const double* __restrict__ xk = &X[size_t(k) * n];
        for (int r = 0; r < h && i0 + r <= k; ++r) {
          const double xki = xk[i0 + r];
          double* __restrict__ ai = A + size_t(i0 + r) * n;
          for (int j = 0; j <= k; ++j) ai[j] += xki * xk[j];
        }
      }
    }
  });
  return true;
}

#define GRID_STRIDE(i, n) \
  _Pragma("unroll 4") for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < (n); i += int64_t(gridDim.x) * blockDim.x)

// y = A x on the node graph, FEVbr point layout: the NEQ rows of a node are
// contiguous (row r, neighbour slot s, component c at r*S*NEQ + s*NEQ + c);
// FP64 accumulation, fixed-order warp reduction.
//
// NEQ = 4 (the coupled tetrahedron system): persistent warps, warp w walking
// the nodes w, w + W, w + 2W, ... (W: warps of the grid) with spmv4_walk, the
// next node's loads in flight while one node is reduced.
template <typename VT, typename MT>
__global__ void __launch_bounds__(256, 3) spmv4_stream_kernel(int64_t N, const int64_t* __restrict__ start,
                                                             const int32_t* __restrict__ adj,
                                                             const MT* __restrict__ vals, const VT* __restrict__ x,
                                                             VT* __restrict__ y, const int* __restrict__ done) {
  if (done && *done) return;
  spmv4_walk<MT, VT, VT>((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5, N,
                         int64_t(gridDim.x) * (blockDim.x >> 5), start, adj, vals, x, y, threadIdx.x & 31);
}

// y = A x for block rows of NEQ <= 3 equations: persistent 8-lane groups, 4 a
// warp, walking the nodes g, g + G, ... (G: groups of the grid) with the next
// node's loads in flight (spmv_group_walk).
template <int NEQ, typename VT, typename MT>
__global__ void __launch_bounds__(256) spmv_small_kernel(int64_t N, const int64_t* __restrict__ start,
                                                         const int32_t* __restrict__ adj, const MT* __restrict__ vals,
                                                         const VT* __restrict__ x, VT* __restrict__ y,
                                                         const int* __restrict__ done) {
  if (done && *done) return;
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  spmv_group_walk<NEQ, MT, VT, VT>(0, N, int64_t(gridDim.x) * (blockDim.x >> 3), t >> 3, int(t & 7), start, adj,
                                   vals, x, y);
}

template <typename MT, typename VT>
__global__ void jacobi_kernel(int64_t n, const int64_t* __restrict__ diagpos, const MT* __restrict__ vals,
                              VT* __restrict__ dinv) {
  GRID_STRIDE(i, n) {
    const double d = double(vals[diagpos[i]]);
    dinv[i] = VT(d != 0.0 ? 1.0 / d : 1.0);
  }
}

// Node-block Jacobi: inverse of each neq x neq diagonal block (Gauss-Jordan with
// partial pivoting), row-major per node.
template <typename MT, typename VT>
__global__ void block_jacobi_kernel(int64_t N, int neq, const int64_t* __restrict__ diagpos,
                                    const MT* __restrict__ vals, VT* __restrict__ binv) {
  GRID_STRIDE(i, N) {
    double a[4][8];
    for (int r = 0; r < neq; ++r) {
      const int64_t d = diagpos[i * neq + r] - r;  // first column of the diagonal block in row r
      for (int c = 0; c < neq; ++c) {
        a[r][c] = double(vals[d + c]);
        a[r][neq + c] = (r == c) ? 1.0 : 0.0;
      }
    }
    for (int c = 0; c < neq; ++c) {
      int piv = c;
      for (int r = c + 1; r < neq; ++r)
        if (fabs(a[r][c]) > fabs(a[piv][c])) piv = r;
      if (piv != c)
        for (int k = 0; k < 2 * neq; ++k) { const double tmp = a[c][k]; a[c][k] = a[piv][k]; a[piv][k] = tmp; }
      const double p = a[c][c];
      const double ip = (p != 0.0) ? 1.0 / p : 0.0;
      for (int k = 0; k < 2 * neq; ++k) a[c][k] *= ip;
      for (int r = 0; r < neq; ++r)
        if (r != c) {
          const double f = a[r][c];
          for (int k = 0; k < 2 * neq; ++k) a[r][k] -= f * a[c][k];
        }
    }
    for (int r = 0; r < neq; ++r)
      for (int c = 0; c < neq; ++c) binv[(i * neq + r) * neq + c] = VT(a[r][neq + c]);
  }
}

template <typename VT>
__global__ void precond_kernel(int64_t n, int neq, int kind, const VT* __restrict__ dinv, const VT* __restrict__ v,
                               VT* __restrict__ z, const int* __restrict__ done) {
  if (done && *done) return;
  GRID_STRIDE(i, n) {
    if (kind == 0) {
      z[i] = v[i];
    } else if (kind == 1) {
      z[i] = dinv[i] * v[i];
    } else {
      const int64_t node = i / neq;
      const int r = int(i - node * neq);
      double s = 0.0;
      for (int c = 0; c < neq; ++c) s += double(dinv[(node * neq + r) * neq + c]) * double(v[node * neq + c]);
      z[i] = VT(s);
    }
  }
}

// part[j * nblk + b] = block b's share of V_j . w, for j < k (grid.y = k).
template <typename VT>
__global__ void dot_partials_kernel(int64_t n, const VT* __restrict__ V, int64_t ldv, const VT* __restrict__ w,
                                    double* __restrict__ part, const int* __restrict__ done) {
  if (done && *done) return;
  __shared__ double sm[32];
  const int j = blockIdx.y;
  const VT* v = V + int64_t(j) * ldv;
  double s = 0.0;
  GRID_STRIDE(i, n) s += double(v[i]) * double(w[i]);
  s = block_sum(s, sm);
  if (threadIdx.x == 0) part[int64_t(j) * gridDim.x + blockIdx.x] = s;
}

// out[j] = sum_b part[j * nblk + b] in a fixed order; one block per j.
__global__ void reduce_partials_kernel(int nblk, const double* __restrict__ part, double* __restrict__ out,
                                       const int* __restrict__ done) {
  if (done && *done) return;
  __shared__ double sm[32];
  const int j = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += part[int64_t(j) * nblk + b];
  s = block_sum(s, sm);
  if (threadIdx.x == 0) out[j] = s;
}

// w -= sum_{j<k} h_j V_j ; optionally block partials of ||w||^2.
template <typename VT>
__global__ void multi_axpy_kernel(int64_t n, int k, const VT* __restrict__ V, int64_t ldv,
                                  const double* __restrict__ h, VT* __restrict__ w, double* __restrict__ normpart,
                                  const int* __restrict__ done) {
  if (done && *done) return;
  __shared__ double sm[32];
  double s2 = 0.0;
  GRID_STRIDE(i, n) {
    double acc = double(w[i]);
    for (int j = 0; j < k; ++j) acc -= h[j] * double(V[int64_t(j) * ldv + i]);
    const VT wv = VT(acc);
    w[i] = wv;
    s2 += double(wv) * double(wv);
  }
  if (normpart) {
    s2 = block_sum(s2, sm);
    if (threadIdx.x == 0) normpart[blockIdx.x] = s2;
  }
}

// t = V y (first k columns, k read from ictl[1]).
template <typename VT>
__global__ void combine_kernel(int64_t n, const VT* __restrict__ V, int64_t ldv, const double* __restrict__ y,
                               const int* __restrict__ ictl, VT* __restrict__ t) {
  const int k = ictl[1];
  GRID_STRIDE(i, n) {
    double acc = 0.0;
    for (int j = 0; j < k; ++j) acc += y[j] * double(V[int64_t(j) * ldv + i]);
    t[i] = VT(acc);
  }
}

// Arnoldi step j: H(:,j) = h1 + h2, H(j+1,j) = ||w||, Givens update, convergence.
__global__ void givens_kernel(int j, int m, const double* __restrict__ hbuf, const double* __restrict__ normpart,
                              int nblk, double* __restrict__ H, double* __restrict__ cs, double* __restrict__ sn,
                              double* __restrict__ g, double* __restrict__ dctl, int* __restrict__ ictl, double tol,
                              int last) {
  if (ictl[0]) return;
  double nn = 0.0;
  for (int b = 0; b < nblk; ++b) nn += normpart[b];
  const double hnext = sqrt(nn);
  for (int i = 0; i <= j; ++i) H[i * m + j] = hbuf[i] + hbuf[(m + 2) + i];
  H[(j + 1) * m + j] = hnext;
  for (int i = 0; i < j; ++i) {
    const double a = H[i * m + j], b = H[(i + 1) * m + j];
    H[i * m + j] = cs[i] * a + sn[i] * b;
    H[(i + 1) * m + j] = -sn[i] * a + cs[i] * b;
  }
  const double a = H[j * m + j], b = H[(j + 1) * m + j];
  const double den = sqrt(a * a + b * b);
  const double c = den != 0.0 ? a / den : 1.0;
  const double s = den != 0.0 ? b / den : 0.0;
  cs[j] = c;
  sn[j] = s;
  H[j * m + j] = den;
  H[(j + 1) * m + j] = 0.0;
  g[j + 1] = -s * g[j];
  g[j] = c * g[j];
  const double res = fabs(g[j + 1]);
  dctl[kEst] = res;
  dctl[kHnext] = hnext;
  ictl[1] = j + 1;
  if (!isfinite(res) || !isfinite(hnext) || den == 0.0) {
    ictl[0] = 1;
    ictl[2] = 3;
  } else if (res <= tol * dctl[kBnorm] || hnext <= 1e-300 * dctl[kBnorm] || last) {
    ictl[0] = 1;
  }
}

// dst = src * (1 / dctl[idx])
template <typename VT>
__global__ void scale_kernel(int64_t n, const VT* __restrict__ src, VT* __restrict__ dst,
                             const double* __restrict__ dctl, int idx, const int* __restrict__ done) {
  if (done && *done) return;
  const double inv = 1.0 / dctl[idx];
  GRID_STRIDE(i, n) dst[i] = VT(double(src[i]) * inv);
}

// r = b * bscale - w with block partials of ||r||^2 and (optionally) ||b||^2.
template <typename VT, typename BT>
__global__ void residual_kernel(int64_t n, const BT* __restrict__ b, const VT* __restrict__ w, VT* __restrict__ r,
                                double* __restrict__ normpart, double* __restrict__ bpart) {
  __shared__ double sm[32];
  double s2 = 0.0, b2 = 0.0;
  GRID_STRIDE(i, n) {
    const double bi = double(b[i]);
    const VT ri = VT(bi - double(w[i]));
    r[i] = ri;
    s2 += double(ri) * double(ri);
    b2 += bi * bi;
  }
  s2 = block_sum(s2, sm);
  if (threadIdx.x == 0) normpart[blockIdx.x] = s2;
  if (bpart) {
    b2 = block_sum(b2, sm);
    if (threadIdx.x == 0) bpart[blockIdx.x] = b2;
  }
}

// Partial sums of ||r||^2 and ||b||^2 (per block), no update.
__global__ void norm2_partials_kernel(int64_t n, const double* __restrict__ r, const double* __restrict__ b,
                                      double* __restrict__ rpart, double* __restrict__ bpart) {
  __shared__ double sm[32];
  double s2 = 0.0, b2 = 0.0;
  GRID_STRIDE(i, n) {
    s2 += r[i] * r[i];
    b2 += b[i] * b[i];
  }
  s2 = block_sum(s2, sm);
  if (threadIdx.x == 0) rpart[blockIdx.x] = s2;
  b2 = block_sum(b2, sm);
  if (threadIdx.x == 0) bpart[blockIdx.x] = b2;
}

// Restart: beta = ||r||, g = beta e1, done if converged.
__global__ void restart_setup_kernel(int nblk, int m, const double* __restrict__ normpart,
                                     const double* __restrict__ bpart, int first, double* __restrict__ g,
                                     double* __restrict__ dctl, int* __restrict__ ictl, double tol) {
  double nn = 0.0;
  for (int b = 0; b < nblk; ++b) nn += normpart[b];
  if (first) {
    double bb = 0.0;
    for (int b = 0; b < nblk; ++b) bb += bpart[b];
    dctl[kBnorm] = sqrt(bb);
  }
  const double beta = sqrt(nn);
  dctl[kBeta] = beta;
  dctl[kEst] = beta;
  for (int i = 0; i <= m; ++i) g[i] = 0.0;
  g[0] = beta;
  ictl[0] = 0;
  ictl[1] = 0;
  ictl[2] = 0;
  if (!isfinite(beta)) {
    ictl[0] = 1;
    ictl[2] = 3;
  } else if (beta <= tol * dctl[kBnorm] || beta == 0.0) {
    ictl[0] = 1;
  }
}

__global__ void backsolve_kernel(int m, const double* __restrict__ H, const double* __restrict__ g,
                                 double* __restrict__ y, const int* __restrict__ ictl) {
  const int k = ictl[1];
  for (int i = k - 1; i >= 0; --i) {
    double s = g[i];
    for (int l = i + 1; l < k; ++l) s -= H[i * m + l] * y[l];
    y[i] = s / H[i * m + i];
  }
}

template <typename VT>
__global__ void axpy_kernel(int64_t n, double alpha, const VT* __restrict__ x, VT* __restrict__ y) {
  GRID_STRIDE(i, n) y[i] = VT(double(y[i]) + alpha * double(x[i]));
}

// x64 += dctl[idx] * d32
template <typename VT>
__global__ void add_scaled_kernel(int64_t n, const VT* __restrict__ d, double* __restrict__ x,
                                  const double* __restrict__ dctl, int idx) {
  const double sc = dctl[idx];
  GRID_STRIDE(i, n) x[i] += sc * double(d[i]);
}

template <typename VT>
__global__ void fill_kernel(int64_t n, VT v, VT* __restrict__ x) {
  GRID_STRIDE(i, n) x[i] = v;
}

// dctl[idx] = (sqrt) sum of nblk partials
__global__ void finalize_norm_kernel(int nblk, const double* __restrict__ part, double* __restrict__ dctl, int idx,
                                     int take_sqrt) {
  __shared__ double sm[32];
  double s = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += part[b];
  s = block_sum(s, sm);
  if (threadIdx.x == 0) dctl[idx] = take_sqrt ? sqrt(s) : s;
}

// ---- BiCGStab kernels ---------------------------------------------------------
// Scalars in dctl: rho (= rh.r of the current residual), rho_old, alpha, omega.
// Each reduction's last block folds the block partials in a fixed order and
// computes the next scalar (the single-block "reduce" kernels do the same where
// the workspace has no fold counter), so an iteration is seven launches, and
// thirteen with the two-level preconditioner's coarse correction.

// p = r + beta (p - omega v), beta = (rho/rho_old)(alpha/omega); ph = M^-1 p
// (point Jacobi or identity inline; block Jacobi applied by precond_kernel).
template <typename VT>
__global__ void bicg_p_kernel(int64_t n, int pkind, const VT* __restrict__ dinv, const VT* __restrict__ r,
                              const VT* __restrict__ v, VT* __restrict__ p, VT* __restrict__ ph,
                              const double* __restrict__ dctl, const int* __restrict__ ictl) {
  if (ictl[0]) return;
  const double beta = (dctl[kRho] / dctl[kRhoOld]) * (dctl[kAlpha] / dctl[kOmega]);
  const double om = dctl[kOmega];
  GRID_STRIDE(i, n) {
    const VT pi = VT(double(r[i]) + beta * (double(p[i]) - om * double(v[i])));
    p[i] = pi;
    if (pkind != 2) ph[i] = (pkind == 1) ? VT(dinv[i] * pi) : pi;
  }
}

// alpha = rho / (rh . v), given d = rh . v (one thread).
__device__ __forceinline__ void bicg_alpha_update(double d, double* __restrict__ dctl, int* __restrict__ ictl,
                                                  double alpha_max) {
  dctl[kRhV] = d;
  if (d == 0.0 || !isfinite(d)) {
    ictl[0] = 1;
    ictl[2] = isfinite(d) ? 2 : 3;
    return;
  }
  const double a = dctl[kRho] / d;
  if (!(fabs(a) < alpha_max)) {  // (rh, v) ~ 0: the step would overflow the vector type
    ictl[0] = 1;
    ictl[2] = 2;
    return;
  }
  dctl[kAlpha] = a;
}

// alpha from the block partials of rh . v (a fixed-order fold).
__global__ void bicg_alpha_kernel(int nblk, const double* __restrict__ part, double* __restrict__ dctl,
                                  int* __restrict__ ictl, double alpha_max) {
  if (ictl[0]) return;
  __shared__ double sm[32];
  double sv = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) sv += part[b];
  const double d = block_sum(sv, sm);
  if (threadIdx.x != 0) return;
  bicg_alpha_update(d, dctl, ictl, alpha_max);
}

// s = r - alpha v ; sh = M^-1 s
template <typename VT>
__global__ void bicg_s_kernel(int64_t n, int pkind, const VT* __restrict__ dinv, const VT* __restrict__ r,
                              const VT* __restrict__ v, VT* __restrict__ s, VT* __restrict__ sh,
                              const double* __restrict__ dctl, const int* __restrict__ ictl) {
  if (ictl[0]) return;
  const double al = dctl[kAlpha];
  GRID_STRIDE(i, n) {
    const VT si = VT(double(r[i]) - al * double(v[i]));
    s[i] = si;
    if (pkind != 2) sh[i] = (pkind == 1) ? VT(dinv[i] * si) : si;
  }
}

// block partials of t.s (part[0..nblk)) and t.t (part[nblk..2nblk))
template <typename VT>
__global__ void dot2_partials_kernel(int64_t n, const VT* __restrict__ t, const VT* __restrict__ s,
                                     double* __restrict__ part, const int* __restrict__ ictl) {
  if (ictl[0]) return;
  __shared__ double sm[32];
  double ts = 0.0, tt = 0.0;
  GRID_STRIDE(i, n) {
    const double ti = double(t[i]);
    ts += ti * double(s[i]);
    tt += ti * ti;
  }
  ts = block_sum(ts, sm);
  tt = block_sum(tt, sm);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = ts;
    part[gridDim.x + blockIdx.x] = tt;
  }
}

// omega = (t . s) / (t . t) (one thread).
__device__ __forceinline__ void bicg_omega_update(double ts, double tt, double* __restrict__ dctl,
                                                  int* __restrict__ ictl) {
  const double om = (tt != 0.0) ? ts / tt : 0.0;
  dctl[kTS] = ts;
  dctl[kTT] = tt;
  dctl[kOmega] = om;
  if (!isfinite(om)) {
    ictl[0] = 1;
    ictl[2] = 3;
  } else if (om == 0.0 && tt != 0.0) {
    // t.s = 0 with t != 0: the next beta would divide by omega (breakdown);
    // x is still advanced by alpha*ph in bicg_xr_kernel before stopping
    ictl[2] = 2;
  }
}

__global__ void bicg_omega_kernel(int nblk, const double* __restrict__ part, double* __restrict__ dctl,
                                  int* __restrict__ ictl) {
  if (ictl[0]) return;
  __shared__ double sm[32];
  double a = 0.0, b = 0.0;
  for (int k = threadIdx.x; k < nblk; k += blockDim.x) {
    a += part[k];
    b += part[nblk + k];
  }
  const double ts = block_sum(a, sm);
  const double tt = block_sum(b, sm);
  if (threadIdx.x != 0) return;
  bicg_omega_update(ts, tt, dctl, ictl);
}

// x += alpha ph + omega sh ; r = s - omega t ; partials of r.r and rh.r
template <typename VT>
__global__ void bicg_xr_kernel(int64_t n, const VT* __restrict__ ph, const VT* __restrict__ sh,
                               const VT* __restrict__ s, const VT* __restrict__ t, const VT* __restrict__ rh,
                               VT* __restrict__ x, VT* __restrict__ r, const double* __restrict__ dctl,
                               const int* __restrict__ ictl, double* __restrict__ part) {
  if (ictl[0]) return;
  __shared__ double sm[32];
  const double al = dctl[kAlpha], om = dctl[kOmega];
  double rr = 0.0, hr = 0.0;
  GRID_STRIDE(i, n) {
    x[i] = VT(double(x[i]) + al * double(ph[i]) + om * double(sh[i]));
    const VT ri = VT(double(s[i]) - om * double(t[i]));
    r[i] = ri;
    rr += double(ri) * double(ri);
    hr += double(rh[i]) * double(ri);
  }
  rr = block_sum(rr, sm);
  hr = block_sum(hr, sm);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = rr;
    part[gridDim.x + blockIdx.x] = hr;
  }
}

// ||r|| and the next rho = rh . r; convergence and iteration count (one thread).
__device__ __forceinline__ void bicg_end_update(double nn, double rho_new, double* __restrict__ dctl,
                                                int* __restrict__ ictl, double tol, int maxit) {
  const double rn = sqrt(nn);
  dctl[kEst] = rn;
  dctl[kRhoOld] = dctl[kRho];
  dctl[kRho] = rho_new;
  ictl[3] += 1;
  if (ictl[2] == 2) {  // omega breakdown flagged this iteration
    ictl[0] = 1;
  } else if (!isfinite(rn) || !isfinite(rho_new)) {
    ictl[0] = 1;
    ictl[2] = 3;
  } else if (rn <= tol * dctl[kBnorm]) {
    ictl[0] = 1;
  } else if (rho_new == 0.0) {
    ictl[0] = 1;
    ictl[2] = 2;
  } else if (ictl[3] >= maxit) {
    ictl[0] = 1;
    ictl[2] = 1;
  }
}

__global__ void bicg_end_kernel(int nblk, const double* __restrict__ part, double* __restrict__ dctl,
                                int* __restrict__ ictl, double tol, int maxit) {
  if (ictl[0]) return;
  __shared__ double sm[32];
  double a = 0.0, b = 0.0;
  for (int k = threadIdx.x; k < nblk; k += blockDim.x) {
    a += part[k];
    b += part[nblk + k];
  }
  const double nn = block_sum(a, sm);
  const double rho_new = block_sum(b, sm);
  if (threadIdx.x != 0) return;
  bicg_end_update(nn, rho_new, dctl, ictl, tol, maxit);
}

// rho = ||r0||^2 (rh = r0), rho_old = alpha = omega = 1, converged test.
__global__ void bicg_init_kernel(double* dctl, int* ictl, double tol) {
  dctl[kRho] = dctl[kBeta] * dctl[kBeta];
  dctl[kRhoOld] = 1.0;
  dctl[kAlpha] = 1.0;
  dctl[kOmega] = 1.0;
  ictl[0] = (dctl[kBeta] <= tol * dctl[kBnorm] || dctl[kBnorm] == 0.0) ? 1 : 0;
  ictl[2] = isfinite(dctl[kBeta]) ? 0 : 3;
  if (ictl[2]) ictl[0] = 1;
  ictl[3] = 0;
}

// ---- CG kernels (symmetric positive definite systems) -------------------------
// Scalars in dctl: rho = r . z, alpha, omega slot = beta.  Five launches per
// iteration: SpMV, p.q partials, alpha, x/r/z update with r.r and r.z
// partials, and the fold that tests convergence and forms beta; the direction
// update is folded into the next iteration's first kernel.

// p = z + beta p (skipped on the first iteration: beta = 0, p = z).
template <typename VT>
__global__ void cg_p_kernel(int64_t n, const VT* __restrict__ z, VT* __restrict__ p,
                            const double* __restrict__ dctl, const int* __restrict__ ictl) {
  if (ictl[0]) return;
  const double beta = dctl[kOmega];
  GRID_STRIDE(i, n) p[i] = VT(double(z[i]) + beta * double(p[i]));
}

// alpha = rho / (p . q); a non-positive p . q stops the solve (not SPD).
__global__ void cg_alpha_kernel(int nblk, const double* __restrict__ part, double* __restrict__ dctl,
                                int* __restrict__ ictl) {
  if (ictl[0]) return;
  __shared__ double sm[32];
  double sv = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) sv += part[b];
  const double d = block_sum(sv, sm);
  if (threadIdx.x != 0) return;
  if (!isfinite(d)) {
    ictl[0] = 1;
    ictl[2] = 3;
    return;
  }
  if (!(d > 0.0)) {
    ictl[0] = 1;
    ictl[2] = 2;
    return;
  }
  dctl[kAlpha] = dctl[kRho] / d;
}

// x += alpha p ; r -= alpha q ; z = M^-1 r (point Jacobi or identity inline) ;
// partials of r.r and r.z.  With block Jacobi (pkind 2) z is formed afterwards.
template <typename VT>
__global__ void cg_xr_kernel(int64_t n, int pkind, const VT* __restrict__ dinv, const VT* __restrict__ p,
                             const VT* __restrict__ q, VT* __restrict__ x, VT* __restrict__ r, VT* __restrict__ z,
                             const double* __restrict__ dctl, const int* __restrict__ ictl,
                             double* __restrict__ part) {
  if (ictl[0]) return;
  __shared__ double sm[32];
  const double al = dctl[kAlpha];
  double rr = 0.0, rz = 0.0;
  GRID_STRIDE(i, n) {
    x[i] = VT(double(x[i]) + al * double(p[i]));
    const VT ri = VT(double(r[i]) - al * double(q[i]));
    r[i] = ri;
    rr += double(ri) * double(ri);
    if (pkind != 2) {
      const VT zi = (pkind == 1) ? VT(dinv[i] * ri) : ri;
      z[i] = zi;
      rz += double(ri) * double(zi);
    }
  }
  rr = block_sum(rr, sm);
  rz = block_sum(rz, sm);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = rr;
    part[gridDim.x + blockIdx.x] = rz;
  }
}

// ||r||, rho_new = r . z, beta = rho_new / rho; convergence and iteration count.
__global__ void cg_end_kernel(int nblk, const double* __restrict__ part, double* __restrict__ dctl,
                              int* __restrict__ ictl, double tol, int maxit) {
  if (ictl[0]) return;
  __shared__ double sm[32];
  double a = 0.0, b = 0.0;
  for (int k = threadIdx.x; k < nblk; k += blockDim.x) {
    a += part[k];
    b += part[nblk + k];
  }
  const double nn = block_sum(a, sm);
  const double rho_new = block_sum(b, sm);
  if (threadIdx.x != 0) return;
  const double rn = sqrt(nn);
  dctl[kEst] = rn;
  dctl[kOmega] = rho_new / dctl[kRho];
  dctl[kRho] = rho_new;
  ictl[3] += 1;
  if (!isfinite(rn) || !isfinite(rho_new)) {
    ictl[0] = 1;
    ictl[2] = 3;
  } else if (rn <= tol * dctl[kBnorm]) {
    ictl[0] = 1;
  } else if (!(rho_new > 0.0)) {  // indefinite preconditioner or exact breakdown
    ictl[0] = 1;
    ictl[2] = 2;
  } else if (ictl[3] >= maxit) {
    ictl[0] = 1;
    ictl[2] = 1;
  }
}

// rho = r0 . z0 (from the partials), beta = 0, converged test.
__global__ void cg_init_kernel(int nblk, const double* __restrict__ part, double* dctl, int* ictl, double tol) {
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += part[b];
  dctl[kRho] = s;
  dctl[kOmega] = 0.0;
  ictl[0] = (dctl[kBeta] <= tol * dctl[kBnorm] || dctl[kBnorm] == 0.0) ? 1 : 0;
  ictl[2] = isfinite(dctl[kBeta]) ? 0 : 3;
  if (ictl[2]) ictl[0] = 1;
  ictl[3] = 0;
}

// ---- fused CG iteration (point Jacobi or no preconditioner) ------------------
// Each reduction kernel writes its block partials, and the last block to finish
// (an atomic ticket on a per-solve counter, reset by that block) folds them in
// block order and updates the scalars: deterministic, and no block waits for
// another.  Four launches per iteration: p update, SpMV, p.q with the alpha
// fold, x/r/z update with the convergence/beta fold.

__device__ __forceinline__ bool last_block(int* counter, int* s_flag) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) *s_flag = (atomicAdd(counter, 1) == int(gridDim.x) - 1) ? 1 : 0;
  __syncthreads();
  if (*s_flag == 0) return false;
  __threadfence();
  if (threadIdx.x == 0) *counter = 0;  // ready for the next launch
  return true;
}

// BiCGStab's reductions with their scalar updates folded in: the launch's last
// block (an atomic ticket, reset by that block; no block waits for another)
// folds the block partials exactly as the separate single-block kernels do --
// the same grid, the same 256-thread strided sums and block tree -- so the
// arithmetic is theirs, bitwise, with one launch fewer per reduction.

// rh . v partials, then alpha
template <typename VT>
__global__ void bicg_vdot_fold_kernel(int64_t n, const VT* __restrict__ rh, const VT* __restrict__ v,
                                      double* __restrict__ part, int* __restrict__ counter,
                                      double* __restrict__ dctl, int* __restrict__ ictl, double alpha_max) {
  if (ictl[0]) return;  // read before any block of this launch can change it
  __shared__ double sm[32];
  __shared__ int flag;
  double s = 0.0;
  GRID_STRIDE(i, n) s += double(rh[i]) * double(v[i]);
  s = block_sum(s, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
  if (!last_block(counter, &flag)) return;
  double sv = 0.0;
  for (int b = threadIdx.x; b < int(gridDim.x); b += blockDim.x) sv += __ldcg(part + b);
  const double d = block_sum(sv, sm);
  if (threadIdx.x != 0) return;
  bicg_alpha_update(d, dctl, ictl, alpha_max);
}

// t . s and t . t partials, then omega
template <typename VT>
__global__ void bicg_ts_fold_kernel(int64_t n, const VT* __restrict__ t, const VT* __restrict__ s,
                                    double* __restrict__ part, int* __restrict__ counter,
                                    double* __restrict__ dctl, int* __restrict__ ictl) {
  if (ictl[0]) return;
  __shared__ double sm[32];
  __shared__ int flag;
  double ts = 0.0, tt = 0.0;
  GRID_STRIDE(i, n) {
    const double ti = double(t[i]);
    ts += ti * double(s[i]);
    tt += ti * ti;
  }
  ts = block_sum(ts, sm);
  tt = block_sum(tt, sm);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = ts;
    part[gridDim.x + blockIdx.x] = tt;
  }
  if (!last_block(counter, &flag)) return;
  const int nb = int(gridDim.x);
  double a = 0.0, b = 0.0;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {
    a += __ldcg(part + k);
    b += __ldcg(part + nb + k);
  }
  const double fts = block_sum(a, sm);
  const double ftt = block_sum(b, sm);
  if (threadIdx.x != 0) return;
  bicg_omega_update(fts, ftt, dctl, ictl);
}

// x += alpha ph + omega sh ; r = s - omega t with the partials of r.r and
// rh.r, then the convergence test and the next rho
template <typename VT>
__global__ void bicg_xr_fold_kernel(int64_t n, const VT* __restrict__ ph, const VT* __restrict__ sh,
                                    const VT* __restrict__ s, const VT* __restrict__ t, const VT* __restrict__ rh,
                                    VT* __restrict__ x, VT* __restrict__ r, double* __restrict__ dctl,
                                    int* __restrict__ ictl, double* __restrict__ part, int* __restrict__ counter,
                                    double tol, int maxit) {
  if (ictl[0]) return;
  __shared__ double sm[32];
  __shared__ int flag;
  const double al = dctl[kAlpha], om = dctl[kOmega];
  double rr = 0.0, hr = 0.0;
  GRID_STRIDE(i, n) {
    x[i] = VT(double(x[i]) + al * double(ph[i]) + om * double(sh[i]));
    const VT ri = VT(double(s[i]) - om * double(t[i]));
    r[i] = ri;
    rr += double(ri) * double(ri);
    hr += double(rh[i]) * double(ri);
  }
  rr = block_sum(rr, sm);
  hr = block_sum(hr, sm);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = rr;
    part[gridDim.x + blockIdx.x] = hr;
  }
  if (!last_block(counter, &flag)) return;
  const int nb = int(gridDim.x);
  double a = 0.0, b = 0.0;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {
    a += __ldcg(part + k);
    b += __ldcg(part + nb + k);
  }
  const double nn = block_sum(a, sm);
  const double rho_new = block_sum(b, sm);
  if (threadIdx.x != 0) return;
  bicg_end_update(nn, rho_new, dctl, ictl, tol, maxit);
}

// Last block of a CG iteration: ||r|| and rho_new = r.z from the block partials
// part[0..grid) and part[grid..2 grid), beta, convergence and iteration count.
__device__ __forceinline__ void cg_fold_end(const double* __restrict__ part, double* __restrict__ dctl,
                                            int* __restrict__ ictl, double tol, int maxit, double* sm) {
  double a = 0.0, b = 0.0;
  for (int k = threadIdx.x; k < int(gridDim.x); k += blockDim.x) {
    a += __ldcg(part + k);
    b += __ldcg(part + gridDim.x + k);
  }
  const double nn = block_sum(a, sm);
  const double rho_new = block_sum(b, sm);
  if (threadIdx.x != 0) return;
  const double rn = sqrt(nn);
  dctl[kEst] = rn;
  dctl[kOmega] = rho_new / dctl[kRho];
  dctl[kRho] = rho_new;
  ictl[3] += 1;
  if (!isfinite(rn) || !isfinite(rho_new)) {
    ictl[0] = 1;
    ictl[2] = 3;
  } else if (rn <= tol * dctl[kBnorm]) {
    ictl[0] = 1;
  } else if (!(rho_new > 0.0)) {
    ictl[0] = 1;
    ictl[2] = 2;
  } else if (ictl[3] >= maxit) {
    ictl[0] = 1;
    ictl[2] = 1;
  }
}

template <typename VT>
__global__ void cg_pq_fold_kernel(int64_t n, const VT* __restrict__ p, const VT* __restrict__ q,
                                  double* __restrict__ part, int* __restrict__ counter, double* __restrict__ dctl,
                                  int* __restrict__ ictl) {
  if (ictl[0]) return;  // read before any block of this launch can change it
  __shared__ double sm[32];
  __shared__ int flag;
  double s = 0.0;
  GRID_STRIDE(i, n) s += double(p[i]) * double(q[i]);
  s = block_sum(s, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
  if (!last_block(counter, &flag)) return;
  double sv = 0.0;
  for (int b = threadIdx.x; b < int(gridDim.x); b += blockDim.x) sv += __ldcg(part + b);
  const double d = block_sum(sv, sm);
  if (threadIdx.x != 0) return;
  if (!isfinite(d)) {
    ictl[0] = 1;
    ictl[2] = 3;
  } else if (!(d > 0.0)) {
    ictl[0] = 1;
    ictl[2] = 2;
  } else {
    dctl[kAlpha] = dctl[kRho] / d;
  }
}

template <typename VT>
__global__ void cg_xr_fold_kernel(int64_t n, int pkind, const VT* __restrict__ dinv, const VT* __restrict__ p,
                                  const VT* __restrict__ q, VT* __restrict__ x, VT* __restrict__ r,
                                  VT* __restrict__ z, double* __restrict__ part, int* __restrict__ counter,
                                  double* __restrict__ dctl, int* __restrict__ ictl, double tol, int maxit) {
  if (ictl[0]) return;
  __shared__ double sm[32];
  __shared__ int flag;
  const double al = dctl[kAlpha];
  double rr = 0.0, rz = 0.0;
  GRID_STRIDE(i, n) {
    x[i] = VT(double(x[i]) + al * double(p[i]));
    const VT ri = VT(double(r[i]) - al * double(q[i]));
    r[i] = ri;
    const VT zi = (pkind == 1) ? VT(dinv[i] * ri) : ri;
    z[i] = zi;
    rr += double(ri) * double(ri);
    rz += double(ri) * double(zi);
  }
  rr = block_sum(rr, sm);
  rz = block_sum(rz, sm);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = rr;
    part[gridDim.x + blockIdx.x] = rz;
  }
  if (!last_block(counter, &flag)) return;
  cg_fold_end(part, dctl, ictl, tol, maxit, sm);
}

// x += alpha p ; r -= alpha q ; partials of r.r (the z update follows the
// coarse correction of the two-level preconditioner).
template <typename VT>
__global__ void cg_xr_plain_kernel(int64_t n, const VT* __restrict__ p, const VT* __restrict__ q, VT* __restrict__ x,
                                   VT* __restrict__ r, double* __restrict__ part, const double* __restrict__ dctl,
                                   const int* __restrict__ ictl) {
  if (ictl[0]) return;
  __shared__ double sm[32];
  const double al = dctl[kAlpha];
  double rr = 0.0;
  GRID_STRIDE(i, n) {
    x[i] = VT(double(x[i]) + al * double(p[i]));
    const VT ri = VT(double(r[i]) - al * double(q[i]));
    r[i] = ri;
    rr += double(ri) * double(ri);
  }
  rr = block_sum(rr, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = rr;
}

// Threads of the restriction and coarse-product blocks.
constexpr int kCoarseThreads = 128;

// c[I] = sum of r over the rows of aggregate I, one block per aggregate (a fixed
// thread partition and block tree: deterministic).
template <typename VT>
__global__ void __launch_bounds__(kCoarseThreads)
    restrict_kernel(int nc, const int32_t* __restrict__ agg_ptr, const int32_t* __restrict__ agg_rows,
                    const VT* __restrict__ r, double* __restrict__ c, const int* __restrict__ done) {
  if (done && *done) return;
  __shared__ double sm[32];
  const int I = blockIdx.x;
  double s = 0.0;
  for (int k = agg_ptr[I] + threadIdx.x; k < agg_ptr[I + 1]; k += blockDim.x) s += double(r[agg_rows[k]]);
  s = block_sum(s, sm);
  if (threadIdx.x == 0) c[I] = s;
}

// y = Ac^-1 c, one block per coarse row.
__global__ void __launch_bounds__(kCoarseThreads)
    coarse_kernel(int nc, const double* __restrict__ ainv, const double* __restrict__ c, double* __restrict__ y,
                  const int* __restrict__ done) {
  if (done && *done) return;
  __shared__ double sm[32];
  const int I = blockIdx.x;
  double s = 0.0;
  for (int J = threadIdx.x; J < nc; J += blockDim.x) s += ainv[int64_t(I) * nc + J] * c[J];
  s = block_sum(s, sm);
  if (threadIdx.x == 0) y[I] = s;
}

// z = D^-1 r + y[agg]
template <typename VT>
__global__ void prolong_kernel(int64_t n, const VT* __restrict__ dinv, const int32_t* __restrict__ agg,
                               const double* __restrict__ y, const VT* __restrict__ r, VT* __restrict__ z) {
  GRID_STRIDE(i, n) {
    const int a = agg[i];
    z[i] = VT(double(dinv[i]) * double(r[i]) + (a >= 0 ? y[a] : 0.0));
  }
}

// z += y[agg] on the rows of the coarse space (the coupled two-level form:
// z already holds D^-1 r).
template <typename VT>
__global__ void prolong_add_kernel(int64_t n, const int32_t* __restrict__ agg, const double* __restrict__ y,
                                   VT* __restrict__ z, const int* __restrict__ done) {
  if (done && *done) return;
  GRID_STRIDE(i, n) {
    const int a = agg[i];
    if (a >= 0) z[i] = VT(double(z[i]) + y[a]);
  }
}

// Coarse pressure matrix of the coupled two-level form: ac[dst[q]] = the sum of
// the values at the segment's sorted CSR positions (one warp per segment; the
// lane partition and the shuffle tree are fixed, so the sum is deterministic).
__global__ void coarse_matrix_kernel(int nseg, const int32_t* __restrict__ seg, const int32_t* __restrict__ dst,
                                     const int64_t* __restrict__ pos, const double* __restrict__ vals,
                                     double* __restrict__ ac) {
  const int q = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (q >= nseg) return;  // whole warps
  double s = 0.0;
  for (int k = seg[q] + lane; k < seg[q + 1]; k += 32) s += vals[pos[k]];
  s = warp_sum(s);
  if (lane == 0) ac[dst[q]] = s;
}

// z = D^-1 r + y[agg] ; partials of r.z ; the last block folds r.r (written by
// cg_xr_plain_kernel with the same grid) and r.z into the convergence test and beta.
template <typename VT>
__global__ void cg_prolong_fold_kernel(int64_t n, const VT* __restrict__ dinv, const int32_t* __restrict__ agg,
                                       const double* __restrict__ y, const VT* __restrict__ r, VT* __restrict__ z,
                                       double* __restrict__ part, int* __restrict__ counter,
                                       double* __restrict__ dctl, int* __restrict__ ictl, double tol, int maxit) {
  if (ictl[0]) return;
  __shared__ double sm[32];
  __shared__ int flag;
  double rz = 0.0;
  GRID_STRIDE(i, n) {
    const int a = agg[i];
    const double ri = double(r[i]);
    const VT zi = VT(double(dinv[i]) * ri + (a >= 0 ? y[a] : 0.0));
    z[i] = zi;
    rz += ri * double(zi);
  }
  rz = block_sum(rz, sm);
  if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = rz;
  if (!last_block(counter, &flag)) return;
  cg_fold_end(part, dctl, ictl, tol, maxit, sm);
}

// ---------------------------------------------------------------------------
template <typename T>
int dalloc(T** p, size_t count) {
  if (*p) return UFEM_OK;
  DeviceLock lk(device_mutex());
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess)
    return set_error(UFEM_ERR_NOMEM, std::string("cudaMalloc (Krylov workspace): ") + cudaGetErrorString(e));
  return UFEM_OK;
}

template <typename T>
void dfree(T*& p) {
  DeviceLock lk(device_mutex());
  if (p) cudaFree(p);
  p = nullptr;
}

int ensure_work(ufem_ns_handle* h, int m, bool need32, bool bicg) {
  if (!h->kw) h->kw = new KrylovWork();
  KrylovWork& kw = *h->kw;
  const int64_t n = h->nrows;
  if (kw.m < m && (kw.V || kw.V32 || kw.part)) {  // a longer restart: reallocate the basis-sized buffers
    dfree(kw.V); dfree(kw.V32); dfree(kw.part); dfree(kw.hbuf); dfree(kw.H);
    dfree(kw.cs); dfree(kw.sn); dfree(kw.g); dfree(kw.y);
  }
  kw.m = std::max(kw.m, m);
  kw.n = n;
  kw.nblk = red_blocks(n);
  kw.cg_nblk = int(std::min<int64_t>(kCGMaxBlocks, std::max<int64_t>(1, (n + 511) / 512)));
  const int M = kw.m;
  const size_t nd = size_t(n);
  const size_t ndinv = size_t(h->N) * h->neq * h->neq;
  const size_t npart = std::max(size_t(M + 2) * kw.nblk, size_t(2) * kCGMaxBlocks);
  int rc;
  if (!kw.cg_counter) {
    if ((rc = dalloc(&kw.cg_counter, 1))) return rc;
    UFEM_CUDA_TRY(cudaMemset(kw.cg_counter, 0, sizeof(int)));
  }
  if ((rc = dalloc(&kw.w, nd)) || (rc = dalloc(&kw.z, nd)) || (rc = dalloc(&kw.t, nd)) || (rc = dalloc(&kw.r, nd)) ||
      (rc = dalloc(&kw.dinv, ndinv)) || (rc = dalloc(&kw.part, npart)) ||
      (rc = dalloc(&kw.hbuf, size_t(2) * (M + 2))) || (rc = dalloc(&kw.H, size_t(M + 1) * M)) ||
      (rc = dalloc(&kw.cs, size_t(M))) || (rc = dalloc(&kw.sn, size_t(M))) || (rc = dalloc(&kw.g, size_t(M + 1))) ||
      (rc = dalloc(&kw.y, size_t(M))) || (rc = dalloc(&kw.dctl, 16)) || (rc = dalloc(&kw.ictl, 8)))
    return rc;
  if (!kw.h_dctl) {
    DeviceLock lk(device_mutex());
    UFEM_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&kw.h_dctl), 16 * sizeof(double)));
    UFEM_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&kw.h_ictl), 8 * sizeof(int)));
  }
  if (!bicg) {
    if (need32) {
      if ((rc = dalloc(&kw.V32, size_t(M + 1) * nd))) return rc;
    } else {
      if ((rc = dalloc(&kw.V, size_t(M + 1) * nd))) return rc;
    }
  }
  if (need32 && (rc = dalloc(&h->d_vals32, size_t(h->nnz)))) return rc;
  if (need32 && !bicg) {  // mixed GMRES runs its inner solve on FP32 vectors
    if ((rc = dalloc(&kw.w32, nd)) || (rc = dalloc(&kw.z32, nd)) || (rc = dalloc(&kw.t32, nd)) ||
        (rc = dalloc(&kw.r32, nd)) || (rc = dalloc(&kw.x32, nd)) || (rc = dalloc(&kw.q32, nd)) ||
        (rc = dalloc(&kw.dinv32, ndinv)))
      return rc;
  }
  if (bicg) {  // FP64 vectors, also for the mixed path (FP32 operator only)
    if ((rc = dalloc(&kw.bp, nd)) || (rc = dalloc(&kw.bv, nd)) || (rc = dalloc(&kw.bs, nd)) ||
        (rc = dalloc(&kw.bt, nd)) || (rc = dalloc(&kw.brh, nd)) || (rc = dalloc(&kw.bph, nd)) ||
        (rc = dalloc(&kw.bsh, nd)))
      return rc;
  }
  return UFEM_OK;
}

inline unsigned grid_for(int64_t n, int threads, int64_t cap = 8 * 148) {
  return unsigned(std::max<int64_t>(1, std::min<int64_t>(cap, (n + threads - 1) / threads)));
}

template <typename VT, typename MT>
int spmv(ufem_ns_handle* h, const MT* vals, const VT* x, VT* y, const int* done, cudaStream_t s) {
  const int64_t threads = h->N * 32;
  const unsigned grid = unsigned((threads + 255) / 256);
  const unsigned grid8 = unsigned((h->N * 8 + 255) / 256);  // 8 lanes per node
  if (h->neq == 4) {
    // resident grid of the persistent kernel (the device's SM count, queried once)
    static const unsigned resident = [] {
      int b = 0, dev = 0, sms = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, spmv4_stream_kernel<VT, MT>, 256, 0) != cudaSuccess)
        b = 1;
      if (cudaGetDevice(&dev) != cudaSuccess ||
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        sms = 1;
      return unsigned(std::max(1, b) * std::max(1, sms));
    }();
    spmv4_stream_kernel<VT, MT><<<std::min(grid, resident), 256, 0, s>>>(h->N, h->d_start, h->d_adj, vals, x, y,
                                                                          done);
  } else {
    // resident grid of the persistent group kernel (queried once per instantiation)
    auto resident_of = [](auto kernel) {
      int b = 0, dev = 0, sms = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, 256, 0) != cudaSuccess) b = 1;
      if (cudaGetDevice(&dev) != cudaSuccess ||
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        sms = 1;
      return unsigned(std::max(1, b) * std::max(1, sms));
    };
    if (h->neq == 3) {
      static const unsigned r3 = resident_of(spmv_small_kernel<3, VT, MT>);
      spmv_small_kernel<3, VT, MT><<<std::min(grid8, r3), 256, 0, s>>>(h->N, h->d_start, h->d_adj, vals, x, y, done);
    } else if (h->neq == 2) {
      static const unsigned r2 = resident_of(spmv_small_kernel<2, VT, MT>);
      spmv_small_kernel<2, VT, MT><<<std::min(grid8, r2), 256, 0, s>>>(h->N, h->d_start, h->d_adj, vals, x, y, done);
    } else {
      static const unsigned r1 = resident_of(spmv_small_kernel<1, VT, MT>);
      spmv_small_kernel<1, VT, MT><<<std::min(grid8, r1), 256, 0, s>>>(h->N, h->d_start, h->d_adj, vals, x, y, done);
    }
  }
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

template <typename VT, typename MT>
int setup_precond(ufem_ns_handle* h, int kind, const MT* vals, VT* dinv, cudaStream_t s) {
  if (kind == 1 || kind == 3 || kind == 4)
    jacobi_kernel<MT, VT><<<grid_for(h->nrows, 256), 256, 0, s>>>(h->nrows, h->d_diagpos, vals, dinv);
  else if (kind == 2)
    block_jacobi_kernel<MT, VT><<<grid_for(h->N, 128), 128, 0, s>>>(h->N, h->neq, h->d_diagpos, vals, dinv);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

// z += R Ac^-1 R^T v: the coarse correction of the coupled two-level form.
template <typename VT>
int coarse_correct(ufem_ns_handle* h, const VT* v, VT* z, const int* done, cudaStream_t s) {
  KrylovWork& kw = *h->kw;
  restrict_kernel<VT><<<unsigned(kw.nc), kCoarseThreads, 0, s>>>(kw.nc, kw.agg_ptr, kw.agg_rows, v, kw.cvec, done);
  coarse_kernel<<<unsigned(kw.nc), kCoarseThreads, 0, s>>>(kw.nc, kw.ainv, kw.cvec, kw.yvec, done);
  prolong_add_kernel<VT><<<unsigned(kw.nblk), kRedThreads, 0, s>>>(h->nrows, kw.agg, kw.yvec, z, done);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

template <typename VT>
int precond(ufem_ns_handle* h, int kind, const VT* dinv, const VT* v, VT* z, const int* done, cudaStream_t s) {
  precond_kernel<VT><<<grid_for(h->nrows, 256), 256, 0, s>>>(h->nrows, h->neq, kind == 4 ? 1 : kind, dinv, v, z,
                                                              done);
  UFEM_CUDA_TRY(cudaGetLastError());
  if (kind == 4) return coarse_correct<VT>(h, v, z, done, s);
  return UFEM_OK;
}

struct SolveResult {
  int iters = 0;
  int status = 0;  // 0 ok, 1 max iterations, 2 breakdown, 3 non-finite
  double relres = 0.0;
  bool converged = false;
};

// Final FP64-or-VT true residual ||b - A x|| / ||b|| into res.
template <typename VT, typename MT, typename BT>
int true_residual(ufem_ns_handle* h, KrylovWork& kw, const MT* vals, const BT* b, const VT* x, VT* w, VT* r,
                  double bnorm, cudaStream_t s, double* out) {
  int rc;
  if ((rc = spmv<VT, MT>(h, vals, x, w, nullptr, s))) return rc;
  residual_kernel<VT, BT><<<unsigned(kw.nblk), kRedThreads, 0, s>>>(h->nrows, b, w, r, kw.part, nullptr);
  finalize_norm_kernel<<<1, kRedThreads, 0, s>>>(kw.nblk, kw.part, kw.dctl, kTrue, 1);
  UFEM_CUDA_TRY(cudaMemcpyAsync(kw.h_dctl, kw.dctl, 16 * sizeof(double), cudaMemcpyDeviceToHost, s));
  UFEM_CUDA_TRY(cudaStreamSynchronize(s));
  // a zero RHS has the zero solution; a non-finite ||b|| never counts as converged
  *out = bnorm > 0.0 ? kw.h_dctl[kTrue] / bnorm : (bnorm == 0.0 ? 0.0 : NAN);
  return UFEM_OK;
}

// Right-preconditioned restarted GMRES(m) with CGS2 orthogonalisation:
// A M^-1 u = b, x = x0 + M^-1 V y.  One host synchronisation per restart cycle.
template <typename VT, typename MT, typename BT>
int gmres(ufem_ns_handle* h, const MT* vals, const BT* b, VT* x, VT* V, VT* w, VT* z, VT* t, VT* r, VT* dinv,
          int pkind, double tol, int maxit, int m, cudaStream_t s, SolveResult& res) {
  KrylovWork& kw = *h->kw;
  const int64_t n = h->nrows;
  const int nblk = kw.nblk;
  const unsigned g1 = unsigned(nblk);
  int rc;
  if ((rc = setup_precond<VT, MT>(h, pkind, vals, dinv, s))) return rc;
  res = SolveResult();
  bool first = true;
  double bnorm = 0.0;
  while (true) {
    if ((rc = spmv<VT, MT>(h, vals, x, w, nullptr, s))) return rc;
    residual_kernel<VT, BT><<<g1, kRedThreads, 0, s>>>(n, b, w, r, kw.part, first ? kw.part + nblk : nullptr);
    restart_setup_kernel<<<1, 1, 0, s>>>(nblk, m, kw.part, kw.part + nblk, first ? 1 : 0, kw.g, kw.dctl, kw.ictl, tol);
    scale_kernel<VT><<<g1, kRedThreads, 0, s>>>(n, r, V, kw.dctl, kBeta, kw.ictl);
    UFEM_CUDA_TRY(cudaGetLastError());
    first = false;
    const int budget = std::max(1, std::min(m, maxit - res.iters));
    for (int j = 0; j < budget; ++j) {
      const VT* vj = V + int64_t(j) * n;
      if ((rc = precond<VT>(h, pkind, dinv, vj, z, kw.ictl, s))) return rc;
      if ((rc = spmv<VT, MT>(h, vals, z, w, kw.ictl, s))) return rc;
      for (int pass = 0; pass < 2; ++pass) {  // classical Gram-Schmidt, twice
        double* hb = kw.hbuf + pass * (kw.m + 2);
        dot_partials_kernel<VT><<<dim3(g1, unsigned(j + 1)), kRedThreads, 0, s>>>(n, V, n, w, kw.part, kw.ictl);
        reduce_partials_kernel<<<unsigned(j + 1), 256, 0, s>>>(nblk, kw.part, hb, kw.ictl);
        multi_axpy_kernel<VT><<<g1, kRedThreads, 0, s>>>(n, j + 1, V, n, hb, w, pass == 1 ? kw.part : nullptr,
                                                          kw.ictl);
      }
      givens_kernel<<<1, 1, 0, s>>>(j, kw.m, kw.hbuf, kw.part, nblk, kw.H, kw.cs, kw.sn, kw.g, kw.dctl, kw.ictl, tol,
                                    j + 1 == budget ? 1 : 0);
      scale_kernel<VT><<<g1, kRedThreads, 0, s>>>(n, w, V + int64_t(j + 1) * n, kw.dctl, kHnext, kw.ictl);
      UFEM_CUDA_TRY(cudaGetLastError());
    }
    backsolve_kernel<<<1, 1, 0, s>>>(kw.m, kw.H, kw.g, kw.y, kw.ictl);
    combine_kernel<VT><<<g1, kRedThreads, 0, s>>>(n, V, n, kw.y, kw.ictl, t);
    if ((rc = precond<VT>(h, pkind, dinv, t, z, nullptr, s))) return rc;
    UFEM_CUDA_TRY(cudaMemcpyAsync(kw.h_ictl, kw.ictl, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
    UFEM_CUDA_TRY(cudaMemcpyAsync(kw.h_dctl, kw.dctl, 16 * sizeof(double), cudaMemcpyDeviceToHost, s));
    UFEM_CUDA_TRY(cudaStreamSynchronize(s));
    const int jc = kw.h_ictl[1];
    bnorm = kw.h_dctl[kBnorm];
    if (kw.h_ictl[2] == 3) {
      res.status = 3;
      res.relres = NAN;
      return UFEM_OK;
    }
    if (bnorm == 0.0) {
      fill_kernel<VT><<<g1, kRedThreads, 0, s>>>(n, VT(0), x);
      UFEM_CUDA_TRY(cudaGetLastError());
      res.converged = true;
      return UFEM_OK;
    }
    if (jc > 0) {
      axpy_kernel<VT><<<g1, kRedThreads, 0, s>>>(n, 1.0, z, x);
      UFEM_CUDA_TRY(cudaGetLastError());
    }
    res.iters += jc;
    if (jc == 0) {  // converged at the restart residual (exact)
      res.converged = kw.h_dctl[kBeta] <= tol * bnorm;
      res.relres = kw.h_dctl[kBeta] / bnorm;
      res.status = res.converged ? 0 : 2;
      return UFEM_OK;
    }
    if (res.iters >= maxit) {
      double rr;
      if ((rc = true_residual<VT, MT, BT>(h, kw, vals, b, x, w, r, bnorm, s, &rr))) return rc;
      res.relres = rr;
      res.converged = rr <= tol;
      res.status = res.converged ? 0 : 1;
      return UFEM_OK;
    }
  }
}

// Right-preconditioned BiCGStab with device-side scalars; the host checks the
// done flag between blocks of iterations of growing length.
template <typename VT, typename MT, typename BT>
int bicgstab(ufem_ns_handle* h, KrylovWork& kw, const MT* vals, const BT* b, VT* x, VT* r, VT* rh, VT* p, VT* v,
             VT* sv, VT* tv, VT* ph, VT* sh, VT* dinv, int pkind, double tol, int maxit, cudaStream_t st,
             SolveResult& res) {
  const int64_t n = h->nrows;
  const int nblk = kw.nblk;
  const unsigned g1 = unsigned(nblk);
  int rc;
  if ((rc = setup_precond<VT, MT>(h, pkind, vals, dinv, st))) return rc;
  res = SolveResult();
  if ((rc = spmv<VT, MT>(h, vals, x, v, nullptr, st))) return rc;
  residual_kernel<VT, BT><<<g1, kRedThreads, 0, st>>>(n, b, v, r, kw.part, kw.part + nblk);
  finalize_norm_kernel<<<1, kRedThreads, 0, st>>>(nblk, kw.part, kw.dctl, kBeta, 1);
  finalize_norm_kernel<<<1, kRedThreads, 0, st>>>(nblk, kw.part + nblk, kw.dctl, kBnorm, 1);
  UFEM_CUDA_TRY(cudaMemcpyAsync(rh, r, n * sizeof(VT), cudaMemcpyDeviceToDevice, st));
  fill_kernel<VT><<<g1, kRedThreads, 0, st>>>(n, VT(0), p);
  fill_kernel<VT><<<g1, kRedThreads, 0, st>>>(n, VT(0), v);
  bicg_init_kernel<<<1, 1, 0, st>>>(kw.dctl, kw.ictl, tol);
  UFEM_CUDA_TRY(cudaGetLastError());
  const double alpha_max = std::is_same<VT, float>::value ? 1e20 : 1e150;
  // the reductions with their scalar updates folded in (three launches fewer an
  // iteration), where the workspace has the fold counter (not the
  // allocation-free solve's)
  const bool fused = kw.cg_counter != nullptr;
  auto iteration = [&](cudaStream_t s2) -> int {
    int irc;
    const int pk = pkind == 4 ? 1 : pkind;  // the two-level form: point Jacobi plus the coarse correction
    bicg_p_kernel<VT><<<g1, kRedThreads, 0, s2>>>(n, pk, dinv, r, v, p, ph, kw.dctl, kw.ictl);
    if (pkind == 2 && (irc = precond<VT>(h, pkind, dinv, p, ph, kw.ictl, s2))) return irc;
    if (pkind == 4 && (irc = coarse_correct<VT>(h, p, ph, kw.ictl, s2))) return irc;
    if ((irc = spmv<VT, MT>(h, vals, ph, v, kw.ictl, s2))) return irc;
    if (fused) {
      bicg_vdot_fold_kernel<VT><<<g1, kRedThreads, 0, s2>>>(n, rh, v, kw.part, kw.cg_counter, kw.dctl, kw.ictl,
                                                           alpha_max);
    } else {
      dot_partials_kernel<VT><<<dim3(g1, 1), kRedThreads, 0, s2>>>(n, rh, n, v, kw.part, kw.ictl);
      bicg_alpha_kernel<<<1, 256, 0, s2>>>(nblk, kw.part, kw.dctl, kw.ictl, alpha_max);
    }
    bicg_s_kernel<VT><<<g1, kRedThreads, 0, s2>>>(n, pk, dinv, r, v, sv, sh, kw.dctl, kw.ictl);
    if (pkind == 2 && (irc = precond<VT>(h, pkind, dinv, sv, sh, kw.ictl, s2))) return irc;
    if (pkind == 4 && (irc = coarse_correct<VT>(h, sv, sh, kw.ictl, s2))) return irc;
    if ((irc = spmv<VT, MT>(h, vals, sh, tv, kw.ictl, s2))) return irc;
    if (fused) {
      bicg_ts_fold_kernel<VT><<<g1, kRedThreads, 0, s2>>>(n, tv, sv, kw.part, kw.cg_counter, kw.dctl, kw.ictl);
      bicg_xr_fold_kernel<VT><<<g1, kRedThreads, 0, s2>>>(n, ph, sh, sv, tv, rh, x, r, kw.dctl, kw.ictl, kw.part,
                                                         kw.cg_counter, tol, maxit);
    } else {
      dot2_partials_kernel<VT><<<g1, kRedThreads, 0, s2>>>(n, tv, sv, kw.part, kw.ictl);
      bicg_omega_kernel<<<1, 256, 0, s2>>>(nblk, kw.part, kw.dctl, kw.ictl);
      bicg_xr_kernel<VT><<<g1, kRedThreads, 0, s2>>>(n, ph, sh, sv, tv, rh, x, r, kw.dctl, kw.ictl, kw.part);
      bicg_end_kernel<<<1, 256, 0, s2>>>(nblk, kw.part, kw.dctl, kw.ictl, tol, maxit);
    }
    UFEM_CUDA_TRY(cudaGetLastError());
    return UFEM_OK;
  };
  // Blocks of 8 iterations, captured once per operand set in a CUDA graph and
  // replayed (the same launches in the same order: the same arithmetic).
  constexpr int kBlock = 8;
  KrylovWork::CGGraph* gr = nullptr;
  if (kw.use_graph) {
    gr = &kw.bicg_graph[std::is_same<MT, float>::value ? 1 : 0];
    const void* key[16] = {vals, b, x, r, rh, p, v, sv, tv, ph, sh, dinv, h->d_start,
                           reinterpret_cast<const void*>(intptr_t(pkind == 4 ? kw.coarse_version : 0))};
    const bool cached = gr->exec && gr->pkind == pkind && gr->tol == tol && gr->maxit == maxit &&
                        std::equal(key, key + 16, gr->key);
    if (!cached) {
      DeviceLock lk(device_mutex());  // no implicit device synchronisation from other threads during capture
      if (gr->exec) {
        cudaGraphExecDestroy(gr->exec);
        gr->exec = nullptr;
      }
      if (!kw.capture_stream) UFEM_CUDA_TRY(cudaStreamCreateWithFlags(&kw.capture_stream, cudaStreamNonBlocking));
      cudaGraph_t g = nullptr;
      UFEM_CUDA_TRY(cudaStreamBeginCapture(kw.capture_stream, cudaStreamCaptureModeThreadLocal));
      int crc = UFEM_OK;
      for (int k = 0; k < kBlock && crc == UFEM_OK; ++k) crc = iteration(kw.capture_stream);
      const cudaError_t ce = cudaStreamEndCapture(kw.capture_stream, &g);
      if (crc) {
        if (g) cudaGraphDestroy(g);
        return crc;
      }
      if (ce != cudaSuccess) return set_error(UFEM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
      const cudaError_t ie = cudaGraphInstantiate(&gr->exec, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess)
        return set_error(UFEM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
      gr->pkind = pkind;
      gr->tol = tol;
      gr->maxit = maxit;
      std::copy(key, key + 16, gr->key);
    }
  }
  // The host reads the done flag first after the previous solve's iteration
  // count (rounded down to a block of 8; 8 for the handle's first solve), then
  // after 8, 16, 32 and at most 64 more iterations: few synchronisations on
  // long solves, little overshoot on short ones or ones like the last
  // (iterations after convergence return at once on the device flag, so the
  // cadence changes no result).
  int& expect = kw.bicg_expect[std::is_same<MT, float>::value ? 1 : 0];
  int check = std::max(kBlock, expect / kBlock * kBlock);
  for (int it = 0, next = kBlock; it < maxit; it += check, check = next, next = std::min(2 * next, 64)) {
    for (int k = 0; k < check; k += kBlock) {
      if (gr) {
        UFEM_CUDA_TRY(cudaGraphLaunch(gr->exec, st));
      } else {
        for (int j = 0; j < kBlock; ++j)
          if ((rc = iteration(st))) return rc;
      }
    }
    UFEM_CUDA_TRY(cudaMemcpyAsync(kw.h_ictl, kw.ictl, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
    UFEM_CUDA_TRY(cudaStreamSynchronize(st));
    if (kw.h_ictl[0]) break;
  }
  UFEM_CUDA_TRY(cudaMemcpyAsync(kw.h_ictl, kw.ictl, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
  UFEM_CUDA_TRY(cudaMemcpyAsync(kw.h_dctl, kw.dctl, 16 * sizeof(double), cudaMemcpyDeviceToHost, st));
  UFEM_CUDA_TRY(cudaStreamSynchronize(st));
  res.iters = kw.h_ictl[3];
  res.status = kw.h_ictl[2];
  expect = res.iters;
  const double bnorm = kw.h_dctl[kBnorm];
  if (bnorm == 0.0) {
    fill_kernel<VT><<<g1, kRedThreads, 0, st>>>(n, VT(0), x);
    UFEM_CUDA_TRY(cudaGetLastError());
    res.converged = true;
    res.status = 0;
    return UFEM_OK;
  }
  double rr;
  if ((rc = true_residual<VT, MT, BT>(h, kw, vals, b, x, v, r, bnorm, st, &rr))) return rc;
  res.relres = rr;
  res.converged = rr <= tol;
  if (res.converged) res.status = 0;
  else if (res.status == 0) res.status = 1;
  return UFEM_OK;
}

// One CG iteration (five launches; a sixth and seventh with block Jacobi).
template <typename VT, typename MT>
int cg_iteration(ufem_ns_handle* h, KrylovWork& kw, const MT* vals, VT* x, VT* r, VT* z, VT* p, VT* q, VT* dinv,
                 int pkind, double tol, int maxit, cudaStream_t st) {
  const int64_t n = h->nrows;
  const int nblk = kw.nblk;
  const unsigned g1 = unsigned(nblk);
  int rc;
  if (pkind == 3) {
    const unsigned gc = unsigned(kw.cg_nblk);
    const unsigned gw = unsigned(kw.nc);  // one block per aggregate / coarse row
    cg_p_kernel<VT><<<gc, kRedThreads, 0, st>>>(n, z, p, kw.dctl, kw.ictl);
    if ((rc = spmv<VT, MT>(h, vals, p, q, kw.ictl, st))) return rc;
    cg_pq_fold_kernel<VT><<<gc, kRedThreads, 0, st>>>(n, p, q, kw.part, kw.cg_counter, kw.dctl, kw.ictl);
    cg_xr_plain_kernel<VT><<<gc, kRedThreads, 0, st>>>(n, p, q, x, r, kw.part, kw.dctl, kw.ictl);
    restrict_kernel<VT><<<gw, kCoarseThreads, 0, st>>>(kw.nc, kw.agg_ptr, kw.agg_rows, r, kw.cvec, kw.ictl);
    coarse_kernel<<<gw, kCoarseThreads, 0, st>>>(kw.nc, kw.ainv, kw.cvec, kw.yvec, kw.ictl);
    cg_prolong_fold_kernel<VT><<<gc, kRedThreads, 0, st>>>(n, dinv, kw.agg, kw.yvec, r, z, kw.part, kw.cg_counter,
                                                          kw.dctl, kw.ictl, tol, maxit);
    UFEM_CUDA_TRY(cudaGetLastError());
    return UFEM_OK;
  }
  if (pkind != 2) {
    const unsigned gc = unsigned(kw.cg_nblk);
    cg_p_kernel<VT><<<gc, kRedThreads, 0, st>>>(n, z, p, kw.dctl, kw.ictl);
    if ((rc = spmv<VT, MT>(h, vals, p, q, kw.ictl, st))) return rc;
    cg_pq_fold_kernel<VT><<<gc, kRedThreads, 0, st>>>(n, p, q, kw.part, kw.cg_counter, kw.dctl, kw.ictl);
    cg_xr_fold_kernel<VT><<<gc, kRedThreads, 0, st>>>(n, pkind, dinv, p, q, x, r, z, kw.part, kw.cg_counter,
                                                     kw.dctl, kw.ictl, tol, maxit);
    UFEM_CUDA_TRY(cudaGetLastError());
    return UFEM_OK;
  }
  cg_p_kernel<VT><<<g1, kRedThreads, 0, st>>>(n, z, p, kw.dctl, kw.ictl);
  if ((rc = spmv<VT, MT>(h, vals, p, q, kw.ictl, st))) return rc;
  dot_partials_kernel<VT><<<dim3(g1, 1), kRedThreads, 0, st>>>(n, p, n, q, kw.part, kw.ictl);
  cg_alpha_kernel<<<1, 256, 0, st>>>(nblk, kw.part, kw.dctl, kw.ictl);
  cg_xr_kernel<VT><<<g1, kRedThreads, 0, st>>>(n, pkind, dinv, p, q, x, r, z, kw.dctl, kw.ictl, kw.part);
  if (pkind == 2) {
    if ((rc = precond<VT>(h, pkind, dinv, r, z, kw.ictl, st))) return rc;
    dot_partials_kernel<VT><<<dim3(g1, 1), kRedThreads, 0, st>>>(n, r, n, z, kw.part + nblk, kw.ictl);
  }
  cg_end_kernel<<<1, 256, 0, st>>>(nblk, kw.part, kw.dctl, kw.ictl, tol, maxit);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

// Preconditioned conjugate gradients with device-side scalars (the Belos
// "Block CG" of the reference's semi-implicit velocity and pressure solves,
// block size 1).  The iterations are small, latency-bound launches on
// systems of a few hundred thousand rows, so a block of 8 is captured once in
// a CUDA graph (per operand set) and replayed between host checks of the done
// flag: first as many blocks as the previous solve needed, then 1, 2, 4 and
// then 8; iterations after convergence return at once.
template <typename VT, typename MT, typename BT>
int cg(ufem_ns_handle* h, KrylovWork& kw, const MT* vals, const BT* b, VT* x, VT* r, VT* z, VT* p, VT* q, VT* dinv,
       int pkind, double tol, int maxit, cudaStream_t st, SolveResult& res) {
  constexpr int kCGBlock = 8;
  const int64_t n = h->nrows;
  const int nblk = kw.nblk;
  const unsigned g1 = unsigned(nblk);
  int rc;
  if ((rc = setup_precond<VT, MT>(h, pkind, vals, dinv, st))) return rc;
  res = SolveResult();
  if ((rc = spmv<VT, MT>(h, vals, x, q, nullptr, st))) return rc;
  residual_kernel<VT, BT><<<g1, kRedThreads, 0, st>>>(n, b, q, r, kw.part, kw.part + nblk);
  finalize_norm_kernel<<<1, kRedThreads, 0, st>>>(nblk, kw.part, kw.dctl, kBeta, 1);
  finalize_norm_kernel<<<1, kRedThreads, 0, st>>>(nblk, kw.part + nblk, kw.dctl, kBnorm, 1);
  if (pkind == 3) {
    const unsigned gw = unsigned(kw.nc);  // one block per aggregate / coarse row
    restrict_kernel<VT><<<gw, kCoarseThreads, 0, st>>>(kw.nc, kw.agg_ptr, kw.agg_rows, r, kw.cvec, nullptr);
    coarse_kernel<<<gw, kCoarseThreads, 0, st>>>(kw.nc, kw.ainv, kw.cvec, kw.yvec, nullptr);
    prolong_kernel<VT><<<g1, kRedThreads, 0, st>>>(n, dinv, kw.agg, kw.yvec, r, z);
    UFEM_CUDA_TRY(cudaGetLastError());
  } else if ((rc = precond<VT>(h, pkind, dinv, r, z, nullptr, st))) {
    return rc;
  }
  dot_partials_kernel<VT><<<dim3(g1, 1), kRedThreads, 0, st>>>(n, r, n, z, kw.part, nullptr);
  cg_init_kernel<<<1, 1, 0, st>>>(nblk, kw.part, kw.dctl, kw.ictl, tol);
  fill_kernel<VT><<<g1, kRedThreads, 0, st>>>(n, VT(0), p);
  UFEM_CUDA_TRY(cudaGetLastError());
  KrylovWork::CGGraph& gr = kw.cg_graph[std::is_same<MT, float>::value ? 1 : 0];
  const void* key[16] = {vals, b, x, r, z, p, q, dinv, h->d_start,
                         reinterpret_cast<const void*>(intptr_t(pkind == 3 ? kw.coarse_version : 0))};
  const bool cached = gr.exec && gr.pkind == pkind && gr.tol == tol && gr.maxit == maxit &&
                      std::equal(key, key + 16, gr.key);
  if (!cached) {
    DeviceLock lk(device_mutex());  // no implicit device synchronisation from other threads during capture
    if (gr.exec) {
      cudaGraphExecDestroy(gr.exec);
      gr.exec = nullptr;
    }
    if (!kw.capture_stream) UFEM_CUDA_TRY(cudaStreamCreateWithFlags(&kw.capture_stream, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    UFEM_CUDA_TRY(cudaStreamBeginCapture(kw.capture_stream, cudaStreamCaptureModeThreadLocal));
    int crc = UFEM_OK;
    for (int k = 0; k < kCGBlock && crc == UFEM_OK; ++k)
      crc = cg_iteration<VT, MT>(h, kw, vals, x, r, z, p, q, dinv, pkind, tol, maxit, kw.capture_stream);
    const cudaError_t ce = cudaStreamEndCapture(kw.capture_stream, &g);
    if (crc) {
      if (g) cudaGraphDestroy(g);
      return crc;
    }
    if (ce != cudaSuccess) return set_error(UFEM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    const cudaError_t ie = cudaGraphInstantiate(&gr.exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return set_error(UFEM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    gr.pkind = pkind;
    gr.tol = tol;
    gr.maxit = maxit;
    std::copy(key, key + 16, gr.key);
  }
  // first look at the done flag after the previous solve's iteration count
  // (rounded down to a block), then after 1, 2, 4 and at most 8 more blocks
  int& expect = kw.cg_expect[std::is_same<MT, float>::value ? 1 : 0];
  int reps = std::max(1, expect / kCGBlock);
  for (int it = 0, next = 1; it < maxit; it += reps * kCGBlock, reps = next, next = std::min(2 * next, 8)) {
    for (int k = 0; k < reps; ++k) UFEM_CUDA_TRY(cudaGraphLaunch(gr.exec, st));
    UFEM_CUDA_TRY(cudaMemcpyAsync(kw.h_ictl, kw.ictl, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
    UFEM_CUDA_TRY(cudaStreamSynchronize(st));
    if (kw.h_ictl[0]) break;
  }
  UFEM_CUDA_TRY(cudaMemcpyAsync(kw.h_ictl, kw.ictl, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
  UFEM_CUDA_TRY(cudaMemcpyAsync(kw.h_dctl, kw.dctl, 16 * sizeof(double), cudaMemcpyDeviceToHost, st));
  UFEM_CUDA_TRY(cudaStreamSynchronize(st));
  res.iters = kw.h_ictl[3];
  res.status = kw.h_ictl[2];
  expect = res.iters;
  const double bnorm = kw.h_dctl[kBnorm];
  if (bnorm == 0.0) {
    fill_kernel<VT><<<g1, kRedThreads, 0, st>>>(n, VT(0), x);
    UFEM_CUDA_TRY(cudaGetLastError());
    res.converged = true;
    res.status = 0;
    return UFEM_OK;
  }
  double rr;
  if ((rc = true_residual<VT, MT, BT>(h, kw, vals, b, x, q, r, bnorm, st, &rr))) return rc;
  res.relres = rr;
  res.converged = rr <= tol;
  if (res.converged) res.status = 0;
  else if (res.status == 0) res.status = 1;
  return UFEM_OK;
}

// dst32 = src64 * (1 / dctl[idx])
__global__ void to32_scaled_kernel(int64_t n, const double* __restrict__ src, float* __restrict__ dst,
                                   const double* __restrict__ dctl, int idx) {
  const double inv = dctl[idx] > 0.0 ? 1.0 / dctl[idx] : 0.0;
  GRID_STRIDE(i, n) dst[i] = float(src[i] * inv);
}

__global__ void vals_to32_kernel(int64_t n, const double* __restrict__ v, float* __restrict__ v32) {
  GRID_STRIDE(i, n) v32[i] = float(v[i]);
}

}  // namespace

namespace {

// Aggregates of the coupled two-level form: k^dim boxes of the mesh's bounding
// box (k chosen for at least 64 nodes a box, at most max_side_3d boxes a side
// in 3D and max_side_2d in 2D, so the coarse matrix stays small enough to invert
// on the host at every solve); the coarse space holds the pressure rows of the
// nodes whose pressure is neither a Dirichlet dof nor a periodic slave.  Built
// once per condition list: the aggregate of each row, the rows of each aggregate, and
// the pressure-pressure CSR positions sorted by (row aggregate, column
// aggregate, position) with their segments.
int coupled_coarse_build(ufem_ns_handle* h, int max_side_2d, int max_side_3d) {
  KrylovWork& kw = *h->kw;
  if (kw.cp_thread.joinable()) kw.cp_thread.join();
  kw.cp_pending = false;
  kw.cp_lag_ready = false;
  if (kw.h_ac2) {
    DeviceLock lk(device_mutex());
    cudaFreeHost(kw.h_ac2);
    kw.h_ac2 = nullptr;
  }
  kw.cp_caps = max_side_2d * 1000 + max_side_3d;
  dfree(kw.agg); dfree(kw.agg_ptr); dfree(kw.agg_rows); dfree(kw.ainv); dfree(kw.cvec); dfree(kw.yvec);
  dfree(kw.cp_pos); dfree(kw.cp_seg); dfree(kw.cp_dst); dfree(kw.acd);
  if (kw.h_ac) {
    DeviceLock lk(device_mutex());
    cudaFreeHost(kw.h_ac);
    kw.h_ac = nullptr;
  }
  kw.nc = 0;
  kw.cp_nseg = 0;
  kw.cp_bc_version = h->bc_list_version;
  ++kw.coarse_version;
  const int dim = h->dim, neq = h->neq;
  const int64_t N = h->N;
  if (int64_t(h->coords_h.size()) != N * dim) return UFEM_OK;  // no coordinates: point Jacobi
  std::vector<char> in(size_t(N), 1);
  for (const auto& bc : h->bcs)
    if (bc.comp == dim) in[bc.node] = 0;
  if (!h->p2m_h.empty())
    for (int64_t i = 0; i < N; ++i)
      if (h->p2m_h[size_t(i)] != uint32_t(i)) in[size_t(i)] = 0;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t i = 0; i < N; ++i)
    for (int d = 0; d < dim; ++d) {
      lo[d] = std::min(lo[d], h->coords_h[size_t(i * dim + d)]);
      hi[d] = std::max(hi[d], h->coords_h[size_t(i * dim + d)]);
    }
  int k = int(std::floor(std::pow(double(N) / 64.0, 1.0 / dim)));
  k = std::max(1, std::min(k, dim == 3 ? max_side_3d : max_side_2d));
  std::vector<int32_t> box(size_t(N), -1), id(size_t(std::pow(k, dim)) + 1, -1);
  int nc = 0;
  for (int64_t i = 0; i < N; ++i) {
    if (!in[size_t(i)]) continue;
    int b = 0, mul = 1;
    for (int d = 0; d < dim; ++d) {
      const double span = hi[d] > lo[d] ? hi[d] - lo[d] : 1.0;
      const int c = std::min(k - 1, std::max(0, int((h->coords_h[size_t(i * dim + d)] - lo[d]) / span * k)));
      b += c * mul;
      mul *= k;
    }
    if (id[size_t(b)] < 0) id[size_t(b)] = nc++;
    box[size_t(i)] = id[size_t(b)];
  }
  if (nc == 0) return UFEM_OK;
  std::vector<int32_t> agg(size_t(h->nrows), -1), ptr(size_t(nc) + 1, 0), rows;
  for (int64_t i = 0; i < N; ++i)
    if (box[size_t(i)] >= 0) {
      agg[size_t(i * neq + dim)] = box[size_t(i)];
      ++ptr[size_t(box[size_t(i)]) + 1];
    }
  for (int a = 0; a < nc; ++a) ptr[size_t(a) + 1] += ptr[size_t(a)];
  rows.resize(size_t(ptr[size_t(nc)]));
  {
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int64_t i = 0; i < N; ++i)  // ascending rows within each aggregate
      if (box[size_t(i)] >= 0) rows[size_t(fill[size_t(box[size_t(i)])]++)] = int32_t(i * neq + dim);
  }
  std::vector<int64_t> pos_sorted, starts;
  // counting sort by (row aggregate, column aggregate): the positions are
  // generated in ascending order (nodes and slots ascending), so each key's
  // positions stay ascending
  const int64_t nkey = int64_t(nc) * nc;
  std::vector<int64_t> cnt(size_t(nkey) + 1, 0);
  for (int pass = 0; pass < 2; ++pass) {
    for (int64_t i = 0; i < N; ++i) {
      if (box[size_t(i)] < 0) continue;
      const int64_t s0 = h->start_h[size_t(i)], S = h->start_h[size_t(i) + 1] - s0;
      const int64_t rowkey = int64_t(box[size_t(i)]) * nc;
      for (int64_t q = 0; q < S; ++q) {
        const int32_t j = h->adj_h[size_t(s0 + q)];
        if (box[size_t(j)] < 0) continue;
        const int64_t key = rowkey + box[size_t(j)];
        if (pass == 0) ++cnt[size_t(key) + 1];
        else pos_sorted[size_t(cnt[size_t(key)]++)] = int64_t(neq) * neq * s0 + (int64_t(dim) * S + q) * neq + dim;
      }
    }
    if (pass == 0) {
      for (int64_t k = 0; k < nkey; ++k) cnt[size_t(k) + 1] += cnt[size_t(k)];
      pos_sorted.resize(size_t(cnt[size_t(nkey)]));
      starts.assign(cnt.begin(), cnt.end());
    }
  }
  std::vector<int64_t>& pos = pos_sorted;
  std::vector<int32_t> seg, dst;
  for (int64_t k = 0; k < nkey; ++k)
    if (starts[size_t(k) + 1] > starts[size_t(k)]) {
      seg.push_back(int32_t(starts[size_t(k)]));
      dst.push_back(int32_t(k));
    }
  seg.push_back(int32_t(pos.size()));
  int rc;
  if ((rc = dalloc(&kw.agg, agg.size())) || (rc = dalloc(&kw.agg_ptr, ptr.size())) ||
      (rc = dalloc(&kw.agg_rows, std::max<size_t>(rows.size(), 1))) || (rc = dalloc(&kw.ainv, size_t(nc) * nc)) ||
      (rc = dalloc(&kw.cvec, size_t(nc))) || (rc = dalloc(&kw.yvec, size_t(nc))) ||
      (rc = dalloc(&kw.cp_pos, std::max<size_t>(pos.size(), 1))) || (rc = dalloc(&kw.cp_seg, seg.size())) ||
      (rc = dalloc(&kw.cp_dst, std::max<size_t>(dst.size(), 1))) || (rc = dalloc(&kw.acd, size_t(nc) * nc)))
    return rc;
  {
    DeviceLock lk(device_mutex());
    UFEM_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&kw.h_ac), size_t(nc) * nc * sizeof(double)));
  }
  UFEM_CUDA_TRY(cudaMemcpy(kw.agg, agg.data(), agg.size() * 4, cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemcpy(kw.agg_ptr, ptr.data(), ptr.size() * 4, cudaMemcpyHostToDevice));
  if (!rows.empty()) UFEM_CUDA_TRY(cudaMemcpy(kw.agg_rows, rows.data(), rows.size() * 4, cudaMemcpyHostToDevice));
  if (!pos.empty()) UFEM_CUDA_TRY(cudaMemcpy(kw.cp_pos, pos.data(), pos.size() * 8, cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemcpy(kw.cp_seg, seg.data(), seg.size() * 4, cudaMemcpyHostToDevice));
  if (!dst.empty()) UFEM_CUDA_TRY(cudaMemcpy(kw.cp_dst, dst.data(), dst.size() * 4, cudaMemcpyHostToDevice));
  kw.cp_nseg = int(dst.size());
  kw.nc = nc;
  return UFEM_OK;
}

// The coarse matrix of the current system (FP64 values, after the Dirichlet
// pass), its inverse on the host, uploaded for the solve; cp_spd false (point
// Jacobi for this solve) when it is not positive definite.
int coupled_coarse_refresh(ufem_ns_handle* h, cudaStream_t s, int max_side_2d = kCoarseSide2D,
                           int max_side_3d = kCoarseSide3D,
                           bool* rebuilt = nullptr, bool lag = false) {
  KrylovWork& kw = *h->kw;
  int rc;
  const bool stale = kw.cp_bc_version != h->bc_list_version || kw.cp_caps != max_side_2d * 1000 + max_side_3d;
  if (rebuilt) *rebuilt = stale;
  if (stale && (rc = coupled_coarse_build(h, max_side_2d, max_side_3d))) return rc;  // (joins the thread)
  const int nc = kw.nc;
  if (nc == 0) {
    kw.cp_spd = false;
    return UFEM_OK;
  }
  const size_t bytes = size_t(nc) * nc * sizeof(double);
  // lagged: an inverse of the previous solve's coarse matrix exists (on the
  // device, or on its way from the host thread); this solve uses it
  const bool lagged = lag && !stale && (kw.cp_pending || kw.cp_lag_ready);
  if (lagged && kw.cp_pending) {
    kw.cp_thread.join();
    kw.cp_pending = false;
    kw.cp_spd = kw.cp_next_spd;
    if (kw.cp_spd) UFEM_CUDA_TRY(cudaMemcpyAsync(kw.ainv, kw.h_ac2, bytes, cudaMemcpyHostToDevice, s));
  }
  UFEM_CUDA_TRY(cudaMemsetAsync(kw.acd, 0, bytes, s));
  if (kw.cp_nseg > 0)
    coarse_matrix_kernel<<<unsigned((int64_t(kw.cp_nseg) * 32 + 255) / 256), 256, 0, s>>>(
        kw.cp_nseg, kw.cp_seg, kw.cp_dst, kw.cp_pos, h->d_vals, kw.acd);
  UFEM_CUDA_TRY(cudaGetLastError());
  UFEM_CUDA_TRY(cudaMemcpyAsync(kw.h_ac, kw.acd, bytes, cudaMemcpyDeviceToHost, s));
  if (!lagged) {  // invert this solve's own matrix before the solve starts
    UFEM_CUDA_TRY(cudaStreamSynchronize(s));
    kw.cp_spd = spd_invert(kw.h_ac, nc);
    if (kw.cp_spd) UFEM_CUDA_TRY(cudaMemcpyAsync(kw.ainv, kw.h_ac, bytes, cudaMemcpyHostToDevice, s));
    kw.cp_lag_ready = lag;  // the next lagged solve keeps this inverse
    return UFEM_OK;
  }
  // the next solve's inverse: this solve's matrix, inverted on a host thread
  // once its copy has landed, while this solve runs
  if (!kw.h_ac2) {
    DeviceLock lk(device_mutex());
    UFEM_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&kw.h_ac2), bytes));
  }
  if (!kw.cp_event) UFEM_CUDA_TRY(cudaEventCreateWithFlags(&kw.cp_event, cudaEventDisableTiming));
  UFEM_CUDA_TRY(cudaEventRecord(kw.cp_event, s));
  double* src = kw.h_ac;
  double* dst = kw.h_ac2;
  cudaEvent_t ev = kw.cp_event;
  KrylovWork* kwp = &kw;
  kw.cp_thread = std::thread([src, dst, bytes, nc, ev, kwp]() {
    const bool ok = cudaEventSynchronize(ev) == cudaSuccess;
    if (ok) std::memcpy(dst, src, bytes);
    kwp->cp_next_spd = ok && spd_invert(dst, nc);
  });
  kw.cp_pending = true;
  kw.cp_lag_ready = false;
  return UFEM_OK;
}

}  // namespace

int krylov_prepare(ufem_ns_handle* h, const ufem_krylov_opts* ko, int batched) {
  ufem_krylov_opts o = *ko;
  if (o.restart <= 0) o.restart = 30;
  int rc;
  if (!batched) {
    if ((rc = ensure_work(h, o.restart, o.mixed != 0, o.method != 0))) return rc;
  } else {
    if (!h->kw) h->kw = new KrylovWork();  // batch members keep their vectors in the batch
    if (o.mixed != 0 && (rc = dalloc(&h->d_vals32, size_t(h->nnz)))) return rc;
  }
  KrylovWork& kw = *h->kw;
  if (o.precond == 4 && h->neq > 1) {
    const int s2 = batched ? kBatchCoarseSide2D : kCoarseSide2D, s3 = batched ? kBatchCoarseSide3D : kCoarseSide3D;
    if ((kw.cp_bc_version != h->bc_list_version || kw.cp_caps != s2 * 1000 + s3) &&
        (rc = coupled_coarse_build(h, s2, s3)))
      return rc;
    if (!batched && h->conditioned) {
      // the coarse inverse of the system as it stands, which the next solve
      // takes as its lagged inverse: the first solve after this does not wait
      // for a host inversion (on a private stream; nothing else is touched)
      cudaStream_t ps = nullptr;
      UFEM_CUDA_TRY(cudaStreamCreateWithFlags(&ps, cudaStreamNonBlocking));
      rc = coupled_coarse_refresh(h, ps, s2, s3, nullptr, true);
      const cudaError_t ce = cudaStreamSynchronize(ps);
      cudaStreamDestroy(ps);
      if (rc) return rc;
      if (ce != cudaSuccess) return set_error(UFEM_ERR_CUDA, std::string("prepare: ") + cudaGetErrorString(ce));
    }
  }
  return UFEM_OK;
}

int krylov_coupled_coarse_members(ufem_ns_handle* const* hs, const int32_t* active, int n, cudaStream_t s,
                                  int max_side_2d, int max_side_3d, bool* rebuilt, CoarseView* views) {
  // (1) every active member's coarse matrix, summed on the device and copied
  // to its pinned host buffer, all on `s`
  int rc;
  for (int m = 0; m < n; ++m) {
    rebuilt[m] = false;
    if (!active[m]) continue;
    ufem_ns_handle* h = hs[m];
    if (!h->kw) h->kw = new KrylovWork();  // coarse data only: batch members keep their vectors in the batch
    KrylovWork& kw = *h->kw;
    if (kw.cp_pending) {  // a lagged inversion from solves of the handle on its own
      kw.cp_thread.join();
      kw.cp_pending = false;
    }
    const bool stale = kw.cp_bc_version != h->bc_list_version || kw.cp_caps != max_side_2d * 1000 + max_side_3d;
    rebuilt[m] = stale;
    if (stale && (rc = coupled_coarse_build(h, max_side_2d, max_side_3d))) return rc;
    if (kw.nc == 0) continue;
    const size_t bytes = size_t(kw.nc) * kw.nc * sizeof(double);
    UFEM_CUDA_TRY(cudaMemsetAsync(kw.acd, 0, bytes, s));
    if (kw.cp_nseg > 0)
      coarse_matrix_kernel<<<unsigned((int64_t(kw.cp_nseg) * 32 + 255) / 256), 256, 0, s>>>(
          kw.cp_nseg, kw.cp_seg, kw.cp_dst, kw.cp_pos, h->d_vals, kw.acd);
    UFEM_CUDA_TRY(cudaGetLastError());
    UFEM_CUDA_TRY(cudaMemcpyAsync(kw.h_ac, kw.acd, bytes, cudaMemcpyDeviceToHost, s));
  }
  // (2) one synchronisation, (3) the inversions on host threads, one member
  // per thread at a time (each inversion's arithmetic is the one-handle
  // refresh's: the same inverse, bitwise), (4) the inverses uploaded
  UFEM_CUDA_TRY(cudaStreamSynchronize(s));
  std::vector<int> todo;
  for (int m = 0; m < n; ++m)
    if (active[m] && hs[m]->kw->nc > 0) todo.push_back(m);
  std::vector<char> spd(size_t(n), 0);
  const int extra = todo.size() > 1 ? acquire_spare_threads(int(todo.size()) - 1) : 0;
  const int nt = 1 + extra;
  std::atomic<size_t> next{0};
  auto work = [&]() {
    for (size_t q = next++; q < todo.size(); q = next++) {
      const int m = todo[q];
      KrylovWork& kw = *hs[m]->kw;
      spd[size_t(m)] = spd_invert(kw.h_ac, kw.nc, 1) ? 1 : 0;
    }
  };
  {
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(work);
    work();  // the calling thread takes members too
    for (auto& x : th) x.join();
  }
  release_spare_threads(extra);
  for (int m = 0; m < n; ++m) {
    views[m] = CoarseView{};
    if (!active[m]) continue;
    KrylovWork& kw = *hs[m]->kw;
    if (kw.nc == 0) {
      kw.cp_spd = false;
    } else {
      kw.cp_spd = spd[size_t(m)] != 0;
      if (kw.cp_spd)
        UFEM_CUDA_TRY(cudaMemcpyAsync(kw.ainv, kw.h_ac, size_t(kw.nc) * kw.nc * sizeof(double),
                                      cudaMemcpyHostToDevice, s));
      kw.cp_lag_ready = false;
    }
    views[m].nc = kw.cp_spd ? kw.nc : 0;
    views[m].agg = kw.agg;
    views[m].agg_ptr = kw.agg_ptr;
    views[m].agg_rows = kw.agg_rows;
    views[m].ainv = kw.ainv;
  }
  return UFEM_OK;
}

int krylov_coupled_coarse(ufem_ns_handle* h, cudaStream_t s, int max_side_2d, int max_side_3d, bool* rebuilt,
                          CoarseView* view, bool lag) {
  if (!h->kw) h->kw = new KrylovWork();  // coarse data only: batch members keep their vectors in the batch
  int rc;
  if ((rc = coupled_coarse_refresh(h, s, max_side_2d, max_side_3d, rebuilt, lag))) return rc;
  const KrylovWork& kw = *h->kw;
  view->nc = kw.cp_spd ? kw.nc : 0;
  view->agg = kw.agg;
  view->agg_ptr = kw.agg_ptr;
  view->agg_rows = kw.agg_rows;
  view->ainv = kw.ainv;
  return UFEM_OK;
}

int krylov_solve(ufem_ns_handle* h, const ufem_krylov_opts* ko, ufem_krylov_status* st, cudaStream_t s) {
  ufem_krylov_opts o = *ko;
  if (o.restart <= 0) o.restart = 30;
  if (o.max_iters <= 0) o.max_iters = 3000;
  if (o.tol <= 0) o.tol = 1e-10;
  if (o.max_refine <= 0) o.max_refine = 20;
  if (o.inner_tol <= 0) o.inner_tol = 1e-3;
  if (o.precond < 0 || o.precond > 4) return set_error(UFEM_ERR_ARG, "precond must be 0, 1, 2, 3 or 4");
  if (o.precond == 4 && (h->neq < 2 || o.method == 2))
    return set_error(UFEM_ERR_ARG, "the coupled two-level preconditioner (4) is for BiCGStab or GMRES on the coupled system");
  if (o.precond == 3 && (o.method != 2 || h->neq != 1 || !h->kw || h->kw->nc == 0))
    return set_error(UFEM_ERR_ARG, "the two-level preconditioner needs CG on a one-equation system with aggregates set");
  if (o.method < 0 || o.method > 2)
    return set_error(UFEM_ERR_ARG, "method must be 0 (GMRES), 1 (BiCGStab) or 2 (CG)");
  if (o.mixed < 0 || o.mixed > 2) return set_error(UFEM_ERR_ARG, "mixed must be 0, 1 or 2");
  const bool mixed = o.mixed != 0;
  const bool use_cg = o.method == 2;
  const bool bicg = o.method == 1 || use_cg;  // CG uses the BiCGStab work vectors
  int rc;
  if ((rc = ensure_work(h, o.restart, mixed, bicg))) return rc;
  if (o.precond == 4) {  // coarse matrix of this system; point Jacobi when it is not positive definite
    // lagged: from the second solve on, each solve uses the previous solve's coarse
    // inverse while its own matrix is inverted on a host thread for the next one
    if ((rc = coupled_coarse_refresh(h, s, kCoarseSide2D, kCoarseSide3D, nullptr, true))) return rc;
    if (!h->kw->cp_spd) o.precond = 1;
  }
  KrylovWork& kw = *h->kw;
  const int64_t n = h->nrows;
  const unsigned g1 = unsigned(kw.nblk);
  ufem_krylov_status out{};
  if (!mixed) {
    SolveResult r;
    if (use_cg) {
      rc = cg<double, double, double>(h, kw, h->d_vals, h->d_rhs, h->d_sol, kw.r, kw.bs, kw.bp, kw.bv, kw.dinv,
                                      o.precond, o.tol, o.max_iters, s, r);
    } else if (bicg) {
      // A breakdown (rho or omega ~ 0) leaves a finite iterate: restart from it
      // while iterations remain.
      int used = 0;
      for (int restarts = 0;; ++restarts) {
        rc = bicgstab<double, double, double>(h, kw, h->d_vals, h->d_rhs, h->d_sol, kw.r, kw.brh, kw.bp, kw.bv, kw.bs,
                                              kw.bt, kw.bph, kw.bsh, kw.dinv, o.precond, o.tol, o.max_iters - used, s, r);
        if (rc) return rc;
        used += r.iters;
        // also restart a solve that stopped early because its recursive
        // residual met the tolerance while the true one had drifted above it
        if ((r.status == 2 || r.status == 1) && !r.converged && std::isfinite(r.relres) && used < o.max_iters &&
            restarts < kMaxRestarts)
          continue;
        break;
      }
      r.iters = used;
    } else {
      rc = gmres<double, double, double>(h, h->d_vals, h->d_rhs, h->d_sol, kw.V, kw.w, kw.z, kw.t, kw.r, kw.dinv,
                                         o.precond, o.tol, o.max_iters, o.restart, s, r);
    }
    if (rc) return rc;
    out.converged = r.converged;
    out.status = r.status;
    out.iterations = r.iters;
    out.refinements = 0;
    out.rel_residual = r.relres;
  } else {
    // FP64 iterative refinement around an FP32 inner Krylov solve.  The FP32
    // matrix copy is written by the assembly kernel (or converted here).
    if (!h->vals32_valid) {
      vals_to32_kernel<<<grid_for(h->nnz, 256), 256, 0, s>>>(h->nnz, h->d_vals, h->d_vals32);
      UFEM_CUDA_TRY(cudaGetLastError());
      h->vals32_valid = true;
    }
    double bnorm = -1.0;
    int total = 0;
    int status = 0;
    int ref = 0;
    double relres = 0.0;
    bool conv = false;
    for (ref = 0; ref <= o.max_refine; ++ref) {
      if (o.mixed == 2) {
        // r = b - M x of the FP64 system from the FP64 element pass (no FP64
        // matrix needed: the stored one may hold FP32 element arithmetic);
        // ||b|| is taken from the assembled RHS
        if ((rc = launch_mf_residual(h, kw.w, kw.r, s))) return rc;
        norm2_partials_kernel<<<g1, kRedThreads, 0, s>>>(n, kw.r, h->d_rhs, kw.part, kw.part + kw.nblk);
      } else {
        // r = b - A x in FP64
        if ((rc = spmv<double, double>(h, h->d_vals, h->d_sol, kw.w, nullptr, s))) return rc;
        residual_kernel<double, double><<<g1, kRedThreads, 0, s>>>(n, h->d_rhs, kw.w, kw.r, kw.part,
                                                                   kw.part + kw.nblk);
      }
      finalize_norm_kernel<<<1, kRedThreads, 0, s>>>(kw.nblk, kw.part, kw.dctl, kScale, 1);
      finalize_norm_kernel<<<1, kRedThreads, 0, s>>>(kw.nblk, kw.part + kw.nblk, kw.dctl, kR2, 1);
      UFEM_CUDA_TRY(cudaMemcpyAsync(kw.h_dctl, kw.dctl, 16 * sizeof(double), cudaMemcpyDeviceToHost, s));
      UFEM_CUDA_TRY(cudaStreamSynchronize(s));
      if (bnorm < 0) bnorm = kw.h_dctl[kR2];
      const double rn = kw.h_dctl[kScale];
      if (!std::isfinite(rn)) { status = 3; relres = NAN; break; }
      relres = bnorm > 0 ? rn / bnorm : 0.0;
      if (bnorm == 0.0) {
        fill_kernel<double><<<g1, kRedThreads, 0, s>>>(n, 0.0, h->d_sol);
        UFEM_CUDA_TRY(cudaGetLastError());
        conv = true;
        break;
      }
      if (relres <= o.tol) { conv = true; break; }
      if (ref == o.max_refine || total >= o.max_iters * (o.max_refine + 1)) { status = 1; break; }
      // inner: A32 d = r / ||r||, d0 = 0
      // keep ||r|| for the update: the inner solve reuses the scalar slots
      UFEM_CUDA_TRY(cudaMemcpyAsync(kw.dctl + 14, kw.dctl + kScale, sizeof(double), cudaMemcpyDeviceToDevice, s));
      SolveResult ir;
      // Each inner solve is short: FP32 Krylov recurrences stagnate near the
      // FP32-attainable accuracy, so a capped inner solve followed by a fresh
      // FP64 residual makes steadier progress than one long FP32 run.
      const int inner_iters = std::min(o.max_iters, kInnerIterCap);
      if (use_cg) {
        // FP32 operator, FP64 vectors and scalars (as for BiCGStab below)
        scale_kernel<double><<<g1, kRedThreads, 0, s>>>(n, kw.r, kw.t, kw.dctl, kScale, nullptr);
        fill_kernel<double><<<g1, kRedThreads, 0, s>>>(n, 0.0, kw.z);
        UFEM_CUDA_TRY(cudaGetLastError());
        rc = cg<double, float, double>(h, kw, h->d_vals32, kw.t, kw.z, kw.w, kw.bs, kw.bp, kw.bv, kw.dinv,
                                       o.precond, o.inner_tol, inner_iters, s, ir);
      } else if (bicg) {
        // FP32 operator (half the SpMV traffic), FP64 vectors and scalars: the
        // recurrences keep FP64 accuracy, only the operator is rounded, so the
        // refinement contracts by about cond(A) * 2^-24 per pass.
        scale_kernel<double><<<g1, kRedThreads, 0, s>>>(n, kw.r, kw.t, kw.dctl, kScale, nullptr);
        fill_kernel<double><<<g1, kRedThreads, 0, s>>>(n, 0.0, kw.z);
        UFEM_CUDA_TRY(cudaGetLastError());
        rc = bicgstab<double, float, double>(h, kw, h->d_vals32, kw.t, kw.z, kw.w, kw.brh, kw.bp, kw.bv, kw.bs, kw.bt,
                                             kw.bph, kw.bsh, kw.dinv, o.precond, o.inner_tol, inner_iters, s, ir);
      } else {
        to32_scaled_kernel<<<g1, kRedThreads, 0, s>>>(n, kw.r, kw.r32, kw.dctl, kScale);
        fill_kernel<float><<<g1, kRedThreads, 0, s>>>(n, 0.0f, kw.x32);
        UFEM_CUDA_TRY(cudaGetLastError());
        rc = gmres<float, float, float>(h, h->d_vals32, kw.r32, kw.x32, kw.V32, kw.w32, kw.z32, kw.t32, kw.q32,
                                        kw.dinv32, o.precond, o.inner_tol, inner_iters, o.restart, s, ir);
      }
      if (rc) return rc;
      total += ir.iters;
      // A breakdown (status 2) leaves a finite, partially converged correction:
      // apply it and let the next FP64 residual restart the inner solve.  A
      // non-finite inner iterate is never applied.
      if (ir.status == 3 || !std::isfinite(ir.relres)) { status = 3; relres = NAN; break; }
      if (bicg)
        add_scaled_kernel<double><<<g1, kRedThreads, 0, s>>>(n, kw.z, h->d_sol, kw.dctl, 14);
      else
        add_scaled_kernel<float><<<g1, kRedThreads, 0, s>>>(n, kw.x32, h->d_sol, kw.dctl, 14);
      UFEM_CUDA_TRY(cudaGetLastError());
    }
    out.converged = conv;
    out.status = conv ? 0 : (status ? status : 1);
    out.iterations = total;
    out.refinements = ref;
    out.rel_residual = relres;
  }
  if (st) *st = out;
  return UFEM_OK;
}

int ensure_vals32(ufem_ns_handle* h, cudaStream_t s) {
  if (h->d_vals32 == nullptr) {
    int rc;
    if ((rc = dalloc(&h->d_vals32, size_t(h->nnz)))) return rc;
    vals_to32_kernel<<<grid_for(h->nnz, 256), 256, 0, s>>>(h->nnz, h->d_vals, h->d_vals32);
    UFEM_CUDA_TRY(cudaGetLastError());
    h->vals32_valid = true;
  }
  return UFEM_OK;
}

namespace {

// In-place inverse of an SPD matrix through its Cholesky factor; false if a
// pivot is not positive (the coarse matrix of a system without conditions
// that fix its constant mode is singular).
bool spd_inverse(std::vector<double>& A, int n) { return spd_invert(A.data(), n); }

}  // namespace

int krylov_set_coarse(ufem_ns_handle* h, const std::vector<int32_t>& agg, int nc, cudaStream_t s) {
  if (h->neq != 1) return set_error(UFEM_ERR_ARG, "aggregates are defined for one-equation systems");
  if (int64_t(agg.size()) != h->nrows) return set_error(UFEM_ERR_ARG, "one aggregate id per row expected");
  int rc;
  if ((rc = ensure_work(h, 30, false, true))) return rc;
  KrylovWork& kw = *h->kw;
  dfree(kw.agg); dfree(kw.agg_ptr); dfree(kw.agg_rows); dfree(kw.ainv); dfree(kw.cvec); dfree(kw.yvec);
  kw.nc = 0;
  ++kw.coarse_version;
  if (nc <= 0) return UFEM_OK;
  std::vector<int32_t> ptr(size_t(nc) + 1, 0), rows;
  for (int32_t a : agg) {
    if (a >= nc) return set_error(UFEM_ERR_ARG, "aggregate id out of range");
    if (a >= 0) ++ptr[size_t(a) + 1];
  }
  for (int I = 0; I < nc; ++I) ptr[size_t(I) + 1] += ptr[size_t(I)];
  rows.resize(size_t(ptr[size_t(nc)]));
  {
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int64_t i = 0; i < h->nrows; ++i)
      if (agg[size_t(i)] >= 0) rows[size_t(fill[size_t(agg[size_t(i)])]++)] = int32_t(i);
  }
  // Galerkin coarse matrix R^T A R from the system's current values, summed in
  // row and column order on the host (deterministic), then inverted.
  std::vector<double> vals(size_t(h->nnz));
  UFEM_CUDA_TRY(cudaStreamSynchronize(s));
  UFEM_CUDA_TRY(cudaMemcpy(vals.data(), h->d_vals, size_t(h->nnz) * 8, cudaMemcpyDeviceToHost));
  std::vector<double> A(size_t(nc) * nc, 0.0);
  for (int64_t i = 0; i < h->nrows; ++i) {
    const int32_t I = agg[size_t(i)];
    if (I < 0) continue;
    for (int64_t q = h->start_h[size_t(i)]; q < h->start_h[size_t(i) + 1]; ++q) {
      const int32_t J = agg[size_t(h->adj_h[size_t(q)])];
      if (J >= 0) A[size_t(I) * nc + J] += vals[size_t(q)];
    }
  }
  if (!spd_inverse(A, nc)) return UFEM_OK;  // nc stays 0: the caller falls back to point Jacobi
  if ((rc = dalloc(&kw.agg, size_t(h->nrows))) || (rc = dalloc(&kw.agg_ptr, ptr.size())) ||
      (rc = dalloc(&kw.agg_rows, std::max<size_t>(rows.size(), 1))) || (rc = dalloc(&kw.ainv, A.size())) ||
      (rc = dalloc(&kw.cvec, size_t(nc))) || (rc = dalloc(&kw.yvec, size_t(nc))))
    return rc;
  UFEM_CUDA_TRY(cudaMemcpy(kw.agg, agg.data(), agg.size() * 4, cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemcpy(kw.agg_ptr, ptr.data(), ptr.size() * 4, cudaMemcpyHostToDevice));
  if (!rows.empty()) UFEM_CUDA_TRY(cudaMemcpy(kw.agg_rows, rows.data(), rows.size() * 4, cudaMemcpyHostToDevice));
  UFEM_CUDA_TRY(cudaMemcpy(kw.ainv, A.data(), A.size() * 8, cudaMemcpyHostToDevice));
  kw.nc = nc;
  return UFEM_OK;
}

int krylov_coarse_size(const ufem_ns_handle* h) { return h->kw ? h->kw->nc : 0; }

int krylov_fp64_residual(ufem_ns_handle* h, double* r_host, cudaStream_t s) {
  int rc;
  if ((rc = ensure_work(h, 30, false, true))) return rc;
  KrylovWork& kw = *h->kw;
  if ((rc = launch_mf_residual(h, kw.w, kw.r, s))) return rc;
  UFEM_CUDA_TRY(cudaMemcpyAsync(r_host, kw.r, size_t(h->nrows) * 8, cudaMemcpyDeviceToHost, s));
  UFEM_CUDA_TRY(cudaStreamSynchronize(s));
  return UFEM_OK;
}

int krylov_apply(ufem_ns_handle* h, const double* d_x, double* d_y, cudaStream_t s) {
  return spmv<double, double>(h, h->d_vals, d_x, d_y, nullptr, s);
}

int64_t krylov_device_bytes(const ufem_ns_handle* h) {
  if (!h->kw) return 0;
  const KrylovWork& k = *h->kw;
  const int64_t R = h->nrows;
  int64_t b = 0;
  for (const double* p : {k.w, k.z, k.t, k.r, k.dinv, k.bp, k.bv, k.bs, k.bt, k.brh, k.bph, k.bsh})
    if (p) b += R * 8;
  for (const float* p : {k.w32, k.z32, k.t32, k.r32, k.x32, k.q32, k.dinv32})
    if (p) b += R * 4;
  if (k.V) b += int64_t(k.m + 1) * R * 8;    // GMRES basis
  if (k.V32) b += int64_t(k.m + 1) * R * 4;
  if (k.agg) b += R * 4 * 2;                // aggregate of each row, members of each aggregate
  if (k.ainv) b += int64_t(k.nc) * k.nc * 8 * 2;  // coarse inverse and coarse matrix
  if (k.cp_pos) b += int64_t(k.cp_nseg) * 12 + R * 8;  // coarse-matrix segments (an upper bound)
  return b;
}

void krylov_free(ufem_ns_handle* h) {
  if (!h->kw) return;
  KrylovWork& k = *h->kw;
  dfree(k.V); dfree(k.w); dfree(k.z); dfree(k.t); dfree(k.r); dfree(k.dinv);
  dfree(k.V32); dfree(k.w32); dfree(k.z32); dfree(k.t32); dfree(k.r32); dfree(k.x32); dfree(k.q32); dfree(k.dinv32);
  dfree(k.bp); dfree(k.bv); dfree(k.bs); dfree(k.bt); dfree(k.brh); dfree(k.bph); dfree(k.bsh);
  dfree(k.part); dfree(k.hbuf); dfree(k.H); dfree(k.cs); dfree(k.sn); dfree(k.g); dfree(k.y);
  dfree(k.dctl); dfree(k.ictl); dfree(k.cg_counter);
  dfree(k.agg); dfree(k.agg_ptr); dfree(k.agg_rows); dfree(k.ainv); dfree(k.cvec); dfree(k.yvec);
  if (k.cp_thread.joinable()) k.cp_thread.join();
  dfree(k.cp_pos); dfree(k.cp_seg); dfree(k.cp_dst); dfree(k.acd);
  DeviceLock lk(device_mutex());
  if (k.h_ac) cudaFreeHost(k.h_ac);
  if (k.h_ac2) cudaFreeHost(k.h_ac2);
  if (k.cp_event) cudaEventDestroy(k.cp_event);
  for (auto& g : k.cg_graph)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  for (auto& g : k.bicg_graph)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (k.capture_stream) cudaStreamDestroy(k.capture_stream);
  if (k.h_dctl) cudaFreeHost(k.h_dctl);
  if (k.h_ictl) cudaFreeHost(k.h_ictl);
  delete h->kw;
  h->kw = nullptr;
}

// ---------------------------------------------------------------------------
// Allocation-free solve.  Its Krylov vectors, block partials and scalars live
// in one fixed array of this file instead of memory obtained from cudaMalloc.
// Layout (doubles): 9 vectors of UFEM_NOALLOC_MAX_ROWS (r, r^, p, v, s, t, p^,
// s^, inverse diagonal), 2 * kMaxPartials partials, 16 scalars, 8 for the
// integer flags.
// ---------------------------------------------------------------------------
constexpr int64_t kNoAllocRows = UFEM_NOALLOC_MAX_ROWS;
constexpr int kMaxPartials = kRedBlocksMax;  // the largest block count red_blocks gives
constexpr int64_t kNoAllocDoubles = 9 * kNoAllocRows + 2 * kMaxPartials + 16 + 8;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

namespace {
constexpr int kMaxDevices = 64;

// Device address of g_noalloc_scratch on the current device, looked up once per
// device (the host-side symbol is only a stand-in and must not reach a kernel).
// The cache is read and written under a mutex, so first calls from several host
// threads do not race.  cudaDeviceReset ends every handle of the library and the
// cached addresses with them: the library is not used after a reset.
int noalloc_scratch(double** out) {
  static std::mutex mu;
  static double* addr[kMaxDevices] = {};
  int dev = 0;
  UFEM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return set_error(UFEM_ERR_LIMIT, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    UFEM_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    addr[dev] = static_cast<double*>(p);
  }
  *out = addr[dev];
  return UFEM_OK;
}
}  // namespace

}  // namespace ufem

extern "C" int ufem_ns_solve_noalloc(ufem_ns_handle* h, const ufem_krylov_opts* kopts, ufem_krylov_status* status,
                                     void* stream) {
  using namespace ufem;
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  ufem_krylov_opts o;
  ufem_krylov_default_opts(&o);
  if (kopts) o = *kopts;
  if (o.method != 1) return set_error(UFEM_ERR_ARG, "ufem_ns_solve_noalloc supports BiCGStab (method 1) only");
  if (o.precond != 0 && o.precond != 1)
    return set_error(UFEM_ERR_ARG, "ufem_ns_solve_noalloc supports no preconditioner or point Jacobi only");
  if (o.mixed != 0) return set_error(UFEM_ERR_ARG, "ufem_ns_solve_noalloc solves in FP64 only (mixed = 0)");
  if (o.max_iters <= 0) o.max_iters = 3000;
  if (o.tol <= 0) o.tol = 1e-10;
  const int64_t n = h->nrows;
  if (n > kNoAllocRows)
    return set_error(UFEM_ERR_LIMIT, "system has " + std::to_string(n) + " rows; ufem_ns_solve_noalloc handles at most " +
                                         std::to_string(kNoAllocRows));
  double* base = nullptr;
  int rc;
  if ((rc = noalloc_scratch(&base))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double h_d[16];
  int h_i[8];
  KrylovWork kw;  // a view of the fixed scratch; owns nothing
  kw.use_graph = false;  // graph instantiation would allocate
  kw.n = n;
  kw.nblk = red_blocks(n);
  double* vec[9];
  for (int k = 0; k < 9; ++k) vec[k] = base + k * kNoAllocRows;
  kw.part = base + 9 * kNoAllocRows;
  kw.dctl = kw.part + 2 * kMaxPartials;
  kw.ictl = reinterpret_cast<int*>(kw.dctl + 16);
  kw.h_dctl = h_d;
  kw.h_ictl = h_i;
  SolveResult r;
  // the restart rule of ufem_ns_solve: after a breakdown, or when the recursive
  // residual met the tolerance while the true one had drifted above it, restart
  // from the current iterate while iterations remain
  int used = 0;
  for (int restarts = 0;; ++restarts) {
    rc = bicgstab<double, double, double>(h, kw, h->d_vals, h->d_rhs, h->d_sol, vec[0], vec[1], vec[2], vec[3], vec[4],
                                          vec[5], vec[6], vec[7], vec[8], o.precond, o.tol, o.max_iters - used, s, r);
    if (rc) return rc;
    used += r.iters;
    if ((r.status == 2 || r.status == 1) && !r.converged && std::isfinite(r.relres) && used < o.max_iters &&
        restarts < kMaxRestarts)
      continue;
    break;
  }
  r.iters = used;
  ufem_krylov_status st{};
  st.converged = r.converged;
  st.status = r.status;
  st.iterations = r.iters;
  st.rel_residual = r.relres;
  if (status) *status = st;
  if (!st.converged)
    return set_error(UFEM_ERR_SOLVE, "Krylov solve did not converge, relative residual " + std::to_string(st.rel_residual));
  return UFEM_OK;
}
