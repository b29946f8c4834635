// semi.cu -- the semi-implicit (pressure-correction) Navier-Stokes scheme of the
// UFEM plugin on P1 triangles and tetrahedra: per-element velocity matrix and
// right-hand sides, the simplified pressure Laplacian, the lumped mass, and the
// inner predictor/corrector loop of one time step.
//
// Reference (plugins/UFEM/src/UFEM/ns_semi_implicit/):
//   MatrixAssembly.hpp:52-149   VelocityAssembly (T + theta dt M)
//   MatrixAssembly.hpp:153-210  PressureRHS
//   MatrixAssembly.hpp:212-360  VelocityRHS (with the body force overload)
//   MatrixAssembly.hpp:364-404  ApplyAup
//   MatrixAssembly.hpp:409-500  the element expressions and their tau inputs
//   PressureSystem.cpp:110-140  pressure matrix theta (tau_ps + dt) grad N^T grad N
//   implementation/NavierStokesSemiImplicit.cpp:96-198   InnerLoop::execute
//   implementation/NavierStokesSemiImplicit.cpp:238-247  lumped mass reciprocal
//   implementation/NavierStokesSemiImplicit.cpp:329-375  per-step action order
//   implementation/NavierStokesSemiImplicit.cpp:400-455  initial conditions
// Triangles and tetrahedra take IntegralOrder 1 (MatrixAssembly.hpp:28-46): one
// centroid point for the operators, the order-2 rule for the mass terms.
//
// Layout.  A base handle holds the mesh, the node fields and the node graph
// with the element incidences of every row (ascending element id).  Two views
// share that graph: the velocity system (dim equations per node) and the
// pressure system (one), in the point-CSR layout of the coupled system, so the
// Krylov solvers and the symmetric-Dirichlet kernels run on them unchanged.
// The LSS vectors of the inner loop (u, p, a, the pressure increment sum, the
// lumped mass inverse) are node-major arrays of the same row numbering.
//
// Every element quantity is evaluated by the thread that owns the row (one
// thread per node, its incidences in ascending element order), so each global
// entry is a sum over elements in the order the reference adds them: no
// atomics, deterministic results.  Linked (periodic) nodes keep identity rows
// with a zero right-hand side; their values are copied from the master row
// after every solve, so element gathers may read any node's own row.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "element.cuh"
#include "internal.h"

struct ufem_nssi_handle {
  ufem_ns_handle* base = nullptr;  // mesh, fields (u, p, u_adv, history, nu, force), graph, incidences
  ufem_ns_handle* us = nullptr;    // velocity system (neq = dim): matrix T + theta dt M, rhs, delta_a
  ufem_ns_handle* ps = nullptr;    // pressure system (neq = 1): matrix, rhs, delta_p
  int nb_iterations = 2;           // NavierStokesSemiImplicit.cpp:290-293
  ufem_krylov_opts ku{}, kp{};
  double* d_uvec = nullptr;        // N x dim: u of the inner loop
  double* d_a = nullptr;           // N x dim: accumulated acceleration a
  double* d_minv = nullptr;        // N x dim: reciprocal lumped mass
  double* d_pvec = nullptr;        // N: p of the inner loop
  double* d_dpsum = nullptr;       // N: sum of the pressure increments
  bool initialized = false;        // pressure matrix and lumped mass assembled
  ufem_krylov_status last_u{}, last_p{};
  // two-level pressure preconditioner: the geometric box of every node (k^dim
  // boxes over the mesh's bounding box) and whether the coarse space matches
  // the current pressure matrix and conditions
  std::vector<int32_t> box;
  int nbox = 0;
  bool coarse_ready = false;
  bool coarse_ok = false;
};

namespace ufem {
namespace {

constexpr int kSIThreads = 128;

// Inputs every element routine reads.
struct SIArgs {
  const double* coords;    // N x 4
  const double* uadv;      // N x 4 (u_adv, nu_eff at 3)
  const double* state;     // N x 4 (u, p at dim)
  const double* force;     // N x 4 or null
  const int4* conn;        // E (triangles padded)
  const int32_t* row_inc;  // N + 1
  const int32_t* inc_elem;
  const uint32_t* inc_info;
  const int64_t* start;    // node graph, N + 1
  int64_t N;
  NSParams p;
};

template <int D>
struct SIGeom {
  Elem<D, double> el;  // relative coordinates, tau velocity, nodal nu
  double G[D][D + 1];  // shape-function gradients
  double det;
  double tps, tsu, tbu;
  double nu_c;         // nu_eff at the centroid
  double uc[D];        // tau velocity at the centroid
};

__device__ __forceinline__ void load_ids(const int4* __restrict__ conn, int64_t e, int (&ids)[4]) {
  const int4 c = __ldg(conn + e);
  ids[0] = c.x;
  ids[1] = c.y;
  ids[2] = c.z;
  ids[3] = c.w;
}

// Geometry, gradients and ComputeTauImpl::compute_coefficients (SUPG.hpp:140-219)
// evaluated on the velocity `vel` (N x 4 records: u_adv or the solution u).
template <int D>
__device__ __forceinline__ void si_element(const SIArgs& A, const KParams<double>& kp, const int (&ids)[4],
                                           const double* __restrict__ vel, SIGeom<D>& g) {
  constexpr int n = D + 1;
  double X0[4];
  ld4(A.coords + 4ll * ids[0], X0[0], X0[1], X0[2], X0[3]);
#pragma unroll
  for (int b = 0; b < n; ++b) {
    double x[4], u[4], w[4];
    ld4(A.coords + 4ll * ids[b], x[0], x[1], x[2], x[3]);
    ld4(vel + 4ll * ids[b], u[0], u[1], u[2], u[3]);
    ld4(A.uadv + 4ll * ids[b], w[0], w[1], w[2], w[3]);
#pragma unroll
    for (int k = 0; k < D; ++k) {
      g.el.Xr[b][k] = x[k] - X0[k];
      g.el.U[b][k] = u[k];
    }
    g.el.NU[b] = w[3];
  }
  double J[D][D], Ji[D][D];
#pragma unroll
  for (int r = 0; r < D; ++r)
#pragma unroll
    for (int c = 0; c < D; ++c) J[r][c] = g.el.Xr[r + 1][c];
  inverse_det<double>(J, Ji, g.det);
#pragma unroll
  for (int r = 0; r < D; ++r) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < D; ++k) s += Ji[r][k] * -1.0;
    g.G[r][0] = s;
#pragma unroll
    for (int b = 1; b <= D; ++b) g.G[r][b] = Ji[r][b - 1];
  }
  double Nc[n];
  centroid_N<D, double>(Nc);
  double nsum = 0.0, nuc = 0.0;
#pragma unroll
  for (int b = 0; b < n; ++b) {
    nsum += g.el.NU[b];
    nuc += Nc[b] * g.el.NU[b];
  }
  g.nu_c = nuc;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    double s = 0.0;
#pragma unroll
    for (int b = 0; b < n; ++b) s += Nc[b] * g.el.U[b][k];
    g.uc[k] = s;
  }
  double gm[D][D];
  metric_tensor<D, double>(g.G, 0, gm);
  compute_tau<D, double>(kp, g.el, g.uc, fabs(nsum / n), g.G, gm, g.det, g.tps, g.tsu, g.tbu);
}

template <int D>
__device__ __forceinline__ constexpr double w1_ref() { return D == 2 ? 0.5 : 1.0 / 6.0; }
template <int D>
__device__ __forceinline__ constexpr double w2_ref() { return D == 2 ? 1.0 / 6.0 : 1.0 / 24.0; }
template <int D>
__device__ __forceinline__ constexpr int n_gauss2() { return D == 2 ? 3 : 4; }

// ---------------------------------------------------------------------------
// Velocity matrix T + theta dt M (VelocityAssembly, MatrixAssembly.hpp:52-149):
// T the consistent mass (order-2 rule) on the diagonal component blocks,
// M = nu_c grad N^T grad N (diagonal blocks) + tau_bulk dN/dx_i^T dN/dx_j (all
// blocks) at the centroid; tau from u_adv.  One thread per node writes its
// dim rows (zeroed first; ZeroLSS).
template <int D>
__global__ void __launch_bounds__(kSIThreads) si_velocity_matrix_kernel(SIArgs A, const int64_t* __restrict__ rowptr,
                                                                        double* __restrict__ vals) {
  constexpr int n = D + 1;
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= A.N) return;
  const KParams<double> kp = make_kparams<double>(A.p);
  const int64_t S = A.start[i + 1] - A.start[i];
  const int64_t r0 = rowptr[i * D];
  for (int64_t q = r0; q < r0 + int64_t(D) * D * S; ++q) vals[q] = 0.0;
  const double thdt = kp.theta * kp.dt;
  for (int32_t p = A.row_inc[i]; p < A.row_inc[i + 1]; ++p) {
    const int64_t e = A.inc_elem[p];
    const uint32_t info = A.inc_info[p];
    const int a = int(info >> 24);
    int ids[4];
    load_ids(A.conn, e, ids);
    SIGeom<D> g;
    si_element<D>(A, kp, ids, A.uadv, g);
    const double w1 = w1_ref<D>() * g.det, w2 = w2_ref<D>() * g.det;
    double Tm[n];
#pragma unroll
    for (int b = 0; b < n; ++b) Tm[b] = 0.0;
#pragma unroll
    for (int qp = 0; qp < n_gauss2<D>(); ++qp) {
      double Nq[n];
      gauss_N<D, double>(qp, Nq);
      const double wa = w2 * sel<n>(Nq, a);
#pragma unroll
      for (int b = 0; b < n; ++b) Tm[b] += wa * Nq[b];
    }
    double Ga[D];
#pragma unroll
    for (int k = 0; k < D; ++k) Ga[k] = sel<n>(g.G[k], a);
    const double lapc = w1 * g.nu_c, bulkc = w1 * g.tbu;
#pragma unroll
    for (int b = 0; b < n; ++b) {
      const int slot = int((info >> (6 * b)) & 63u);
      double dot = 0.0;
#pragma unroll
      for (int k = 0; k < D; ++k) dot += Ga[k] * g.G[k][b];
      const double lap = lapc * dot;
#pragma unroll
      for (int r = 0; r < D; ++r) {
        const double br = bulkc * Ga[r];
        double* row = vals + r0 + int64_t(r) * D * S + int64_t(slot) * D;
#pragma unroll
        for (int c = 0; c < D; ++c) {
          const double bulk = br * g.G[c][b];
          const double M = (r == c) ? lap + bulk : bulk;
          const double T = (r == c) ? Tm[b] : 0.0;
          row[c] += T + thdt * M;
        }
      }
    }
  }
}

// Pressure matrix theta (tau_ps + dt) grad N^T grad N (PressureSystem.cpp:110-140),
// tau from the velocity solution u; order-2 rule.
template <int D>
__global__ void __launch_bounds__(kSIThreads) si_pressure_matrix_kernel(SIArgs A, double* __restrict__ vals) {
  constexpr int n = D + 1;
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= A.N) return;
  const KParams<double> kp = make_kparams<double>(A.p);
  const int64_t s0 = A.start[i], S = A.start[i + 1] - s0;
  for (int64_t q = 0; q < S; ++q) vals[s0 + q] = 0.0;
  for (int32_t p = A.row_inc[i]; p < A.row_inc[i + 1]; ++p) {
    const int64_t e = A.inc_elem[p];
    const uint32_t info = A.inc_info[p];
    const int a = int(info >> 24);
    int ids[4];
    load_ids(A.conn, e, ids);
    SIGeom<D> g;
    si_element<D>(A, kp, ids, A.state, g);
    const double coef = kp.theta * (g.tps + kp.dt);
    const double w2 = w2_ref<D>() * g.det;
#pragma unroll
    for (int b = 0; b < n; ++b) {
      double dot = 0.0;
#pragma unroll
      for (int k = 0; k < D; ++k) dot += sel<n>(g.G[k], a) * g.G[k][b];
      double Ab = 0.0;
#pragma unroll
      for (int qp = 0; qp < n_gauss2<D>(); ++qp) Ab += w2 * dot;
      const int slot = int((info >> (6 * b)) & 63u);
      vals[s0 + slot] += coef * Ab;
    }
  }
}

// Lumped mass (row-sum lumping of the order-2 consistent mass, the same value
// for every velocity component) and its reciprocal
// (NavierStokesSemiImplicit.cpp:238-247 and MatrixAssembly.hpp:411-420).
template <int D>
__global__ void __launch_bounds__(kSIThreads) si_lumped_mass_kernel(SIArgs A, double* __restrict__ minv) {
  constexpr int n = D + 1;
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= A.N) return;
  double acc = 0.0;
  for (int32_t p = A.row_inc[i]; p < A.row_inc[i + 1]; ++p) {
    const int64_t e = A.inc_elem[p];
    const int a = int(A.inc_info[p] >> 24);
    int ids[4];
    load_ids(A.conn, e, ids);
    double X0[4], J[D][D], Ji[D][D], det;
    ld4(A.coords + 4ll * ids[0], X0[0], X0[1], X0[2], X0[3]);
#pragma unroll
    for (int r = 0; r < D; ++r) {
      double x[4];
      ld4(A.coords + 4ll * ids[r + 1], x[0], x[1], x[2], x[3]);
#pragma unroll
      for (int c = 0; c < D; ++c) J[r][c] = x[c] - X0[c];
    }
    inverse_det<double>(J, Ji, det);
    const double w2 = w2_ref<D>() * det;
    double M[n];
#pragma unroll
    for (int b = 0; b < n; ++b) M[b] = 0.0;
#pragma unroll
    for (int qp = 0; qp < n_gauss2<D>(); ++qp) {
      double Nq[n];
      gauss_N<D, double>(qp, Nq);
      const double wa = w2 * sel<n>(Nq, a);
#pragma unroll
      for (int b = 0; b < n; ++b) M[b] += wa * Nq[b];
    }
    double rowsum = 0.0;
#pragma unroll
    for (int b = 0; b < n; ++b) rowsum += M[b];
    acc += rowsum;
  }
  const double r = 1.0 / acc;  // rows without incidences (linked nodes) are overwritten from their master
#pragma unroll
  for (int k = 0; k < D; ++k) minv[i * D + k] = r;
}

// Velocity right-hand side (VelocityRHS, MatrixAssembly.hpp:212-360) with
// a_vec = a, dt_a_min_u = dt (1 - theta) a - u, p_plus_dp = (1 - theta) dpsum - p
// (the arguments of MatrixAssembly.hpp:440-462); tau from u_adv.
template <int D>
__global__ void __launch_bounds__(kSIThreads) si_velocity_rhs_kernel(SIArgs A, const double* __restrict__ avec,
                                                                     const double* __restrict__ uvec,
                                                                     const double* __restrict__ pvec,
                                                                     const double* __restrict__ dpsum,
                                                                     double* __restrict__ rhs) {
  constexpr int n = D + 1;
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= A.N) return;
  const KParams<double> kp = make_kparams<double>(A.p);
  const double dtl = kp.dt * (1.0 - kp.theta), omt = 1.0 - kp.theta;
  double acc[D];
#pragma unroll
  for (int k = 0; k < D; ++k) acc[k] = 0.0;
  for (int32_t p = A.row_inc[i]; p < A.row_inc[i + 1]; ++p) {
    const int64_t e = A.inc_elem[p];
    const int a = int(A.inc_info[p] >> 24);
    int ids[4];
    load_ids(A.conn, e, ids);
    SIGeom<D> g;
    si_element<D>(A, kp, ids, A.uadv, g);
    double AV[n][D], DAU[n][D], PP[n];
#pragma unroll
    for (int b = 0; b < n; ++b) {
#pragma unroll
      for (int k = 0; k < D; ++k) {
        const double av = avec[int64_t(ids[b]) * D + k];
        AV[b][k] = av;
        DAU[b][k] = dtl * av - uvec[int64_t(ids[b]) * D + k];
      }
      PP[b] = omt * dpsum[ids[b]] - pvec[ids[b]];
    }
    double div = 0.0;  // sum_i grad N_i . dt_a_min_u_i
#pragma unroll
    for (int k = 0; k < D; ++k) {
      double s = 0.0;
#pragma unroll
      for (int b = 0; b < n; ++b) s += g.G[k][b] * DAU[b][k];
      div += s;
    }
    double Ga[D];
#pragma unroll
    for (int k = 0; k < D; ++k) Ga[k] = sel<n>(g.G[k], a);
    double contrib[D];
#pragma unroll
    for (int k = 0; k < D; ++k) contrib[k] = 0.0;
    // mass-type terms, order-2 rule (MatrixAssembly.hpp:256-287)
    const double w2 = w2_ref<D>() * g.det;
#pragma unroll
    for (int qp = 0; qp < n_gauss2<D>(); ++qp) {
      double Nq[n];
      gauss_N<D, double>(qp, Nq);
      double uq[D];
#pragma unroll
      for (int k = 0; k < D; ++k) {
        double s = 0.0;
#pragma unroll
        for (int b = 0; b < n; ++b) s += Nq[b] * g.el.U[b][k];
        uq[k] = s;
      }
      double adv[n];
#pragma unroll
      for (int b = 0; b < n; ++b) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) s += uq[k] * g.G[k][b];
        adv[b] = s;
      }
      const double npa = g.tsu * sel<n>(adv, a) + sel<n>(Nq, a);
      const double fs = 0.5 * (div * w2);
#pragma unroll
      for (int k = 0; k < D; ++k) {
        double c = 0.0, ee = 0.0;
#pragma unroll
        for (int b = 0; b < n; ++b) {
          c += Nq[b] * AV[b][k];
          ee += adv[b] * DAU[b][k];
        }
        contrib[k] += npa * ((-w2 * c + w2 * ee) + fs * uq[k]);
      }
    }
    // operator terms at the centroid (MatrixAssembly.hpp:289-341, IntegralOrder 1)
    {
      const double w1 = w1_ref<D>() * g.det;
      const double wv = w1 * g.nu_c, tw = w1 * g.tsu;
      double Nc[n];
      centroid_N<D, double>(Nc);
      double adv[n];
#pragma unroll
      for (int b = 0; b < n; ++b) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) s += g.uc[k] * g.G[k][b];
        adv[b] = s;
      }
      double np = 0.0;
#pragma unroll
      for (int b = 0; b < n; ++b) np += Nc[b] * PP[b];
      const double bb = -w1 * np;
      const double fb = g.tbu * (div * w1);
      const double adva = sel<n>(adv, a);
#pragma unroll
      for (int k = 0; k < D; ++k) {
        double gp = 0.0;
#pragma unroll
        for (int b = 0; b < n; ++b) gp += g.G[k][b] * PP[b];
        const double av = tw * gp;
        double visc = 0.0;
#pragma unroll
        for (int m = 0; m < D; ++m) {
          double s = 0.0;
#pragma unroll
          for (int b = 0; b < n; ++b) s += g.G[m][b] * DAU[b][k];
          visc += Ga[m] * (wv * s);
        }
        contrib[k] += (adva * av + Ga[k] * (bb + fb)) + visc;
      }
    }
    // body force, order-2 rule (MatrixAssembly.hpp:344-360)
    if (A.force) {
      double F[n][D];
#pragma unroll
      for (int b = 0; b < n; ++b)
#pragma unroll
        for (int k = 0; k < D; ++k) F[b][k] = A.force[4ll * ids[b] + k];
#pragma unroll
      for (int qp = 0; qp < n_gauss2<D>(); ++qp) {
        double Nq[n];
        gauss_N<D, double>(qp, Nq);
        const double na = sel<n>(Nq, a);
#pragma unroll
        for (int k = 0; k < D; ++k) {
          double s = 0.0;
#pragma unroll
          for (int b = 0; b < n; ++b) s += Nq[b] * F[b][k];
          contrib[k] += na * s * w2;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < D; ++k) acc[k] += contrib[k];
  }
#pragma unroll
  for (int k = 0; k < D; ++k) rhs[i * D + k] = acc[k];
}

// Pressure right-hand side (PressureRHS, MatrixAssembly.hpp:153-210) with the
// element velocity u_adv, tau_ps from the solution u (MatrixAssembly.hpp:465-472),
// u_plus_dt_da = u + dt delta_a, a_plus_da = a + delta_a.
template <int D>
__global__ void __launch_bounds__(kSIThreads) si_pressure_rhs_kernel(SIArgs A, const double* __restrict__ uvec,
                                                                     const double* __restrict__ avec,
                                                                     const double* __restrict__ da,
                                                                     const double* __restrict__ pvec,
                                                                     double* __restrict__ rhs) {
  constexpr int n = D + 1;
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= A.N) return;
  const KParams<double> kp = make_kparams<double>(A.p);
  double acc = 0.0;
  for (int32_t p = A.row_inc[i]; p < A.row_inc[i + 1]; ++p) {
    const int64_t e = A.inc_elem[p];
    const int a = int(A.inc_info[p] >> 24);
    int ids[4];
    load_ids(A.conn, e, ids);
    SIGeom<D> g;
    si_element<D>(A, kp, ids, A.state, g);  // tau_ps from the solution u
    double Nc[n];
    centroid_N<D, double>(Nc);
    double ua[n][D], UP[n][D], APD[n][D], PV[n];
#pragma unroll
    for (int b = 0; b < n; ++b) {
      double w[4];
      ld4(A.uadv + 4ll * ids[b], w[0], w[1], w[2], w[3]);
#pragma unroll
      for (int k = 0; k < D; ++k) {
        const int64_t r = int64_t(ids[b]) * D + k;
        const double d = da[r];
        ua[b][k] = w[k];
        UP[b][k] = uvec[r] + kp.dt * d;
        APD[b][k] = avec[r] + d;
      }
      PV[b] = pvec[ids[b]];
    }
    double uac[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
      double s = 0.0;
#pragma unroll
      for (int b = 0; b < n; ++b) s += Nc[b] * ua[b][k];
      uac[k] = g.tps * s;
    }
    double adv[n];
#pragma unroll
    for (int b = 0; b < n; ++b) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < D; ++k) s += uac[k] * g.G[k][b];
      adv[b] = s;
    }
    const double w1 = w1_ref<D>() * g.det, tw = w1 * g.tps;
    const double na = sel<n>(Nc, a), adva = sel<n>(adv, a);
    double contrib = 0.0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
      double sa = 0.0, sb = 0.0, sc = 0.0;
#pragma unroll
      for (int b = 0; b < n; ++b) {
        sa += g.G[k][b] * UP[b][k];
        sb += adv[b] * UP[b][k];
        sc += Nc[b] * APD[b][k];
      }
      const double av = w1 * sa, bv = w1 * sb, cv = tw * sc;
      contrib -= av * (na + adva * 0.5) + (bv + cv) * sel<n>(g.G[k], a);
    }
    double app = 0.0;  // (App p)_a, App = tau_ps w grad N^T grad N
#pragma unroll
    for (int b = 0; b < n; ++b) {
      double dot = 0.0;
#pragma unroll
      for (int k = 0; k < D; ++k) dot += sel<n>(g.G[k], a) * g.G[k][b];
      app += (tw * dot) * PV[b];
    }
    contrib -= app;
    acc += contrib;
  }
  rhs[i] = acc;
}

// A_up delta_p (ApplyAup, MatrixAssembly.hpp:364-404), tau_su from u_adv.
template <int D>
__global__ void __launch_bounds__(kSIThreads) si_apply_aup_kernel(SIArgs A, const double* __restrict__ dp,
                                                                  double* __restrict__ rhs) {
  constexpr int n = D + 1;
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= A.N) return;
  const KParams<double> kp = make_kparams<double>(A.p);
  double acc[D];
#pragma unroll
  for (int k = 0; k < D; ++k) acc[k] = 0.0;
  for (int32_t p = A.row_inc[i]; p < A.row_inc[i + 1]; ++p) {
    const int64_t e = A.inc_elem[p];
    const int a = int(A.inc_info[p] >> 24);
    int ids[4];
    load_ids(A.conn, e, ids);
    SIGeom<D> g;
    si_element<D>(A, kp, ids, A.uadv, g);
    double Nc[n], P[n];
    centroid_N<D, double>(Nc);
#pragma unroll
    for (int b = 0; b < n; ++b) P[b] = dp[ids[b]];
    const double w = kp.theta * w1_ref<D>() * g.det;
    const double ws = w * g.tsu;
    double adva = 0.0;
#pragma unroll
    for (int k = 0; k < D; ++k) adva += g.uc[k] * sel<n>(g.G[k], a);
    adva *= ws;
    double np = 0.0;
#pragma unroll
    for (int b = 0; b < n; ++b) np += Nc[b] * P[b];
    const double bb = -w * np;
#pragma unroll
    for (int k = 0; k < D; ++k) {
      double gp = 0.0;
#pragma unroll
      for (int b = 0; b < n; ++b) gp += g.G[k][b] * P[b];
      acc[k] += gp * adva + bb * sel<n>(g.G[k], a);
    }
  }
#pragma unroll
  for (int k = 0; k < D; ++k) rhs[i * D + k] = acc[k];
}

// ---- vector kernels ------------------------------------------------------------
#define SI_GRID_STRIDE(i, n) \
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < (n); i += int64_t(gridDim.x) * blockDim.x)

__global__ void si_scale_kernel(int64_t n, double s, double* __restrict__ v) {
  SI_GRID_STRIDE(i, n) v[i] *= s;
}

__global__ void si_zero_dofs_kernel(int64_t nbc, const int64_t* __restrict__ dofs, double* __restrict__ v) {
  SI_GRID_STRIDE(i, nbc) v[dofs[i]] = 0.0;
}

__global__ void si_fill_kernel(int64_t n, double* __restrict__ v) {
  SI_GRID_STRIDE(i, n) v[i] = 0.0;
}

// u and p of the inner loop from the fields, a = 0, dpsum = 0
// (SetSolution, NavierStokesSemiImplicit.cpp:362-364; InnerLoop::execute :109-112).
__global__ void si_load_kernel(int64_t N, int dim, const double* __restrict__ state, double* __restrict__ uvec,
                               double* __restrict__ avec, double* __restrict__ pvec, double* __restrict__ dpsum) {
  SI_GRID_STRIDE(i, N) {
    for (int k = 0; k < dim; ++k) {
      uvec[i * dim + k] = state[4 * i + k];
      avec[i * dim + k] = 0.0;
    }
    pvec[i] = state[4 * i + dim];
    dpsum[i] = 0.0;
  }
}

// delta_a = delta_a_star - Ml^-1 (A_up delta_p) (NavierStokesSemiImplicit.cpp:177).
__global__ void si_correct_kernel(int64_t n, const double* __restrict__ minv, const double* __restrict__ aup,
                                  double* __restrict__ da) {
  SI_GRID_STRIDE(i, n) da[i] = da[i] - minv[i] * aup[i];
}

// a += delta_a ; u += dt delta_a ; p += delta_p ; dpsum += delta_p
// (NavierStokesSemiImplicit.cpp:183-186).
__global__ void si_accumulate_kernel(int64_t N, int dim, double dt, const double* __restrict__ da,
                                     const double* __restrict__ dp, double* __restrict__ avec,
                                     double* __restrict__ uvec, double* __restrict__ pvec,
                                     double* __restrict__ dpsum) {
  SI_GRID_STRIDE(i, N) {
    for (int k = 0; k < dim; ++k) {
      const int64_t r = i * dim + k;
      avec[r] = avec[r] + da[r];
      uvec[r] = uvec[r] + dt * da[r];
    }
    pvec[i] = pvec[i] + dp[i];
    dpsum[i] = dpsum[i] + dp[i];
  }
}

// Update (NavierStokesSemiImplicit.cpp:373): u3 = u2, u2 = u1, u1 = u, u = u_lss, p = p_lss.
__global__ void si_update_kernel(int64_t N, int dim, const double* __restrict__ uvec, const double* __restrict__ pvec,
                                 double* __restrict__ state, double* __restrict__ hist) {
  SI_GRID_STRIDE(i, N) {
    double* u1 = hist + 4 * i;
    double* u2 = hist + 4 * N + 4 * i;
    double* u3 = hist + 8 * N + 4 * i;
    for (int k = 0; k < dim; ++k) {
      u3[k] = u2[k];
      u2[k] = u1[k];
      u1[k] = state[4 * i + k];
      state[4 * i + k] = uvec[i * dim + k];
    }
    state[4 * i + dim] = pvec[i];
  }
}

// Initial conditions: nu_eff into the u_adv records and, with `reset`, the
// linearised velocity u_adv = u1 = u2 = u3 = u (NavierStokesSemiImplicit.cpp:400-409).
__global__ void si_history_kernel(int64_t N, int dim, int reset, const double* __restrict__ state,
                                  const double* __restrict__ nu, double* __restrict__ uadv,
                                  double* __restrict__ hist) {
  SI_GRID_STRIDE(i, N) {
    uadv[4 * i + 3] = nu[i];
    if (!reset) continue;
    for (int k = 0; k < dim; ++k) {
      const double u = state[4 * i + k];
      uadv[4 * i + k] = u;
      hist[4 * i + k] = u;
      hist[4 * N + 4 * i + k] = u;
      hist[8 * N + 4 * i + k] = u;
    }
  }
}

// Linked nodes: copy the master's values (tie = slave, master pairs).
__global__ void si_sync_kernel(int64_t ntie, int neq, const int32_t* __restrict__ tie, double* __restrict__ v) {
  SI_GRID_STRIDE(t, ntie) {
    const int64_t s = tie[2 * t], m = tie[2 * t + 1];
    for (int c = 0; c < neq; ++c) v[s * neq + c] = v[m * neq + c];
  }
}

// Linked nodes: identity rows with a zero right-hand side (decoupled; the
// systems stay symmetric for CG).
__global__ void si_identity_rows_kernel(int64_t ntie, int neq, const int32_t* __restrict__ tie,
                                        const int64_t* __restrict__ rowptr, const int64_t* __restrict__ diagpos,
                                        double* __restrict__ vals, double* __restrict__ rhs) {
  SI_GRID_STRIDE(t, ntie * neq) {
    const int64_t s = tie[2 * (t / neq)];
    const int64_t r = s * neq + t % neq;
    for (int64_t q = rowptr[r]; q < rowptr[r + 1]; ++q) vals[q] = (q == diagpos[r]) ? 1.0 : 0.0;
    if (rhs) rhs[r] = 0.0;
  }
}

inline unsigned si_blocks(int64_t n, int threads = kSIThreads) {
  return unsigned(std::max<int64_t>(1, (n + threads - 1) / threads));
}
inline unsigned si_vec_blocks(int64_t n) { return unsigned(std::max<int64_t>(1, std::min<int64_t>(8 * 148, (n + 255) / 256))); }

SIArgs make_args(const ufem_ns_handle* b) {
  SIArgs A;
  A.coords = b->d_coords;
  A.uadv = b->d_uadv;
  A.state = b->d_state;
  A.force = b->d_force;
  A.conn = reinterpret_cast<const int4*>(b->d_conn);
  A.row_inc = b->d_row_inc;
  A.inc_elem = b->d_inc_elem;
  A.inc_info = b->d_inc_info;
  A.start = b->d_start;
  A.N = b->N;
  fill_params(b, A.p);
  return A;
}

int sync_slaves(const ufem_ns_handle* sys, double* v, cudaStream_t s) {
  if (sys->ntie == 0) return UFEM_OK;
  si_sync_kernel<<<si_vec_blocks(sys->ntie), 256, 0, s>>>(sys->ntie, sys->neq, sys->d_tie, v);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

int identity_rows(ufem_ns_handle* sys, cudaStream_t s) {
  if (sys->ntie == 0) return UFEM_OK;
  si_identity_rows_kernel<<<si_vec_blocks(sys->ntie * sys->neq), 256, 0, s>>>(
      sys->ntie, sys->neq, sys->d_tie, sys->d_rowptr, sys->d_diagpos, sys->d_vals, sys->d_rhs);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

int zero_bc_dofs(ufem_ns_handle* sys, double* v, cudaStream_t s) {
  const DirichletPlan& bp = sys->bcp;
  if (bp.nbc == 0) return UFEM_OK;
  si_zero_dofs_kernel<<<si_vec_blocks(bp.nbc), 256, 0, s>>>(bp.nbc, bp.bc_dof, v);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

template <int D>
int launch_velocity_matrix(ufem_nssi_handle* h, cudaStream_t s) {
  si_velocity_matrix_kernel<D><<<si_blocks(h->base->N), kSIThreads, 0, s>>>(make_args(h->base), h->us->d_rowptr,
                                                                            h->us->d_vals);
  UFEM_CUDA_TRY(cudaGetLastError());
  return identity_rows(h->us, s);
}

template <int D>
int launch_initial(ufem_nssi_handle* h, cudaStream_t s) {
  const SIArgs A = make_args(h->base);
  si_pressure_matrix_kernel<D><<<si_blocks(A.N), kSIThreads, 0, s>>>(A, h->ps->d_vals);
  si_lumped_mass_kernel<D><<<si_blocks(A.N), kSIThreads, 0, s>>>(A, h->d_minv);
  UFEM_CUDA_TRY(cudaGetLastError());
  int rc;
  if ((rc = identity_rows(h->ps, s))) return rc;
  return sync_slaves(h->us, h->d_minv, s);
}

template <int D>
int launch_velocity_rhs(ufem_nssi_handle* h, cudaStream_t s) {
  si_velocity_rhs_kernel<D><<<si_blocks(h->base->N), kSIThreads, 0, s>>>(make_args(h->base), h->d_a, h->d_uvec,
                                                                         h->d_pvec, h->d_dpsum, h->us->d_rhs);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

template <int D>
int launch_pressure_rhs(ufem_nssi_handle* h, cudaStream_t s) {
  si_pressure_rhs_kernel<D><<<si_blocks(h->base->N), kSIThreads, 0, s>>>(make_args(h->base), h->d_uvec, h->d_a,
                                                                         h->us->d_sol, h->d_pvec, h->ps->d_rhs);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

template <int D>
int launch_apply_aup(ufem_nssi_handle* h, cudaStream_t s) {
  si_apply_aup_kernel<D><<<si_blocks(h->base->N), kSIThreads, 0, s>>>(make_args(h->base), h->ps->d_sol,
                                                                      h->us->d_rhs);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

void fold_status(ufem_krylov_status& acc, const ufem_krylov_status& s, bool first) {
  if (first) {
    acc = s;
    return;
  }
  acc.converged = acc.converged && s.converged;
  acc.status = std::max(acc.status, s.status);
  acc.iterations += s.iterations;
  acc.refinements += s.refinements;
  acc.rel_residual = std::max(acc.rel_residual, s.rel_residual);
}

// Aggregates of the pressure rows: the node's box, except rows the conditions
// or the periodic links decouple (identity rows); empty boxes are dropped.
int build_pressure_coarse(ufem_nssi_handle* h, cudaStream_t s) {
  ufem_ns_handle* ps = h->ps;
  const int64_t N = ps->N;
  std::vector<int32_t> agg(h->box);
  for (const auto& e : ps->bcs) agg[ps->p2m_h.empty() ? e.node : ps->p2m_h[e.node]] = -1;
  if (!ps->p2m_h.empty())
    for (int64_t i = 0; i < N; ++i)
      if (ps->p2m_h[size_t(i)] != uint32_t(i)) agg[size_t(i)] = -1;
  std::vector<int32_t> ren(size_t(h->nbox), -1);
  int nc = 0;
  for (int32_t& a : agg)
    if (a >= 0) {
      if (ren[size_t(a)] < 0) ren[size_t(a)] = nc++;
      a = ren[size_t(a)];
    }
  int rc;
  if ((rc = krylov_set_coarse(ps, agg, nc, s))) return rc;
  h->coarse_ok = krylov_coarse_size(ps) > 0;
  h->coarse_ready = true;
  return UFEM_OK;
}

template <int D>
int step_one(ufem_nssi_handle* h, cudaStream_t s) {
  ufem_ns_handle* b = h->base;
  ufem_ns_handle* us = h->us;
  ufem_ns_handle* ps = h->ps;
  const double dt = b->opt.dt;
  const int64_t N = b->N;
  int rc;
  if ((rc = launch_linearize(b, s))) return rc;                 // LinearizeU
  if ((rc = launch_velocity_matrix<D>(h, s))) return rc;        // VelocityLSS: ZeroLSS + Assembly
  si_load_kernel<<<si_vec_blocks(N), 256, 0, s>>>(N, D, b->d_state, h->d_uvec, h->d_a, h->d_pvec, h->d_dpsum);
  UFEM_CUDA_TRY(cudaGetLastError());
  for (int it = 0; it < h->nb_iterations; ++it) {
    // velocity predictor: delta_a_star
    if ((rc = launch_velocity_rhs<D>(h, s))) return rc;
    if (it == 0) {  // the velocity BC acts on velocities: scale the acceleration RHS around it
      si_scale_kernel<<<si_vec_blocks(us->nrows), 256, 0, s>>>(us->nrows, dt, us->d_rhs);
      us->time = b->time;  // function values at the step's start time
      if ((rc = launch_dirichlet_functions(us, s))) return rc;
      if ((rc = launch_dirichlet(us, s))) return rc;
      si_scale_kernel<<<si_vec_blocks(us->nrows), 256, 0, s>>>(us->nrows, 1.0 / dt, us->d_rhs);
      UFEM_CUDA_TRY(cudaGetLastError());
    } else if ((rc = zero_bc_dofs(us, us->d_rhs, s))) {
      return rc;
    }
    si_fill_kernel<<<si_vec_blocks(us->nrows), 256, 0, s>>>(us->nrows, us->d_sol);
    UFEM_CUDA_TRY(cudaGetLastError());
    ufem_krylov_status st{};
    if ((rc = krylov_solve(us, &h->ku, &st, s))) return rc;
    fold_status(h->last_u, st, it == 0);
    if ((rc = sync_slaves(us, us->d_sol, s))) return rc;
    // pressure: delta_p
    if ((rc = launch_pressure_rhs<D>(h, s))) return rc;
    si_fill_kernel<<<si_vec_blocks(ps->nrows), 256, 0, s>>>(ps->nrows, ps->d_sol);
    UFEM_CUDA_TRY(cudaGetLastError());
    if (it == 0) {
      ps->time = b->time;
      if ((rc = launch_dirichlet_functions(ps, s))) return rc;
      if ((rc = launch_dirichlet(ps, s))) return rc;
      // the pressure matrix is final once its conditions are applied: (re)build
      // the coarse space of the two-level preconditioner from it
      if (h->kp.precond == 3 && !h->coarse_ready && (rc = build_pressure_coarse(h, s))) return rc;
    } else if ((rc = zero_bc_dofs(ps, ps->d_rhs, s))) {
      return rc;
    }
    ufem_krylov_opts kp = h->kp;
    if (kp.precond == 3 && !h->coarse_ok) kp.precond = 1;  // singular coarse matrix: point Jacobi
    if ((rc = krylov_solve(ps, &kp, &st, s))) return rc;
    fold_status(h->last_p, st, it == 0);
    if ((rc = sync_slaves(ps, ps->d_sol, s))) return rc;
    // corrector: delta_a = delta_a_star - Ml^-1 A_up delta_p
    if ((rc = launch_apply_aup<D>(h, s))) return rc;
    if ((rc = zero_bc_dofs(us, us->d_rhs, s))) return rc;
    si_correct_kernel<<<si_vec_blocks(us->nrows), 256, 0, s>>>(us->nrows, h->d_minv, us->d_rhs, us->d_sol);
    UFEM_CUDA_TRY(cudaGetLastError());
    if ((rc = sync_slaves(us, us->d_sol, s))) return rc;
    si_accumulate_kernel<<<si_vec_blocks(N), 256, 0, s>>>(N, D, dt, us->d_sol, ps->d_sol, h->d_a, h->d_uvec,
                                                         h->d_pvec, h->d_dpsum);
    UFEM_CUDA_TRY(cudaGetLastError());
  }
  si_update_kernel<<<si_vec_blocks(N), 256, 0, s>>>(N, D, h->d_uvec, h->d_pvec, b->d_state, b->d_hist);
  UFEM_CUDA_TRY(cudaGetLastError());
  b->time += dt;
  return UFEM_OK;
}

int ensure_plans(ufem_nssi_handle* h) {
  int rc;
  for (ufem_ns_handle* sys : {h->us, h->ps})
    if (sys->bcp.dirty && (rc = build_bc_plan(sys))) return rc;
  return UFEM_OK;
}

template <typename T>
int si_alloc(T** p, size_t count) {
  DeviceLock lk(device_mutex());
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) return set_error(UFEM_ERR_NOMEM, std::string("cudaMalloc (semi-implicit vectors): ") +
                                                             cudaGetErrorString(e));
  return UFEM_OK;
}

void si_destroy(ufem_nssi_handle* h) {
  if (!h) return;
  {
    DeviceLock lk(device_mutex());
    for (double* p : {h->d_uvec, h->d_a, h->d_minv, h->d_pvec, h->d_dpsum})
      if (p) cudaFree(p);
  }
  destroy_handle(h->us);
  destroy_handle(h->ps);
  destroy_handle(h->base);
  delete h;
}

}  // namespace
}  // namespace ufem

using namespace ufem;

extern "C" {

int ufem_nssi_create(const ufem_mesh* mesh, const ufem_ns_options* opts, int32_t nb_iterations,
                     const uint32_t* slaves, const uint32_t* masters, int64_t nlinks, ufem_nssi_handle** out) {
  if (!out) return set_error(UFEM_ERR_ARG, "out handle pointer is NULL");
  *out = nullptr;
  if (!opts) return set_error(UFEM_ERR_ARG, "options are NULL");
  if (nb_iterations < 1) return set_error(UFEM_ERR_ARG, "nb_iterations must be at least 1");
  ufem_ns_options o = *opts;
  o.precision = 0;  // the semi-implicit element expressions are evaluated in FP64
  ufem_nssi_handle* h = new ufem_nssi_handle();
  h->nb_iterations = nb_iterations;
  int rc;
  if ((rc = create_base(mesh, &o, slaves, masters, nlinks, &h->base))) {
    si_destroy(h);
    return rc;
  }
  const int D = h->base->dim;
  const int64_t N = h->base->N;
  if ((rc = make_system_view(h->base, D, 0, &h->us)) || (rc = make_system_view(h->base, 1, D, &h->ps)) ||
      (rc = si_alloc(&h->d_uvec, size_t(N) * D)) || (rc = si_alloc(&h->d_a, size_t(N) * D)) ||
      (rc = si_alloc(&h->d_minv, size_t(N) * D)) || (rc = si_alloc(&h->d_pvec, size_t(N))) ||
      (rc = si_alloc(&h->d_dpsum, size_t(N)))) {
    si_destroy(h);
    return rc;
  }
  // Both systems are symmetric positive definite after the symmetric Dirichlet
  // conditions: CG (the reference's tests pick Belos Block CG for the velocity
  // and ML-preconditioned CG for the pressure).  Velocity: point Jacobi (the
  // mass matrix dominates).  Pressure: the two-level preconditioner, point
  // Jacobi plus a coarse correction on geometric aggregates of about 64 or
  // more nodes (at most 512 in 3D, 484 in 2D), which removes the slow
  // near-constant modes of a Laplacian fixed at few nodes.
  ufem_krylov_default_opts(&h->ku);
  h->ku.method = 2;
  h->kp = h->ku;
  h->kp.precond = 3;
  {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t i = 0; i < N; ++i)
      for (int c = 0; c < D; ++c) {
        lo[c] = std::min(lo[c], mesh->coords[i * D + c]);
        hi[c] = std::max(hi[c], mesh->coords[i * D + c]);
      }
    const int kmax = D == 3 ? 8 : 22;
    const int k = std::max(1, std::min(kmax, int(std::floor(std::pow(double(N) / 64.0, 1.0 / D)))));
    h->nbox = D == 3 ? k * k * k : k * k;
    h->box.resize(size_t(N));
    for (int64_t i = 0; i < N; ++i) {
      int id = 0, mul = 1;
      for (int c = 0; c < D; ++c) {
        const double ext = hi[c] - lo[c];
        int b = ext > 0 ? int((mesh->coords[i * D + c] - lo[c]) / ext * k) : 0;
        b = std::min(std::max(b, 0), k - 1);
        id += b * mul;
        mul *= k;
      }
      h->box[size_t(i)] = id;
    }
  }
  *out = h;
  return UFEM_OK;
}

void ufem_nssi_destroy(ufem_nssi_handle* h) { si_destroy(h); }

int ufem_nssi_set_krylov(ufem_nssi_handle* h, const ufem_krylov_opts* velocity, const ufem_krylov_opts* pressure) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (velocity && (velocity->method < 0 || velocity->method > 2 || velocity->precond < 0 || velocity->precond > 2))
    return set_error(UFEM_ERR_ARG, "invalid velocity Krylov options");
  if (pressure && (pressure->method < 0 || pressure->method > 2 || pressure->precond < 0 || pressure->precond > 3 ||
                   (pressure->precond == 3 && pressure->method != 2)))
    return set_error(UFEM_ERR_ARG, "invalid pressure Krylov options (precond 3 needs CG)");
  if (velocity) h->ku = *velocity;
  if (pressure) h->kp = *pressure;
  return UFEM_OK;
}

int ufem_nssi_set_state(ufem_nssi_handle* h, const double* up, const double* lin, const double* nu,
                        const double* force) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  return ufem_ns_set_state(h->base, up, lin, nu, force);
}

int ufem_nssi_get_state(ufem_nssi_handle* h, double* up, double* lin) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  return ufem_ns_get_state(h->base, up, lin);
}

int ufem_nssi_add_velocity_dirichlet(ufem_nssi_handle* h, const uint32_t* nodes, int64_t n, int32_t comp,
                                     const double* values) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  return ufem_ns_add_dirichlet(h->us, nodes, n, comp, values);
}

int ufem_nssi_add_pressure_dirichlet(ufem_nssi_handle* h, const uint32_t* nodes, int64_t n, const double* values) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  h->coarse_ready = false;
  return ufem_ns_add_dirichlet(h->ps, nodes, n, 0, values);
}

int ufem_nssi_add_velocity_dirichlet_function(ufem_nssi_handle* h, const uint32_t* nodes, int64_t n, int32_t comp,
                                              const char* expr) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  return ufem_ns_add_dirichlet_function(h->us, nodes, n, comp, expr);
}

int ufem_nssi_add_pressure_dirichlet_function(ufem_nssi_handle* h, const uint32_t* nodes, int64_t n,
                                              const char* expr) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  h->coarse_ready = false;
  return ufem_ns_add_dirichlet_function(h->ps, nodes, n, 0, expr);
}

int ufem_nssi_set_time(ufem_nssi_handle* h, double t) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  return ufem_ns_set_time(h->base, t);
}

// Restart files of the fields the reference lists as the solver's restart
// tags (NavierStokesSemiImplicit.cpp:277-278: u, p, linearized velocity,
// viscosity; plus the body force when set).  After reading, the caller runs
// ufem_nssi_initialize(h, 0, ...) as the reference's initial conditions do
// after their Restarts component: the pressure matrix then follows the
// restarted velocity.
int ufem_nssi_write_restart(ufem_nssi_handle* h, const char* path, double current_time, double time_step,
                            int64_t iteration) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  return ufem_ns_write_restart(h->base, path, current_time, time_step, iteration);
}

int ufem_nssi_read_restart(ufem_nssi_handle* h, const char* path, double* current_time, double* time_step,
                           int64_t* iteration) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  h->initialized = false;
  return ufem_ns_read_restart(h->base, path, current_time, time_step, iteration);
}

int ufem_nssi_clear_dirichlet(ufem_nssi_handle* h) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  int rc;
  if ((rc = ufem_ns_clear_dirichlet(h->us)) || (rc = ufem_ns_clear_dirichlet(h->ps))) return rc;
  h->coarse_ready = false;
  return UFEM_OK;
}

int ufem_nssi_initialize(ufem_nssi_handle* h, int32_t reset_history, void* stream) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  ufem_ns_handle* b = h->base;
  if (!b->state_set) return set_error(UFEM_ERR_STATE, "set the state before ufem_nssi_initialize");
  si_history_kernel<<<si_vec_blocks(b->N), 256, 0, s>>>(b->N, b->dim, reset_history ? 1 : 0, b->d_state, b->d_nu,
                                                        b->d_uadv, b->d_hist);
  UFEM_CUDA_TRY(cudaGetLastError());
  const int rc = b->dim == 2 ? launch_initial<2>(h, s) : launch_initial<3>(h, s);
  if (rc) return rc;
  h->initialized = true;
  h->coarse_ready = false;  // new pressure matrix
  return UFEM_OK;
}

int ufem_nssi_step(ufem_nssi_handle* h, int32_t nsteps, ufem_krylov_status* velocity, ufem_krylov_status* pressure,
                   void* stream) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (!h->initialized) return set_error(UFEM_ERR_STATE, "ufem_nssi_initialize must run before the first step");
  if (nsteps < 0) return set_error(UFEM_ERR_ARG, "nsteps must be >= 0");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc;
  if ((rc = ensure_plans(h))) return rc;
  ufem_krylov_status vu{}, vp{};
  for (int k = 0; k < nsteps; ++k) {
    rc = h->base->dim == 2 ? step_one<2>(h, s) : step_one<3>(h, s);
    if (rc) return rc;
    fold_status(vu, h->last_u, k == 0);
    fold_status(vp, h->last_p, k == 0);
  }
  UFEM_CUDA_TRY(cudaStreamSynchronize(s));
  if (velocity) *velocity = vu;
  if (pressure) *pressure = vp;
  return UFEM_OK;
}

int ufem_nssi_get_time(const ufem_nssi_handle* h, double* t) {
  if (!h || !t) return set_error(UFEM_ERR_ARG, "NULL argument");
  *t = h->base->time;
  return UFEM_OK;
}

int ufem_nssi_sizes(const ufem_nssi_handle* h, int64_t* velocity_nnz, int64_t* pressure_nnz) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  if (velocity_nnz) *velocity_nnz = h->us->nnz;
  if (pressure_nnz) *pressure_nnz = h->ps->nnz;
  return UFEM_OK;
}

// Debug/parity access to the two systems: which = 0 velocity, 1 pressure.
int ufem_nssi_get_system(ufem_nssi_handle* h, int32_t which, int64_t* rowptr, int32_t* colidx, double* vals,
                         double* rhs, double* sol) {
  if (!h || (which != 0 && which != 1)) return set_error(UFEM_ERR_ARG, "invalid arguments");
  ufem_ns_handle* sys = which == 0 ? h->us : h->ps;
  UFEM_CUDA_TRY(cudaDeviceSynchronize());
  if (rowptr) UFEM_CUDA_TRY(cudaMemcpy(rowptr, sys->d_rowptr, size_t(sys->nrows + 1) * 8, cudaMemcpyDeviceToHost));
  if (colidx) UFEM_CUDA_TRY(cudaMemcpy(colidx, sys->d_colidx, size_t(sys->nnz) * 4, cudaMemcpyDeviceToHost));
  if (vals) UFEM_CUDA_TRY(cudaMemcpy(vals, sys->d_vals, size_t(sys->nnz) * 8, cudaMemcpyDeviceToHost));
  if (rhs) UFEM_CUDA_TRY(cudaMemcpy(rhs, sys->d_rhs, size_t(sys->nrows) * 8, cudaMemcpyDeviceToHost));
  if (sol) UFEM_CUDA_TRY(cudaMemcpy(sol, sys->d_sol, size_t(sys->nrows) * 8, cudaMemcpyDeviceToHost));
  return UFEM_OK;
}

// The velocity matrix of the current state (LinearizeU + VelocityAssembly),
// without boundary conditions: for parity tests of the element expressions.
int ufem_nssi_assemble_velocity_matrix(ufem_nssi_handle* h, void* stream) {
  if (!h) return set_error(UFEM_ERR_ARG, "NULL handle");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc;
  if ((rc = launch_linearize(h->base, s))) return rc;
  rc = h->base->dim == 2 ? launch_velocity_matrix<2>(h, s) : launch_velocity_matrix<3>(h, s);
  if (rc) return rc;
  UFEM_CUDA_TRY(cudaStreamSynchronize(s));
  return UFEM_OK;
}

// The lumped-mass reciprocal (N x dim), after ufem_nssi_initialize.
int ufem_nssi_get_lumped_inverse(ufem_nssi_handle* h, double* minv) {
  if (!h || !minv) return set_error(UFEM_ERR_ARG, "NULL argument");
  UFEM_CUDA_TRY(cudaDeviceSynchronize());
  UFEM_CUDA_TRY(cudaMemcpy(minv, h->d_minv, size_t(h->base->N) * h->base->dim * 8, cudaMemcpyDeviceToHost));
  return UFEM_OK;
}

int64_t ufem_nssi_device_bytes(const ufem_nssi_handle* h) {
  if (!h) return 0;
  const ufem_ns_handle* b = h->base;
  const int64_t N = b->N, E = b->E, D = b->dim;
  // base: node records (coords, state, 3 history, u_adv), nu, connectivity,
  // graph, incidences, staging, force, tie list
  int64_t bytes = N * (32 + 32 + 96 + 32 + 8) + E * 16 + (N + 1) * 12 + b->bnnz * 4 + E * b->nn * 8 +
                  N * 4 * D * 8 + (b->d_force ? N * 32 : 0) + b->ntie * 8;
  for (const ufem_ns_handle* sys : {h->us, h->ps}) {
    const int64_t R = sys->nrows, Z = sys->nnz;
    bytes += (R + 1) * 8 + Z * 12 + R * 24 + (sys->kw ? R * 8 * 13 : 0);
    bytes += sys->bcp.nbc * 40 + sys->bcp.nfix_rows * 16 + sys->bcp.nfix * 12;
  }
  return bytes + N * (3 * D + 2) * 8;  // inner-loop vectors
}

}  // extern "C"
