// assembly.cu -- sm_100a kernels of the UFEM Navier-Stokes step, except the Krylov solve.
//
// Row-owner assembly.  The reference loops over elements and adds each element
// matrix into the FEVbr block rows it touches (Proto/ElementLooper.hpp:173-179,
// TrilinosFEVbrMatrix.cpp:271-357).  Here every CTA owns a contiguous range of
// CSR block rows ("chunk").  Phase 1: one thread per incidence (row node i,
// element e containing i at local position a) gathers the element's nodal data,
// evaluates the element's row block a -- the neq x (n*neq) slice of
// invdt*T + theta*A and the neq entries of -A*x + a -- and stages it in shared
// memory.  Phase 2: one thread per (row, neighbour slot, equation) sums the
// staged contributions of the row's incidences in ascending element order (the
// order in which the reference adds them) and writes each CSR value exactly
// once, coalesced.  No floating-point atomics, no element matrices in HBM.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <type_traits>

#include "internal.h"
#include "element.cuh"

namespace ufem {
namespace {

// Stores one row (neq values) of a staged element block: contiguous and
// vectorised when the staging pitch CH is 1 (warp kernel, 16-byte aligned
// rows), strided otherwise (chunk kernel, value-major staging).
template <int NEQ, typename T>
__device__ __forceinline__ void put_row(T* __restrict__ st, int idx, int CH, const T (&v)[NEQ]) {
  if (NEQ == 4 && CH == 1) {
    if constexpr (std::is_same<T, float>::value) {
      *reinterpret_cast<float4*>(st + idx) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
      reinterpret_cast<double2*>(st + idx)[0] = make_double2(v[0], v[1]);
      reinterpret_cast<double2*>(st + idx)[1] = make_double2(v[2], v[3]);
    }
  } else {
#pragma unroll
    for (int c = 0; c < NEQ; ++c) st[(idx + c) * CH] = v[c];
  }
}

// Where the element routines send their results.  StageSink stages each row
// of the element row block and the RHS row in shared memory for the reduction
// (put_row); the residual kernel's sink folds them into b - M dx instead.
template <typename T>
struct StageSink {
  T* __restrict__ st;
  T* __restrict__ rst;
  int CH;
  template <int NEQ>
  __device__ __forceinline__ void row(int idx, const T (&v)[NEQ]) { put_row<NEQ, T>(st, idx, CH, v); }
  template <int NEQ>
  __device__ __forceinline__ void rhs(const T (&v)[NEQ]) { put_row<NEQ, T>(rst, 0, CH, v); }
};

// Shared tail of both element forms: rhs row a, M = invdt*T + theta*A with the
// p row of A divided by theta first (NavierStokesAssembly.hpp:69-71), staged.
template <int D, typename T, typename Sink>
__device__ __forceinline__ void stage_block(const T (&A)[D + 1][D + 1], const T (&Tm)[D + 1][D + 1],
                                            const T (&xb)[D + 1], const KParams<T>& kp, T (&rhs)[D + 1],
                                            Sink& sk, int b) {
  constexpr int neq = D + 1;
#pragma unroll
  for (int r = 0; r < neq; ++r) {
    T s = 0;
#pragma unroll
    for (int c = 0; c < neq; ++c) s += -A[r][c] * xb[c];
    rhs[r] += s;
    T row[neq];
#pragma unroll
    for (int c = 0; c < neq; ++c) {
      const T a = (r == D) ? A[r][c] * kp.inv_theta : A[r][c];  // _A(p) / theta
      row[c] = kp.invdt * Tm[r][c] + kp.theta * a;
    }
    sk.template row<neq>((b * neq + r) * neq, row);
  }
}

template <int D, typename T>
__device__ __forceinline__ void load_state(const NodeData& nd, int node, T (&x)[D + 1]) {
  if constexpr (std::is_same<T, float>::value) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(nd.node32) + 2ll * node + 1);
    const float vv[4] = {v.x, v.y, v.z, v.w};
    // (u, v, [w], p): p sits at index D of the padded record
#pragma unroll
    for (int k = 0; k < D; ++k) x[k] = vv[k];
    x[D] = vv[3];
  } else {
    double s[4];
    ld4(nd.state + 4ll * node, s[0], s[1], s[2], s[3]);
#pragma unroll
    for (int k = 0; k <= D; ++k) x[k] = T(s[k]);
  }
}

// ---------------------------------------------------------------------------
// Generic expression (NavierStokesAssembly.hpp:51-67) for the row node, which
// the caller has placed at local position 0.  The reference integrates it with
// the order-2 Gauss rule (Proto/ElementIntegration.hpp:236-258, weight
// w_q det J).  For P1 elements the gradients G are constant and every integrand
// is a polynomial of degree <= 2 in the barycentric coordinates, which that
// rule integrates exactly, so the sums are evaluated here in closed form with
//   int N_k = m1 = V/n,   int N_k N_l = m2 (1 + d_kl),   m2 = V/(n(n+1)),
// c_kb = U_k . G_b (U: nodal u_adv), ubar = mean U, alpha_b = ubar . G_b,
// w_k = c_k0 and q = sum_k w_k U_k:
//   int adv_b          = V alpha_b
//   int N_0 adv_b      = m2 (n alpha_b + c_0b)
//   int adv_0 adv_b    = m2 (n^2 alpha_0 alpha_b + q . G_b)
//   int adv_0 N_b      = m2 (n alpha_0 + w_b)
//   int ua_i S_0       = m2 (n ubar_i + U_0i) + tau_su m2 (n^2 ubar_i alpha_0 + q_i)
//   int S_0 g_i        = m2 (n gbar_i + g_0i) + tau_su m2 (n^2 gbar_i alpha_0 + sum_k w_k g_ki)
// (tests/test_gpu_parity.py checks the result against the oracle's literal
// quadrature).
// ---------------------------------------------------------------------------
template <int D, typename T, typename Sink>
__device__ __forceinline__ void generic_row(const int (&ids)[4], int a, const NodeData& nd,
                                            const double* __restrict__ force, const KParams<T>& kp, Sink& sk) {
  constexpr int n = D + 1, neq = D + 1;
  const T inv_n = T(1.0 / n);
  const T nT = T(n), n2 = T(n * n);
  Elem<D, T> el;
  gather_geometry_uadv<D, T>(ids, nd, el);
  // tau inputs: |mean nodal nu| and u_adv at the centroid (SUPG.hpp:110-116, 145-147)
  T nsum = 0;
#pragma unroll
  for (int b = 0; b < n; ++b) nsum += el.NU[b];
  const T nu_bar = nsum * inv_n;
  T Nc[n];
  centroid_N<D, T>(Nc);
  T uc[D], ub[D];
#pragma unroll
  for (int k = 0; k < D; ++k) {
    T s = 0, m = 0;
#pragma unroll
    for (int b = 0; b < n; ++b) {
      if constexpr (D == 2) s += Nc[b] * el.U[b][k];
      m += el.U[b][k];
    }
    ub[k] = m * inv_n;
    // tetrahedra: N_b(centroid) = 1/4 exactly, so the centroid value is the mean
    uc[k] = (D == 3) ? ub[k] : s;
  }
  T J[D][D], Ji[D][D], det;
#pragma unroll
  for (int r = 0; r < D; ++r)
#pragma unroll
    for (int c = 0; c < D; ++c) J[r][c] = el.Xr[r + 1][c];
  inverse_det<T>(J, Ji, det);
  T G[D][n];
#pragma unroll
  for (int r = 0; r < D; ++r) {
    T s = -Ji[r][0];
#pragma unroll
    for (int k = 1; k < D; ++k) s -= Ji[r][k];
    G[r][0] = s;
#pragma unroll
    for (int b = 1; b <= D; ++b) G[r][b] = Ji[r][b - 1];
  }
  T g[D][D];
  metric_tensor<D, T>(G, a, g);
  T tps, tsu, tbu;
  compute_tau<D, T>(kp, el, uc, tabs(nu_bar), G, g, det, tps, tsu, tbu);
  const T V = det * T(D == 2 ? 0.5 : 1.0 / 6.0);
  const T m1 = V * inv_n;
  const T m2 = V * T(1.0 / (n * (n + 1)));
  T alpha[n], w[n], c0[n], D0[n];
#pragma unroll
  for (int b = 0; b < n; ++b) {
    T a = 0, ww = 0, cc = 0, dd = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
      a += ub[k] * G[k][b];
      ww += el.U[b][k] * G[k][0];
      cc += el.U[0][k] * G[k][b];
      dd += G[k][0] * G[k][b];
    }
    alpha[b] = a;
    w[b] = ww;
    c0[b] = cc;
    D0[b] = dd;
  }
  T q[D];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    T s = 0;
#pragma unroll
    for (int k = 0; k < n; ++k) s += w[k] * el.U[k][i];
    q[i] = s;
  }
  const T tsum2 = tsu * m2;
  const T sWS = m1 + tsu * V * alpha[0];
  const T sWSp = m1 + T(0.5) * tps * V * alpha[0];
  T gam[D], au[D];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    gam[i] = tbu * V * G[i][0] + T(0.5) * (m2 * (nT * ub[i] + el.U[0][i]) + tsum2 * (n2 * ub[i] * alpha[0] + q[i]));
    au[i] = 0;
  }
  if (kp.has_force) {
    T F[n][D];
#pragma unroll
    for (int b = 0; b < n; ++b) {
      double f[4];
      ld4(force + 4ll * ids[b], f[0], f[1], f[2], f[3]);
#pragma unroll
      for (int k = 0; k < D; ++k) F[b][k] = T(f[k]);
    }
#pragma unroll
    for (int i = 0; i < D; ++i) {
      T gs = 0, gw = 0;
#pragma unroll
      for (int k = 0; k < n; ++k) {
        gs += F[k][i];
        gw += w[k] * F[k][i];
      }
      const T gbar = gs * inv_n;
      au[i] = m2 * (nT * gbar + F[0][i]) + tsum2 * (n2 * gbar * alpha[0] + gw);
    }
  }
  // nodal state (u, p) of the element: A x for the RHS
  T xs[n][neq];
#pragma unroll
  for (int b = 0; b < n; ++b) load_state<D, T>(nd, ids[b], xs[b]);
  T div = 0, gradp[D], kx[D], ax[D];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    gradp[i] = 0;
    kx[i] = 0;
    ax[i] = 0;
  }
  const T theta = kp.theta, invdt = kp.invdt, inv_rho = kp.inv_rho;
  const T thS = theta * sWS * inv_rho;  // u rows, p column: theta * G_ib * sWS / rho
  const T tpv = tps * inv_rho * V;      // p row, p column: tps * D0_b * V / rho
  T cj[D], ej[D];                        // p row, u_j columns: G_jb sWSp + cj Vab + ej
#pragma unroll
  for (int j = 0; j < D; ++j) {
    cj[j] = tps * G[j][0];
    ej[j] = invdt * (cj[j] * m1);
  }
#pragma unroll
  for (int b = 0; b < n; ++b) {
    const T Kd = nu_bar * V * D0[b] + m2 * (nT * alpha[b] + c0[b]);
    T qg = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) qg += q[k] * G[k][b];
    const T Kdb = Kd + tsum2 * (n2 * alpha[0] * alpha[b] + qg);
    const T Tuu = m2 * (b == 0 ? T(2) : T(1)) + tsum2 * (nT * alpha[0] + w[b]);
    const T Vab = V * alpha[b];
    // rows u_i: M = invdt*T + theta*A
    const T diag = theta * Kdb + invdt * Tuu;
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const T tg = theta * gam[i];
      T row[neq];
#pragma unroll
      for (int j = 0; j < D; ++j) row[j] = tg * G[j][b] + (i == j ? diag : T(0));
      row[D] = G[i][b] * thS;
      sk.template row<neq>((b * neq + i) * neq, row);
    }
    // row p: theta * (A / theta) + invdt * T = A + invdt * T
    {
      T row[neq];
#pragma unroll
      for (int j = 0; j < D; ++j) row[j] = G[j][b] * sWSp + (cj[j] * Vab + ej[j]);
      row[D] = D0[b] * tpv;
      sk.template row<neq>((b * neq + D) * neq, row);
    }
    // pieces of A x
#pragma unroll
    for (int k = 0; k < D; ++k) {
      div += G[k][b] * xs[b][k];
      gradp[k] += G[k][b] * xs[b][D];
      kx[k] += Kdb * xs[b][k];
      ax[k] += Vab * xs[b][k];
    }
  }
  // rhs row 0 = a - A x  (A before the theta combination)
  T rrow[neq];
#pragma unroll
  for (int i = 0; i < D; ++i) rrow[i] = au[i] - (kx[i] + gam[i] * div + sWS * inv_rho * gradp[i]);
  T g0ax = 0, g0gp = 0;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    g0ax += G[k][0] * ax[k];
    g0gp += G[k][0] * gradp[k];
  }
  rrow[D] = -(sWSp * div + tps * g0ax + tps * V * inv_rho * g0gp);
  sk.template rhs<neq>(rrow);
}

// ---------------------------------------------------------------------------
// Specialised triangles, NavierStokesSpecializations.hpp:37-147, for the row
// node at local position 0 (ai: the relabel key, used by the metric tau only).
// Each entry receives its terms in the reference's order.
// ---------------------------------------------------------------------------
template <int D, typename T>
__device__ __forceinline__ void spec_tau_common(const KParams<T>& kp, const Elem<D, T>& el, int a,
                                                const NodeData& nd, const int (&ids)[4], T nu,
                                                const T (&Ji)[D][D], T det, T (&xs)[D + 1][D + 1],
                                                T& tps, T& tsu, T& tbu) {
  // tau of the solution velocity u; the nodal states are returned in xs (the
  // caller's A x needs them) and J^-1, det J come from the caller
  constexpr int n = D + 1;
  T Nc[n];
  centroid_N<D, T>(Nc);
  T uc[D];
#pragma unroll
  for (int k = 0; k < D; ++k) uc[k] = 0;
#pragma unroll
  for (int b = 0; b < n; ++b) {
    load_state<D, T>(nd, ids[b], xs[b]);
#pragma unroll
    for (int k = 0; k < D; ++k) uc[k] += Nc[b] * xs[b][k];
  }
  T G[D][D + 1];
#pragma unroll
  for (int r = 0; r < D; ++r) {
    T s = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) s += Ji[r][k] * T(-1);
    G[r][0] = s;
#pragma unroll
    for (int b = 1; b <= D; ++b) G[r][b] = Ji[r][b - 1];
  }
  T g[D][D];
  metric_tensor<D, T>(G, a, g);
  // a default ComputeTauImpl: METRIC, c1 = 1 (4 c1^2 / dt^2 = 4 / dt^2), c2 = 16, alphas 1
  KParams<T> dk = kp;
  dk.supg_type = 1;
  dk.c2 = T(16);
  dk.tau_c1 = kp.tau_std;
  dk.a_ps = dk.a_su = dk.a_bu = T(1);
  compute_tau<D, T>(dk, el, uc, nu, G, g, det, tps, tsu, tbu);
}

template <typename T, typename Sink>
__device__ __forceinline__ void spec_tri_row(const int (&ids)[4], int ai, const NodeData& nd, const KParams<T>& kp,
                                             Sink& sk) {
  Elem<2, T> el;
  gather_geometry_uadv<2, T>(ids, nd, el);
  T u_avg[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    T s = 0;
#pragma unroll
    for (int b = 0; b < 3; ++b) s += el.U[b][k];
    u_avg[k] = s / T(3);
  }
  const auto& X = el.Xr;
  const T volume = T(0.5) * ((X[1][0] - X[0][0]) * (X[2][1] - X[0][1]) - (X[2][0] - X[0][0]) * (X[1][1] - X[0][1]));
  const T fc = T(0.5);
  T nsum = 0;
#pragma unroll
  for (int b = 0; b < 3; ++b) nsum += el.NU[b];
  const T nu = tabs(nsum / T(3));
  T nx[3], ny[3];
  nx[0] = X[1][1] - X[2][1]; ny[0] = X[2][0] - X[1][0];
  nx[1] = X[2][1] - X[0][1]; ny[1] = X[0][0] - X[2][0];
  nx[2] = X[0][1] - X[1][1]; ny[2] = X[1][0] - X[0][0];
  T tau_ps, tau_su, tau_bulk;
  T J[2][2], Ji[2][2], det;
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int c = 0; c < 2; ++c) J[r][c] = X[r + 1][c];
  inverse_det<T>(J, Ji, det);
  T xs[3][3];
  spec_tau_common<2, T>(kp, el, ai, nd, ids, nu, Ji, det, xs, tau_ps, tau_su, tau_bulk);
  const T nix = nx[0], niy = ny[0];  // row node at local position 0
  const T u_ni = u_avg[0] * nix + u_avg[1] * niy;
  const T rho = kp.rho;
  // j-independent factors evaluated once (the same expressions as below)
  const T su4 = tau_su / (T(4) * volume), ps4 = tau_ps / (T(4) * volume);
  const T fsu4 = fc * tau_su / (T(4) * volume), fps4 = fc * tau_ps / (T(4) * volume);
  const T nu4 = nu / (T(4) * volume), rho6 = T(1) / (T(6) * rho);
  const T surho4 = tau_su / (T(4) * rho * volume), lap4 = T(1) / (T(4) * rho * volume);
  const T bulk4 = tau_bulk / (T(4) * volume), v12 = volume / T(12);
  const T su6 = tau_su / T(6), ps6 = tau_ps / T(6);
  const T third = T(1. / 3.);  // the reference divides these products by 3
  T rhs[3] = {0, 0, 0};
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    T A[3][3], Tm[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) { A[r][c] = 0; Tm[r][c] = 0; }
    const T uk = u_avg[0], vk = u_avg[1];
    const T uknj = uk * nx[j] + vk * ny[j];
    T val = T(1. / 6.) * uknj;
    val += su4 * uknj * u_ni;
    A[0][0] += val; A[1][1] += val;
    val = ps4 * uknj;
    A[2][0] += val * nix; A[2][1] += val * niy;
    val = fc / T(6);
    val += fsu4 * u_ni;
    A[0][0] += val * uk * nx[j]; A[0][1] += val * uk * ny[j];
    A[1][0] += val * vk * nx[j]; A[1][1] += val * vk * ny[j];
    val = fps4;
    A[2][0] += val * nix * uk * nx[j]; A[2][1] += val * nix * uk * ny[j];
    A[2][0] += val * niy * vk * nx[j]; A[2][1] += val * niy * vk * ny[j];
    val = nu4;
    A[0][0] += val * (T(4. / 3.) * nix * nx[j] + niy * ny[j]);
    A[0][1] += val * nix * ny[j] * third;
    A[1][0] += val * niy * nx[j] * third;
    A[1][1] += val * (nix * nx[j] + T(4. / 3.) * niy * ny[j]);
    val = rho6;
    val += surho4 * u_ni;
    A[0][2] += nx[j] * val; A[1][2] += ny[j] * val;
    const T laplacian = lap4 * (nix * nx[j] + niy * ny[j]);
    A[2][2] += tau_ps * laplacian;
    val = T(1. / 6.);
    A[2][0] += val * nx[j]; A[2][1] += val * ny[j];
    val = bulk4;
    A[0][0] += val * nix * nx[j]; A[0][1] += val * nix * ny[j];
    A[1][0] += val * niy * nx[j]; A[1][1] += val * niy * ny[j];
    val = v12 * (T(1) + (j == 0 ? T(1) : T(0)));
    val += su6 * u_ni;
    Tm[0][0] += val; Tm[1][1] += val;
    val = ps6;
    Tm[2][0] += val * nix; Tm[2][1] += val * niy;
    stage_block<2, T>(A, Tm, xs[j], kp, rhs, sk, j);
  }
  sk.template rhs<3>(rhs);
}

// Specialised tetrahedra, NavierStokesSpecializations.hpp:150-302, row i = a,
// including the reference's use of vk in the W rows (:224-226, :236-238).
template <typename T, typename Sink>
__device__ __forceinline__ void spec_tet_row(const int (&ids)[4], int ai, const NodeData& nd, const KParams<T>& kp,
                                             Sink& sk) {
  Elem<3, T> el;
  gather_geometry_uadv<3, T>(ids, nd, el);
  T u_avg[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    T s = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b) s += el.U[b][k];
    u_avg[k] = s / T(4);
  }
  const auto& X = el.Xr;
  T J[3][3], Ji[3][3], det;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) J[r][c] = X[r + 1][c];
  inverse_det<T>(J, Ji, det);
  const T volume = det / T(6);
  const T fc = T(0.5);
  T nsum = 0;
#pragma unroll
  for (int b = 0; b < 4; ++b) nsum += el.NU[b];
  const T nu = tabs(nsum / T(4));
  T nr[4][3];
  const int XX = 0, YY = 1, ZZ = 2;
  nr[0][XX] = ((X[3][YY]-X[1][YY])*(X[2][ZZ]-X[1][ZZ]) - (X[2][YY]-X[1][YY])*(X[3][ZZ]-X[1][ZZ])) / T(2);
  nr[0][YY] = ((X[3][ZZ]-X[1][ZZ])*(X[2][XX]-X[1][XX]) - (X[2][ZZ]-X[1][ZZ])*(X[3][XX]-X[1][XX])) / T(2);
  nr[0][ZZ] = ((X[3][XX]-X[1][XX])*(X[2][YY]-X[1][YY]) - (X[2][XX]-X[1][XX])*(X[3][YY]-X[1][YY])) / T(2);
  nr[1][XX] = ((X[2][YY]-X[0][YY])*(X[3][ZZ]-X[0][ZZ]) - (X[3][YY]-X[0][YY])*(X[2][ZZ]-X[0][ZZ])) / T(2);
  nr[1][YY] = ((X[2][ZZ]-X[0][ZZ])*(X[3][XX]-X[0][XX]) - (X[3][ZZ]-X[0][ZZ])*(X[2][XX]-X[0][XX])) / T(2);
  nr[1][ZZ] = ((X[2][XX]-X[0][XX])*(X[3][YY]-X[0][YY]) - (X[3][XX]-X[0][XX])*(X[2][YY]-X[0][YY])) / T(2);
  nr[2][XX] = ((X[3][YY]-X[0][YY])*(X[1][ZZ]-X[0][ZZ]) - (X[1][YY]-X[0][YY])*(X[3][ZZ]-X[0][ZZ])) / T(2);
  nr[2][YY] = ((X[3][ZZ]-X[0][ZZ])*(X[1][XX]-X[0][XX]) - (X[1][ZZ]-X[0][ZZ])*(X[3][XX]-X[0][XX])) / T(2);
  nr[2][ZZ] = ((X[3][XX]-X[0][XX])*(X[1][YY]-X[0][YY]) - (X[1][XX]-X[0][XX])*(X[3][YY]-X[0][YY])) / T(2);
  nr[3][XX] = ((X[1][YY]-X[0][YY])*(X[2][ZZ]-X[0][ZZ]) - (X[2][YY]-X[0][YY])*(X[1][ZZ]-X[0][ZZ])) / T(2);
  nr[3][YY] = ((X[1][ZZ]-X[0][ZZ])*(X[2][XX]-X[0][XX]) - (X[2][ZZ]-X[0][ZZ])*(X[1][XX]-X[0][XX])) / T(2);
  nr[3][ZZ] = ((X[1][XX]-X[0][XX])*(X[2][YY]-X[0][YY]) - (X[2][XX]-X[0][XX])*(X[1][YY]-X[0][YY])) / T(2);
  T tau_ps, tau_su, tau_bulk;
  T xs[4][4];
  spec_tau_common<3, T>(kp, el, ai, nd, ids, nu, Ji, det, xs, tau_ps, tau_su, tau_bulk);
  T ni[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    T col[4] = {nr[0][k], nr[1][k], nr[2][k], nr[3][k]};
    ni[k] = col[0];  // row node at local position 0
  }
  const T u_ni = u_avg[XX] * ni[XX] + u_avg[YY] * ni[YY] + u_avg[ZZ] * ni[ZZ];
  const T rho = kp.rho;
  // The reference's j-independent factors, evaluated once (the same expressions
  // as in the loop below, so the same values); FP64 divisions are expensive.
  const T su9 = tau_su / (T(9) * volume), ps9 = tau_ps / (T(9) * volume);
  const T fsu9 = fc * tau_su / (T(9) * volume), fps9 = fc * tau_ps / (T(9) * volume);
  const T nu9 = nu / (T(9) * volume), rho12 = T(1) / (T(12) * rho);
  const T surho9 = tau_su / (T(9) * rho * volume), psrho9 = tau_ps / (T(9) * rho * volume);
  const T bulk9 = tau_bulk / (T(9) * volume), v20 = volume / T(20);
  const T su12 = tau_su / T(12), ps12 = tau_ps / T(12);
  const T third = T(1. / 3.);  // the reference divides these products by 3
  T rhs[4] = {0, 0, 0, 0};
  // local rows/cols: 0 = U, 1 = V, 2 = W, 3 = P
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    T A[4][4], Tm[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) { A[r][c] = 0; Tm[r][c] = 0; }
    const T uk = u_avg[XX], vk = u_avg[YY], wk = u_avg[ZZ];
    const T* nj = nr[j];
    const T uknj = uk * nj[XX] + vk * nj[YY] + wk * nj[ZZ];
    T val = T(1. / 12.) * uknj;
    val += su9 * uknj * u_ni;
    A[0][0] += val; A[1][1] += val; A[2][2] += val;
    val = ps9 * uknj;
    A[3][0] += val * ni[XX]; A[3][1] += val * ni[YY]; A[3][2] += val * ni[ZZ];
    val = fc / T(12);
    val += fsu9 * u_ni;
    A[0][0] += val * uk * nj[XX]; A[0][1] += val * uk * nj[YY]; A[0][2] += val * uk * nj[ZZ];
    A[1][0] += val * vk * nj[XX]; A[1][1] += val * vk * nj[YY]; A[1][2] += val * vk * nj[ZZ];
    A[2][0] += val * vk * nj[XX]; A[2][1] += val * vk * nj[YY]; A[2][2] += val * vk * nj[ZZ];
    val = fps9;
    A[3][0] += val * ni[XX] * uk * nj[XX]; A[3][1] += val * ni[XX] * uk * nj[YY];
    A[3][2] += val * ni[XX] * uk * nj[ZZ]; A[3][0] += val * ni[YY] * vk * nj[XX];
    A[3][1] += val * ni[YY] * vk * nj[YY]; A[3][2] += val * ni[YY] * vk * nj[ZZ];
    A[3][0] += val * ni[ZZ] * vk * nj[XX]; A[3][1] += val * ni[ZZ] * vk * nj[YY];
    A[3][2] += val * ni[ZZ] * vk * nj[ZZ];
    val = nu9;
    A[0][0] += val * (T(4. / 3.) * ni[XX] * nj[XX] + ni[YY] * nj[YY] + ni[ZZ] * nj[ZZ]);
    A[0][1] += val * ni[XX] * nj[YY] * third;
    A[0][2] += val * ni[XX] * nj[ZZ] * third;
    A[1][0] += val * ni[YY] * nj[XX] * third;
    A[1][1] += val * (ni[XX] * nj[XX] + T(4. / 3.) * ni[YY] * nj[YY] + ni[ZZ] * nj[ZZ]);
    A[1][2] += val * ni[YY] * nj[ZZ] * third;
    A[2][0] += val * ni[ZZ] * nj[XX] * third;
    A[2][1] += val * ni[ZZ] * nj[YY] * third;
    A[2][2] += val * (ni[XX] * nj[XX] + ni[YY] * nj[YY] + T(4. / 3.) * ni[ZZ] * nj[ZZ]);
    val = rho12;
    val += surho9 * u_ni;
    A[0][3] += nj[XX] * val; A[1][3] += nj[YY] * val; A[2][3] += nj[ZZ] * val;
    val = psrho9 * (ni[XX] * nj[XX] + ni[YY] * nj[YY] + ni[ZZ] * nj[ZZ]);
    A[3][3] += val;
    val = T(1. / 12.);
    A[3][0] += val * nj[XX]; A[3][1] += val * nj[YY]; A[3][2] += val * nj[ZZ];
    val = bulk9;
    A[0][0] += val * ni[XX] * nj[XX]; A[0][1] += val * ni[XX] * nj[YY];
    A[0][2] += val * ni[XX] * nj[ZZ]; A[1][0] += val * ni[YY] * nj[XX];
    A[1][1] += val * ni[YY] * nj[YY]; A[1][2] += val * ni[YY] * nj[ZZ];
    A[2][0] += val * ni[ZZ] * nj[XX]; A[2][1] += val * ni[ZZ] * nj[YY];
    A[2][2] += val * ni[ZZ] * nj[ZZ];
    val = v20 * (T(1) + (j == 0 ? T(1) : T(0)));
    val += su12 * u_ni;
    Tm[0][0] += val; Tm[1][1] += val; Tm[2][2] += val;
    val = ps12;
    Tm[3][0] += val * ni[XX]; Tm[3][1] += val * ni[YY]; Tm[3][2] += val * ni[ZZ];
    stage_block<3, T>(A, Tm, xs[j], kp, rhs, sk, j);
  }
  sk.template rhs<4>(rhs);
}

// Shared memory of one chunk: staged row blocks [value][incidence] (T), staged
// RHS rows, the permuted slot word of every incidence, per-row offsets, and one
// 64-bit contributor mask per (row, neighbour slot).
template <int D, typename T, int CH>
constexpr size_t assembly_smem_bytes() {
  return size_t(P1<D>::nvals + P1<D>::neq) * CH * sizeof(T) +  // st, rst
         size_t(CH) * 8 +                                     // s_mask (sum of row slots <= CH)
         size_t(CH) * 4 +                                     // s_info
         size_t(5 * CH + 3) * 4;                              // s_rowinc, s_pref, s_spref, s_slots, s_self
}

// The row-owner assembly kernel.  One CTA per chunk of whole block rows.
template <int D, typename T, int CH, bool SPEC>
__global__ void __launch_bounds__(CH) ns_assembly_kernel(
    const int2* __restrict__ chunk_rows, const int32_t* __restrict__ row_inc,
    const int32_t* __restrict__ inc_elem, const uint32_t* __restrict__ inc_info, const int4* __restrict__ conn,
    const double* __restrict__ coords, const double* __restrict__ uadv, const double* __restrict__ state,
    const float* __restrict__ node32, const double* __restrict__ force, const int64_t* __restrict__ start,
    NSParams p, double* __restrict__ vals,
    float* __restrict__ vals32, double* __restrict__ rhs) {
  constexpr int n = P1<D>::n, neq = P1<D>::neq, nvals = P1<D>::nvals;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* st = reinterpret_cast<T*>(smem_raw);
  T* rst = st + nvals * CH;
  unsigned long long* s_mask = reinterpret_cast<unsigned long long*>(rst + neq * CH);  // CH
  uint32_t* s_info = reinterpret_cast<uint32_t*>(s_mask + CH);                         // CH
  int* s_rowinc = reinterpret_cast<int*>(s_info + CH);                                 // CH + 1
  int* s_pref = s_rowinc + CH + 1;                                                     // CH + 1
  int* s_spref = s_pref + CH + 1;                                                      // CH + 1
  int* s_slots = s_spref + CH + 1;                                                     // CH
  int* s_self = s_slots + CH;                                                          // CH: slot of the row node

  const int2 cr = chunk_rows[blockIdx.x];
  const int row0 = cr.x, row1 = cr.y;
  const int R = row1 - row0;  // 1 <= R <= K <= CH (every node has an incidence)
  const int inc0 = row_inc[row0];
  const int K = row_inc[row1] - inc0;
  const int t = threadIdx.x;

  // Row metadata and zeroed contributor masks
  for (int rl = t; rl <= R; rl += CH) s_rowinc[rl] = row_inc[row0 + rl] - inc0;
  for (int rl = t; rl < R; rl += CH) s_slots[rl] = int(start[row0 + rl + 1] - start[row0 + rl]);
  for (int k = t; k < CH; k += CH) s_mask[k] = 0ull;
  __syncthreads();
  if (t == 0) {
    int items = 0, slots = 0;
    s_pref[0] = 0;
    s_spref[0] = 0;
    for (int rl = 0; rl < R; ++rl) {
      items += (s_slots[rl] - 1) * neq;  // off-diagonal blocks
      slots += s_slots[rl];
      s_pref[rl + 1] = items;
      s_spref[rl + 1] = slots;
    }
  }
  __syncthreads();

  // Phase 1: element row blocks, one thread per incidence.  The element's
  // nodes are relabelled by the even permutation k -> k ^ a (tetrahedra) or the
  // rotation k -> (k + a) mod 3 (triangles), which brings the row node to local
  // position 0 and leaves det J, the orientation and the symmetric order-2 Gauss
  // rules unchanged; the element routines then see a compile-time row index.
  if (t < K) {
    const int k = inc0 + t;
    const int e = __ldg(inc_elem + k);
    const uint32_t info = __ldg(inc_info + k);
    const int a = int(info >> 24) & 3;
    const int4 cn = __ldg(conn + e);
    const int ids0[4] = {cn.x, cn.y, cn.z, cn.w};
    int ids[4];
    uint32_t pslots = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int src = (D == 3) ? (q ^ a) : (q < 3 ? (q + a) % 3 : 3);
      ids[q] = ids0[src];
      const uint32_t sl = (q < n) ? ((info >> (6 * src)) & 63u) : 0xFFu;
      pslots |= sl << (8 * q);
    }
    s_info[t] = pslots;
    const KParams<T> kp = make_kparams<T>(p);
    const NodeData nd{coords, uadv, state, node32};
    StageSink<T> sk{st + t, rst + t, CH};
    if constexpr (SPEC) {
      if constexpr (D == 2) spec_tri_row<T>(ids, a, nd, kp, sk);
      else spec_tet_row<T>(ids, a, nd, kp, sk);
    } else {
      generic_row<D, T>(ids, a, nd, force, kp, sk);
    }
    // contributor masks: bit = position of this incidence within its row
    int lo = 0, hi = R - 1;
    while (lo < hi) {  // last rl with s_rowinc[rl] <= t
      const int mid = (lo + hi + 1) >> 1;
      if (s_rowinc[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const int bit = t - s_rowinc[lo];
    if (bit == 0) s_self[lo] = int(pslots & 0xFFu);  // relabelled node 0 is the row node
    if (bit < 64) {
      const int sb = s_spref[lo];
#pragma unroll
      for (int q = 1; q < n; ++q) {  // off-diagonal slots; the diagonal block takes every incidence
        unsigned* word = reinterpret_cast<unsigned*>(s_mask + sb + int((pslots >> (8 * q)) & 0xFFu)) + (bit >> 5);
        atomicOr(word, 1u << (bit & 31));
      }
    }
  }
  __syncthreads();

  // Phase 2a: off-diagonal CSR blocks, one thread per (row, equation,
  // neighbour slot != self); the slot's contributors are visited in ascending
  // element order.  Off-diagonal slots have a few contributors each, so the
  // warps stay converged; the diagonal blocks (every incidence of the row)
  // follow in phase 2b.
  const int nitems = s_pref[R];
  for (int it = t; it < nitems; it += CH) {
    int lo = 0, hi = R - 1;
    while (lo < hi) {  // last rl with s_pref[rl] <= it
      const int mid = (lo + hi + 1) >> 1;
      if (s_pref[mid] <= it) lo = mid; else hi = mid - 1;
    }
    const int rl = lo;
    const int S = s_slots[rl];
    const int local = it - s_pref[rl];
    const int r = local / (S - 1);
    const int s1 = local - r * (S - 1);
    const int s = s1 + (s1 >= s_self[rl] ? 1 : 0);
    const int kb = s_rowinc[rl], ke = s_rowinc[rl + 1];
    const uint32_t key = uint32_t(s) * 0x01010101u;
    double acc[neq];
#pragma unroll
    for (int c = 0; c < neq; ++c) acc[c] = 0.0;
    if (ke - kb <= 64) {
      unsigned long long m = s_mask[s_spref[rl] + s];
      while (m) {
        const int kk = kb + __ffsll(static_cast<long long>(m)) - 1;
        m &= m - 1;
        const int b = (__ffs(__vcmpeq4(s_info[kk], key)) - 1) >> 3;
        const T* src = st + ((b * neq + r) * neq) * CH + kk;
#pragma unroll
        for (int c = 0; c < neq; ++c) acc[c] += double(src[c * CH]);
      }
    } else {  // rows with more than 64 incident elements: scan
      for (int kk = kb; kk < ke; ++kk) {
        const uint32_t eq = __vcmpeq4(s_info[kk], key);
        if (eq) {
          const int b = (__ffs(eq) - 1) >> 3;
          const T* src = st + ((b * neq + r) * neq) * CH + kk;
#pragma unroll
          for (int c = 0; c < neq; ++c) acc[c] += double(src[c * CH]);
        }
      }
    }
    const int64_t base = int64_t(neq) * neq * start[row0 + rl] + int64_t(r * S + s) * neq;
#pragma unroll
    for (int c = 0; c < neq; ++c) vals[base + c] = acc[c];
    if (vals32 != nullptr) {
#pragma unroll
      for (int c = 0; c < neq; ++c) vals32[base + c] = float(acc[c]);
    }
  }
  // Phase 2b: diagonal blocks and RHS, one thread per (row, equation): every
  // incidence of the row contributes, with the row node at local position 0.
  for (int it = t; it < R * neq; it += CH) {
    const int rl = it / neq, r = it - rl * neq;
    const int kb = s_rowinc[rl], ke = s_rowinc[rl + 1];
    double acc[neq];
#pragma unroll
    for (int c = 0; c < neq; ++c) acc[c] = 0.0;
    double racc = 0.0;
    const T* src = st + (r * neq) * CH;  // b = 0
    for (int kk = kb; kk < ke; ++kk) {
#pragma unroll
      for (int c = 0; c < neq; ++c) acc[c] += double(src[c * CH + kk]);
      racc += double(rst[r * CH + kk]);
    }
    const int S = s_slots[rl];
    const int64_t base = int64_t(neq) * neq * start[row0 + rl] + int64_t(r * S + s_self[rl]) * neq;
#pragma unroll
    for (int c = 0; c < neq; ++c) vals[base + c] = acc[c];
    if (vals32 != nullptr) {
#pragma unroll
      for (int c = 0; c < neq; ++c) vals32[base + c] = float(acc[c]);
    }
    rhs[int64_t(row0 + rl) * neq + r] = racc;
  }
}

// ---------------------------------------------------------------------------
// Warp-per-row-group assembly.  A warp owns a range of consecutive block rows
// with at most 32 incidences in total; lane l evaluates incidence l of the
// range (incidences are sorted by row, then element id) and stages its element
// row block in the warp's shared-memory slice, value-major with a 33-element
// pitch (conflict-free for both the per-lane writes and the per-value reads).
// Contributor masks (bit = lane) are built with shared atomicOr, one word per
// neighbour slot.  The lanes then own CSR items: a diagonal entry or an RHS
// entry (sum over all lanes of the row) or an off-diagonal (row, equation,
// slot) quad (sum over the mask bits).  Lanes are visited in ascending order,
// i.e. every CSR value is the element-ordered sum of its contributions, as in
// the chunk kernel, and each value is written once.
// ---------------------------------------------------------------------------
// Lane pitch of the staging slice, in elements of T: 16-byte aligned rows
// whose quarter-warp 16-byte accesses hit distinct banks (3D), odd for the
// scalar accesses of the 2D layout.
template <int D, typename T>
constexpr int warp_lane_pitch() {
  return D == 3 ? (sizeof(T) == 4 ? 68 : 70) : 31;
}

constexpr size_t kDescSlot = (sizeof(AsmDesc) + 15) / 16 * 16;

// KC: lanes that evaluate incidences (group capacity); the staging holds KC lanes.
template <int D, typename T, int KC = 32, bool BATCH = false>
constexpr size_t warp_stage_bytes() {
  return size_t(KC) * warp_lane_pitch<D, T>() * sizeof(T) +  // staged row blocks + RHS rows, one slice per lane
         size_t(D * 64 + 32 + 36 + 36) * 4 +                  // slot masks per local position, pslots, prefix, offsets
         (BATCH ? 2 * kDescSlot : 0);                         // batch: descriptors of the current and next mesh
}
static_assert(warp_stage_bytes<2, float>() % 16 == 0 && warp_stage_bytes<2, double>() % 16 == 0 &&
                  warp_stage_bytes<3, float>() % 16 == 0 && warp_stage_bytes<3, double>() % 16 == 0 &&
                  warp_stage_bytes<3, float, 24>() % 16 == 0 && warp_stage_bytes<3, double, 24>() % 16 == 0 &&
                  warp_stage_bytes<2, float, 32, true>() % 16 == 0 && warp_stage_bytes<2, double, 32, true>() % 16 == 0 &&
                  warp_stage_bytes<3, float, 32, true>() % 16 == 0 && warp_stage_bytes<3, double, 32, true>() % 16 == 0,
              "per-warp staging slices must stay 16-byte aligned");

// Resident-CTA hints (register budgets) of the 24-lane tetrahedron variants:
// FP32 20 warps (<= 102 registers); FP64 14 warps, which with 4-warp CTAs asks
// for 3 CTAs (12 warps, no register cap: the variant's smaller staging then
// leaves more of the SM's shared/L1 array to the node-data gathers than the
// 32-lane kernel at the same warps) and with 2-warp CTAs for 7 (a 128-register
// budget that spills; the autotuner passes it over).  The 32-lane variants keep
// the compiler's choice (their staging caps the warps anyway).
template <int D, typename T, int KC, int WPB>
constexpr int warp_min_blocks() {
  if (D != 3 || KC == 32) return 0;  // 0: no hint
  const int warps = sizeof(T) == 8 ? 14 : 20;
  return warps / WPB > 0 ? warps / WPB : 1;
}

// Loads NV consecutive staged values (16-byte aligned when NV is a multiple of 4).
template <int NV, typename T>
__device__ __forceinline__ void load_run(const T* __restrict__ src, T (&v)[NV]) {
  if constexpr (NV % 4 == 0 && std::is_same<T, float>::value) {
#pragma unroll
    for (int q = 0; q < NV / 4; ++q) {
      const float4 x = reinterpret_cast<const float4*>(src)[q];
      v[4 * q] = x.x; v[4 * q + 1] = x.y; v[4 * q + 2] = x.z; v[4 * q + 3] = x.w;
    }
  } else if constexpr (NV % 2 == 0 && std::is_same<T, double>::value && NV % 4 == 0) {
#pragma unroll
    for (int q = 0; q < NV / 2; ++q) {
      const double2 x = reinterpret_cast<const double2*>(src)[q];
      v[2 * q] = x.x; v[2 * q + 1] = x.y;
    }
  } else {
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = src[q];
  }
}

template <int D, typename T, bool SPEC, int WPB, bool BATCH, int KC>
__global__ void __launch_bounds__(32 * WPB, warp_min_blocks<D, T, KC, WPB>()) ns_assembly_warp_kernel(
    int ngroups, int nmesh, const AsmDesc* __restrict__ descs, const int* __restrict__ gprefix,
    // one-mesh launch (BATCH false): the mesh's arrays as separate parameters
    const int4* __restrict__ groups_1, const int32_t* __restrict__ row_inc_1, const int32_t* __restrict__ inc_elem_1,
    const uint32_t* __restrict__ inc_info_1, const int4* __restrict__ conn_1, const double* __restrict__ coords_1,
    const double* __restrict__ uadv_1, const double* __restrict__ state_1, const float* __restrict__ node32_1,
    const double* __restrict__ force_1, const int64_t* __restrict__ start_1, NSParams p_1,
    double* __restrict__ vals_1, float* __restrict__ vals32_1, double* __restrict__ rhs_1) {
  constexpr int n = P1<D>::n, neq = P1<D>::neq, nvals = P1<D>::nvals;
  constexpr int LS = warp_lane_pitch<D, T>();
  constexpr int RPI = (D == 3) ? 2 : 3;      // equations (CSR rows) per off-diagonal item
  constexpr int RG = neq / RPI;              // items per (row, slot)
  constexpr int NV = RPI * neq;              // values per off-diagonal item
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* stage = reinterpret_cast<T*>(smem_raw + size_t(warp) * warp_stage_bytes<D, T, KC, BATCH>());
  uint32_t* s_mask = reinterpret_cast<uint32_t*>(stage + KC * LS);  // D x 64: local position 1..n-1, slot
  uint32_t* s_pslots = s_mask + D * 64;                              // 32
  int* s_pref = reinterpret_cast<int*>(s_pslots + 32);               // 33 (+3 pad)
  int* s_off = s_pref + 36;                                          // 33 (+3 pad): lane offset of each row
  // Mesh descriptors: a one-mesh launch reads its descriptor from the kernel
  // parameters; a batch keeps the descriptors of the current and the next
  // group's mesh in the warp's slice (copied when the mesh changes).
  AsmDesc* s_desc = reinterpret_cast<AsmDesc*>(reinterpret_cast<unsigned char*>(s_off + 36));
  int mesh0 = -1, mesh1 = -1;  // mesh held by descriptor slot 0 / 1
  auto load_desc = [&](int m, int slot) {
    if constexpr (BATCH) {
      const int held = slot ? mesh1 : mesh0;
      if (held != m) {  // warp-uniform
        constexpr int W = int(sizeof(AsmDesc) / 8);
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(descs + m);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(s_desc + slot);
        for (int q = lane; q < W; q += 32) dst[q] = __ldg(src + q);
        if (slot) mesh1 = m; else mesh0 = m;
        __syncwarp();
      }
    }
  };
  // Field f of the mesh in descriptor slot `slot`: a batch reads its shared
  // descriptor copy, a one-mesh launch its own parameters.
#define UFEM_F(slot, f) (BATCH ? s_desc[(slot)].f : f##_1)

  // Persistent warps: a warp walks the global groups g, g + stride, ... of all
  // meshes of the launch (mesh m owns groups [gprefix[m], gprefix[m + 1])).
  // While it reduces one group it already loads the incidence records
  // (element id, slot word) and the connectivity of the next, so the next
  // element phase starts with only the node gathers outstanding.
  int g = blockIdx.x * WPB + warp;
  if (g >= ngroups) return;  // whole warp; no CTA-wide barrier below
  const int gstride = gridDim.x * WPB;
  auto mesh_of = [&](int q) {  // last m with gprefix[m] <= q
    int lo = 0, hi = nmesh - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(gprefix + mid) <= q) lo = mid; else hi = mid - 1;
    }
    return lo;
  };
  int cm = BATCH ? mesh_of(g) : 0;
  int cs = 0;  // descriptor slot of the current mesh
  load_desc(cm, cs);
  // first row, end row, first incidence, incidences
  int4 G = BATCH ? __ldg(UFEM_F(cs, groups) + (g - __ldg(gprefix + cm))) : groups_1[g];
  int pe = 0, poff = 0, pitems = 0;
  uint32_t pinfo = 0;
  int4 pcn = make_int4(0, 0, 0, 0);
  auto fetch_records = [&](const int4& q, const int32_t* inc_elem, const uint32_t* inc_info,
                           const int32_t* row_inc, const int64_t* start) {
    if (lane < q.w) {
      pe = __ldg(inc_elem + q.z + lane);
      pinfo = __ldg(inc_info + q.z + lane);
    }
    if (lane < q.y - q.x) {
      poff = __ldg(row_inc + q.x + lane) - q.z;
      pitems = int(__ldg(start + q.x + lane + 1) - __ldg(start + q.x + lane) - 1) * RG;
    }
  };
  fetch_records(G, UFEM_F(cs, inc_elem), UFEM_F(cs, inc_info), UFEM_F(cs, row_inc), UFEM_F(cs, start));
  if (lane < G.w) pcn = __ldg(UFEM_F(cs, conn) + pe);
  for (;;) {
    const int row0 = G.x, R = G.y - G.x, K = G.w;  // 1 <= R <= K <= KC
    const int gn = g + gstride;
    const int mn = (BATCH && gn < ngroups) ? mesh_of(gn) : cm;
    const int ns = (mn == cm) ? cs : 1 - cs;  // descriptor slot of the next group's mesh
    int4 Gn = make_int4(0, 0, 0, 0);
    if constexpr (!BATCH) {
      if (gn < ngroups) Gn = groups_1[gn];
    }
    __syncwarp();  // the previous group's reads of the shared slice are complete
    if constexpr (BATCH) {
      load_desc(mn, ns);
      if (gn < ngroups) Gn = __ldg(s_desc[ns].groups + (gn - __ldg(gprefix + mn)));
    }
    const int64_t* __restrict__ start = UFEM_F(cs, start);
    int pref = lane < R ? pitems : 0;  // inclusive scan of the off-diagonal item counts
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(FULL, pref, o);
      if (lane >= o) pref += v;
    }
    const int nitems = __shfl_sync(FULL, pref, R - 1);
    if (lane < R) {
      s_pref[lane + 1] = pref;
      s_off[lane] = poff;
    }
    if (lane == 0) {
      s_pref[0] = 0;
      s_off[R] = K;
    }
#pragma unroll
    for (int q = 0; q < D * 2; ++q) s_mask[q * 32 + lane] = 0u;
    __syncwarp();

    // Phase 1: one lane per incidence; the row node is relabelled to local
    // position 0 exactly as in the chunk kernel.  Lane k stages its block
    // (local column node b, equation r, component c) at k*LS + (b*neq + r)*neq + c
    // and its RHS row at k*LS + nvals + r.
    uint32_t pslots = 0xFFFFFFFFu;
    if (lane < K) {
      const uint32_t info = pinfo;
      const int a = int(info >> 24) & 3;
      const int ids0[4] = {pcn.x, pcn.y, pcn.z, pcn.w};
      int ids[4];
      pslots = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int src = (D == 3) ? (q ^ a) : (q < 3 ? (q + a) % 3 : 3);
        ids[q] = ids0[src];
        const uint32_t sl = (q < n) ? ((info >> (6 * src)) & 63u) : 0xFFu;
        pslots |= sl << (8 * q);
      }
      T* st = stage + lane * LS;
      const KParams<T> kp = make_kparams<T>(UFEM_F(cs, p));
      const NodeData nd{UFEM_F(cs, coords), UFEM_F(cs, uadv), UFEM_F(cs, state), UFEM_F(cs, node32)};
      StageSink<T> sk{st, st + nvals, 1};
      if constexpr (SPEC) {
        if constexpr (D == 2) spec_tri_row<T>(ids, a, nd, kp, sk);
        else spec_tet_row<T>(ids, a, nd, kp, sk);
      } else {
        generic_row<D, T>(ids, a, nd, UFEM_F(cs, force), kp, sk);
      }
#pragma unroll
      for (int q = 1; q < n; ++q) atomicOr(s_mask + (q - 1) * 64 + ((pslots >> (8 * q)) & 0xFFu), 1u << lane);
    }
    s_pslots[lane] = pslots;
    __syncwarp();
    fetch_records(Gn, UFEM_F(ns, inc_elem), UFEM_F(ns, inc_info), UFEM_F(ns, row_inc),
                  UFEM_F(ns, start));  // next group's records load while this group is reduced
    double* __restrict__ vals = UFEM_F(cs, vals);
    float* __restrict__ vals32 = UFEM_F(cs, vals32);
    double* __restrict__ rhs = UFEM_F(cs, rhs);

    // Phase 2a: diagonal entries and RHS entries, neq * (neq + 1) items per row,
    // each the sum over the row's lanes in element order.
    constexpr int ND = neq * (neq + 1);
    for (int it = lane; it < R * ND; it += 32) {
      const int rl = it / ND, j = it - rl * ND;
      const int kb = s_off[rl], ke = s_off[rl + 1];  // lanes of row rl
      const int row = row0 + rl;
      const T* src = stage + (j < neq * neq ? j : nvals + (j - neq * neq));  // b = 0 block, or the RHS row
      double acc = 0.0;
#pragma unroll 8
      for (int k = kb; k < ke; ++k) acc += double(src[k * LS]);
      if (j < neq * neq) {
        const int r = j / neq, c = j - r * neq;
        const int64_t s0 = __ldg(start + row);
        const int S = int(__ldg(start + row + 1) - s0);
        const int self = int(s_pslots[kb] & 0xFFu);
        const int64_t pos = int64_t(neq) * neq * s0 + int64_t(r * S + self) * neq + c;
        __stcs(vals + pos, acc);  // streamed: keep L2 for the node data the element phase gathers
        if (vals32 != nullptr) __stcs(vals32 + pos, float(acc));
      } else {
        __stcs(rhs + int64_t(row) * neq + (j - neq * neq), acc);
      }
    }

    if (lane < Gn.w) pcn = __ldg(UFEM_F(ns, conn) + pe);

    // Phase 2b: off-diagonal items (row, slot != self, group of RPI equations):
    // the contributors of slot s are the row's lanes holding s at local position
    // b = 1..n-1, visited in ascending lane (= element) order.
    for (int it = lane; it < nitems; it += 32) {
      int lo = 0, hi = R - 1;
      while (lo < hi) {  // last rl with s_pref[rl] <= it
        const int mid = (lo + hi + 1) >> 1;
        if (s_pref[mid] <= it) lo = mid; else hi = mid - 1;
      }
      const int rl = lo;
      const int row = row0 + rl;
      const int64_t s0 = __ldg(start + row);
      const int S = int(__ldg(start + row + 1) - s0);
      const int local = it - s_pref[rl];
      const int s1 = local / RG;
      const int rg = local - s1 * RG;
      const int kb = s_off[rl], ke = s_off[rl + 1];
      const int self = int(s_pslots[kb] & 0xFFu);
      const int s = s1 + (s1 >= self ? 1 : 0);
      const unsigned rowmask = unsigned((1ull << ke) - (1ull << kb));
      const unsigned m1 = s_mask[s] & rowmask;
      const unsigned m2 = s_mask[64 + s] & rowmask;
      const unsigned m3 = (D == 3) ? (s_mask[128 + s] & rowmask) : 0u;
      unsigned m = m1 | m2 | m3;
      double acc[NV];
#pragma unroll
      for (int q = 0; q < NV; ++q) acc[q] = 0.0;
      while (m) {
        const int k = __ffs(m) - 1;
        m &= m - 1;
        const int b = 1 + int((m2 >> k) & 1u) + 2 * int((m3 >> k) & 1u);
        T v[NV];
        load_run<NV, T>(stage + k * LS + (b * neq + rg * RPI) * neq, v);
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] += double(v[q]);
      }
#pragma unroll
      for (int rr = 0; rr < RPI; ++rr) {
        const int r = rg * RPI + rr;
        const int64_t pos = int64_t(neq) * neq * s0 + int64_t(r * S + s) * neq;
        if constexpr (neq == 4) {
          __stcs(reinterpret_cast<double2*>(vals + pos), make_double2(acc[4 * rr], acc[4 * rr + 1]));
          __stcs(reinterpret_cast<double2*>(vals + pos) + 1, make_double2(acc[4 * rr + 2], acc[4 * rr + 3]));
          if (vals32 != nullptr)
            __stcs(reinterpret_cast<float4*>(vals32 + pos),
                   make_float4(float(acc[4 * rr]), float(acc[4 * rr + 1]), float(acc[4 * rr + 2]), float(acc[4 * rr + 3])));
        } else {
#pragma unroll
          for (int c = 0; c < neq; ++c) __stcs(vals + pos + c, acc[rr * neq + c]);
          if (vals32 != nullptr) {
#pragma unroll
            for (int c = 0; c < neq; ++c) __stcs(vals32 + pos + c, float(acc[rr * neq + c]));
          }
        }
      }
    }
    if (gn >= ngroups) break;
    g = gn;
    G = Gn;
    cm = mn;
    cs = ns;
  }
#undef UFEM_F
}

// LinearizeU (NavierStokes.cpp:105), evaluated left to right without FMA
// contraction: u_adv = ((2.1875u - 2.1875u1) + 1.3125u2) - 0.3125u3.  Also
// copies nu_eff into the node record read by the assembly.
__global__ void linearize_kernel(int64_t N, int dim, const double* __restrict__ state,
                                 const double* __restrict__ u1, const double* __restrict__ u2,
                                 const double* __restrict__ u3, const double* __restrict__ nu,
                                 double* __restrict__ uadv, float* __restrict__ node32) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double out[4] = {0, 0, 0, 0};
  for (int k = 0; k < dim; ++k) {
    const int64_t o = 4 * i + k;
    double v = __dsub_rn(__dmul_rn(2.1875, state[o]), __dmul_rn(2.1875, u1[o]));
    v = __dadd_rn(v, __dmul_rn(1.3125, u2[o]));
    v = __dsub_rn(v, __dmul_rn(0.3125, u3[o]));
    out[k] = v;
  }
  out[3] = nu[i];
  reinterpret_cast<double2*>(uadv + 4 * i)[0] = make_double2(out[0], out[1]);
  reinterpret_cast<double2*>(uadv + 4 * i)[1] = make_double2(out[2], out[3]);
  if (node32 != nullptr) {  // FP32 copy for the FP32 element path: (u_adv, nu), (u, p)
    float4* q = reinterpret_cast<float4*>(node32) + 2 * i;
    q[0] = make_float4(float(out[0]), float(out[1]), float(out[2]), float(out[3]));
    const double* x = state + 4 * i;
    q[1] = make_float4(float(x[0]), float(x[1]), dim == 3 ? float(x[2]) : 0.0f, float(x[dim]));
  }
}

// UpdateActions (NavierStokes.cpp:172-179): u3=u2, u2=u1, u1=u, u+=du, p+=dp.
__global__ void update_kernel(int64_t N, int dim, double* __restrict__ state, double* __restrict__ u1,
                              double* __restrict__ u2, double* __restrict__ u3, const double* __restrict__ sol) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int neq = dim + 1;
  for (int k = 0; k < dim; ++k) {
    const int64_t o = 4 * i + k;
    u3[o] = u2[o];
    u2[o] = u1[o];
    const double u = state[o];
    u1[o] = u;
    state[o] = __dadd_rn(u, sol[i * neq + k]);
  }
  state[4 * i + dim] = __dadd_rn(state[4 * i + dim], sol[i * neq + dim]);
}

// Point CSR from the node graph: row node*neq + r, columns adj*neq + c.
__global__ void build_csr_kernel(int64_t N, int neq, const int64_t* __restrict__ start,
                                 const int32_t* __restrict__ adj, int64_t* __restrict__ rowptr,
                                 int32_t* __restrict__ colidx, int64_t* __restrict__ diagpos) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int64_t s0 = start[i];
  const int S = int(start[i + 1] - s0);
  const int64_t base = int64_t(neq) * neq * s0;
  int self = 0;
  for (int s = 0; s < S; ++s)
    if (adj[s0 + s] == i) self = s;
  for (int r = 0; r < neq; ++r) {
    const int64_t rb = base + int64_t(r) * S * neq;
    rowptr[i * neq + r] = rb;
    diagpos[i * neq + r] = rb + int64_t(self) * neq + r;
    for (int s = 0; s < S; ++s) {
      const int32_t cn = adj[s0 + s] * neq;
      for (int c = 0; c < neq; ++c) colidx[rb + int64_t(s) * neq + c] = cn + c;
    }
  }
  if (i == N - 1) rowptr[N * neq] = int64_t(neq) * neq * start[N];
}

// Symmetric Dirichlet, part 1: per-step values v = value - old for the first
// and last application of every constrained dof.
__global__ void dirichlet_values_kernel(int64_t nbc, int neq, const int64_t* __restrict__ bc_dof,
                                        const double* __restrict__ first, const double* __restrict__ state,
                                        double* __restrict__ vfirst) {
  const int64_t u = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (u >= nbc) return;
  const int64_t dof = bc_dof[u];
  const int64_t node = dof / neq;
  const int comp = int(dof - node * neq);
  vfirst[u] = __dsub_rn(first[u], state[4 * node + comp]);
}

// Part 2: rows that are not constrained move their constrained columns to the
// RHS in first-application order (the order of the sequential reference).
// Eight lanes per row, four rows per warp: the lanes load eight of the row's
// constrained entries at a time, the terms are added to the RHS one by one in
// first-application order (the rounding of the sequential form: no FMA, no
// reassociation), then the lanes zero the entries.
__global__ void dirichlet_columns_kernel(int64_t nrows, const int64_t* __restrict__ fix_row,
                                         const int64_t* __restrict__ fix_ptr, const int64_t* __restrict__ fix_pos,
                                         const int32_t* __restrict__ fix_bc, const double* __restrict__ vfirst,
                                         double* __restrict__ vals, float* __restrict__ vals32,
                                         double* __restrict__ rhs) {
  constexpr unsigned FULL = 0xffffffffu;
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if ((t >> 5) * 4 >= nrows) return;  // whole warp
  const int64_t q = t >> 3;
  const int sub = int(t & 7), gbase = int(threadIdx.x & 31) & ~7;
  const bool valid = q < nrows;
  int64_t row = 0, k0 = 0;
  int len = 0;
  double r = 0.0;
  if (valid) {
    row = fix_row[q];
    k0 = fix_ptr[q];
    len = int(fix_ptr[q + 1] - k0);
    r = rhs[row];
  }
  int maxlen = len;  // the warp's longest row: every lane runs the same shuffles
  maxlen = max(maxlen, __shfl_xor_sync(FULL, maxlen, 8));
  maxlen = max(maxlen, __shfl_xor_sync(FULL, maxlen, 16));
  for (int kb = 0; kb < maxlen; kb += 8) {
    const int n = len - kb;  // this row's terms left
    double term = 0.0;
    int64_t pos = -1;
    if (sub < n) {
      pos = fix_pos[k0 + kb + sub];
      term = __dmul_rn(-vals[pos], vfirst[fix_bc[k0 + kb + sub]]);
    }
    for (int j = 0; j < 8; ++j) {  // added one by one, in first-application order
      const double tj = __shfl_sync(FULL, term, gbase + j);
      if (j < n) r = __dadd_rn(r, tj);
    }
    if (sub < n) {
      vals[pos] = 0.0;
      if (vals32) vals32[pos] = 0.0f;
    }
  }
  if (valid && sub == 0) rhs[row] = r;
}

// Part 3: constrained rows become identity rows; rhs = sol = last value - old.
// Eight lanes per constrained dof: the lanes zero the row (the diagonal entry is
// written 1 in the same pass, so no ordering between lanes is needed).
__global__ void dirichlet_rows_kernel(int64_t nbc, int neq, const int64_t* __restrict__ bc_dof,
                                      const double* __restrict__ last, const int64_t* __restrict__ bc_diag,
                                      const int64_t* __restrict__ rowptr, const double* __restrict__ state,
                                      double* __restrict__ vals, float* __restrict__ vals32,
                                      double* __restrict__ rhs, double* __restrict__ sol) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t u = t >> 3;  // eight lanes per constrained dof
  const int sub = int(t & 7);
  if (u >= nbc) return;
  const int64_t dof = bc_dof[u];
  const int64_t diag = bc_diag[u];
  for (int64_t p = rowptr[dof] + sub; p < rowptr[dof + 1]; p += 8) {
    const double v = (p == diag) ? 1.0 : 0.0;
    vals[p] = v;
    if (vals32) vals32[p] = float(v);
  }
  if (sub == 0) {
    const int64_t node = dof / neq;
    const int comp = int(dof - node * neq);
    const double v = __dsub_rn(last[u], state[4 * node + comp]);
    rhs[dof] = v;
    sol[dof] = v;
  }
}

}  // namespace

void fill_params(const ufem_ns_handle* h, NSParams& p) {
  const double dt = h->opt.dt, c1 = h->opt.c1;
  p.theta = h->opt.theta; p.inv_theta = 1.0 / h->opt.theta; p.dt = dt; p.invdt = 1.0 / dt;
  p.rho = h->opt.rho; p.inv_rho = 1.0 / h->opt.rho;
  p.tau_c1 = 4. * c1 * c1 / (dt * dt);  // SUPG.hpp:184
  p.tau_std = 4. / (dt * dt);           // SUPG.hpp:188
  p.two_dt = 2. / dt;                   // SUPG.hpp:169
  p.c2 = h->opt.c2; p.a_ps = h->opt.alpha_ps; p.a_su = h->opt.alpha_su;
  p.a_bu = h->opt.alpha_bu; p.u_ref = h->opt.u_ref; p.supg_type = h->opt.supg_type;
  p.has_force = h->d_force != nullptr;
}

void fill_desc(const ufem_ns_handle* h, bool write32, AsmDesc& d, const WarpPlan* plan) {
  d.coords = h->d_coords;
  d.uadv = h->d_uadv;
  d.state = h->d_state;
  d.node32 = h->d_node32;
  d.force = h->d_force;
  d.start = h->d_start;
  d.row_inc = h->d_row_inc;
  d.inc_elem = h->d_inc_elem;
  d.inc_info = h->d_inc_info;
  d.conn = reinterpret_cast<const int4*>(h->d_conn);
  d.groups = (plan ? plan : &h->wplan)->groups;
  d.vals = h->d_vals;
  d.vals32 = write32 ? h->d_vals32 : nullptr;
  d.rhs = h->d_rhs;
  fill_params(h, d.p);
}

namespace {

template <int D, typename T, int CH, bool SPEC>
int launch_chunk_t(const ufem_ns_handle* h, const AssemblyPlan& plan, const NSParams& p, cudaStream_t s,
                   bool write32) {
  if (plan.nchunks == 0) return UFEM_OK;
  constexpr size_t smem = assembly_smem_bytes<D, T, CH>();
  if (plan.cap != CH) return set_error(UFEM_ERR_STATE, "assembly plan does not match the kernel width");
  ns_assembly_kernel<D, T, CH, SPEC><<<plan.nchunks, CH, smem, s>>>(
      plan.chunks, h->d_row_inc, h->d_inc_elem, h->d_inc_info, reinterpret_cast<const int4*>(h->d_conn),
      h->d_coords, h->d_uadv, h->d_state, h->d_node32, h->d_force, h->d_start, p, h->d_vals,
      write32 ? h->d_vals32 : nullptr,
      h->d_rhs);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

// Resident CTAs of a kernel on the current device (persistent-warp grids).
template <typename K>
int resident_ctas(K kernel, int threads, size_t smem) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
    return 0;
  return sms * per_sm;
}

template <int D, typename T, bool SPEC, int WPB, bool BATCH, int KC>
int launch_warp_t(int ngroups, int nmesh, const AsmDesc* descs, const int* gprefix, const AsmDesc& one,
                  cudaStream_t s) {
  if (ngroups == 0) return UFEM_OK;
  constexpr size_t smem = warp_stage_bytes<D, T, KC, BATCH>() * WPB;
  static const int resident = resident_ctas(ns_assembly_warp_kernel<D, T, SPEC, WPB, BATCH, KC>, 32 * WPB, smem);
  if (resident <= 0) return set_error(UFEM_ERR_CUDA, "occupancy query of the warp assembly kernel failed");
  const unsigned grid = unsigned(std::min<int64_t>((ngroups + WPB - 1) / WPB, resident));
  ns_assembly_warp_kernel<D, T, SPEC, WPB, BATCH, KC><<<grid, 32 * WPB, smem, s>>>(
      ngroups, nmesh, descs, gprefix, one.groups, one.row_inc, one.inc_elem, one.inc_info, one.conn, one.coords,
      one.uadv, one.state, one.node32, one.force, one.start, one.p, one.vals, one.vals32, one.rhs);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

template <int D, typename T, bool SPEC, bool BATCH, int KC = 32>
int launch_warp_w(int warps, int ngroups, int nmesh, const AsmDesc* descs, const int* gprefix, const AsmDesc& one,
                  cudaStream_t s) {
  switch (warps) {
    case 2: return launch_warp_t<D, T, SPEC, 2, BATCH, KC>(ngroups, nmesh, descs, gprefix, one, s);
    case 8: return launch_warp_t<D, T, SPEC, 8, BATCH, KC>(ngroups, nmesh, descs, gprefix, one, s);
    default: return launch_warp_t<D, T, SPEC, 4, BATCH, KC>(ngroups, nmesh, descs, gprefix, one, s);
  }
}

template <int D, typename T, int CH, bool SPEC>
int launch_assembly_t(ufem_ns_handle* h, cudaStream_t s, bool write32) {
  NSParams p;
  fill_params(h, p);
  constexpr bool f32 = std::is_same<T, float>::value;
  if (h->asm_variant == kAsmChunk) return launch_chunk_t<D, T, CH, SPEC>(h, f32 ? h->plan32 : h->plan64, p, s, write32);
  int rc;
  const bool w24 = D == 3 && h->asm_variant == kAsmWarp24;
  const WarpPlan& wp = w24 ? h->wplan24 : h->wplan;
  AsmDesc one;  // this handle's descriptor, passed as a kernel parameter
  fill_desc(h, write32, one, &wp);
  if constexpr (D == 3) {
    if (w24) rc = launch_warp_w<D, T, SPEC, false, 24>(h->asm_warps, wp.ngroups, 1, nullptr, nullptr, one, s);
    else rc = launch_warp_w<D, T, SPEC, false, 32>(h->asm_warps, wp.ngroups, 1, nullptr, nullptr, one, s);
  } else {
    rc = launch_warp_w<D, T, SPEC, false, 32>(h->asm_warps, wp.ngroups, 1, nullptr, nullptr, one, s);
  }
  if (rc) return rc;
  return launch_chunk_t<D, T, CH, SPEC>(h, f32 ? wp.big32 : wp.big64, p, s, write32);
}

template <int D, typename T, bool SPEC, bool BATCH, int KC>
int set_warp_smem_attr() {
  UFEM_CUDA_TRY(cudaFuncSetAttribute(ns_assembly_warp_kernel<D, T, SPEC, 2, BATCH, KC>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(2 * warp_stage_bytes<D, T, KC, BATCH>())));
  UFEM_CUDA_TRY(cudaFuncSetAttribute(ns_assembly_warp_kernel<D, T, SPEC, 4, BATCH, KC>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(4 * warp_stage_bytes<D, T, KC, BATCH>())));
  UFEM_CUDA_TRY(cudaFuncSetAttribute(ns_assembly_warp_kernel<D, T, SPEC, 8, BATCH, KC>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(8 * warp_stage_bytes<D, T, KC, BATCH>())));
  return UFEM_OK;
}

template <int D, typename T, int CH, bool SPEC>
int set_smem_attr() {
  constexpr size_t smem = assembly_smem_bytes<D, T, CH>();
  UFEM_CUDA_TRY(cudaFuncSetAttribute(ns_assembly_kernel<D, T, CH, SPEC>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  int rc;
  if ((rc = set_warp_smem_attr<D, T, SPEC, false, 32>()) || (rc = set_warp_smem_attr<D, T, SPEC, true, 32>()))
    return rc;
  if constexpr (D == 3) {
    if ((rc = set_warp_smem_attr<D, T, SPEC, false, 24>())) return rc;
  }
  return UFEM_OK;
}

// ---------------------------------------------------------------------------
// Matrix-free FP64 residual.  The refinement residual of the mixed-precision
// solve when the element matrices are assembled in FP32: for the current
// increment dx, r = b - M dx of the FP64 system that the FP64 assembly and the
// symmetric Dirichlet conditions would have built, evaluated element by element
// without forming M.  Per incidence (row node, element) the FP64 element
// routines run with a sink that applies each row of M = invdt T + theta A
// (NavierStokesAssembly.hpp:69-71) to the element's increment instead of staging
// it, and keeps the RHS row a - A x (the reference's system_rhs += -_A _x + _a,
// :69); the rows' contributions are then summed in element order.
// Constrained columns take the value of their dof's first application (what the
// symmetric Dirichlet pass moves to the RHS), constrained rows get r = 0 (their
// increment already holds the row value, which the inner corrections keep).
// ---------------------------------------------------------------------------
template <int D>
struct ResidSink {
  double dl[D + 1][D + 1];  // increment of the relabelled element nodes (u, v, [w], p)
  double acc[D + 1];        // (M dx) of the row
  double rr[D + 1];         // a - A x of the row
  template <int NEQ>
  __device__ __forceinline__ void row(int idx, const double (&v)[NEQ]) {
    const int b = idx / (NEQ * NEQ), r = (idx / NEQ) % NEQ;
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < NEQ; ++c) s += v[c] * dl[b][c];
    acc[r] += s;
  }
  template <int NEQ>
  __device__ __forceinline__ void rhs(const double (&v)[NEQ]) {
#pragma unroll
    for (int r = 0; r < NEQ; ++r) rr[r] = v[r];
  }
};

// One CTA per chunk of whole rows (the chunk plan), one thread per incidence.
template <int D, int CH, bool SPEC>
__global__ void __launch_bounds__(CH) ns_residual_kernel(
    const int2* __restrict__ chunk_rows, const int32_t* __restrict__ row_inc, const int32_t* __restrict__ inc_elem,
    const uint32_t* __restrict__ inc_info, const int4* __restrict__ conn, const double* __restrict__ coords,
    const double* __restrict__ uadv, const double* __restrict__ state, const double* __restrict__ force, NSParams p,
    const double* __restrict__ dx, double* __restrict__ res) {
  constexpr int n = D + 1, neq = D + 1;
  __shared__ double s_res[neq * CH];
  __shared__ int s_rowinc[CH + 1];
  const int2 cr = chunk_rows[blockIdx.x];
  const int row0 = cr.x, R = cr.y - cr.x;  // 1 <= R <= K <= CH
  const int inc0 = row_inc[row0];
  const int K = row_inc[cr.y] - inc0;
  const int t = threadIdx.x;
  for (int rl = t; rl <= R; rl += CH) s_rowinc[rl] = row_inc[row0 + rl] - inc0;
  if (t < K) {
    const int k = inc0 + t;
    const int e = __ldg(inc_elem + k);
    const int a = int(__ldg(inc_info + k) >> 24) & 3;
    const int4 cn = __ldg(conn + e);
    const int ids0[4] = {cn.x, cn.y, cn.z, cn.w};
    int ids[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) ids[q] = ids0[(D == 3) ? (q ^ a) : (q < 3 ? (q + a) % 3 : 3)];
    ResidSink<D> sk;
#pragma unroll
    for (int q = 0; q < n; ++q)
#pragma unroll
      for (int c = 0; c < neq; ++c) sk.dl[q][c] = __ldg(dx + int64_t(ids[q]) * neq + c);
#pragma unroll
    for (int r = 0; r < neq; ++r) sk.acc[r] = 0.0;
    const KParams<double> kp = make_kparams<double>(p);
    const NodeData nd{coords, uadv, state, nullptr};
    if constexpr (SPEC) {
      if constexpr (D == 2) spec_tri_row<double>(ids, a, nd, kp, sk);
      else spec_tet_row<double>(ids, a, nd, kp, sk);
    } else {
      generic_row<D, double>(ids, a, nd, force, kp, sk);
    }
#pragma unroll
    for (int r = 0; r < neq; ++r) s_res[r * CH + t] = sk.rr[r] - sk.acc[r];
  }
  __syncthreads();
  for (int it = t; it < R * neq; it += CH) {  // sums over the row's incidences in element order
    const int rl = it / neq, r = it - rl * neq;
    double acc = 0.0;
    for (int kk = s_rowinc[rl]; kk < s_rowinc[rl + 1]; ++kk) acc += s_res[r * CH + kk];
    res[int64_t(row0 + rl) * neq + r] = acc;
  }
}

// dx' = dx with each constrained dof replaced by its first application's value
// (value - old), the column value the symmetric Dirichlet pass moves to the RHS.
__global__ void mf_columns_kernel(int64_t nbc, const int64_t* __restrict__ bc_dof, const double* __restrict__ vfirst,
                                  double* __restrict__ dxp) {
  const int64_t u = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (u < nbc) dxp[bc_dof[u]] = vfirst[u];
}

__global__ void mf_rows_kernel(int64_t nbc, const int64_t* __restrict__ bc_dof, double* __restrict__ res) {
  const int64_t u = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (u < nbc) res[bc_dof[u]] = 0.0;
}

template <int D, int CH, bool SPEC>
int launch_residual_t(ufem_ns_handle* h, const double* dxp, double* res, cudaStream_t s) {
  NSParams p;
  fill_params(h, p);
  if (h->plan64.cap != CH) return set_error(UFEM_ERR_STATE, "chunk plan does not match the residual kernel width");
  ns_residual_kernel<D, CH, SPEC><<<h->plan64.nchunks, CH, 0, s>>>(
      h->plan64.chunks, h->d_row_inc, h->d_inc_elem, h->d_inc_info, reinterpret_cast<const int4*>(h->d_conn),
      h->d_coords, h->d_uadv, h->d_state, h->d_force, p, dxp, res);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

constexpr int kChunk2D = 256;
constexpr int kChunk3D64 = 128;
constexpr int kChunk3D32 = 256;

}  // namespace

int assembly_chunk_capacity(int dim, int precision) {
  if (dim == 2) return kChunk2D;
  return precision == 1 ? kChunk3D32 : kChunk3D64;
}

int configure_kernels() {
  static bool done = false;
  if (done) return UFEM_OK;
  int rc;
  if ((rc = set_smem_attr<2, double, kChunk2D, false>())) return rc;
  if ((rc = set_smem_attr<2, double, kChunk2D, true>())) return rc;
  if ((rc = set_smem_attr<2, float, kChunk2D, false>())) return rc;
  if ((rc = set_smem_attr<2, float, kChunk2D, true>())) return rc;
  if ((rc = set_smem_attr<3, double, kChunk3D64, false>())) return rc;
  if ((rc = set_smem_attr<3, double, kChunk3D64, true>())) return rc;
  if ((rc = set_smem_attr<3, float, kChunk3D32, false>())) return rc;
  if ((rc = set_smem_attr<3, float, kChunk3D32, true>())) return rc;
  done = true;
  return UFEM_OK;
}

int launch_assembly(ufem_ns_handle* h, cudaStream_t s, bool write32) {
  const bool spec = h->opt.use_specializations != 0;
  const bool f32 = h->opt.precision == 1;
  if (h->dim == 2) {
    if (f32) return spec ? launch_assembly_t<2, float, kChunk2D, true>(h, s, write32)
                         : launch_assembly_t<2, float, kChunk2D, false>(h, s, write32);
    return spec ? launch_assembly_t<2, double, kChunk2D, true>(h, s, write32)
                : launch_assembly_t<2, double, kChunk2D, false>(h, s, write32);
  }
  if (f32) return spec ? launch_assembly_t<3, float, kChunk3D32, true>(h, s, write32)
                       : launch_assembly_t<3, float, kChunk3D32, false>(h, s, write32);
  return spec ? launch_assembly_t<3, double, kChunk3D64, true>(h, s, write32)
              : launch_assembly_t<3, double, kChunk3D64, false>(h, s, write32);
}

int launch_assembly_batch(int dim, int precision, bool spec, int warps, int ngroups, int nmesh,
                          const AsmDesc* d_descs, const int* d_gprefix, cudaStream_t s) {
  const bool f32 = precision == 1;
  if (dim == 2) {
    if (f32) return spec ? launch_warp_w<2, float, true, true>(warps, ngroups, nmesh, d_descs, d_gprefix, AsmDesc{}, s)
                         : launch_warp_w<2, float, false, true>(warps, ngroups, nmesh, d_descs, d_gprefix, AsmDesc{}, s);
    return spec ? launch_warp_w<2, double, true, true>(warps, ngroups, nmesh, d_descs, d_gprefix, AsmDesc{}, s)
                : launch_warp_w<2, double, false, true>(warps, ngroups, nmesh, d_descs, d_gprefix, AsmDesc{}, s);
  }
  if (f32) return spec ? launch_warp_w<3, float, true, true>(warps, ngroups, nmesh, d_descs, d_gprefix, AsmDesc{}, s)
                       : launch_warp_w<3, float, false, true>(warps, ngroups, nmesh, d_descs, d_gprefix, AsmDesc{}, s);
  return spec ? launch_warp_w<3, double, true, true>(warps, ngroups, nmesh, d_descs, d_gprefix, AsmDesc{}, s)
              : launch_warp_w<3, double, false, true>(warps, ngroups, nmesh, d_descs, d_gprefix, AsmDesc{}, s);
}

int launch_assembly_big_rows(ufem_ns_handle* h, cudaStream_t s, bool write32) {
  NSParams p;
  fill_params(h, p);
  const bool spec = h->opt.use_specializations != 0;
  const bool f32 = h->opt.precision == 1;
  const WarpPlan& w = h->wplan;
  if (h->dim == 2) {
    if (f32) return spec ? launch_chunk_t<2, float, kChunk2D, true>(h, w.big32, p, s, write32)
                         : launch_chunk_t<2, float, kChunk2D, false>(h, w.big32, p, s, write32);
    return spec ? launch_chunk_t<2, double, kChunk2D, true>(h, w.big64, p, s, write32)
                : launch_chunk_t<2, double, kChunk2D, false>(h, w.big64, p, s, write32);
  }
  if (f32) return spec ? launch_chunk_t<3, float, kChunk3D32, true>(h, w.big32, p, s, write32)
                       : launch_chunk_t<3, float, kChunk3D32, false>(h, w.big32, p, s, write32);
  return spec ? launch_chunk_t<3, double, kChunk3D64, true>(h, w.big64, p, s, write32)
              : launch_chunk_t<3, double, kChunk3D64, false>(h, w.big64, p, s, write32);
}

int launch_linearize(ufem_ns_handle* h, cudaStream_t s) {
  const int64_t N = h->N;
  const double* u1 = h->d_hist;
  const double* u2 = h->d_hist + 4 * N;
  const double* u3 = h->d_hist + 8 * N;
  linearize_kernel<<<unsigned((N + 255) / 256), 256, 0, s>>>(N, h->dim, h->d_state, u1, u2, u3, h->d_nu, h->d_uadv,
                                                            h->opt.precision == 1 ? h->d_node32 : nullptr);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

int launch_update(ufem_ns_handle* h, cudaStream_t s) {
  const int64_t N = h->N;
  update_kernel<<<unsigned((N + 255) / 256), 256, 0, s>>>(N, h->dim, h->d_state, h->d_hist, h->d_hist + 4 * N,
                                                        h->d_hist + 8 * N, h->d_sol);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

int launch_build_csr(ufem_ns_handle* h, cudaStream_t s) {
  const int64_t N = h->N;
  build_csr_kernel<<<unsigned((N + 127) / 128), 128, 0, s>>>(N, h->neq, h->d_start, h->d_adj, h->d_rowptr,
                                                           h->d_colidx, h->d_diagpos);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

// Tie rows of linked (periodic) nodes, after the assembly: the element
// contributions at a slave node were assembled into its master's rows and
// columns; the slave's own rows become x_slave - x_master = 0 (identity block
// at the slave, minus identity at the master, rhs 0), so the solution and the
// update give the slave its master's values.
__global__ void tie_rows_kernel(int64_t ntie, int neq, const int32_t* __restrict__ tie,
                                const int64_t* __restrict__ start, const int32_t* __restrict__ adj,
                                double* __restrict__ vals, float* __restrict__ vals32, double* __restrict__ rhs) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= ntie) return;
  const int sl = tie[2 * t], ms = tie[2 * t + 1];
  const int64_t s0 = start[sl];
  const int S = int(start[sl + 1] - s0);
  for (int r = 0; r < neq; ++r) {
    const int64_t rs = int64_t(neq) * neq * s0 + int64_t(r) * S * neq;
    for (int k = 0; k < S; ++k) {
      const int col = adj[s0 + k];
      for (int c = 0; c < neq; ++c) {
        const double v = (c != r) ? 0.0 : (col == sl ? 1.0 : (col == ms ? -1.0 : 0.0));
        vals[rs + k * neq + c] = v;
        if (vals32 != nullptr) vals32[rs + k * neq + c] = float(v);
      }
    }
    rhs[int64_t(sl) * neq + r] = 0.0;
  }
}

int launch_tie_rows(ufem_ns_handle* h, cudaStream_t s, bool write32) {
  if (h->ntie == 0) return UFEM_OK;
  tie_rows_kernel<<<unsigned((h->ntie + 127) / 128), 128, 0, s>>>(h->ntie, h->neq, h->d_tie, h->d_start, h->d_adj,
                                                                  h->d_vals, write32 ? h->d_vals32 : nullptr,
                                                                  h->d_rhs);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

// rhs[dof] += contributions of the constant Neumann faces, in face order.
__global__ void neumann_kernel(int64_t n, const int64_t* __restrict__ dof, const int64_t* __restrict__ ptr,
                               const double* __restrict__ val, double* __restrict__ rhs) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double r = rhs[dof[i]];
  for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k) r = __dadd_rn(r, val[k]);
  rhs[dof[i]] = r;
}

int launch_neumann(ufem_ns_handle* h, cudaStream_t s) {
  const DirichletPlan& bp = h->bcp;
  if (bp.nneu == 0) return UFEM_OK;
  neumann_kernel<<<unsigned((bp.nneu + 255) / 256), 256, 0, s>>>(bp.nneu, bp.neu_dof, bp.neu_ptr, bp.neu_val,
                                                                  h->d_rhs);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

int launch_dirichlet(ufem_ns_handle* h, cudaStream_t s) {
  const DirichletPlan& bp = h->bcp;
  if (bp.nbc == 0) return UFEM_OK;
  dirichlet_values_kernel<<<unsigned((bp.nbc + 255) / 256), 256, 0, s>>>(bp.nbc, h->neq, bp.bc_dof, bp.bc_first,
                                                                         h->d_state, bp.vfirst);
  UFEM_CUDA_TRY(cudaGetLastError());
  if (bp.nfix_rows > 0) {
    dirichlet_columns_kernel<<<unsigned((bp.nfix_rows * 8 + 255) / 256), 256, 0, s>>>(
        bp.nfix_rows, bp.fix_row, bp.fix_ptr, bp.fix_pos, bp.fix_bc, bp.vfirst, h->d_vals, h->d_vals32, h->d_rhs);
    UFEM_CUDA_TRY(cudaGetLastError());
  }
  dirichlet_rows_kernel<<<unsigned((bp.nbc * 8 + 255) / 256), 256, 0, s>>>(bp.nbc, h->neq, bp.bc_dof, bp.bc_last,
                                                                            bp.bc_diag,
                                                        h->d_rowptr, h->d_state, h->d_vals, h->d_vals32, h->d_rhs,
                                                        h->d_sol);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

}  // namespace ufem

namespace ufem {

int launch_mf_residual(ufem_ns_handle* h, double* dx_work, double* res, cudaStream_t s) {
  if (h->ntie > 0)
    return set_error(UFEM_ERR_ARG, "the matrix-free FP64 residual does not support periodic node links");
  const DirichletPlan& bp = h->bcp;
  UFEM_CUDA_TRY(cudaMemcpyAsync(dx_work, h->d_sol, size_t(h->nrows) * 8, cudaMemcpyDeviceToDevice, s));
  if (bp.nbc > 0) {
    mf_columns_kernel<<<unsigned((bp.nbc + 255) / 256), 256, 0, s>>>(bp.nbc, bp.bc_dof, bp.vfirst, dx_work);
    UFEM_CUDA_TRY(cudaGetLastError());
  }
  const bool spec = h->opt.use_specializations != 0;
  int rc;
  if (h->dim == 2)
    rc = spec ? launch_residual_t<2, kChunk2D, true>(h, dx_work, res, s) : launch_residual_t<2, kChunk2D, false>(h, dx_work, res, s);
  else
    rc = spec ? launch_residual_t<3, kChunk3D64, true>(h, dx_work, res, s)
              : launch_residual_t<3, kChunk3D64, false>(h, dx_work, res, s);
  if (rc) return rc;
  if (bp.nneu > 0) {
    neumann_kernel<<<unsigned((bp.nneu + 255) / 256), 256, 0, s>>>(bp.nneu, bp.neu_dof, bp.neu_ptr, bp.neu_val, res);
    UFEM_CUDA_TRY(cudaGetLastError());
  }
  if (bp.nbc > 0) {
    mf_rows_kernel<<<unsigned((bp.nbc + 255) / 256), 256, 0, s>>>(bp.nbc, bp.bc_dof, res);
    UFEM_CUDA_TRY(cudaGetLastError());
  }
  return UFEM_OK;
}

}  // namespace ufem
