// element.cuh -- P1 element helpers shared by the Navier-Stokes kernels (coupled
// and semi-implicit): geometry, stabilisation coefficients, Gauss points.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "internal.h"

namespace ufem {
namespace {

template <int D>
struct P1 {
  static constexpr int n = D + 1;           // nodes per element
  static constexpr int neq = D + 1;         // u, v, [w], p
  static constexpr int nvals = n * neq * neq;  // one element row block
};

template <typename T>
struct KParams {
  T theta, inv_theta, dt, invdt, rho, inv_rho, c2, a_ps, a_su, a_bu, u_ref;
  T tau_c1, tau_std, two_dt;  // 4 c1^2 / dt^2, 4 / dt^2, 2 / dt (computed on the host in FP64)
  int supg_type, has_force;
};

template <typename T>
__device__ __forceinline__ KParams<T> make_kparams(const NSParams& p) {
  KParams<T> k;
  k.theta = T(p.theta); k.inv_theta = T(p.inv_theta); k.dt = T(p.dt); k.invdt = T(p.invdt); k.rho = T(p.rho);
  k.inv_rho = T(p.inv_rho); k.tau_c1 = T(p.tau_c1); k.tau_std = T(p.tau_std); k.two_dt = T(p.two_dt);
  k.c2 = T(p.c2); k.a_ps = T(p.a_ps); k.a_su = T(p.a_su); k.a_bu = T(p.a_bu);
  k.u_ref = T(p.u_ref); k.supg_type = p.supg_type; k.has_force = p.has_force;
  return k;
}

__device__ __forceinline__ double tsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float tsqrt(float x) { return sqrtf(x); }
// 1/sqrt(x) and 1/x through CUDA's reciprocal square root and correctly rounded
// reciprocal: one short dependent sequence each instead of a square root or
// a division followed by another (the element routines are latency-bound)
__device__ __forceinline__ double trsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float trsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double trcp(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float trcp(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double tabs(double x) { return fabs(x); }
__device__ __forceinline__ float tabs(float x) { return fabsf(x); }
__device__ __forceinline__ double tcbrt_pow(double x) { return pow(x, 1. / 3.); }
__device__ __forceinline__ float tcbrt_pow(float x) { return powf(x, 1.f / 3.f); }

// Runtime selection of a[i] for a compile-time-sized array without local memory.
template <int M, typename T>
__device__ __forceinline__ T sel(const T (&arr)[M], int i) {
  T r = arr[0];
#pragma unroll
  for (int k = 1; k < M; ++k)
    if (i == k) r = arr[k];
  return r;
}

__device__ __forceinline__ void ld4(const double* __restrict__ p, double& a, double& b, double& c, double& d) {
  const double2 x = __ldg(reinterpret_cast<const double2*>(p));
  const double2 y = __ldg(reinterpret_cast<const double2*>(p) + 1);
  a = x.x; b = x.y; c = y.x; d = y.y;
}

// Inverse and determinant in the cofactor form (Proto/ElementData.hpp:308-314).
template <typename T>
__device__ __forceinline__ void inverse_det(const T (&J)[2][2], T (&Ji)[2][2], T& det) {
  det = J[0][0] * J[1][1] - J[1][0] * J[0][1];
  const T inv = trcp(det);
  Ji[0][0] = J[1][1] * inv;
  Ji[1][0] = -J[1][0] * inv;
  Ji[0][1] = -J[0][1] * inv;
  Ji[1][1] = J[0][0] * inv;
}
template <typename T>
__device__ __forceinline__ void inverse_det(const T (&m)[3][3], T (&Ji)[3][3], T& det) {
  T cof[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      cof[i][j] = m[i1][j1] * m[i2][j2] - m[i1][j2] * m[i2][j1];
    }
  det = (cof[0][0] * m[0][0] + cof[1][0] * m[1][0]) + cof[2][0] * m[2][0];
  const T inv = trcp(det);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) Ji[j][i] = cof[i][j] * inv;
}

// Element data in the arithmetic type T.  Coordinates are made relative to the
// element's node 0 in FP64 before any conversion, so the FP32 path keeps the
// geometry at full relative accuracy.
template <int D, typename T>
struct Elem {
  T Xr[D + 1][D];
  T U[D + 1][D];   // u_adv
  T NU[D + 1];     // nu_eff
};

// Nodal inputs of the element routines.  FP64 element arithmetic reads the
// FP64 node records; the FP32 path reads node32, an FP32 copy of
// (u_adv, nu_eff, u, p) per node written by the linearisation kernel (the same
// round-to-nearest values a conversion here would give), and keeps only the
// coordinates in FP64 so that differences are formed before rounding.
struct NodeData {
  const double* coords;  // N x 4
  const double* uadv;    // N x 4 (u_adv, nu_eff)
  const double* state;   // N x 4 (u, p)
  const float* node32;   // N x 8 (u_adv, nu_eff, u, p), FP32 path only
};

template <int D, typename T>
__device__ __forceinline__ void gather_geometry_uadv(const int (&ids)[4], const NodeData& nd, Elem<D, T>& el) {
  double X0[4];
  ld4(nd.coords + 4ll * ids[0], X0[0], X0[1], X0[2], X0[3]);
#pragma unroll
  for (int b = 0; b <= D; ++b) {
    double x[4];
    ld4(nd.coords + 4ll * ids[b], x[0], x[1], x[2], x[3]);
#pragma unroll
    for (int k = 0; k < D; ++k) el.Xr[b][k] = T(x[k] - X0[k]);
    if constexpr (std::is_same<T, float>::value) {
      const float4 u = __ldg(reinterpret_cast<const float4*>(nd.node32) + 2ll * ids[b]);
      const float uu[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
      for (int k = 0; k < D; ++k) el.U[b][k] = uu[k];
      el.NU[b] = u.w;
    } else {
      double u[4];
      ld4(nd.uadv + 4ll * ids[b], u[0], u[1], u[2], u[3]);
#pragma unroll
      for (int k = 0; k < D; ++k) el.U[b][k] = T(u[k]);
      el.NU[b] = T(u[3]);
    }
  }
}

// Metric tensor of the METRIC tau, g = J^-T J^-1 = [grad xi_m . grad xi_n], in
// the reference frame of the element's OWN node order (xi_m is the shape
// function of original local node m+1).  The caller has relabelled the nodes
// (row node first): original local node k sits at position k ^ a (tetrahedra)
// or (k - a) mod 3 (triangles), and G holds the gradients in the relabelled
// order.  g depends on the node order, so it is rebuilt from the original one.
template <int D, typename T>
__device__ __forceinline__ void metric_tensor(const T (&G)[D][D + 1], int a, T (&g)[D][D]) {
  T col[D][D];
#pragma unroll
  for (int m = 0; m < D; ++m) {
    const int k = m + 1;
    const int pos = (D == 3) ? (k ^ a) : ((k - a + 3) % 3);
#pragma unroll
    for (int r = 0; r < D; ++r) col[m][r] = sel<D + 1>(G[r], pos);
  }
#pragma unroll
  for (int m = 0; m < D; ++m)
#pragma unroll
    for (int q = m; q < D; ++q) {  // symmetric: the same products in the same order
      T s = 0;
#pragma unroll
      for (int r = 0; r < D; ++r) s += col[m][r] * col[q][r];
      g[m][q] = s;
      g[q][m] = s;
    }
}

// ComputeTauImpl::compute_coefficients (SUPG.hpp:140-219).  G: node gradients
// (any order), g: metric tensor in the element's own frame, det: det J.
template <int D, typename T>
__device__ __forceinline__ void compute_tau(const KParams<T>& kp, const Elem<D, T>& el, const T (&uc)[D],
                                            T element_nu, const T (&G)[D][D + 1], const T (&g)[D][D], T det,
                                            T& tps, T& tsu, T& tbu) {
  constexpr int n = D + 1;
  const int type = kp.supg_type;
  const T c2 = kp.c2, u_ref = kp.u_ref, dt = kp.dt;
  if (type == 0) {  // TEZDUYAR
    T h = T(1e10);
#pragma unroll
    for (int i = 0; i < n; ++i)
#pragma unroll
      for (int j = 0; j < n; ++j)
        if (i != j) {
          T s = 0;
#pragma unroll
          for (int k = 0; k < D; ++k) { const T d = el.Xr[i][k] - el.Xr[j][k]; s += d * d; }
          h = s < h ? s : h;
        }
    h = tsqrt(h);
    T um2 = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) um2 += uc[k] * uc[k];
    const T umag = tsqrt(um2);
    tsu = T(1) / ((T(2) * umag) / h + kp.two_dt + (T(4) * element_nu) / (h * h));
    tps = tsu;
    tbu = tsu * umag * umag;
  } else if (type == 1) {  // METRIC
    T adv = 0, sq = 0, tr = 0;
#pragma unroll
    for (int b = 0; b < D; ++b) {
      T s = 0;
#pragma unroll
      for (int a = 0; a < D; ++a) s += uc[a] * g[a][b];
      adv += s * uc[b];
    }
#pragma unroll
    for (int a = 0; a < D; ++a) {
      tr += g[a][a];
#pragma unroll
      for (int b = 0; b < D; ++b) sq += g[a][b] * g[a][b];
    }
    const T adv_sq = tabs(adv);
    const T diff = element_nu * element_nu * sq;
    tsu = trsqrt(kp.tau_c1 + adv_sq + c2 * diff);  // tau_c1 = 4 c1^2 / dt^2
    tps = tsu;
    // 1 / tau_su of the standard constants (tau_std = 4 / dt^2)
    tbu = tsqrt(kp.tau_std + adv_sq + T(16) * diff) * trcp(tr);
  } else {  // CF2
    const T volume = (D == 2) ? det / T(2) : det / T(6);
    const T pi = T(3.141592654);
    const T he = (D == 2) ? tsqrt(T(4) / pi * volume) : tcbrt_pow(T(3) / T(4) / pi * volume);
    const T ree = u_ref * he / (T(2) * element_nu);
    const T xi = ree < T(3) ? ree / T(3) : T(1);
    tps = he * xi / (T(2) * u_ref);
    tbu = he * u_ref / xi;
    tsu = 0;
    T um2 = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) um2 += uc[k] * uc[k];
    const T umag = tsqrt(um2);
    if (umag > T(1e-10)) {
      // sum over nodes of u . grad N_b (a rounding-level number for P1)
      T s = 0;
#pragma unroll
      for (int b = 0; b <= D; ++b) {
        T t = 0;
#pragma unroll
        for (int k = 0; k < D; ++k) t += uc[k] * G[k][b];
        s += t;
      }
      const T h = T(2) * umag / s;
      const T tau_adv = h / (T(2) * umag);
      const T tau_time = T(0.5) * dt;
      const T tau_diff = h * h / (T(4) * element_nu);
      tsu = T(1) / (T(1) / tau_adv + T(1) / tau_time + T(1) / tau_diff);
    }
  }
  tps *= kp.a_ps;
  tsu *= kp.a_su;
  tbu *= kp.a_bu;
}

template <int D, typename T>
__device__ __forceinline__ void centroid_N(T (&Nc)[D + 1]) {
  const T mu = (D == 2) ? T(0.3333333333333333333333333) : T(0.25);
  T s = 1;
#pragma unroll
  for (int k = 0; k < D; ++k) s -= mu;
  Nc[0] = s;
#pragma unroll
  for (int k = 1; k <= D; ++k) Nc[k] = mu;
}

// Order-2 Gauss points (GaussImplementation.hpp:195-226 and :395-428).
template <int D, typename T>
__device__ __forceinline__ void gauss_N(int q, T (&N)[D + 1]) {
  T xi[D];
  if (D == 2) {
    const T p[3][2] = {{T(0.5), T(0.0)}, {T(0.5), T(0.5)}, {T(0.0), T(0.5)}};
#pragma unroll
    for (int k = 0; k < D; ++k) xi[k] = p[q][k];
  } else {
    const T mu = T(0.13819660112501051517954131656);
#pragma unroll
    for (int k = 0; k < D; ++k) xi[k] = mu;
    if (q > 0) xi[q - 1] = T(1) - T(3) * mu;
  }
  T s = 1;
#pragma unroll
  for (int k = 0; k < D; ++k) s -= xi[k];
  N[0] = s;
#pragma unroll
  for (int k = 0; k < D; ++k) N[k + 1] = xi[k];
}

}  // namespace
}  // namespace ufem
