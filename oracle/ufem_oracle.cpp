// ufem_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the parity oracle).
//
// A serial FP64 CPU restatement of COOLFluiD 3's UFEM Navier-Stokes time step
// (ZeroLSS -> LinearizeU -> Assembly -> symmetric Dirichlet -> solve -> update),
// written from the reference sources cited per function below.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library; the
// product (coolfluid3_b200) never links, loads or calls it.
//
// Parity status: the reference cannot be compiled in this environment (Boost,
// Eigen3, Trilinos and MPI are absent), and the reference repository holds no
// numeric golden vectors for NS element matrices (its spec-vs-generic test is
// commented out, plugins/UFEM/test/utest-proto-ns-assembly.cpp:158-203).  The
// element arithmetic is therefore "parity unpinned" against reference outputs;
// what IS pinned against the reference's own tests: the sparsity structure
// (utest-ufem-buildsparsity.cpp:99-101), the symmetric-Dirichlet known-answer
// test (test/math/utest-lss-symmetric-dirichlet.cpp:146-210), and closed-form
// P1 integrals that the quadrature must reproduce (tests/test_oracle.py).
//
// Conventions (same as the reference):
//   element dof order (Proto, ElementMatrix.hpp:384-414, ElementData.hpp:1228-1246):
//       u_1..u_n, v_1..v_n, [w_1..w_n], p_1..p_n
//   global dof = node*neq + comp (BlockAccumulator.hpp:147-156, FEVbr point order)
//   CSR row r has columns adj(node)*neq + c, adj sorted ascending incl. self
//       (SparsityBuilder.cpp:157-189 expanded as TrilinosDetail.cpp:251-311)

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <set>
#include <thread>
#include <vector>

extern "C" {

// Same layout as ufem_ns_options in include/ufem_b200.h (kept separate so the
// oracle builds without the product headers).
typedef struct orc_options {
  double theta;               // NavierStokes.cpp:85 (default 1)
  double dt;                  // LSSActionUnsteady::dt()
  double rho;                 // NavierStokesPhysics density
  int32_t supg_type;          // 0 tezduyar, 1 metric, 2 cf2 (SUPG.cpp:15-32)
  int32_t use_specializations;// NavierStokes.cpp:74 (default true)
  double c1, c2;              // SUPG.hpp:100-101
  double alpha_ps, alpha_su, alpha_bu;  // SUPG.hpp:95-97
  double u_ref;               // SUPG.hpp:102
  int32_t precision;          // ignored by the oracle (always FP64)
  int32_t reserved;
} orc_options;

}  // extern "C"

namespace {

// One Line2D face of a constant Neumann condition (BCNeumannConstant).
struct NeumannFace {
  uint32_t a, b;
  int comp;
  double flux;
};

struct BC {
  uint32_t node;
  int comp;
  double value;
};

struct Oracle {
  int dim = 0, nn = 0, neq = 0;  // nn = nodes per element
  int64_t N = 0, E = 0;
  std::vector<double> coords;    // N x dim
  std::vector<uint32_t> conn;    // E x nn
  orc_options o{};
  // node graph (SparsityBuilder.cpp:157-189)
  std::vector<int64_t> start;    // N+1
  std::vector<uint32_t> adj;
  // point CSR
  std::vector<int64_t> rowptr;
  std::vector<int32_t> colidx;
  std::vector<double> vals, rhs, sol;
  // fields (Solver.cpp:358-464 field tags)
  std::vector<double> up;        // navier_stokes_solution N x neq (u, v, [w], p)
  std::vector<double> lin;       // linearized_velocity N x 4d (u_adv, u1, u2, u3)
  std::vector<double> nu;        // navier_stokes_viscosity N
  std::vector<double> force;     // body_force N x dim (empty = zero)
  std::vector<BC> bcs;
  std::vector<NeumannFace> neumann;
  // periodic links: LSS row node of each mesh node (empty: identity)
  std::vector<uint32_t> p2m;
  uint32_t row_of(uint32_t node) const { return p2m.empty() ? node : p2m[node]; }
  // node -> incident elements (for the node-partitioned multi-thread baseline)
  std::vector<int64_t> inc_start;
  std::vector<uint32_t> inc_elem;
  // solver statistics
  int last_iters = 0;
  double last_relres = 0.0;
};

// ---------------------------------------------------------------------------
// Mesh generators (fixtures).  create_rectangle_tris follows
// cf3/Tools/MeshGeneration/MeshGeneration.cpp:209-253.  The tetrahedral cube is
// the Kuhn 6-tet split of each hexahedral cell.  Jitter uses a counter-based
// splitmix64 hash so that any implementation can reproduce it bit-exactly.
// ---------------------------------------------------------------------------
inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
inline double uniform01(uint64_t seed, uint64_t idx) {
  const uint64_t z = mix64(seed + (idx + 1) * 0x9E3779B97F4A7C15ULL);
  return static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);
}

// ---------------------------------------------------------------------------
// Small dense helpers mirroring the reference's Eigen fixed-size operations.
// Inverse/determinant follow the cofactor form of
// computeInverseAndDetWithCheck (Proto/ElementData.hpp:308-314).
// ---------------------------------------------------------------------------
template <int D>
void inverse_det(const double J[D][D], double Ji[D][D], double& det);

template <>
void inverse_det<2>(const double J[2][2], double Ji[2][2], double& det) {
  det = J[0][0] * J[1][1] - J[1][0] * J[0][1];
  const double inv = 1.0 / det;
  Ji[0][0] = J[1][1] * inv;
  Ji[1][0] = -J[1][0] * inv;
  Ji[0][1] = -J[0][1] * inv;
  Ji[1][1] = J[0][0] * inv;
}

template <>
void inverse_det<3>(const double m[3][3], double Ji[3][3], double& det) {
  auto cof = [&](int i, int j) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return m[i1][j1] * m[i2][j2] - m[i1][j2] * m[i2][j1];
  };
  const double c00 = cof(0, 0), c10 = cof(1, 0), c20 = cof(2, 0);
  det = (c00 * m[0][0] + c10 * m[1][0]) + c20 * m[2][0];
  const double inv = 1.0 / det;
  // result(j,i) = cofactor(i,j) / det
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Ji[j][i] = cof(i, j) * inv;
}

// P1 Jacobian J[r][c] = dx_c/dxi_r (Triag2D.cpp:134-140, Tetra3D.cpp:135-171)
template <int D>
void jacobian(const double X[D + 1][D], double J[D][D]) {
  for (int r = 0; r < D; ++r)
    for (int c = 0; c < D; ++c) J[r][c] = X[r + 1][c] - X[0][c];
}

// Shape functions N and dN/dxi (Triag.cpp:24-43, Tetra.cpp:24-48)
template <int D>
void shape_values(const double* xi, double* N) {
  double s = 1.0;
  for (int k = 0; k < D; ++k) s -= xi[k];
  N[0] = s;
  for (int k = 0; k < D; ++k) N[k + 1] = xi[k];
}

// Gradient G = Jinv * dN/dxi (Proto/ElementData.hpp:576-581)
template <int D>
void gradient(const double Ji[D][D], double G[D][D + 1]) {
  for (int r = 0; r < D; ++r) {
    double s = 0.0;
    for (int k = 0; k < D; ++k) s += Ji[r][k] * -1.0;
    G[r][0] = s;
    for (int b = 1; b <= D; ++b) G[r][b] = Ji[r][b - 1];
  }
}

// Gauss rules (GaussImplementation.hpp:170-226 triangles, :370-428 tetrahedra)
template <int D>
struct Gauss2;
template <>
struct Gauss2<2> {
  static constexpr int np = 3;
  static void point(int q, double* xi) {
    static const double p[3][2] = {{0.5, 0.0}, {0.5, 0.5}, {0.0, 0.5}};
    xi[0] = p[q][0];
    xi[1] = p[q][1];
  }
  static double weight() { return 1.0 / 6.0; }
};
template <>
struct Gauss2<3> {
  static constexpr int np = 4;
  static void point(int q, double* xi) {
    const double mu = 0.13819660112501051517954131656;
    xi[0] = mu; xi[1] = mu; xi[2] = mu;
    if (q > 0) xi[q - 1] = 1. - 3. * mu;
  }
  static double weight() { return 0.04166666666666666666666666666666666667; }
};
template <int D>
void centroid(double* xi) {
  const double mu = (D == 2) ? 0.3333333333333333333333333 : 0.25;
  for (int k = 0; k < D; ++k) xi[k] = mu;
}

// Volumes used by the specialised path (Triag2D.cpp:44-53,153-156; Tetra3D.cpp:104-128,203-208)
double volume_tri(const double X[3][2]) {
  const double x0 = X[0][0], x1 = X[1][0], x2 = X[2][0];
  const double y0 = X[0][1], y1 = X[1][1], y2 = X[2][1];
  return 0.5 * ((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0));
}
double volume_tet(const double X[4][3]) {
  const double x0 = X[0][0], y0 = X[0][1], z0 = X[0][2];
  const double x1 = X[1][0], y1 = X[1][1], z1 = X[1][2];
  const double x2 = X[2][0], y2 = X[2][1], z2 = X[2][2];
  const double x3 = X[3][0], y3 = X[3][1], z3 = X[3][2];
  const double det =
      x2*y1*z0 - x3*y1*z0 - x1*y2*z0 + x3*y2*z0 + x1*y3*z0 -
      x2*y3*z0 - x2*y0*z1 + x3*y0*z1 + x0*y2*z1 - x3*y2*z1 -
      x0*y3*z1 + x2*y3*z1 + x1*y0*z2 - x3*y0*z2 - x0*y1*z2 +
      x3*y1*z2 + x0*y3*z2 - x1*y3*z2 - x1*y0*z3 + x2*y0*z3 +
      x0*y1*z3 - x2*y1*z3 - x0*y2*z3 + x1*y2*z3;
  return det / 6.;
}

// ---------------------------------------------------------------------------
// Stabilisation coefficients: ComputeTauImpl::compute_coefficients
// (plugins/UFEM/src/UFEM/SUPG.hpp:140-219).  uc = velocity variable evaluated at
// the centroid (order-1 Gauss point, SUPG.hpp:145-147).
// ---------------------------------------------------------------------------
struct TauParams {
  int type;
  double c1, c2, a_ps, a_su, a_bu, u_ref;
};

template <int D>
void compute_tau(const TauParams& tp, const double X[D + 1][D], const double uc[D], double element_nu,
                 double dt, double& tau_ps, double& tau_su, double& tau_bulk) {
  constexpr int n = D + 1;
  if (tp.type == 0) {  // TEZDUYAR, SUPG.hpp:149-175
    double h_rgn = 1e10;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        if (i != j) {
          double s = 0.0;
          for (int k = 0; k < D; ++k) { const double d = X[i][k] - X[j][k]; s += d * d; }
          h_rgn = std::min(h_rgn, s);
        }
    h_rgn = std::sqrt(h_rgn);
    double umag2 = 0.0;
    for (int k = 0; k < D; ++k) umag2 += uc[k] * uc[k];
    const double umag = std::sqrt(umag2);
    const double h_ugn = h_rgn;
    const double tau_adv_inv = (2. * umag) / h_ugn;
    const double tau_time_inv = 2. / dt;
    const double tau_diff_inv = (4. * element_nu) / (h_rgn * h_rgn);
    tau_su = 1. / (tau_adv_inv + tau_time_inv + tau_diff_inv);
    tau_ps = tau_su;
    tau_bulk = tau_su * umag * umag;
  } else if (tp.type == 1) {  // METRIC, SUPG.hpp:176-190
    double J[D][D], Ji[D][D], det;
    jacobian<D>(X, J);
    inverse_det<D>(J, Ji, det);
    double g[D][D];
    for (int a = 0; a < D; ++a)
      for (int b = 0; b < D; ++b) {
        double s = 0.0;
        for (int k = 0; k < D; ++k) s += Ji[k][a] * Ji[k][b];
        g[a][b] = s;
      }
    double ug[D];
    for (int b = 0; b < D; ++b) {
      double s = 0.0;
      for (int a = 0; a < D; ++a) s += uc[a] * g[a][b];
      ug[b] = s;
    }
    double adv = 0.0;
    for (int b = 0; b < D; ++b) adv += ug[b] * uc[b];
    const double tau_adv_sq = std::fabs(adv);
    double sq = 0.0, tr = 0.0;
    for (int a = 0; a < D; ++a) {
      tr += g[a][a];
      for (int b = 0; b < D; ++b) sq += g[a][b] * g[a][b];
    }
    const double tau_diff = element_nu * element_nu * sq;
    tau_su = 1. / std::sqrt((4. * tp.c1 * tp.c1 / (dt * dt)) + tau_adv_sq + tp.c2 * tau_diff);
    tau_ps = tau_su;
    const double tau_su_std = 1. / std::sqrt((4. / (dt * dt)) + tau_adv_sq + 16. * tau_diff);
    tau_bulk = (1. / tau_su_std) / tr;
  } else {  // CF2, SUPG.hpp:191-210
    double J[D][D], Ji[D][D], det;
    jacobian<D>(X, J);
    inverse_det<D>(J, Ji, det);
    const double volume = (D == 2) ? det / 2.0 : det / 6.0;
    const double he = D == 2 ? std::sqrt(4. / 3.141592654 * volume)
                             : std::pow(3. / 4. / 3.141592654 * volume, 1. / 3.);
    const double ree = tp.u_ref * he / (2. * element_nu);
    const double xi = ree < 3. ? ree / 3. : 1.;
    tau_ps = he * xi / (2. * tp.u_ref);
    tau_bulk = he * tp.u_ref / xi;
    tau_su = 0.;
    double umag2 = 0.0;
    for (int k = 0; k < D; ++k) umag2 += uc[k] * uc[k];
    const double umag = std::sqrt(umag2);
    if (umag > 1e-10) {
      // (u.eval()*u.nabla()).sum(): sum over nodes of u.grad(N_b).  The reference
      // reads the gradient through the support's Jacobian inverse; for P1 the
      // sum is a rounding-level quantity, so h is effectively infinite and
      // tau_su ~ dt/2.  The element's own gradient is used here.
      double G[D][D + 1];
      gradient<D>(Ji, G);
      double s = 0.0;
      for (int b = 0; b <= D; ++b) {
        double t = 0.0;
        for (int k = 0; k < D; ++k) t += uc[k] * G[k][b];
        s += t;
      }
      const double h = 2. * umag / s;
      const double tau_adv = h / (2. * umag);
      const double tau_time = 0.5 * dt;
      const double tau_diff = h * h / (4. * element_nu);
      tau_su = 1. / (1. / tau_adv + 1. / tau_time + 1. / tau_diff);
    }
  }
  tau_ps *= tp.a_ps;
  tau_su *= tp.a_su;
  tau_bulk *= tp.a_bu;
}

// Gather of one element's nodal data (Proto/ElementData.hpp:191-197, 462-466)
template <int D>
struct ElemData {
  static constexpr int n = D + 1;
  double X[n][D];
  double U[n][D];    // u_adv
  double Us[n][D];   // u (solution velocity)
  double P[n];       // p
  double NU[n];      // nu_eff
  double F[n][D];    // body force
};

template <int D>
void gather(const Oracle& S, int64_t e, ElemData<D>& ed) {
  constexpr int n = D + 1;
  for (int b = 0; b < n; ++b) {
    const int64_t node = S.conn[e * n + b];
    for (int k = 0; k < D; ++k) {
      ed.X[b][k] = S.coords[node * D + k];
      ed.U[b][k] = S.lin[node * 4 * D + k];
      ed.Us[b][k] = S.up[node * S.neq + k];
      ed.F[b][k] = S.force.empty() ? 0.0 : S.force[node * D + k];
    }
    ed.P[b] = S.up[node * S.neq + D];
    ed.NU[b] = S.nu[node];
  }
}

// ---------------------------------------------------------------------------
// Generic element expression: NavierStokesAssembly.hpp:51-67 evaluated by the
// Proto quadrature loop (ElementIntegration.hpp:236-258, weight = w_q * detJ at
// :199).  A, T are (n*(D+1))^2 row-major, a is n*(D+1), element-major order.
// ---------------------------------------------------------------------------
template <int D>
void generic_element(const Oracle& S, const ElemData<D>& ed, double* A, double* T, double* av) {
  constexpr int n = D + 1;
  constexpr int nd = n * (D + 1);
  const int pofs = D * n;
  std::fill(A, A + nd * nd, 0.0);
  std::fill(T, T + nd * nd, 0.0);
  std::fill(av, av + nd, 0.0);
  const TauParams tp{S.o.supg_type, S.o.c1, S.o.c2, S.o.alpha_ps, S.o.alpha_su, S.o.alpha_bu, S.o.u_ref};
  // compute_tau.apply(u_adv, nu_eff, dt, ...) (NavierStokesAssembly.hpp:54, SUPG.hpp:110-116)
  double nsum = 0.0;
  for (int b = 0; b < n; ++b) nsum += ed.NU[b];
  const double element_nu = std::fabs(nsum / n);
  double xi_c[D], Nc[n], uc[D];
  centroid<D>(xi_c);
  shape_values<D>(xi_c, Nc);
  for (int k = 0; k < D; ++k) {
    double s = 0.0;
    for (int b = 0; b < n; ++b) s += Nc[b] * ed.U[b][k];
    uc[k] = s;
  }
  double tau_ps, tau_su, tau_bulk;
  compute_tau<D>(tp, ed.X, uc, element_nu, S.o.dt, tau_ps, tau_su, tau_bulk);
  // geometry (constant for P1)
  double J[D][D], Ji[D][D], det;
  jacobian<D>(ed.X, J);
  inverse_det<D>(J, Ji, det);
  double G[D][n];
  gradient<D>(Ji, G);
  double Dm[n][n];
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      double s = 0.0;
      for (int k = 0; k < D; ++k) s += G[k][a] * G[k][b];
      Dm[a][b] = s;
    }
  const double rho = S.o.rho;
  for (int q = 0; q < Gauss2<D>::np; ++q) {
    double xi[D], N[n];
    Gauss2<D>::point(q, xi);
    shape_values<D>(xi, N);
    const double W = Gauss2<D>::weight() * det;
    double ua[D], gq[D], nuq = 0.0;
    for (int k = 0; k < D; ++k) {
      double s = 0.0, f = 0.0;
      for (int b = 0; b < n; ++b) { s += N[b] * ed.U[b][k]; f += N[b] * ed.F[b][k]; }
      ua[k] = s;
      gq[k] = f;
    }
    for (int b = 0; b < n; ++b) nuq += N[b] * ed.NU[b];
    double adv[n], Sv[n];
    for (int b = 0; b < n; ++b) {
      double s = 0.0;
      for (int k = 0; k < D; ++k) s += ua[k] * G[k][b];
      adv[b] = s;
      Sv[b] = N[b] + tau_su * adv[b];
    }
    for (int a = 0; a < n; ++a) {
      const double Sp = N[a] + tau_ps * adv[a] * 0.5;
      for (int b = 0; b < n; ++b) {
        // _A(p, u[_i]) : continuity + PSPG advection
        for (int i = 0; i < D; ++i)
          A[(pofs + a) * nd + i * n + b] += W * (Sp * G[i][b] + tau_ps * G[i][a] * adv[b]);
        // _A(p, p) : PSPG
        A[(pofs + a) * nd + pofs + b] += W * (tau_ps * Dm[a][b] / rho);
        // _A(u[_i], u[_i]) : diffusion + advection
        const double kd = nuq * Dm[a][b] + Sv[a] * adv[b];
        for (int i = 0; i < D; ++i) A[(i * n + a) * nd + i * n + b] += W * kd;
        // _A(u[_i], p) : pressure gradient
        for (int i = 0; i < D; ++i) A[(i * n + a) * nd + pofs + b] += W * (Sv[a] * G[i][b] / rho);
        // _A(u[_i], u[_j]) : bulk viscosity + skew-symmetric advection
        for (int i = 0; i < D; ++i) {
          const double l = tau_bulk * G[i][a] + 0.5 * ua[i] * Sv[a];
          for (int j = 0; j < D; ++j) A[(i * n + a) * nd + j * n + b] += W * (l * G[j][b]);
        }
        // _T(p, u[_i]) : time, PSPG
        for (int i = 0; i < D; ++i) T[(pofs + a) * nd + i * n + b] += W * (tau_ps * G[i][a] * N[b]);
        // _T(u[_i], u[_i]) : time, standard + SUPG
        for (int i = 0; i < D; ++i) T[(i * n + a) * nd + i * n + b] += W * (Sv[a] * N[b]);
      }
      // _a[u[_i]] : body force
      for (int i = 0; i < D; ++i) av[i * n + a] += W * (Sv[a] * gq[i]);
    }
  }
}

// ---------------------------------------------------------------------------
// Specialised closed forms: NavierStokesSpecializations.hpp:37-147 (triangles)
// and :150-302 (tetrahedra), including the reference's 3D W-row use of vk.
// tau comes from a default ComputeTauImpl (METRIC, c1=1, c2=16) applied to the
// solution velocity u (:57-58, :177-178).
// ---------------------------------------------------------------------------
void specialized_tri(const ElemData<2>& ed, double dt, double rho, double* A, double* T) {
  constexpr int n = 3, nd = 9;
  std::fill(A, A + nd * nd, 0.0);
  std::fill(T, T + nd * nd, 0.0);
  auto a = [&](int r, int c) -> double& { return A[r * nd + c]; };
  auto t = [&](int r, int c) -> double& { return T[r * nd + c]; };
  double u_avg[2] = {0, 0};
  for (int k = 0; k < 2; ++k) {
    double s = 0.0;
    for (int b = 0; b < n; ++b) s += ed.U[b][k];
    u_avg[k] = s / n;
  }
  const double volume = volume_tri(ed.X);
  const double fc = 0.5;
  double nsum = 0.0;
  for (int b = 0; b < n; ++b) nsum += ed.NU[b];
  const double nu = std::fabs(nsum / n);
  double nr[3][2];
  const auto& X = ed.X;
  nr[0][0] = X[1][1] - X[2][1]; nr[0][1] = X[2][0] - X[1][0];
  nr[1][0] = X[2][1] - X[0][1]; nr[1][1] = X[0][0] - X[2][0];
  nr[2][0] = X[0][1] - X[1][1]; nr[2][1] = X[1][0] - X[0][0];
  double tau_ps, tau_su, tau_bulk;
  {
    double xi_c[2], Nc[3], uc[2];
    centroid<2>(xi_c);
    shape_values<2>(xi_c, Nc);
    for (int k = 0; k < 2; ++k) {
      double s = 0.0;
      for (int b = 0; b < n; ++b) s += Nc[b] * ed.Us[b][k];
      uc[k] = s;
    }
    const TauParams tp{1, 1., 16., 1., 1., 1., 1.};
    compute_tau<2>(tp, ed.X, uc, nu, dt, tau_ps, tau_su, tau_bulk);
  }
  for (int i = 0; i < 3; ++i) {
    const int Pi = i + 3 * 2, Ui = i, Vi = Ui + 3;
    const double u_ni = u_avg[0] * nr[i][0] + u_avg[1] * nr[i][1];
    for (int j = 0; j < 3; ++j) {
      const int Pj = j + 3 * 2, Uj = j, Vj = Uj + 3;
      const double uk = u_avg[0], vk = u_avg[1];
      const double uknj = uk * nr[j][0] + vk * nr[j][1];
      double val = 1. / 6. * uknj;
      val += tau_su / (4. * volume) * uknj * u_ni;
      a(Ui, Uj) += val; a(Vi, Vj) += val;
      val = tau_ps / (4. * volume) * uknj;
      a(Pi, Uj) += val * nr[i][0]; a(Pi, Vj) += val * nr[i][1];
      val = fc / 6.;
      val += fc * tau_su / (4. * volume) * u_ni;
      a(Ui, Uj) += val * uk * nr[j][0]; a(Ui, Vj) += val * uk * nr[j][1];
      a(Vi, Uj) += val * vk * nr[j][0]; a(Vi, Vj) += val * vk * nr[j][1];
      val = fc * tau_ps / (4. * volume);
      a(Pi, Uj) += val * nr[i][0] * uk * nr[j][0]; a(Pi, Vj) += val * nr[i][0] * uk * nr[j][1];
      a(Pi, Uj) += val * nr[i][1] * vk * nr[j][0]; a(Pi, Vj) += val * nr[i][1] * vk * nr[j][1];
      val = nu / (4. * volume);
      a(Ui, Uj) += val * (4. / 3. * nr[i][0] * nr[j][0] + nr[i][1] * nr[j][1]);
      a(Ui, Vj) += val * nr[i][0] * nr[j][1] / 3.;
      a(Vi, Uj) += val * nr[i][1] * nr[j][0] / 3.;
      a(Vi, Vj) += val * (nr[i][0] * nr[j][0] + 4. / 3. * nr[i][1] * nr[j][1]);
      val = 1. / (6. * rho);
      val += tau_su / (4. * rho * volume) * u_ni;
      a(Ui, Pj) += nr[j][0] * val; a(Vi, Pj) += nr[j][1] * val;
      const double laplacian = 1. / (4. * rho * volume) * (nr[i][0] * nr[j][0] + nr[i][1] * nr[j][1]);
      a(Pi, Pj) += tau_ps * laplacian;
      val = 1. / 6.;
      a(Pi, Uj) += val * nr[j][0]; a(Pi, Vj) += val * nr[j][1];
      val = tau_bulk / (4. * volume);
      a(Ui, Uj) += val * nr[i][0] * nr[j][0]; a(Ui, Vj) += val * nr[i][0] * nr[j][1];
      a(Vi, Uj) += val * nr[i][1] * nr[j][0]; a(Vi, Vj) += val * nr[i][1] * nr[j][1];
      val = volume / 12. * (1. + ((i) == (j) ? 1. : 0.));
      val += tau_su / 6. * u_ni;
      t(Ui, Uj) += val; t(Vi, Vj) += val;
      val = tau_ps / 6.;
      t(Pi, Uj) += val * nr[i][0]; t(Pi, Vj) += val * nr[i][1];
    }
  }
}

void specialized_tet(const ElemData<3>& ed, double dt, double rho, double* A, double* T) {
  constexpr int n = 4, nd = 16;
  std::fill(A, A + nd * nd, 0.0);
  std::fill(T, T + nd * nd, 0.0);
  auto a = [&](int r, int c) -> double& { return A[r * nd + c]; };
  auto t = [&](int r, int c) -> double& { return T[r * nd + c]; };
  double u_avg[3];
  for (int k = 0; k < 3; ++k) {
    double s = 0.0;
    for (int b = 0; b < n; ++b) s += ed.U[b][k];
    u_avg[k] = s / n;
  }
  const double volume = volume_tet(ed.X);
  const double fc = 0.5;
  double nsum = 0.0;
  for (int b = 0; b < n; ++b) nsum += ed.NU[b];
  const double nu = std::fabs(nsum / n);
  const auto& X = ed.X;
  double nr[4][3];
  const int XX = 0, YY = 1, ZZ = 2;
  nr[0][XX] = ((X[3][YY]-X[1][YY])*(X[2][ZZ]-X[1][ZZ]) - (X[2][YY]-X[1][YY])*(X[3][ZZ]-X[1][ZZ])) / 2.0;
  nr[0][YY] = ((X[3][ZZ]-X[1][ZZ])*(X[2][XX]-X[1][XX]) - (X[2][ZZ]-X[1][ZZ])*(X[3][XX]-X[1][XX])) / 2.0;
  nr[0][ZZ] = ((X[3][XX]-X[1][XX])*(X[2][YY]-X[1][YY]) - (X[2][XX]-X[1][XX])*(X[3][YY]-X[1][YY])) / 2.0;
  nr[1][XX] = ((X[2][YY]-X[0][YY])*(X[3][ZZ]-X[0][ZZ]) - (X[3][YY]-X[0][YY])*(X[2][ZZ]-X[0][ZZ])) / 2.0;
  nr[1][YY] = ((X[2][ZZ]-X[0][ZZ])*(X[3][XX]-X[0][XX]) - (X[3][ZZ]-X[0][ZZ])*(X[2][XX]-X[0][XX])) / 2.0;
  nr[1][ZZ] = ((X[2][XX]-X[0][XX])*(X[3][YY]-X[0][YY]) - (X[3][XX]-X[0][XX])*(X[2][YY]-X[0][YY])) / 2.0;
  nr[2][XX] = ((X[3][YY]-X[0][YY])*(X[1][ZZ]-X[0][ZZ]) - (X[1][YY]-X[0][YY])*(X[3][ZZ]-X[0][ZZ])) / 2.0;
  nr[2][YY] = ((X[3][ZZ]-X[0][ZZ])*(X[1][XX]-X[0][XX]) - (X[1][ZZ]-X[0][ZZ])*(X[3][XX]-X[0][XX])) / 2.0;
  nr[2][ZZ] = ((X[3][XX]-X[0][XX])*(X[1][YY]-X[0][YY]) - (X[1][XX]-X[0][XX])*(X[3][YY]-X[0][YY])) / 2.0;
  nr[3][XX] = ((X[1][YY]-X[0][YY])*(X[2][ZZ]-X[0][ZZ]) - (X[2][YY]-X[0][YY])*(X[1][ZZ]-X[0][ZZ])) / 2.0;
  nr[3][YY] = ((X[1][ZZ]-X[0][ZZ])*(X[2][XX]-X[0][XX]) - (X[2][ZZ]-X[0][ZZ])*(X[1][XX]-X[0][XX])) / 2.0;
  nr[3][ZZ] = ((X[1][XX]-X[0][XX])*(X[2][YY]-X[0][YY]) - (X[2][XX]-X[0][XX])*(X[1][YY]-X[0][YY])) / 2.0;
  double tau_ps, tau_su, tau_bulk;
  {
    double xi_c[3], Nc[4], uc[3];
    centroid<3>(xi_c);
    shape_values<3>(xi_c, Nc);
    for (int k = 0; k < 3; ++k) {
      double s = 0.0;
      for (int b = 0; b < n; ++b) s += Nc[b] * ed.Us[b][k];
      uc[k] = s;
    }
    const TauParams tp{1, 1., 16., 1., 1., 1., 1.};
    compute_tau<3>(tp, ed.X, uc, nu, dt, tau_ps, tau_su, tau_bulk);
  }
  double val;
  for (int i = 0; i < 4; ++i) {
    const int Pi = i + 4 * 3, Ui = i, Vi = Ui + 4, Wi = Vi + 4;
    const double u_ni = u_avg[XX] * nr[i][XX] + u_avg[YY] * nr[i][YY] + u_avg[ZZ] * nr[i][ZZ];
    for (int j = 0; j < 4; ++j) {
      const int Pj = j + 4 * 3, Uj = j, Vj = Uj + 4, Wj = Vj + 4;
      const double uk = u_avg[XX], vk = u_avg[YY], wk = u_avg[ZZ];
      const double uknj = uk * nr[j][XX] + vk * nr[j][YY] + wk * nr[j][ZZ];
      val = 1. / 12. * uknj;
      val += tau_su / (9. * volume) * uknj * u_ni;
      a(Ui, Uj) += val; a(Vi, Vj) += val; a(Wi, Wj) += val;
      val = tau_ps / (9. * volume) * uknj;
      a(Pi, Uj) += val * nr[i][XX]; a(Pi, Vj) += val * nr[i][YY]; a(Pi, Wj) += val * nr[i][ZZ];
      val = fc / 12.;
      val += fc * tau_su / (9. * volume) * u_ni;
      a(Ui, Uj) += val * uk * nr[j][XX]; a(Ui, Vj) += val * uk * nr[j][YY]; a(Ui, Wj) += val * uk * nr[j][ZZ];
      a(Vi, Uj) += val * vk * nr[j][XX]; a(Vi, Vj) += val * vk * nr[j][YY]; a(Vi, Wj) += val * vk * nr[j][ZZ];
      a(Wi, Uj) += val * vk * nr[j][XX]; a(Wi, Vj) += val * vk * nr[j][YY]; a(Wi, Wj) += val * vk * nr[j][ZZ];
      val = fc * tau_ps / (9. * volume);
      a(Pi, Uj) += val * nr[i][XX] * uk * nr[j][XX]; a(Pi, Vj) += val * nr[i][XX] * uk * nr[j][YY];
      a(Pi, Wj) += val * nr[i][XX] * uk * nr[j][ZZ]; a(Pi, Uj) += val * nr[i][YY] * vk * nr[j][XX];
      a(Pi, Vj) += val * nr[i][YY] * vk * nr[j][YY]; a(Pi, Wj) += val * nr[i][YY] * vk * nr[j][ZZ];
      a(Pi, Uj) += val * nr[i][ZZ] * vk * nr[j][XX]; a(Pi, Vj) += val * nr[i][ZZ] * vk * nr[j][YY];
      a(Pi, Wj) += val * nr[i][ZZ] * vk * nr[j][ZZ];
      val = nu / (9. * volume);
      a(Ui, Uj) += val * (4. / 3. * nr[i][XX] * nr[j][XX] + nr[i][YY] * nr[j][YY] + nr[i][ZZ] * nr[j][ZZ]);
      a(Ui, Vj) += val * nr[i][XX] * nr[j][YY] / 3.;
      a(Ui, Wj) += val * nr[i][XX] * nr[j][ZZ] / 3.;
      a(Vi, Uj) += val * nr[i][YY] * nr[j][XX] / 3.;
      a(Vi, Vj) += val * (nr[i][XX] * nr[j][XX] + 4. / 3. * nr[i][YY] * nr[j][YY] + nr[i][ZZ] * nr[j][ZZ]);
      a(Vi, Wj) += val * nr[i][YY] * nr[j][ZZ] / 3.;
      a(Wi, Uj) += val * nr[i][ZZ] * nr[j][XX] / 3.;
      a(Wi, Vj) += val * nr[i][ZZ] * nr[j][YY] / 3.;
      a(Wi, Wj) += val * (nr[i][XX] * nr[j][XX] + nr[i][YY] * nr[j][YY] + 4. / 3. * nr[i][ZZ] * nr[j][ZZ]);
      val = 1. / (12. * rho);
      val += tau_su / (9. * rho * volume) * u_ni;
      a(Ui, Pj) += nr[j][XX] * val; a(Vi, Pj) += nr[j][YY] * val; a(Wi, Pj) += nr[j][ZZ] * val;
      val = tau_ps / (9. * rho * volume) * (nr[i][XX] * nr[j][XX] + nr[i][YY] * nr[j][YY] + nr[i][ZZ] * nr[j][ZZ]);
      a(Pi, Pj) += val;
      val = 1. / 12.;
      a(Pi, Uj) += val * nr[j][XX]; a(Pi, Vj) += val * nr[j][YY]; a(Pi, Wj) += val * nr[j][ZZ];
      val = tau_bulk / (9. * volume);
      a(Ui, Uj) += val * nr[i][XX] * nr[j][XX]; a(Ui, Vj) += val * nr[i][XX] * nr[j][YY];
      a(Ui, Wj) += val * nr[i][XX] * nr[j][ZZ]; a(Vi, Uj) += val * nr[i][YY] * nr[j][XX];
      a(Vi, Vj) += val * nr[i][YY] * nr[j][YY]; a(Vi, Wj) += val * nr[i][YY] * nr[j][ZZ];
      a(Wi, Uj) += val * nr[i][ZZ] * nr[j][XX]; a(Wi, Vj) += val * nr[i][ZZ] * nr[j][YY];
      a(Wi, Wj) += val * nr[i][ZZ] * nr[j][ZZ];
      val = volume / 20. * (1. + (i == j ? 1. : 0.));
      val += tau_su / 12. * u_ni;
      t(Ui, Uj) += val; t(Vi, Vj) += val; t(Wi, Wj) += val;
      val = tau_ps / 12.;
      t(Pi, Uj) += val * nr[i][XX]; t(Pi, Vj) += val * nr[i][YY]; t(Pi, Wj) += val * nr[i][ZZ];
    }
  }
}

// Position of point (row, col) in the CSR, by a linear search of the block row's
// node list as TrilinosFEVbrMatrix::add_values does (TrilinosFEVbrMatrix.cpp:271-357).
inline int64_t csr_pos(const Oracle& S, int64_t rnode, int req, int64_t cnode, int ceq) {
  const int64_t s0 = S.start[rnode], s1 = S.start[rnode + 1];
  for (int64_t k = s0; k < s1; ++k)
    if (S.adj[k] == cnode) return S.rowptr[rnode * S.neq + req] + (k - s0) * S.neq + ceq;
  return -1;
}

// One element: compute, combine (NavierStokesAssembly.hpp:69-71), re-order
// (Proto/BlockAccumulator.hpp:133-184) and scatter the rows whose node lies in
// [own0, own1) -- the owned-rows rule of TrilinosFEVbrMatrix.cpp:287.
template <int D>
void assemble_element(Oracle& S, int64_t e, int64_t own0, int64_t own1) {
  constexpr int n = D + 1, nd = n * (D + 1);
  const int neq = D + 1;
  ElemData<D> ed;
  gather<D>(S, e, ed);
  double A[nd * nd], T[nd * nd], av[nd];
  if (S.o.use_specializations) {
    if constexpr (D == 2) specialized_tri(ed, S.o.dt, S.o.rho, A, T);
    else specialized_tet(ed, S.o.dt, S.o.rho, A, T);
    std::fill(av, av + nd, 0.0);
  } else {
    generic_element<D>(S, ed, A, T, av);
  }
  // element state vector x (FillRhs, ElementData.hpp:1228-1246)
  double x[nd];
  for (int b = 0; b < n; ++b) {
    for (int k = 0; k < D; ++k) x[k * n + b] = ed.Us[b][k];
    x[D * n + b] = ed.P[b];
  }
  // system_rhs += -A*x + a
  double re[nd];
  for (int r = 0; r < nd; ++r) {
    double s = 0.0;
    for (int c = 0; c < nd; ++c) s += -A[r * nd + c] * x[c];
    re[r] = s + av[r];
  }
  // _A(p) = _A(p)/theta ; system_matrix += invdt*T + theta*A
  const double theta = S.o.theta;
  const double invdt = 1.0 / S.o.dt;
  for (int r = D * n; r < nd; ++r)
    for (int c = 0; c < nd; ++c) A[r * nd + c] = A[r * nd + c] / theta;
  double M[nd * nd];
  for (int k = 0; k < nd * nd; ++k) M[k] = invdt * T[k] + theta * A[k];
  // scatter: element row (comp*n + a) -> global (node_a*neq + comp)
  const uint32_t* cn = &S.conn[e * n];
  for (int a = 0; a < n; ++a) {
    const int64_t ra = S.row_of(cn[a]);
    if (ra < own0 || ra >= own1) continue;
    for (int comp = 0; comp < neq; ++comp) {
      const int er = comp * n + a;
      for (int b = 0; b < n; ++b) {
        const int64_t base = csr_pos(S, ra, comp, S.row_of(cn[b]), 0);
        for (int c = 0; c < neq; ++c) S.vals[base + c] += M[er * nd + c * n + b];
      }
      S.rhs[ra * neq + comp] += re[er];
    }
  }
}

void build_graph(Oracle& S) {
  // SparsityBuilder.cpp:157-189: per-node sorted set of nodes sharing an element.
  // With periodic links (LSSAction.cpp:245-269) a node's row is its master's:
  // element nodes are mapped to their rows first; a linked node keeps a row
  // that ties it to its master.
  std::vector<std::set<uint32_t>> sets(S.N);
  for (int64_t e = 0; e < S.E; ++e)
    for (int a = 0; a < S.nn; ++a)
      for (int b = 0; b < S.nn; ++b) sets[S.row_of(S.conn[e * S.nn + a])].insert(S.row_of(S.conn[e * S.nn + b]));
  for (int64_t i = 0; i < S.N; ++i)
    if (S.row_of((uint32_t)i) != (uint32_t)i) {
      sets[i].insert((uint32_t)i);
      sets[i].insert(S.row_of((uint32_t)i));
    }
  S.start.assign(S.N + 1, 0);
  for (int64_t i = 0; i < S.N; ++i) S.start[i + 1] = S.start[i] + (int64_t)sets[i].size();
  S.adj.resize(S.start[S.N]);
  for (int64_t i = 0; i < S.N; ++i) std::copy(sets[i].begin(), sets[i].end(), S.adj.begin() + S.start[i]);
  // point expansion, FEVbr order: row node*neq+eq, columns adj*neq + c
  const int neq = S.neq;
  S.rowptr.assign(S.N * neq + 1, 0);
  for (int64_t i = 0; i < S.N; ++i)
    for (int r = 0; r < neq; ++r)
      S.rowptr[i * neq + r + 1] = S.rowptr[i * neq + r] + (S.start[i + 1] - S.start[i]) * neq;
  S.colidx.resize(S.rowptr.back());
  for (int64_t i = 0; i < S.N; ++i)
    for (int r = 0; r < neq; ++r) {
      int64_t p = S.rowptr[i * neq + r];
      for (int64_t k = S.start[i]; k < S.start[i + 1]; ++k)
        for (int c = 0; c < neq; ++c) S.colidx[p++] = (int32_t)(S.adj[k] * neq + c);
    }
  S.vals.assign(S.colidx.size(), 0.0);
  S.rhs.assign(S.N * neq, 0.0);
  S.sol.assign(S.N * neq, 0.0);
  // node -> elements, elements ascending
  S.inc_start.assign(S.N + 1, 0);
  for (int64_t e = 0; e < S.E; ++e)
    for (int a = 0; a < S.nn; ++a) S.inc_start[S.row_of(S.conn[e * S.nn + a]) + 1]++;
  for (int64_t i = 0; i < S.N; ++i) S.inc_start[i + 1] += S.inc_start[i];
  S.inc_elem.resize(S.inc_start[S.N]);
  std::vector<int64_t> fill(S.inc_start.begin(), S.inc_start.end() - 1);
  for (int64_t e = 0; e < S.E; ++e)
    for (int a = 0; a < S.nn; ++a) S.inc_elem[fill[S.row_of(S.conn[e * S.nn + a])]++] = (uint32_t)e;
}

// LinearizeU (NavierStokes.cpp:105): u_adv = 2.1875u - 2.1875u1 + 1.3125u2 - 0.3125u3
void linearize(Oracle& S) {
  const int D = S.dim;
  for (int64_t i = 0; i < S.N; ++i)
    for (int k = 0; k < D; ++k) {
      const double u = S.up[i * S.neq + k];
      const double u1 = S.lin[i * 4 * D + D + k];
      const double u2 = S.lin[i * 4 * D + 2 * D + k];
      const double u3 = S.lin[i * 4 * D + 3 * D + k];
      S.lin[i * 4 * D + k] = 2.1875 * u - 2.1875 * u1 + 1.3125 * u2 - 0.3125 * u3;
    }
}

void assemble_range(Oracle& S, int64_t own0, int64_t own1, bool all_elements) {
  if (all_elements) {
    for (int64_t e = 0; e < S.E; ++e) {
      if (S.dim == 2) assemble_element<2>(S, e, own0, own1);
      else assemble_element<3>(S, e, own0, own1);
    }
    return;
  }
  // elements touching the owned node range, ascending and unique
  std::vector<uint32_t> elems(S.inc_elem.begin() + S.inc_start[own0], S.inc_elem.begin() + S.inc_start[own1]);
  std::sort(elems.begin(), elems.end());
  elems.erase(std::unique(elems.begin(), elems.end()), elems.end());
  for (uint32_t e : elems) {
    if (S.dim == 2) assemble_element<2>(S, e, own0, own1);
    else assemble_element<3>(S, e, own0, own1);
  }
}

// Tie rows of linked nodes: x_slave - x_master = 0, rhs 0.
void tie_rows(Oracle& S) {
  for (int64_t i = 0; i < S.N; ++i) {
    const uint32_t m = S.row_of((uint32_t)i);
    if (m == (uint32_t)i) continue;
    for (int c = 0; c < S.neq; ++c) {
      S.vals[csr_pos(S, i, c, i, c)] = 1.0;
      S.vals[csr_pos(S, i, c, m, c)] = -1.0;
      S.rhs[i * S.neq + c] = 0.0;
    }
  }
}

// ZeroLSS (math/LSS/ZeroLSS.cpp:56-82, reset_solution=false) + LinearizeU + Assembly
void assemble(Oracle& S, int nthreads) {
  std::fill(S.vals.begin(), S.vals.end(), 0.0);
  std::fill(S.rhs.begin(), S.rhs.end(), 0.0);
  linearize(S);
  if (nthreads <= 1) {
    assemble_range(S, 0, S.N, true);
    tie_rows(S);
    return;
  }
  // Node-partitioned overlap assembly: each thread owns a node range and adds
  // only owned rows, the model of the reference's MPI ranks with a ghost layer.
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t) {
    const int64_t a = S.N * t / nthreads, b = S.N * (t + 1) / nthreads;
    th.emplace_back([&S, a, b] { assemble_range(S, a, b, false); });
  }
  for (auto& x : th) x.join();
  tie_rows(S);
}

// System::dirichlet with preserve_symmetry (System.cpp:240-255) ->
// TrilinosFEVbrMatrix::symmetric_dirichlet (TrilinosFEVbrMatrix.cpp:482-553),
// applied in list order; value = new - old (Proto/DirichletBC.hpp:34-39).
void symmetric_dirichlet(Oracle& S, int64_t b, int c, double v) {
  const int neq = S.neq;
  for (int64_t k = S.start[b]; k < S.start[b + 1]; ++k) {
    const int64_t col = S.adj[k];
    bool row_has_node = false;
    for (int64_t i = S.start[col]; i < S.start[col + 1]; ++i)
      if (S.adj[i] == (uint32_t)b) { row_has_node = true; break; }
    if (!row_has_node) continue;
    for (int j = 0; j < neq; ++j) {
      const int64_t pos = csr_pos(S, col, j, b, c);
      S.rhs[col * neq + j] += -S.vals[pos] * v;
      S.vals[pos] = 0;
    }
    if (col == b) {
      const int64_t r = b * neq + c;
      for (int64_t p = S.rowptr[r]; p < S.rowptr[r + 1]; ++p) S.vals[p] = 0;
      S.vals[csr_pos(S, b, c, b, c)] = 1.;
    }
  }
  S.rhs[b * neq + c] = v;
  S.sol[b * neq + c] = v;
}

// BCNeumannConstant (plugins/UFEM/src/UFEM/BCNeumannConstant.cpp:54-60):
// rhs(var) += integral<1>(transpose(N(var)) * flux * _norm(normal)) over each
// Line2D face.  integral<1> is one Gauss point (xi = 0, weight 2) with the
// weight multiplied by the face's jacobian determinant
// (Proto/ElementIntegration.hpp:200, Line2D.cpp:109-114: |x1 - x0| / 2);
// N = (1/2, 1/2); normal is Line2D::normal (Line2D.cpp:83-87), the unnormalised
// (dy, -dx) / 2.  Evaluated as the reference's expression tree:
// (weight * detJ) * ((N_i * flux) * |normal|), added face by face.
void apply_neumann(Oracle& S) {
  for (const NeumannFace& f : S.neumann) {
    const double* xa = &S.coords[(size_t)f.a * 2];
    const double* xb = &S.coords[(size_t)f.b * 2];
    const double dxdxi = 0.5 * (xb[0] - xa[0]), dydxi = 0.5 * (xb[1] - xa[1]);
    const double detj = std::sqrt(dxdxi * dxdxi + dydxi * dydxi);
    const double nx = 0.5 * (xb[1] - xa[1]), ny = 0.5 * (-xb[0] + xa[0]);
    const double nrm = std::sqrt(nx * nx + ny * ny);
    const double w = 2.0 * detj;
    const double c = w * ((0.5 * f.flux) * nrm);
    S.rhs[(size_t)S.row_of(f.a) * S.neq + f.comp] += c;
    S.rhs[(size_t)S.row_of(f.b) * S.neq + f.comp] += c;
  }
}

// BoundaryConditions in list order: the constant Neumann faces first, then the
// Dirichlet conditions in the order they were added.
void apply_bcs(Oracle& S) {
  apply_neumann(S);
  for (const BC& bc : S.bcs) {  // a linked node's condition acts on its master's row
    const uint32_t row = S.row_of(bc.node);
    const double old = S.up[(int64_t)row * S.neq + bc.comp];
    symmetric_dirichlet(S, row, bc.comp, bc.value - old);
  }
}

// ---------------------------------------------------------------------------
// FP64 reference solve: restarted GMRES(m) with ILU(0) right preconditioning,
// ||r||/||b|| <= tol.  The reference uses Belos GMRES + Ifpack ILU to 1e-10
// (TrilinosStratimikosStrategy.cpp:135-177); the oracle solves tighter so that
// solution differences measure the GPU path, not the oracle.
// ---------------------------------------------------------------------------
struct ILU0 {
  std::vector<double> lu;
  std::vector<int64_t> diag;
};

void ilu0_factor(const Oracle& S, ILU0& f) {
  const int64_t n = (int64_t)S.rowptr.size() - 1;
  f.lu = S.vals;
  f.diag.assign(n, -1);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t p = S.rowptr[i]; p < S.rowptr[i + 1]; ++p)
      if (S.colidx[p] == i) f.diag[i] = p;
  std::vector<int64_t> pos(n, -1);
  for (int64_t i = 0; i < n; ++i) {
    for (int64_t p = S.rowptr[i]; p < S.rowptr[i + 1]; ++p) pos[S.colidx[p]] = p;
    for (int64_t p = S.rowptr[i]; p < S.rowptr[i + 1]; ++p) {
      const int64_t k = S.colidx[p];
      if (k >= i) break;
      const double piv = f.lu[f.diag[k]];
      const double lik = f.lu[p] / piv;
      f.lu[p] = lik;
      for (int64_t q = f.diag[k] + 1; q < S.rowptr[k + 1]; ++q) {
        const int64_t jp = pos[S.colidx[q]];
        if (jp >= 0) f.lu[jp] -= lik * f.lu[q];
      }
    }
    for (int64_t p = S.rowptr[i]; p < S.rowptr[i + 1]; ++p) pos[S.colidx[p]] = -1;
  }
}

void ilu0_apply(const Oracle& S, const ILU0& f, const double* r, double* z) {
  const int64_t n = (int64_t)S.rowptr.size() - 1;
  for (int64_t i = 0; i < n; ++i) {
    double s = r[i];
    for (int64_t p = S.rowptr[i]; p < f.diag[i]; ++p) s -= f.lu[p] * z[S.colidx[p]];
    z[i] = s;
  }
  for (int64_t i = n - 1; i >= 0; --i) {
    double s = z[i];
    for (int64_t p = f.diag[i] + 1; p < S.rowptr[i + 1]; ++p) s -= f.lu[p] * z[S.colidx[p]];
    z[i] = s / f.lu[f.diag[i]];
  }
}

void spmv(const Oracle& S, const double* x, double* y) {
  const int64_t n = (int64_t)S.rowptr.size() - 1;
  for (int64_t i = 0; i < n; ++i) {
    double s = 0.0;
    for (int64_t p = S.rowptr[i]; p < S.rowptr[i + 1]; ++p) s += S.vals[p] * x[S.colidx[p]];
    y[i] = s;
  }
}

double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}

int gmres_ilu0(Oracle& S, double tol, int maxit, int m) {
  const int64_t n = (int64_t)S.rowptr.size() - 1;
  ILU0 f;
  ilu0_factor(S, f);
  std::vector<double>& x = S.sol;
  const double bnorm = std::sqrt(dot(S.rhs, S.rhs));
  if (bnorm == 0.0) {
    std::fill(x.begin(), x.end(), 0.0);
    S.last_iters = 0;
    S.last_relres = 0.0;
    return 0;
  }
  std::vector<std::vector<double>> V(m + 1, std::vector<double>(n)), Z(m, std::vector<double>(n));
  std::vector<double> H((m + 1) * m), cs(m), sn(m), g(m + 1), w(n), r(n);
  int it = 0;
  double relres = 1.0;
  while (it < maxit) {
    spmv(S, x.data(), r.data());
    for (int64_t i = 0; i < n; ++i) r[i] = S.rhs[i] - r[i];
    const double beta = std::sqrt(dot(r, r));
    relres = beta / bnorm;
    if (relres <= tol) break;
    for (int64_t i = 0; i < n; ++i) V[0][i] = r[i] / beta;
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j = 0;
    for (; j < m && it < maxit; ++j, ++it) {
      ilu0_apply(S, f, V[j].data(), Z[j].data());
      spmv(S, Z[j].data(), w.data());
      for (int k = 0; k <= j; ++k) {  // modified Gram-Schmidt
        const double h = dot(w, V[k]);
        H[k * m + j] = h;
        for (int64_t i = 0; i < n; ++i) w[i] -= h * V[k][i];
      }
      const double hn = std::sqrt(dot(w, w));
      H[(j + 1) * m + j] = hn;
      if (hn != 0.0)
        for (int64_t i = 0; i < n; ++i) V[j + 1][i] = w[i] / hn;
      for (int k = 0; k < j; ++k) {
        const double t = cs[k] * H[k * m + j] + sn[k] * H[(k + 1) * m + j];
        H[(k + 1) * m + j] = -sn[k] * H[k * m + j] + cs[k] * H[(k + 1) * m + j];
        H[k * m + j] = t;
      }
      const double a = H[j * m + j], b = H[(j + 1) * m + j];
      const double den = std::sqrt(a * a + b * b);
      cs[j] = a / den;
      sn[j] = b / den;
      H[j * m + j] = den;
      H[(j + 1) * m + j] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      relres = std::fabs(g[j + 1]) / bnorm;
      if (relres <= tol || hn == 0.0) { ++j; ++it; break; }
    }
    // back substitution and update x += Z y
    std::vector<double> y(j);
    for (int k = j - 1; k >= 0; --k) {
      double s = g[k];
      for (int l = k + 1; l < j; ++l) s -= H[k * m + l] * y[l];
      y[k] = s / H[k * m + k];
    }
    for (int k = 0; k < j; ++k)
      for (int64_t i = 0; i < n; ++i) x[i] += y[k] * Z[k][i];
    if (relres <= tol) {
      // confirm with the true residual
      spmv(S, x.data(), r.data());
      for (int64_t i = 0; i < n; ++i) r[i] = S.rhs[i] - r[i];
      relres = std::sqrt(dot(r, r)) / bnorm;
      if (relres <= tol * 10) break;
    }
  }
  S.last_iters = it;
  S.last_relres = relres;
  return relres <= tol * 10 ? 0 : 1;
}

// Update actions (NavierStokes.cpp:172-179): u3=u2, u2=u1, u1=u, u+=du, p+=dp
void update(Oracle& S) {
  const int D = S.dim;
  for (int64_t i = 0; i < S.N; ++i) {
    double* L = &S.lin[i * 4 * D];
    for (int k = 0; k < D; ++k) {
      L[3 * D + k] = L[2 * D + k];
      L[2 * D + k] = L[D + k];
      L[D + k] = S.up[i * S.neq + k];
    }
    for (int k = 0; k <= D; ++k) S.up[i * S.neq + k] += S.sol[i * S.neq + k];
  }
}

}  // namespace

extern "C" {

void orc_mesh_rectangle_tris(int nx, int ny, double jitter, uint64_t seed, double* coords, uint32_t* conn) {
  const double xs = 1.0 / nx, ys = 1.0 / ny;
  for (int j = 0; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i) {
      const int64_t node = (int64_t)j * (nx + 1) + i;
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
      const uint32_t n0 = j * (nx + 1) + i, n1 = n0 + 1, n3 = (j + 1) * (nx + 1) + i, n2 = n3 + 1;
      uint32_t* u = conn + 6 * ((int64_t)j * nx + i);
      u[0] = n0; u[1] = n2; u[2] = n3;  // upper
      u[3] = n0; u[4] = n1; u[5] = n2;  // lower
    }
}

void orc_mesh_cube_tets(int n, double jitter, uint64_t seed, double* coords, uint32_t* conn) {
  const double h = 1.0 / n;
  const int64_t s = n + 1;
  for (int k = 0; k <= n; ++k)
    for (int j = 0; j <= n; ++j)
      for (int i = 0; i <= n; ++i) {
        const int64_t node = ((int64_t)k * s + j) * s + i;
        double p[3] = {i * h, j * h, k * h};
        if (i > 0 && i < n && j > 0 && j < n && k > 0 && k < n)
          for (int c = 0; c < 3; ++c) p[c] += (2.0 * uniform01(seed, node * 4 + c) - 1.0) * jitter * h;
        for (int c = 0; c < 3; ++c) coords[node * 3 + c] = p[c];
      }
  static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  static const int odd[6] = {0, 1, 1, 0, 0, 1};
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        const int64_t cell = ((int64_t)k * n + j) * n + i;
        for (int t = 0; t < 6; ++t) {
          int v[3] = {i, j, k};
          uint32_t ids[4];
          ids[0] = (uint32_t)(((int64_t)v[2] * s + v[1]) * s + v[0]);
          for (int m = 0; m < 3; ++m) {
            v[perm[t][m]] += 1;
            ids[m + 1] = (uint32_t)(((int64_t)v[2] * s + v[1]) * s + v[0]);
          }
          if (odd[t]) std::swap(ids[2], ids[3]);
          for (int m = 0; m < 4; ++m) conn[(cell * 6 + t) * 4 + m] = ids[m];
        }
      }
}

void* orc_create_periodic(int dim, int64_t nb_nodes, int64_t nb_elems, const double* coords, const uint32_t* conn,
                          const orc_options* opts, const uint32_t* slaves, const uint32_t* masters, int64_t nlinks);

void* orc_create(int dim, int64_t nb_nodes, int64_t nb_elems, const double* coords, const uint32_t* conn,
                 const orc_options* opts) {
  return orc_create_periodic(dim, nb_nodes, nb_elems, coords, conn, opts, nullptr, nullptr, 0);
}

// Periodic links slave -> master, chains resolved to the final master.
void* orc_create_periodic(int dim, int64_t nb_nodes, int64_t nb_elems, const double* coords, const uint32_t* conn,
                          const orc_options* opts, const uint32_t* slaves, const uint32_t* masters, int64_t nlinks) {
  if (dim != 2 && dim != 3) return nullptr;
  Oracle* S = new Oracle();
  if (nlinks > 0) {
    std::vector<int64_t> link(nb_nodes, -1);
    for (int64_t i = 0; i < nlinks; ++i) link[slaves[i]] = masters[i];
    S->p2m.resize(nb_nodes);
    for (int64_t i = 0; i < nb_nodes; ++i) {
      int64_t cur = i;
      while (link[cur] >= 0) cur = link[cur];
      S->p2m[i] = (uint32_t)cur;
    }
  }
  S->dim = dim;
  S->nn = dim + 1;
  S->neq = dim + 1;
  S->N = nb_nodes;
  S->E = nb_elems;
  S->coords.assign(coords, coords + nb_nodes * dim);
  S->conn.assign(conn, conn + nb_elems * S->nn);
  S->o = *opts;
  build_graph(*S);
  S->up.assign(S->N * S->neq, 0.0);
  S->lin.assign(S->N * 4 * dim, 0.0);
  S->nu.assign(S->N, 0.0);
  return S;
}

// A bare linear system on a given node graph (no mesh), for the LSS-level
// known-answer tests: LSS::System::create(cp, neq, node_connectivity,
// starting_indices) (System.cpp:82-110).
void* orc_create_lss(int64_t nb_nodes, int neq, const int64_t* start, const uint32_t* adj) {
  Oracle* S = new Oracle();
  S->dim = 0;
  S->neq = neq;
  S->N = nb_nodes;
  S->start.assign(start, start + nb_nodes + 1);
  S->adj.assign(adj, adj + start[nb_nodes]);
  S->rowptr.assign(S->N * neq + 1, 0);
  for (int64_t i = 0; i < S->N; ++i)
    for (int r = 0; r < neq; ++r)
      S->rowptr[i * neq + r + 1] = S->rowptr[i * neq + r] + (S->start[i + 1] - S->start[i]) * neq;
  S->colidx.resize(S->rowptr.back());
  for (int64_t i = 0; i < S->N; ++i)
    for (int r = 0; r < neq; ++r) {
      int64_t p = S->rowptr[i * neq + r];
      for (int64_t k = S->start[i]; k < S->start[i + 1]; ++k)
        for (int c = 0; c < neq; ++c) S->colidx[p++] = (int32_t)(S->adj[k] * neq + c);
    }
  S->vals.assign(S->colidx.size(), 0.0);
  S->rhs.assign(S->N * neq, 0.0);
  S->sol.assign(S->N * neq, 0.0);
  return S;
}

// TrilinosFEVbrMatrix::set_row (TrilinosFEVbrMatrix.cpp:405-450)
void orc_set_row(void* h, int64_t blockrow, int ieq, double diagval, double offdiagval) {
  Oracle* S = static_cast<Oracle*>(h);
  const int64_t r = blockrow * S->neq + ieq;
  for (int64_t p = S->rowptr[r]; p < S->rowptr[r + 1]; ++p) S->vals[p] = offdiagval;
  S->vals[csr_pos(*S, blockrow, ieq, blockrow, ieq)] = diagval;
}

int64_t orc_nrows(void* h) { return static_cast<Oracle*>(h)->N * static_cast<Oracle*>(h)->neq; }

void orc_destroy(void* h) { delete static_cast<Oracle*>(h); }

void orc_set_options(void* h, const orc_options* opts) { static_cast<Oracle*>(h)->o = *opts; }

int64_t orc_nnz(void* h) { return (int64_t) static_cast<Oracle*>(h)->colidx.size(); }
int64_t orc_block_nnz(void* h) { return (int64_t) static_cast<Oracle*>(h)->adj.size(); }

void orc_csr(void* h, int64_t* rowptr, int32_t* colidx) {
  Oracle* S = static_cast<Oracle*>(h);
  std::copy(S->rowptr.begin(), S->rowptr.end(), rowptr);
  std::copy(S->colidx.begin(), S->colidx.end(), colidx);
}

void orc_graph(void* h, int64_t* start, uint32_t* adj) {
  Oracle* S = static_cast<Oracle*>(h);
  std::copy(S->start.begin(), S->start.end(), start);
  std::copy(S->adj.begin(), S->adj.end(), adj);
}

void orc_set_state(void* h, const double* up, const double* lin, const double* nu, const double* force) {
  Oracle* S = static_cast<Oracle*>(h);
  S->up.assign(up, up + S->N * S->neq);
  S->lin.assign(lin, lin + S->N * 4 * S->dim);
  S->nu.assign(nu, nu + S->N);
  if (force) S->force.assign(force, force + S->N * S->dim);
  else S->force.clear();
}

void orc_get_state(void* h, double* up, double* lin) {
  Oracle* S = static_cast<Oracle*>(h);
  if (up) std::copy(S->up.begin(), S->up.end(), up);
  if (lin) std::copy(S->lin.begin(), S->lin.end(), lin);
}

void orc_set_solution(void* h, const double* sol) {
  Oracle* S = static_cast<Oracle*>(h);
  S->sol.assign(sol, sol + S->N * S->neq);
}

void orc_get_solution(void* h, double* sol) {
  Oracle* S = static_cast<Oracle*>(h);
  std::copy(S->sol.begin(), S->sol.end(), sol);
}

void orc_clear_dirichlet(void* h) { static_cast<Oracle*>(h)->bcs.clear(); }
void orc_clear_neumann(void* h) { static_cast<Oracle*>(h)->neumann.clear(); }
// faces: nfaces x 2 node ids (Line2D)
void orc_add_neumann(void* h, const uint32_t* faces, int64_t nfaces, int comp, double flux) {
  Oracle* S = static_cast<Oracle*>(h);
  for (int64_t i = 0; i < nfaces; ++i) S->neumann.push_back({faces[2 * i], faces[2 * i + 1], comp, flux});
}

void orc_add_dirichlet(void* h, const uint32_t* nodes, int64_t n, int comp, const double* values) {
  Oracle* S = static_cast<Oracle*>(h);
  for (int64_t i = 0; i < n; ++i) S->bcs.push_back(BC{nodes[i], comp, values[i]});
}

void orc_add_dirichlet_dofs(void* h, const uint32_t* nodes, const int32_t* comps, const double* values, int64_t n) {
  Oracle* S = static_cast<Oracle*>(h);
  for (int64_t i = 0; i < n; ++i) S->bcs.push_back(BC{nodes[i], comps[i], values[i]});
}

void orc_assemble(void* h, int nthreads) { assemble(*static_cast<Oracle*>(h), nthreads); }
void orc_apply_bcs(void* h) { apply_bcs(*static_cast<Oracle*>(h)); }

// Direct access for the symmetric-Dirichlet known-answer test.
void orc_set_system(void* h, const double* vals, const double* rhs) {
  Oracle* S = static_cast<Oracle*>(h);
  std::copy(vals, vals + S->vals.size(), S->vals.begin());
  std::copy(rhs, rhs + S->rhs.size(), S->rhs.begin());
}
void orc_dirichlet(void* h, int64_t node, int comp, double value) {
  symmetric_dirichlet(*static_cast<Oracle*>(h), node, comp, value);
}

void orc_get_system(void* h, double* vals, double* rhs) {
  Oracle* S = static_cast<Oracle*>(h);
  if (vals) std::copy(S->vals.begin(), S->vals.end(), vals);
  if (rhs) std::copy(S->rhs.begin(), S->rhs.end(), rhs);
}

int orc_solve(void* h, double tol, int maxit, int restart, int* iters, double* relres) {
  Oracle* S = static_cast<Oracle*>(h);
  const int rc = gmres_ilu0(*S, tol, maxit, restart);
  if (iters) *iters = S->last_iters;
  if (relres) *relres = S->last_relres;
  return rc;
}

void orc_update(void* h) { update(*static_cast<Oracle*>(h)); }

// Full time steps: ZeroLSS, LinearizeU, Assembly, BCs, SolveLSS, Update.
int orc_step(void* h, int nsteps, double tol, int maxit, int restart, int nthreads) {
  Oracle* S = static_cast<Oracle*>(h);
  int rc = 0;
  for (int s = 0; s < nsteps; ++s) {
    assemble(*S, nthreads);
    apply_bcs(*S);
    rc |= gmres_ilu0(*S, tol, maxit, restart);
    update(*S);
  }
  return rc;
}

// Wall time (seconds) of `reps` ZeroLSS+LinearizeU+Assembly passes.
double orc_time_assembly(void* h, int nthreads, int reps) {
  Oracle* S = static_cast<Oracle*>(h);
  const auto t0 = std::chrono::steady_clock::now();
  for (int r = 0; r < reps; ++r) assemble(*S, nthreads);
  const auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

// The GPU benchmark's step on the host: ZeroLSS + LinearizeU + assembly
// (nthreads node-partitioned threads) + the symmetric Dirichlet conditions in
// their order, as DirichletBC applies them after the assembly
// (Proto/DirichletBC.hpp:34-51).  Seconds for `reps` steps.
double orc_time_step_assembly(void* h, int nthreads, int reps) {
  Oracle* S = static_cast<Oracle*>(h);
  const auto t0 = std::chrono::steady_clock::now();
  for (int r = 0; r < reps; ++r) {
    assemble(*S, nthreads);
    apply_bcs(*S);
  }
  const auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

// Element-level access for known-answer tests: A, T (nd x nd) and a (nd) of one
// element before the combine step, element-major dof order.
void orc_element(void* h, int64_t e, double* A, double* T, double* av) {
  Oracle* S = static_cast<Oracle*>(h);
  if (S->dim == 2) {
    ElemData<2> ed;
    gather<2>(*S, e, ed);
    if (S->o.use_specializations) { specialized_tri(ed, S->o.dt, S->o.rho, A, T); std::fill(av, av + 9, 0.0); }
    else generic_element<2>(*S, ed, A, T, av);
  } else {
    ElemData<3> ed;
    gather<3>(*S, e, ed);
    if (S->o.use_specializations) { specialized_tet(ed, S->o.dt, S->o.rho, A, T); std::fill(av, av + 16, 0.0); }
    else generic_element<3>(*S, ed, A, T, av);
  }
}

void orc_tau(int dim, int type, const double* X, const double* uc, double nu, double dt, double c1, double c2,
             double* out3) {
  const TauParams tp{type, c1, c2, 1., 1., 1., 1.};
  if (dim == 2) {
    double Xm[3][2];
    for (int i = 0; i < 3; ++i) for (int k = 0; k < 2; ++k) Xm[i][k] = X[i * 2 + k];
    compute_tau<2>(tp, Xm, uc, nu, dt, out3[0], out3[1], out3[2]);
  } else {
    double Xm[4][3];
    for (int i = 0; i < 4; ++i) for (int k = 0; k < 3; ++k) Xm[i][k] = X[i * 3 + k];
    compute_tau<3>(tp, Xm, uc, nu, dt, out3[0], out3[1], out3[2]);
  }
}

}  // extern "C"

// ===========================================================================
// Semi-implicit (pressure-correction) scheme: NavierStokesSemiImplicit
// (plugins/UFEM/src/UFEM/ns_semi_implicit/).  Element expressions from
// MatrixAssembly.hpp, the pressure matrix from PressureSystem.cpp:110-140, the
// step from implementation/NavierStokesSemiImplicit.cpp:96-198 and :329-375.
// Triangles and tetrahedra take IntegralOrder 1 (MatrixAssembly.hpp:28-46):
// the operators at the centroid, the mass terms with the order-2 rule.  Each
// element vector/matrix is formed completely, then added to the global rows in
// element order (as Proto's ElementLooper + BlockAccumulator do).  Linked
// (periodic) nodes keep identity rows with a zero right-hand side and receive
// their master's values after every solve.
// ===========================================================================
namespace {

struct Semi {
  Oracle F;  // mesh, options, fields: up N x (D+1), lin N x 4D, nu, force; periodic map
  Oracle U;  // velocity LSS (neq = D)
  Oracle P;  // pressure LSS (neq = 1)
  int nb_iterations = 2;
  double tol = 1e-13;
  std::vector<double> uvec, avec, pvec, dpsum, minv;
  int iters_u = 0, iters_p = 0;
  double worst_relres = 0.0;
};

void make_lss(const Oracle& F, int neq, Oracle& S) {
  S.dim = F.dim;
  S.nn = F.nn;
  S.neq = neq;
  S.N = F.N;
  S.E = F.E;
  S.coords = F.coords;
  S.conn = F.conn;
  S.o = F.o;
  S.p2m = F.p2m;
  build_graph(S);
}

template <int D>
constexpr double w1_ref() { return D == 2 ? 0.5 : 1.0 / 6.0; }  // GaussMappedCoords<1>: one point

template <int D>
struct SemiElem {
  static constexpr int n = D + 1;
  uint32_t node[n];
  double X[n][D], G[D][n], det;
  double tps, tsu, tbu;
  double nuc;   // nu_eff at the centroid
  double uc[D]; // tau velocity at the centroid
};

// Geometry and ComputeTauImpl (SUPG.hpp:140-219) on u_adv (`adv`) or on the
// velocity solution u.
template <int D>
void semi_elem(const Semi& M, int64_t e, bool adv, SemiElem<D>& s) {
  constexpr int n = D + 1;
  const Oracle& F = M.F;
  double U[n][D], NU[n];
  for (int b = 0; b < n; ++b) {
    const uint32_t node = F.conn[e * n + b];
    s.node[b] = node;
    for (int k = 0; k < D; ++k) {
      s.X[b][k] = F.coords[(size_t)node * D + k];
      U[b][k] = adv ? F.lin[(size_t)node * 4 * D + k] : F.up[(size_t)node * (D + 1) + k];
    }
    NU[b] = F.nu[node];
  }
  double J[D][D], Ji[D][D];
  jacobian<D>(s.X, J);
  inverse_det<D>(J, Ji, s.det);
  gradient<D>(Ji, s.G);
  double xi[D], Nc[n];
  centroid<D>(xi);
  shape_values<D>(xi, Nc);
  double nsum = 0.0;
  s.nuc = 0.0;
  for (int b = 0; b < n; ++b) {
    nsum += NU[b];
    s.nuc += Nc[b] * NU[b];
  }
  for (int k = 0; k < D; ++k) {
    double t = 0.0;
    for (int b = 0; b < n; ++b) t += Nc[b] * U[b][k];
    s.uc[k] = t;
  }
  const TauParams tp{F.o.supg_type, F.o.c1, F.o.c2, F.o.alpha_ps, F.o.alpha_su, F.o.alpha_bu, F.o.u_ref};
  compute_tau<D>(tp, s.X, s.uc, std::fabs(nsum / n), F.o.dt, s.tps, s.tsu, s.tbu);
}

template <int D>
double gdot(const SemiElem<D>& s, int a, int b) {
  double t = 0.0;
  for (int k = 0; k < D; ++k) t += s.G[k][a] * s.G[k][b];
  return t;
}

// Linked nodes: identity rows, zero right-hand side.
void semi_identity_rows(Oracle& S) {
  for (int64_t i = 0; i < S.N; ++i) {
    if (S.row_of((uint32_t)i) == (uint32_t)i) continue;
    for (int c = 0; c < S.neq; ++c) {
      const int64_t r = i * S.neq + c;
      for (int64_t p = S.rowptr[r]; p < S.rowptr[r + 1]; ++p) S.vals[p] = 0.0;
      S.vals[csr_pos(S, i, c, i, c)] = 1.0;
      S.rhs[r] = 0.0;
    }
  }
}

void semi_sync(const Oracle& S, std::vector<double>& v, int neq) {
  for (int64_t i = 0; i < S.N; ++i) {
    const uint32_t m = S.row_of((uint32_t)i);
    if (m == (uint32_t)i) continue;
    for (int c = 0; c < neq; ++c) v[i * neq + c] = v[(int64_t)m * neq + c];
  }
}

// VelocityAssembly (MatrixAssembly.hpp:52-149) + system_matrix += T + theta dt M
// (:428-432), after ZeroLSS of the matrix and the RHS.
template <int D>
void semi_velocity_matrix(Semi& M) {
  constexpr int n = D + 1, nd = n * D;
  Oracle& U = M.U;
  std::fill(U.vals.begin(), U.vals.end(), 0.0);
  std::fill(U.rhs.begin(), U.rhs.end(), 0.0);
  const double thdt = M.F.o.theta * M.F.o.dt;
  for (int64_t e = 0; e < M.F.E; ++e) {
    SemiElem<D> s;
    semi_elem<D>(M, e, true, s);
    double T[nd][nd] = {}, Mm[nd][nd] = {};
    for (int q = 0; q < Gauss2<D>::np; ++q) {  // mass, always order 2
      double xi[D], N[n];
      Gauss2<D>::point(q, xi);
      shape_values<D>(xi, N);
      const double w = Gauss2<D>::weight() * s.det;
      for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) {
          const double v = (w * N[a]) * N[b];
          for (int i = 0; i < D; ++i) T[i * n + a][i * n + b] += v;
        }
    }
    const double w = w1_ref<D>() * s.det;
    const double bulk = w * s.tbu;
    for (int i = 0; i < D; ++i)  // laplacian + diagonal bulk blocks, centroid
      for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b)
          Mm[i * n + a][i * n + b] += (w * s.nuc) * gdot<D>(s, a, b) + (bulk * s.G[i][a]) * s.G[i][b];
    for (int i = 0; i < D; ++i)  // off-diagonal bulk blocks
      for (int j = i + 1; j < D; ++j)
        for (int a = 0; a < n; ++a)
          for (int b = 0; b < n; ++b) {
            const double v = (bulk * s.G[i][a]) * s.G[j][b];
            Mm[i * n + a][j * n + b] += v;
            Mm[j * n + b][i * n + a] += v;
          }
    for (int a = 0; a < n; ++a) {
      const int64_t ra = U.row_of(s.node[a]);
      for (int i = 0; i < D; ++i)
        for (int b = 0; b < n; ++b) {
          const int64_t base = csr_pos(U, ra, i, U.row_of(s.node[b]), 0);
          for (int j = 0; j < D; ++j) U.vals[base + j] += T[i * n + a][j * n + b] + thdt * Mm[i * n + a][j * n + b];
        }
    }
  }
  semi_identity_rows(U);
}

// PressureSystemAssembly::assemble_pp (PressureSystem.cpp:128-140), tau from u.
template <int D>
void semi_pressure_matrix(Semi& M) {
  constexpr int n = D + 1;
  Oracle& P = M.P;
  std::fill(P.vals.begin(), P.vals.end(), 0.0);
  std::fill(P.rhs.begin(), P.rhs.end(), 0.0);
  std::fill(P.sol.begin(), P.sol.end(), 0.0);
  for (int64_t e = 0; e < M.F.E; ++e) {
    SemiElem<D> s;
    semi_elem<D>(M, e, false, s);
    const double coef = M.F.o.theta * (s.tps + M.F.o.dt);
    for (int a = 0; a < n; ++a)
      for (int b = 0; b < n; ++b) {
        double A = 0.0;
        for (int q = 0; q < Gauss2<D>::np; ++q) A += (Gauss2<D>::weight() * s.det) * gdot<D>(s, a, b);
        P.vals[csr_pos(P, P.row_of(s.node[a]), 0, P.row_of(s.node[b]), 0)] += coef * A;
      }
  }
  semi_identity_rows(P);
}

// Lumped mass (MatrixAssembly.hpp:411-420) and its reciprocal
// (NavierStokesSemiImplicit.cpp:238-247).
template <int D>
void semi_lumped_mass(Semi& M) {
  constexpr int n = D + 1;
  std::vector<double> diag(M.F.N * D, 0.0);
  for (int64_t e = 0; e < M.F.E; ++e) {
    SemiElem<D> s;
    semi_elem<D>(M, e, true, s);
    double Me[n][n] = {};
    for (int q = 0; q < Gauss2<D>::np; ++q) {
      double xi[D], N[n];
      Gauss2<D>::point(q, xi);
      shape_values<D>(xi, N);
      const double w = Gauss2<D>::weight() * s.det;
      for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) Me[a][b] += (w * N[a]) * N[b];
    }
    for (int a = 0; a < n; ++a) {
      double rs = 0.0;
      for (int b = 0; b < n; ++b) rs += Me[a][b];
      for (int i = 0; i < D; ++i) diag[(size_t)M.U.row_of(s.node[a]) * D + i] += rs;
    }
  }
  M.minv.assign(M.F.N * D, 0.0);
  for (size_t k = 0; k < diag.size(); ++k) M.minv[k] = 1.0 / diag[k];
  semi_sync(M.U, M.minv, D);
}

// VelocityRHS (MatrixAssembly.hpp:212-360) into U.rhs (zeroed first).
template <int D>
void semi_velocity_rhs(Semi& M) {
  constexpr int n = D + 1;
  Oracle& U = M.U;
  std::fill(U.rhs.begin(), U.rhs.end(), 0.0);
  const double theta = M.F.o.theta, dt = M.F.o.dt;
  const double dtl = dt * (1. - theta), omt = 1. - theta;
  for (int64_t e = 0; e < M.F.E; ++e) {
    SemiElem<D> s;
    semi_elem<D>(M, e, true, s);
    double Ua[n][D], AV[n][D], DAU[n][D], PP[n], Fo[n][D];
    for (int b = 0; b < n; ++b) {
      const uint32_t node = s.node[b];
      for (int k = 0; k < D; ++k) {
        Ua[b][k] = M.F.lin[(size_t)node * 4 * D + k];
        AV[b][k] = M.avec[(size_t)node * D + k];
        DAU[b][k] = dtl * AV[b][k] - M.uvec[(size_t)node * D + k];
        Fo[b][k] = M.F.force.empty() ? 0.0 : M.F.force[(size_t)node * D + k];
      }
      PP[b] = omt * M.dpsum[node] - M.pvec[node];
    }
    double res[D][n] = {};
    for (int q = 0; q < Gauss2<D>::np; ++q) {  // mass part, order 2
      double xi[D], N[n];
      Gauss2<D>::point(q, xi);
      shape_values<D>(xi, N);
      const double w = Gauss2<D>::weight() * s.det;
      double uq[D], adv[n], npa[n];
      for (int k = 0; k < D; ++k) {
        uq[k] = 0.0;
        for (int b = 0; b < n; ++b) uq[k] += N[b] * Ua[b][k];
      }
      for (int b = 0; b < n; ++b) {
        adv[b] = 0.0;
        for (int k = 0; k < D; ++k) adv[b] += uq[k] * s.G[k][b];
        npa[b] = s.tsu * adv[b] + N[b];
      }
      double f = 0.0;
      for (int i = 0; i < D; ++i)
        for (int b = 0; b < n; ++b) f += s.G[i][b] * DAU[b][i];
      f *= w;
      const double fs = 0.5 * f;
      for (int i = 0; i < D; ++i) {
        double c = 0.0, ee = 0.0;
        for (int b = 0; b < n; ++b) {
          c += N[b] * AV[b][i];
          ee += adv[b] * DAU[b][i];
        }
        c = -w * c;
        ee = w * ee;
        for (int a = 0; a < n; ++a) res[i][a] += npa[a] * (c + ee + fs * uq[i]);
      }
    }
    {  // operator part, centroid
      double xi[D], N[n];
      centroid<D>(xi);
      shape_values<D>(xi, N);
      const double w = w1_ref<D>() * s.det;
      const double wv = w * s.nuc, tw = w * s.tsu;
      double adv[n];
      for (int b = 0; b < n; ++b) {
        adv[b] = 0.0;
        for (int k = 0; k < D; ++k) adv[b] += s.uc[k] * s.G[k][b];
      }
      double bb = 0.0;
      for (int b = 0; b < n; ++b) bb += N[b] * PP[b];
      bb = -w * bb;
      double f = 0.0;
      for (int i = 0; i < D; ++i)
        for (int b = 0; b < n; ++b) f += s.G[i][b] * DAU[b][i];
      f *= w;
      const double fb = s.tbu * f;
      for (int i = 0; i < D; ++i) {
        double av = 0.0;
        for (int b = 0; b < n; ++b) av += s.G[i][b] * PP[b];
        av = tw * av;
        double d[D];
        for (int k = 0; k < D; ++k) {
          double t = 0.0;
          for (int b = 0; b < n; ++b) t += s.G[k][b] * DAU[b][i];
          d[k] = wv * t;
        }
        for (int a = 0; a < n; ++a) {
          double visc = 0.0;
          for (int k = 0; k < D; ++k) visc += s.G[k][a] * d[k];
          res[i][a] += adv[a] * av + s.G[i][a] * (bb + fb) + visc;
        }
      }
    }
    if (!M.F.force.empty()) {  // body force, order 2 (MatrixAssembly.hpp:344-360)
      for (int q = 0; q < Gauss2<D>::np; ++q) {
        double xi[D], N[n];
        Gauss2<D>::point(q, xi);
        shape_values<D>(xi, N);
        const double w = Gauss2<D>::weight() * s.det;
        for (int i = 0; i < D; ++i) {
          double g = 0.0;
          for (int b = 0; b < n; ++b) g += N[b] * Fo[b][i];
          for (int a = 0; a < n; ++a) res[i][a] += N[a] * g * w;
        }
      }
    }
    for (int a = 0; a < n; ++a)
      for (int i = 0; i < D; ++i) U.rhs[(size_t)U.row_of(s.node[a]) * D + i] += res[i][a];
  }
}

// PressureRHS (MatrixAssembly.hpp:153-210) into P.rhs (zeroed first); tau_ps from u.
template <int D>
void semi_pressure_rhs(Semi& M) {
  constexpr int n = D + 1;
  Oracle& P = M.P;
  std::fill(P.rhs.begin(), P.rhs.end(), 0.0);
  const double dt = M.F.o.dt;
  for (int64_t e = 0; e < M.F.E; ++e) {
    SemiElem<D> s;
    semi_elem<D>(M, e, false, s);
    double Ua[n][D], UP[n][D], APD[n][D], PV[n];
    for (int b = 0; b < n; ++b) {
      const uint32_t node = s.node[b];
      for (int k = 0; k < D; ++k) {
        const size_t r = (size_t)node * D + k;
        Ua[b][k] = M.F.lin[(size_t)node * 4 * D + k];
        UP[b][k] = M.uvec[r] + dt * M.U.sol[r];
        APD[b][k] = M.avec[r] + M.U.sol[r];
      }
      PV[b] = M.pvec[node];
    }
    double xi[D], N[n];
    centroid<D>(xi);
    shape_values<D>(xi, N);
    const double w = w1_ref<D>() * s.det, tw = w * s.tps;
    double adv[n];
    double ua[D];
    for (int k = 0; k < D; ++k) {
      ua[k] = 0.0;
      for (int b = 0; b < n; ++b) ua[k] += N[b] * Ua[b][k];
    }
    for (int b = 0; b < n; ++b) {
      adv[b] = 0.0;
      for (int k = 0; k < D; ++k) adv[b] += (s.tps * ua[k]) * s.G[k][b];
    }
    double res[n] = {};
    for (int i = 0; i < D; ++i) {
      double av = 0.0, bv = 0.0, cv = 0.0;
      for (int b = 0; b < n; ++b) {
        av += s.G[i][b] * UP[b][i];
        bv += adv[b] * UP[b][i];
        cv += N[b] * APD[b][i];
      }
      av *= w;
      bv *= w;
      cv *= tw;
      for (int a = 0; a < n; ++a) res[a] -= av * (N[a] + adv[a] * 0.5) + (bv + cv) * s.G[i][a];
    }
    for (int a = 0; a < n; ++a) {
      double t = 0.0;
      for (int b = 0; b < n; ++b) t += (tw * gdot<D>(s, a, b)) * PV[b];
      res[a] -= t;
    }
    for (int a = 0; a < n; ++a) P.rhs[P.row_of(s.node[a])] += res[a];
  }
}

// ApplyAup (MatrixAssembly.hpp:364-404) into U.rhs (zeroed first); tau_su from u_adv.
template <int D>
void semi_apply_aup(Semi& M) {
  constexpr int n = D + 1;
  Oracle& U = M.U;
  std::fill(U.rhs.begin(), U.rhs.end(), 0.0);
  for (int64_t e = 0; e < M.F.E; ++e) {
    SemiElem<D> s;
    semi_elem<D>(M, e, true, s);
    double dp[n];
    for (int b = 0; b < n; ++b) dp[b] = M.P.sol[s.node[b]];
    double xi[D], N[n];
    centroid<D>(xi);
    shape_values<D>(xi, N);
    const double w = M.F.o.theta * w1_ref<D>() * s.det;
    double adv[n];
    for (int b = 0; b < n; ++b) {
      double t = 0.0;
      for (int k = 0; k < D; ++k) t += s.uc[k] * s.G[k][b];
      adv[b] = (w * s.tsu) * t;
    }
    double bb = 0.0;
    for (int b = 0; b < n; ++b) bb += N[b] * dp[b];
    bb = -w * bb;
    for (int i = 0; i < D; ++i) {
      double av = 0.0;
      for (int b = 0; b < n; ++b) av += s.G[i][b] * dp[b];
      for (int a = 0; a < n; ++a) U.rhs[(size_t)U.row_of(s.node[a]) * D + i] += av * adv[a] + bb * s.G[i][a];
    }
  }
}

// BoundaryConditions of one system: symmetric Dirichlet in list order with
// value - field (Proto/DirichletBC.hpp:34-39); `field(node, comp)` reads u or p.
template <typename FieldT>
void semi_apply_bcs(Oracle& S, FieldT field) {
  for (const BC& bc : S.bcs) {
    const uint32_t row = S.row_of(bc.node);
    symmetric_dirichlet(S, row, bc.comp, bc.value - field(row, bc.comp));
  }
}

void semi_zero_bc_rows(const Oracle& S, std::vector<double>& v) {
  for (const BC& bc : S.bcs) v[(size_t)S.row_of(bc.node) * S.neq + bc.comp] = 0.0;
}

int semi_solve(Semi& M, Oracle& S, int& iters) {
  const int rc = gmres_ilu0(S, M.tol, 20000, 200);
  iters += S.last_iters;
  M.worst_relres = std::max(M.worst_relres, S.last_relres);
  return rc;
}

// One time step (NavierStokesSemiImplicit.cpp:329-375 with InnerLoop::execute :104-191).
template <int D>
int semi_step(Semi& M) {
  Oracle& F = M.F;
  const int64_t N = F.N;
  const double dt = F.o.dt;
  int rc = 0;
  linearize(F);
  semi_velocity_matrix<D>(M);
  M.uvec.assign(N * D, 0.0);
  M.avec.assign(N * D, 0.0);
  M.pvec.assign(N, 0.0);
  M.dpsum.assign(N, 0.0);
  for (int64_t i = 0; i < N; ++i) {
    for (int k = 0; k < D; ++k) M.uvec[i * D + k] = F.up[i * (D + 1) + k];
    M.pvec[i] = F.up[i * (D + 1) + D];
  }
  auto ufield = [&](uint32_t node, int comp) { return F.up[(size_t)node * (D + 1) + comp]; };
  auto pfield = [&](uint32_t node, int) { return F.up[(size_t)node * (D + 1) + D]; };
  for (int it = 0; it < M.nb_iterations; ++it) {
    semi_velocity_rhs<D>(M);
    if (it == 0) {
      for (double& r : M.U.rhs) r *= dt;
      semi_apply_bcs(M.U, ufield);
      for (double& r : M.U.rhs) r *= 1. / dt;
    } else {
      semi_zero_bc_rows(M.U, M.U.rhs);
    }
    std::fill(M.U.sol.begin(), M.U.sol.end(), 0.0);
    rc |= semi_solve(M, M.U, M.iters_u);
    semi_sync(M.U, M.U.sol, D);
    semi_pressure_rhs<D>(M);
    std::fill(M.P.sol.begin(), M.P.sol.end(), 0.0);
    if (it == 0) semi_apply_bcs(M.P, pfield);
    else semi_zero_bc_rows(M.P, M.P.rhs);
    rc |= semi_solve(M, M.P, M.iters_p);
    semi_sync(M.P, M.P.sol, 1);
    semi_apply_aup<D>(M);
    semi_zero_bc_rows(M.U, M.U.rhs);
    for (int64_t r = 0; r < N * D; ++r) M.U.sol[r] = M.U.sol[r] - M.minv[r] * M.U.rhs[r];
    semi_sync(M.U, M.U.sol, D);
    for (int64_t i = 0; i < N; ++i) {
      for (int k = 0; k < D; ++k) {
        const int64_t r = i * D + k;
        M.avec[r] = M.avec[r] + M.U.sol[r];
        M.uvec[r] = M.uvec[r] + dt * M.U.sol[r];
      }
      M.pvec[i] = M.pvec[i] + M.P.sol[i];
      M.dpsum[i] = M.dpsum[i] + M.P.sol[i];
    }
  }
  for (int64_t i = 0; i < N; ++i) {  // Update
    double* L = &F.lin[i * 4 * D];
    for (int k = 0; k < D; ++k) {
      L[3 * D + k] = L[2 * D + k];
      L[2 * D + k] = L[D + k];
      L[D + k] = F.up[i * (D + 1) + k];
      F.up[i * (D + 1) + k] = M.uvec[i * D + k];
    }
    F.up[i * (D + 1) + D] = M.pvec[i];
  }
  return rc;
}

}  // namespace

extern "C" {

void* orc_semi_create(int dim, int64_t nb_nodes, int64_t nb_elems, const double* coords, const uint32_t* conn,
                      const orc_options* opts, int nb_iterations, const uint32_t* slaves, const uint32_t* masters,
                      int64_t nlinks) {
  Oracle* F = static_cast<Oracle*>(
      orc_create_periodic(dim, nb_nodes, nb_elems, coords, conn, opts, slaves, masters, nlinks));
  if (!F) return nullptr;
  Semi* M = new Semi();
  M->F = std::move(*F);
  delete F;
  M->nb_iterations = nb_iterations;
  make_lss(M->F, dim, M->U);
  make_lss(M->F, 1, M->P);
  return M;
}

void orc_semi_destroy(void* h) { delete static_cast<Semi*>(h); }

void orc_semi_set_state(void* h, const double* up, const double* lin, const double* nu, const double* force) {
  orc_set_state(&static_cast<Semi*>(h)->F, up, lin, nu, force);
}

void orc_semi_get_state(void* h, double* up, double* lin) { orc_get_state(&static_cast<Semi*>(h)->F, up, lin); }

void orc_semi_add_dirichlet(void* h, int which, const uint32_t* nodes, int64_t n, int comp, const double* values) {
  Semi* M = static_cast<Semi*>(h);
  Oracle& S = which == 0 ? M->U : M->P;
  for (int64_t i = 0; i < n; ++i) S.bcs.push_back(BC{nodes[i], comp, values[i]});
}

void orc_semi_clear_dirichlet(void* h, int which) {
  Semi* M = static_cast<Semi*>(h);
  (which == 0 ? M->U : M->P).bcs.clear();
}

void orc_semi_set_fields(void* h, const double* up, const double* lin) {
  Semi* M = static_cast<Semi*>(h);
  M->F.up.assign(up, up + M->F.N * (M->F.dim + 1));
  M->F.lin.assign(lin, lin + M->F.N * 4 * M->F.dim);
}

// Initial conditions (NavierStokesSemiImplicit.cpp:400-455): with reset,
// u_adv = u1 = u2 = u3 = u; the pressure matrix and the lumped mass.
void orc_semi_initialize(void* h, int reset_history) {
  Semi* M = static_cast<Semi*>(h);
  Oracle& F = M->F;
  const int D = F.dim;
  if (reset_history)
    for (int64_t i = 0; i < F.N; ++i)
      for (int j = 0; j < 4; ++j)
        for (int k = 0; k < D; ++k) F.lin[i * 4 * D + j * D + k] = F.up[i * (D + 1) + k];
  if (D == 2) {
    semi_pressure_matrix<2>(*M);
    semi_lumped_mass<2>(*M);
  } else {
    semi_pressure_matrix<3>(*M);
    semi_lumped_mass<3>(*M);
  }
}

// nsteps steps; returns 0 when every solve converged.  iters: (velocity, pressure) totals.
int orc_semi_step(void* h, int nsteps, double tol, int* iters, double* worst_relres) {
  Semi* M = static_cast<Semi*>(h);
  M->tol = tol;
  M->iters_u = M->iters_p = 0;
  M->worst_relres = 0.0;
  int rc = 0;
  for (int k = 0; k < nsteps; ++k) rc |= (M->F.dim == 2 ? semi_step<2>(*M) : semi_step<3>(*M));
  if (iters) {
    iters[0] = M->iters_u;
    iters[1] = M->iters_p;
  }
  if (worst_relres) *worst_relres = M->worst_relres;
  return rc;
}

// The velocity matrix of the current state (LinearizeU + VelocityAssembly), no BCs.
void orc_semi_velocity_matrix(void* h) {
  Semi* M = static_cast<Semi*>(h);
  linearize(M->F);
  if (M->F.dim == 2) semi_velocity_matrix<2>(*M);
  else semi_velocity_matrix<3>(*M);
}

// Element right-hand sides on given inner-loop vectors (parity of the vector
// expressions): kind 0 velocity RHS, 1 pressure RHS (da = delta_a),
// 2 A_up dp.  Results land in the system's rhs (read with orc_semi_get_system).
void orc_semi_rhs(void* h, int kind, const double* uvec, const double* avec, const double* pvec, const double* dpsum,
                  const double* da, const double* dp) {
  Semi* M = static_cast<Semi*>(h);
  const int D = M->F.dim;
  const int64_t N = M->F.N;
  M->uvec.assign(uvec, uvec + N * D);
  M->avec.assign(avec, avec + N * D);
  M->pvec.assign(pvec, pvec + N);
  M->dpsum.assign(dpsum, dpsum + N);
  std::copy(da, da + N * D, M->U.sol.begin());
  std::copy(dp, dp + N, M->P.sol.begin());
  if (kind == 0) (D == 2) ? semi_velocity_rhs<2>(*M) : semi_velocity_rhs<3>(*M);
  else if (kind == 1) (D == 2) ? semi_pressure_rhs<2>(*M) : semi_pressure_rhs<3>(*M);
  else (D == 2) ? semi_apply_aup<2>(*M) : semi_apply_aup<3>(*M);
}

int64_t orc_semi_nnz(void* h, int which) {
  Semi* M = static_cast<Semi*>(h);
  return (int64_t)(which == 0 ? M->U : M->P).vals.size();
}

void orc_semi_get_system(void* h, int which, double* vals, double* rhs, double* sol) {
  Semi* M = static_cast<Semi*>(h);
  const Oracle& S = which == 0 ? M->U : M->P;
  if (vals) std::copy(S.vals.begin(), S.vals.end(), vals);
  if (rhs) std::copy(S.rhs.begin(), S.rhs.end(), rhs);
  if (sol) std::copy(S.sol.begin(), S.sol.end(), sol);
}

void orc_semi_lumped_inverse(void* h, double* out) {
  Semi* M = static_cast<Semi*>(h);
  std::copy(M->minv.begin(), M->minv.end(), out);
}

}  // extern "C"
