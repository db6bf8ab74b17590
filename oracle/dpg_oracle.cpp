// dpg_oracle.cpp — CPU FP64 restatement of Camellia's DPG per-cell assembly.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
// camellia2_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg load it.  The product never links or calls it.
//
// Parity status.  The reference (ApolloFramework/camellia2) cannot be built in
// this environment (Trilinos/Intrepid/Epetra/MOAB absent), so this file restates
// its algorithm.  It is pinned against the reference's own known-answer tests:
//   * unit_tests/BFTests.cpp:28-72, 136-219, 221-300, 302-381 — factoredCholeskySolve
//     golden matrices (tests/test_oracle_golden.py);
//   * drivers/DPGTests/DPGTests.cpp:557-655 — flux stiffness 2/3, 1/3 on the
//     reference quad (side parametrisation, trace basis, side measure);
//   * unit_tests/BasisCacheTests.cpp:60-82 — line cubature exactness, Jacobian of
//     the reference cell;
//   * unit_tests/SolutionTests.cpp:779-810 idea — condensed == uncondensed.
// Entry-level K/G values for the full formulations have no golden vectors in the
// reference; they are pinned by basis-invariant checks (tests/).
//
// Steps restated (file:line in the reference):
//   bases            src/Basis/BasisFactory.cpp:122-420 (HGRAD Cn on spectral =
//                    Gauss-Lobatto points, HDIV In, HVOL = HGRAD C(k-1), traces)
//   cubature         src/Basis/CubatureFactory.cpp:25-53 (tensor Gauss rules,
//                    n = degree/2 + 1 points per direction)
//   degrees          src/Basis/BasisCache.cpp:68-84, 236-267, 198-222
//   geometry         src/Basis/BasisCache.cpp:1325-1406 (J, detJ, J^-1),
//                    1860-1894 (weighted measure), 1798-1858 (side normals),
//                    src/CellTools/CamelliaCellTools.cpp:134-170 (side measure)
//   transforms       src/Basis/BasisEvaluation.cpp:182-390 (HGRAD grad J^-T,
//                    HDIV J v / detJ, div / detJ, HVOL identity)
//   integration      src/ScratchPad/LinearTerm.cpp:427-627, 646-723 (volume and
//                    per-side blocks, weights on the first factor, FLUX parity
//                    1085-1107)
//   B                src/ScratchPad/BF.cpp:575-656 (rowMajor: (C, trial, test))
//   G                src/ScratchPad/IP.cpp:215-292
//   F                src/Problem/RHS.cpp:68-82
//   solve            src/ScratchPad/BF.cpp:924-1018 (DPOEQU, DPOTRF('L'),
//                    unscale, DTRSM, DSYRK + mirror, DTRSM on F, GEMV)
//   condensation     src/Solution/CondensedDofInterpreter.cpp:1063-1225
//                    (Epetra_SerialDenseSolver: optional DGEEQU equilibration,
//                    LU with partial pivoting)
//
// Precision.  The same source builds twice (oracle/build.sh): liboracle.so with
// `real` = double, the FP64 oracle the GPU path is compared with, and
// liboracle_xp.so with `real` = __float128 (113-bit significand, libquadmath), the
// extended-precision truth that measures how far each FP64 code is from the exact
// result of the same double inputs (nodes, coefficients).  Everything between the
// inputs and the outputs -- cubature points and weights, basis tables, geometry,
// products, factorisations -- runs in `real`; the C interface below converts at the
// boundary.
//
// Third-party arithmetic restated here (not present under the reference tree):
// Intrepid (Trilinos, version unpinned by the reference: "a recent version",
// trilinos-fixes targets 12.6.4) bases, cubature and FunctionSpaceTools; LAPACK
// DPOEQU/DPOTRF/DTRSM/DSYRK/DGEEQU/DGETRF semantics.

#include "../include/dpg_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>
#include <string>

#ifdef ORC_QUAD
#include <quadmath.h>
#define ORC_NS orc_xp
#else
#define ORC_NS orc
#endif

namespace ORC_NS {
#ifdef ORC_QUAD
typedef __float128 real;
static inline real r_sqrt(real x) { return sqrtq(x); }
static inline real r_fabs(real x) { return fabsq(x); }
static inline real r_cos(real x) { return cosq(x); }
static inline real r_sin(real x) { return sinq(x); }
static inline real r_pow(real a, real b) { return powq(a, b); }
static inline real r_tgamma(real x) { return tgammaq(x); }
static inline bool r_isnan(real x) { return isnanq(x); }
static const real R_PI = M_PIq;
static const real R_NEWTON_TOL = 1e-32;
#else
typedef double real;
static inline real r_sqrt(real x) { return std::sqrt(x); }
static inline real r_fabs(real x) { return std::fabs(x); }
static inline real r_cos(real x) { return std::cos(x); }
static inline real r_sin(real x) { return std::sin(x); }
static inline real r_pow(real a, real b) { return std::pow(a, b); }
static inline real r_tgamma(real x) { return std::tgamma(x); }
static inline bool r_isnan(real x) { return std::isnan(x); }
static const real R_PI = M_PI;
static const real R_NEWTON_TOL = 1e-16;
#endif
}  // namespace ORC_NS

namespace ORC_NS {

using std::vector;

// ----------------------------------------------------------------------------
// 1D rules
// ----------------------------------------------------------------------------

// Legendre P_n and derivative at x by the three-term recurrence.
static void legendre(int n, real x, real& p, real& dp) {
  real p0 = 1.0, p1 = x;
  if (n == 0) { p = 1.0; dp = 0.0; return; }
  for (int k = 2; k <= n; k++) {
    real pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
    p0 = p1; p1 = pk;
  }
  p = p1;
  dp = (r_fabs(1.0 - x * x) < 1e-300) ? 0.0 : n * (p0 - x * p1) / (1.0 - x * x);
}

// Gauss-Legendre n-point rule on [-1,1], ascending nodes.
void gauss_legendre(int n, real* x, real* w) {
  for (int i = 0; i < n; i++) {
    real xi = -r_cos(R_PI * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; it++) {
      real p, dp;
      legendre(n, xi, p, dp);
      real dx = p / dp;
      xi -= dx;
      if (r_fabs(dx) < R_NEWTON_TOL) break;
    }
    real p, dp;
    legendre(n, xi, p, dp);
    x[i] = xi;
    w[i] = 2.0 / ((1.0 - xi * xi) * dp * dp);
  }
}

// Gauss-Lobatto nodes (p+1 of them) for degree p >= 1: +-1 and the roots of P'_p.
void gauss_lobatto(int p, real* x) {
  x[0] = -1.0;
  x[p] = 1.0;
  for (int i = 1; i < p; i++) {
    real xi = -r_cos(R_PI * i / p);
    for (int it = 0; it < 100; it++) {
      real P, dP;
      legendre(p, xi, P, dP);
      real d2P = (2.0 * xi * dP - p * (p + 1.0) * P) / (1.0 - xi * xi);
      real dx = dP / d2P;
      xi -= dx;
      if (r_fabs(dx) < R_NEWTON_TOL) break;
    }
    x[i] = xi;
  }
}

// Lagrange polynomial i on `nodes` (size m) and its derivative at x.
static void lagrange(const vector<real>& nodes, int i, real x, real& v, real& dv) {
  int m = (int)nodes.size();
  v = 1.0;
  for (int j = 0; j < m; j++)
    if (j != i) v *= (x - nodes[j]) / (nodes[i] - nodes[j]);
  dv = 0.0;
  for (int k = 0; k < m; k++) {
    if (k == i) continue;
    real t = 1.0 / (nodes[i] - nodes[k]);
    for (int j = 0; j < m; j++)
      if (j != i && j != k) t *= (x - nodes[j]) / (nodes[i] - nodes[j]);
    dv += t;
  }
}

// 1D nodal family: "closed" (Gauss-Lobatto, degree n, n+1 nodes) or "open"
// (Gauss-Legendre, degree n, n+1 nodes).  Degree 0 closed = constant.
struct Nodal1D {
  vector<real> nodes;
  void closed(int n) {
    nodes.assign(n + 1, 0.0);
    if (n >= 1) gauss_lobatto(n, nodes.data());
  }
  void open(int n) {
    nodes.assign(n + 1, 0.0);
    vector<real> w(n + 1);
    gauss_legendre(n + 1, nodes.data(), w.data());
  }
  int size() const { return (int)nodes.size(); }
  void eval(int i, real x, real& v, real& dv) const {
    if (nodes.size() == 1) { v = 1.0; dv = 0.0; return; }
    lagrange(nodes, i, x, v, dv);
  }
};

// ----------------------------------------------------------------------------
// Topology
// ----------------------------------------------------------------------------

struct Topo {
  int key = 0, d = 0, nv = 0, nsides = 0, side_nv = 0;
  real v[8][3] = {};
  int sv[6][4] = {};
};

static Topo make_topo(int key) {
  Topo t;
  t.key = key;
  if (key == DPG_TOPO_QUAD) {
    t.d = 2; t.nv = 4; t.nsides = 4; t.side_nv = 2;
    real v[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
    for (int i = 0; i < 4; i++) { t.v[i][0] = v[i][0]; t.v[i][1] = v[i][1]; }
    for (int s = 0; s < 4; s++) { t.sv[s][0] = s; t.sv[s][1] = (s + 1) % 4; }
  } else if (key == DPG_TOPO_HEX) {
    t.d = 3; t.nv = 8; t.nsides = 6; t.side_nv = 4;
    real v[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                      {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
    for (int i = 0; i < 8; i++) for (int k = 0; k < 3; k++) t.v[i][k] = v[i][k];
    // shards Hexahedron<8> face node lists
    int f[6][4] = {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {0, 4, 7, 3}, {0, 3, 2, 1}, {4, 5, 6, 7}};
    for (int s = 0; s < 6; s++) for (int k = 0; k < 4; k++) t.sv[s][k] = f[s][k];
  } else if (key == DPG_TOPO_TRI) {
    t.d = 2; t.nv = 3; t.nsides = 3; t.side_nv = 2;
    real v[3][2] = {{0, 0}, {1, 0}, {0, 1}};
    for (int i = 0; i < 3; i++) { t.v[i][0] = v[i][0]; t.v[i][1] = v[i][1]; }
    for (int s = 0; s < 3; s++) { t.sv[s][0] = s; t.sv[s][1] = (s + 1) % 3; }
  }
  return t;
}

// Vertex shape functions of the geometric map (HGRAD C1, vertex ordered).
static void geom_shape(const Topo& t, const real* xi, real* N, real* dN /*nv x d*/) {
  if (t.key == DPG_TOPO_TRI) {
    N[0] = 1 - xi[0] - xi[1]; N[1] = xi[0]; N[2] = xi[1];
    dN[0] = -1; dN[1] = -1; dN[2] = 1; dN[3] = 0; dN[4] = 0; dN[5] = 1;
    return;
  }
  for (int a = 0; a < t.nv; a++) {
    real f[3], df[3];
    for (int k = 0; k < t.d; k++) {
      f[k] = 0.5 * (1.0 + xi[k] * t.v[a][k]);
      df[k] = 0.5 * t.v[a][k];
    }
    real prod = 1.0;
    for (int k = 0; k < t.d; k++) prod *= f[k];
    N[a] = prod;
    for (int k = 0; k < t.d; k++) {
      real g = df[k];
      for (int m = 0; m < t.d; m++) if (m != k) g *= f[m];
      dN[a * t.d + k] = g;
    }
  }
}

// ----------------------------------------------------------------------------
// Bases: tabulation of reference values at points
// ----------------------------------------------------------------------------

// ----------------------------------------------------------------------------
// Triangle bases.  Intrepid's Basis_HGRAD_TRI_Cn_FEM (POINTTYPE_WARPBLEND,
// BasisFactory.cpp:198-350) is a Lagrange basis on the warp & blend lattice; the
// lattice is restated from the published construction (Warburton 2006;
// Hesthaven & Warburton, "Nodal Discontinuous Galerkin Methods", Nodes2D with the
// optimized alpha table), and the Lagrange functions are built through the
// orthonormal Proriol-Koornwinder-Dubiner (PKD) basis on the biunit triangle.
// Basis_HDIV_TRI_In_FEM spans Raviart-Thomas RT_n (card n(n+2)); this file uses a
// modal basis of the same space: (p, 0), (0, p) for p in P_{n-1}, then x psi for
// the orthonormal PKD polynomials psi of exact degree n-1 (their leading homogeneous
// parts span the homogeneous polynomials of degree n-1; monomials there would make the
// Gram matrix needlessly ill-conditioned at high degree).  A test-space basis change leaves
// K, l and S unchanged (K = B^T G^-1 B is invariant under B -> T^T B, G -> T^T G T).
// ----------------------------------------------------------------------------

// Orthonormal Jacobi polynomial P_n^{(a,b)}(x) on [-1,1] (weight (1-x)^a (1+x)^b).
static real jacobi(real x, real a, real b, int n) {
  real g0 = r_pow(2.0, a + b + 1) / (a + b + 1) * r_tgamma(a + 1) * r_tgamma(b + 1) / r_tgamma(a + b + 1);
  real p0 = 1.0 / r_sqrt(g0);
  if (n == 0) return p0;
  real g1 = (a + 1) * (b + 1) / (a + b + 3) * g0;
  real p1 = ((a + b + 2) * x / 2 + (a - b) / 2) / r_sqrt(g1);
  if (n == 1) return p1;
  real aold = 2.0 / (2 + a + b) * r_sqrt((a + 1) * (b + 1) / (a + b + 3));
  for (int i = 1; i < n; i++) {
    real h1 = 2.0 * i + a + b;
    real anew = 2.0 / (h1 + 2) * r_sqrt((i + 1) * (i + 1 + a + b) * (i + 1 + a) * (i + 1 + b) / (h1 + 1) / (h1 + 3));
    real bnew = -(a * a - b * b) / h1 / (h1 + 2);
    real p2 = (-aold * p0 + (x - bnew) * p1) / anew;
    p0 = p1;
    p1 = p2;
    aold = anew;
  }
  return p1;
}
static real jacobi_d(real x, real a, real b, int n) {
  return n == 0 ? 0.0 : r_sqrt(n * (n + a + b + 1)) * jacobi(x, a + 1, b + 1, n - 1);
}

// PKD mode (i, j) and its (r, s) derivatives at a point of the biunit triangle.
static void pkd_mode(int i, int j, real r, real s, real& v, real& vr, real& vs) {
  real a = (r_fabs(s - 1.0) > 1e-14) ? 2.0 * (1.0 + r) / (1.0 - s) - 1.0 : -1.0, b = s;
  real fa = jacobi(a, 0, 0, i), dfa = jacobi_d(a, 0, 0, i);
  real gb = jacobi(b, 2 * i + 1, 0, j), dgb = jacobi_d(b, 2 * i + 1, 0, j);
  real hb = 0.5 * (1.0 - b);
  v = r_sqrt(2.0) * fa * gb * r_pow(1.0 - b, i);
  real dr = dfa * gb, ds = dfa * gb * 0.5 * (1.0 + a);
  if (i > 0) { dr *= r_pow(hb, i - 1); ds *= r_pow(hb, i - 1); }
  real tmp = dgb * r_pow(hb, i);
  if (i > 0) tmp -= 0.5 * i * gb * r_pow(hb, i - 1);
  ds += fa * tmp;
  const real sc = r_pow(2.0, i + 0.5);
  vr = dr * sc;
  vs = ds * sc;
}

// Warp & blend lattice of degree N on the reference triangle (0,0),(1,0),(0,1):
// Np = (N+1)(N+2)/2 points, bottom row first (eta = 0, xi ascending).
static vector<real> warp_blend_tri(int N) {
  static const real alpopt[15] = {0.0000, 0.0000, 1.4152, 0.1001, 0.2751, 0.9800, 1.0999, 1.2832,
                                    1.3648, 1.4773, 1.4959, 1.5743, 1.5770, 1.6223, 1.6258};
  const real alpha = N < 16 ? alpopt[N - 1] : 5.0 / 3.0;
  vector<real> gll(N + 1);
  gauss_lobatto(N, gll.data());
  auto warpf = [&](real r) {
    // interpolant on equispaced nodes of the GLL displacement, divided by 1 - r^2
    real w = 0.0;
    for (int i = 0; i <= N; i++) {
      real xi_eq = -1.0 + 2.0 * i / N, l = 1.0;
      for (int j = 0; j <= N; j++)
        if (j != i) l *= (r - (-1.0 + 2.0 * j / N)) / (xi_eq - (-1.0 + 2.0 * j / N));
      w += (gll[i] - xi_eq) * l;
    }
    return r_fabs(r) < 1.0 - 1e-10 ? w / (1.0 - r * r) : 0.0;
  };
  vector<real> out;
  const real c2 = r_cos(2 * R_PI / 3), s2 = r_sin(2 * R_PI / 3);
  const real c4 = r_cos(4 * R_PI / 3), s4 = r_sin(4 * R_PI / 3);
  for (int n = 0; n <= N; n++)
    for (int m = 0; m <= N - n; m++) {
      real L1 = (real)n / N, L3 = (real)m / N, L2 = 1.0 - L1 - L3;
      real x = -L2 + L3, y = (-L2 - L3 + 2 * L1) / r_sqrt(3.0);
      real w1 = 4 * L2 * L3 * warpf(L3 - L2) * (1 + (alpha * L1) * (alpha * L1));
      real w2 = 4 * L1 * L3 * warpf(L1 - L3) * (1 + (alpha * L2) * (alpha * L2));
      real w3 = 4 * L1 * L2 * warpf(L2 - L1) * (1 + (alpha * L3) * (alpha * L3));
      x += w1 + c2 * w2 + c4 * w3;
      y += s2 * w2 + s4 * w3;
      // equilateral -> biunit (r, s) -> reference (xi, eta)
      real b1 = (r_sqrt(3.0) * y + 1) / 3, b2 = (-3 * x - r_sqrt(3.0) * y + 2) / 6,
             b3 = (3 * x - r_sqrt(3.0) * y + 2) / 6;
      real r = -b2 + b3 - b1, s = -b2 - b3 + b1;
      out.push_back(0.5 * (1 + r));
      out.push_back(0.5 * (1 + s));
    }
  return out;
}

// Inverse of a dense n x n matrix (Gauss-Jordan, partial pivoting).
static vector<real> invert(vector<real> A, int n) {
  vector<real> X(n * n, 0.0);
  for (int i = 0; i < n; i++) X[i * n + i] = 1.0;
  for (int c = 0; c < n; c++) {
    int piv = c;
    for (int r = c + 1; r < n; r++)
      if (r_fabs(A[r * n + c]) > r_fabs(A[piv * n + c])) piv = r;
    for (int k = 0; k < n; k++) { std::swap(A[c * n + k], A[piv * n + k]); std::swap(X[c * n + k], X[piv * n + k]); }
    real inv = 1.0 / A[c * n + c];
    for (int k = 0; k < n; k++) { A[c * n + k] *= inv; X[c * n + k] *= inv; }
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      real f = A[r * n + c];
      if (f == 0.0) continue;
      for (int k = 0; k < n; k++) { A[r * n + k] -= f * A[c * n + k]; X[r * n + k] -= f * X[c * n + k]; }
    }
  }
  return X;
}

// Lagrange basis of degree N on the warp & blend lattice: phi_k = sum_m psi_m Vinv[m][k].
struct TriLagrange {
  int N = 0, card = 1;
  vector<real> vinv;
  void init(int n) {
    N = n;
    card = (n + 1) * (n + 2) / 2;
    if (n == 0) return;
    vector<real> X = warp_blend_tri(n), V((size_t)card * card);
    for (int p = 0; p < card; p++) {
      int m = 0;
      for (int i = 0; i <= n; i++)
        for (int j = 0; j <= n - i; j++, m++) {
          real v, vr, vs;
          pkd_mode(i, j, 2 * X[2 * p] - 1, 2 * X[2 * p + 1] - 1, v, vr, vs);
          V[(size_t)p * card + m] = v;
        }
    }
    vinv = invert(V, card);
  }
  // values and reference (xi, eta) gradients of all card functions
  void eval(const real* xi, real* val, real* grad) const {
    if (N == 0) {
      if (val) val[0] = 1.0;
      if (grad) { grad[0] = 0.0; grad[1] = 0.0; }
      return;
    }
    vector<real> pv(card), pr(card), ps(card);
    int m = 0;
    for (int i = 0; i <= N; i++)
      for (int j = 0; j <= N - i; j++, m++) pkd_mode(i, j, 2 * xi[0] - 1, 2 * xi[1] - 1, pv[m], pr[m], ps[m]);
    for (int k = 0; k < card; k++) {
      real v = 0, gx = 0, gy = 0;
      for (int mm = 0; mm < card; mm++) {
        real c = vinv[(size_t)mm * card + k];
        v += pv[mm] * c;
        gx += pr[mm] * c;
        gy += ps[mm] * c;
      }
      if (val) val[k] = v;
      if (grad) { grad[2 * k] = 2 * gx; grad[2 * k + 1] = 2 * gy; }  // d/dxi = 2 d/dr
    }
  }
};

// Modal RT_n basis on the reference triangle: values (2 per function) and divergence.
static void tri_rt_eval(int n, const real* xi, real* val, real* div) {
  const int np = n * (n + 1) / 2;  // dim P_{n-1}
  vector<real> pv(np), pr(np), ps(np);
  int m = 0;
  for (int i = 0; i <= n - 1; i++)
    for (int j = 0; j <= n - 1 - i; j++, m++) pkd_mode(i, j, 2 * xi[0] - 1, 2 * xi[1] - 1, pv[m], pr[m], ps[m]);
  int dof = 0;
  for (int c = 0; c < 2; c++)
    for (int k = 0; k < np; k++, dof++) {
      if (val) { val[2 * dof] = c == 0 ? pv[k] : 0.0; val[2 * dof + 1] = c == 1 ? pv[k] : 0.0; }
      if (div) div[dof] = 2 * (c == 0 ? pr[k] : ps[k]);
    }
  for (int j = 0; j < n; j++, dof++) {
    real v, vr, vs;  // PKD polynomial of exact degree n-1; d/dxi = 2 d/dr
    pkd_mode(n - 1 - j, j, 2 * xi[0] - 1, 2 * xi[1] - 1, v, vr, vs);
    if (val) { val[2 * dof] = xi[0] * v; val[2 * dof + 1] = xi[1] * v; }
    if (div) div[dof] = 2 * v + 2 * (xi[0] * vr + xi[1] * vs);
  }
}

struct Basis {
  int topo = 0, space = 0, n = 0;  // n: Cn / In order of the Intrepid basis
  int d = 0, card = 0, rank = 0;   // rank 0 scalar, 1 vector (d comps)
  int ncomp = 1;                   // VECTOR_HVOL copies
  Nodal1D closed, open;            // 1D families
  TriLagrange tri;                 // triangle HGRAD
  // Tabulate at point xi: val[card*vdim], grad[card*d] (HGRAD-type), div[card]
  void eval(const real* xi, real* val, real* grad, real* div) const;
};

// Triangle bases are tabulated through a monomial-coefficient representation.
struct TriPoly {
  // dofs: coefficients in the monomial basis x^a y^b, a+b <= deg
  int deg = 0;
  vector<std::pair<int, int>> mono;
  vector<real> coef;  // card x nmono (scalar) or card x 2 x nmono (vector)
};

static int tensor_card(const Basis& b) {
  if (b.topo == DPG_TOPO_TRI)
    return b.space == DPG_SPACE_HDIV ? b.n * (b.n + 2) : (b.n + 1) * (b.n + 2) / 2 * b.ncomp;
  if (b.topo == DPG_TOPO_QUAD || b.topo == DPG_TOPO_HEX || b.topo == 0) {
    int m = b.closed.size();
    if (b.space == DPG_SPACE_HDIV) {
      int c = b.n + 1, o = b.n;
      return b.d == 2 ? 2 * c * o : 3 * c * o * o;
    }
    int p = 1;
    for (int k = 0; k < b.d; k++) p *= m;
    return p * b.ncomp;
  }
  return 0;
}

static Basis make_basis(int topo, int space, int n, int ncomp = 1) {
  Basis b;
  b.topo = topo; b.space = space; b.n = n; b.ncomp = ncomp;
  b.d = (topo == DPG_TOPO_HEX) ? 3 : (topo == 0 ? 1 : 2);  // topo 0 = line
  if (topo == DPG_TOPO_TRI) {
    b.rank = space == DPG_SPACE_HDIV ? 1 : 0;
    if (space != DPG_SPACE_HDIV) b.tri.init(n);
    b.card = tensor_card(b);
    return b;
  }
  if (space == DPG_SPACE_HDIV) {
    b.rank = 1;
    b.closed.closed(n);
    b.open.open(n - 1);
  } else {
    b.rank = 0;
    b.closed.closed(n);
  }
  b.card = tensor_card(b);
  return b;
}

void Basis::eval(const real* xi, real* val, real* grad, real* div) const {
  int d_ = d;
  if (topo == DPG_TOPO_TRI) {
    if (space == DPG_SPACE_HDIV) {
      tri_rt_eval(n, xi, val, div);
      return;
    }
    const int nper = tri.card;
    vector<real> v(nper), gr(2 * nper);
    tri.eval(xi, v.data(), gr.data());
    for (int c = 0; c < ncomp; c++)
      for (int k = 0; k < nper; k++) {
        const int dof = c * nper + k;
        if (val) val[dof] = v[k];
        if (grad) { grad[dof * 2] = gr[2 * k]; grad[dof * 2 + 1] = gr[2 * k + 1]; }
      }
    return;
  }
  if (space != DPG_SPACE_HDIV) {
    int m = closed.size();
    int nper = 1;
    for (int k = 0; k < d_; k++) nper *= m;
    real v1[3][16], d1[3][16];
    for (int k = 0; k < d_; k++)
      for (int i = 0; i < m; i++) closed.eval(i, xi[k], v1[k][i], d1[k][i]);
    for (int c = 0; c < ncomp; c++) {
      for (int idx = 0; idx < nper; idx++) {
        int ii[3] = {idx % m, (idx / m) % m, idx / (m * m)};
        real v = 1.0;
        for (int k = 0; k < d_; k++) v *= v1[k][ii[k]];
        int dof = c * nper + idx;
        if (val) val[dof] = v;
        if (grad) {
          for (int k = 0; k < d_; k++) {
            real g = d1[k][ii[k]];
            for (int j = 0; j < d_; j++) if (j != k) g *= v1[j][ii[j]];
            grad[dof * d_ + k] = g;
          }
        }
      }
    }
    return;
  }
  // HDIV tensor Raviart-Thomas: component c is closed (degree n) in direction c
  // and open (degree n-1) in the other directions; dofs component-major,
  // x fastest inside a component.
  int c1 = closed.size(), o1 = open.size();
  real cv[3][16], cd[3][16], ov[3][16], od[3][16];
  for (int k = 0; k < d_; k++) {
    for (int i = 0; i < c1; i++) closed.eval(i, xi[k], cv[k][i], cd[k][i]);
    for (int i = 0; i < o1; i++) open.eval(i, xi[k], ov[k][i], od[k][i]);
  }
  int dof = 0;
  for (int comp = 0; comp < d_; comp++) {
    int ext[3];
    for (int k = 0; k < d_; k++) ext[k] = (k == comp) ? c1 : o1;
    int cnt = 1;
    for (int k = 0; k < d_; k++) cnt *= ext[k];
    for (int idx = 0; idx < cnt; idx++) {
      int ii[3];
      int r = idx;
      for (int k = 0; k < d_; k++) { ii[k] = r % ext[k]; r /= ext[k]; }
      real f = 1.0, df = 1.0;
      for (int k = 0; k < d_; k++) {
        real vv = (k == comp) ? cv[k][ii[k]] : ov[k][ii[k]];
        f *= vv;
        if (k == comp) df *= cd[k][ii[k]]; else df *= vv;
      }
      for (int k = 0; k < d_; k++) if (val) val[dof * d_ + k] = (k == comp) ? f : 0.0;
      if (div) div[dof] = df;
      dof++;
    }
  }
}

// ----------------------------------------------------------------------------
// Cubature
// ----------------------------------------------------------------------------

struct Rule {
  int dim = 0;
  vector<real> pts;  // npts x dim
  vector<real> wts;
  int npts() const { return (int)wts.size(); }
};

static int gauss_points_for_degree(int degree) { return degree / 2 + 1; }

static Rule tensor_gauss(int dim, int degree) {
  int n = gauss_points_for_degree(degree);
  vector<real> x(n), w(n);
  gauss_legendre(n, x.data(), w.data());
  Rule r;
  r.dim = dim;
  int total = 1;
  for (int k = 0; k < dim; k++) total *= n;
  r.pts.resize(total * dim);
  r.wts.resize(total);
  for (int idx = 0; idx < total; idx++) {
    int rr = idx;
    real wt = 1.0;
    for (int k = 0; k < dim; k++) {
      int i = rr % n; rr /= n;
      r.pts[idx * dim + k] = x[i];
      wt *= w[i];
    }
    r.wts[idx] = wt;
  }
  return r;
}

// Triangle rule exact to `degree` (Intrepid uses a symmetric rule of the same
// degree; on affine triangles every integrand is a polynomial of at most that
// degree, so any exact rule gives the same integrals): collapsed Gauss-Legendre,
// xi = u (1 - v), eta = v, weight w_u w_v (1 - v) / 4 on [0,1]^2, u fastest.
static Rule tri_rule(int degree) {
  const int nu = degree / 2 + 1, nv = (degree + 1) / 2 + 1;
  vector<real> xu(nu), wu(nu), xv(nv), wv(nv);
  gauss_legendre(nu, xu.data(), wu.data());
  gauss_legendre(nv, xv.data(), wv.data());
  Rule r;
  r.dim = 2;
  for (int j = 0; j < nv; j++)
    for (int i = 0; i < nu; i++) {
      real u = 0.5 * (1 + xu[i]), v = 0.5 * (1 + xv[j]);
      r.pts.push_back(u * (1 - v));
      r.pts.push_back(v);
      r.wts.push_back(0.25 * wu[i] * wv[j] * (1 - v));
    }
  return r;
}

// ----------------------------------------------------------------------------
// Plan
// ----------------------------------------------------------------------------

struct VarLayout {
  int kind, space, k;
  Basis basis;         // volume basis (fields, tests) or side basis (traces)
  int offset;          // first dof
  int per_side;        // dofs per side for traces
  int ndofs;
};

// Reference tabulation of one basis at one point set.
struct RefTab {
  int card = 0, vdim = 1, d = 0;
  vector<real> val, grad, div;  // (npts, card, vdim), (npts, card, d), (npts, card)
};

static RefTab tabulate(const Basis& b, const real* pts, int npts) {
  RefTab t;
  t.card = b.card; t.d = b.d; t.vdim = b.rank ? b.d : 1;
  t.val.assign((size_t)npts * t.card * t.vdim, 0.0);
  if (b.rank) t.div.assign((size_t)npts * t.card, 0.0);
  else t.grad.assign((size_t)npts * t.card * t.d, 0.0);
  for (int q = 0; q < npts; q++)
    b.eval(pts + q * b.d, &t.val[(size_t)q * t.card * t.vdim],
           b.rank ? nullptr : &t.grad[(size_t)q * t.card * t.d],
           b.rank ? &t.div[(size_t)q * t.card] : nullptr);
  return t;
}

struct Plan {
  dpg_bucket_desc desc;
  vector<dpg_var_desc> trial, test;
  vector<dpg_bf_term> bf;
  vector<dpg_ip_entry> ip;
  vector<dpg_rhs_term> rhs;
  Topo topo;
  int d = 0, N = 0, M = 0, nf = 0, nt = 0;
  vector<VarLayout> tv, rv;  // test vars, trial vars
  Rule rG, rB, rS;           // rS in side parameter coordinates
  vector<vector<real>> side_pts;  // per side: Q_side x d volume reference points
  int nIPterms = 0;
  vector<int> ip_ncomp;
  vector<int> is_field;  // per trial dof
  // reference tables: [var][set] with set 0 = G points, 1 = B points, 2+s = side s
  vector<vector<RefTab>> test_tab, field_tab;
  vector<RefTab> trace_tab;  // per trial var (side-parameter points)
  std::string err;
};

static thread_local std::string g_err;

static bool build_plan(Plan& P, const dpg_bucket_desc* desc) {
  P.desc = *desc;
  P.trial.assign(desc->trial, desc->trial + desc->n_trial);
  P.test.assign(desc->test, desc->test + desc->n_test);
  P.bf.assign(desc->bf, desc->bf + desc->n_bf);
  P.ip.assign(desc->ip, desc->ip + desc->n_ip);
  if (desc->n_rhs) P.rhs.assign(desc->rhs, desc->rhs + desc->n_rhs);
  P.topo = make_topo(desc->topology);
  if (P.topo.d == 0) { g_err = "unknown topology"; return false; }
  P.d = P.topo.d;
  int side_topo = (P.d == 2) ? 0 : DPG_TOPO_QUAD;
  // test vars
  int off = 0;
  for (auto& v : P.test) {
    VarLayout L;
    L.kind = v.kind; L.space = v.space; L.k = v.poly_order;
    if (v.space == DPG_SPACE_HGRAD) L.basis = make_basis(P.topo.key, DPG_SPACE_HGRAD, v.poly_order);
    else if (v.space == DPG_SPACE_HDIV) L.basis = make_basis(P.topo.key, DPG_SPACE_HDIV, v.poly_order);
    else { g_err = "test var space must be HGRAD or HDIV"; return false; }
    L.offset = off; L.ndofs = L.basis.card; L.per_side = 0;
    off += L.ndofs;
    P.tv.push_back(L);
  }
  P.N = off;
  off = 0;
  for (auto& v : P.trial) {
    VarLayout L;
    L.kind = v.kind; L.space = v.space; L.k = v.poly_order;
    if (v.kind == DPG_VAR_FIELD) {
      if (v.space == DPG_SPACE_HVOL) L.basis = make_basis(P.topo.key, DPG_SPACE_HGRAD, v.poly_order - 1);
      else if (v.space == DPG_SPACE_VECTOR_HVOL) L.basis = make_basis(P.topo.key, DPG_SPACE_HGRAD, v.poly_order - 1, P.d);
      else { g_err = "field var space must be HVOL or VECTOR_HVOL"; return false; }
      L.ndofs = L.basis.card; L.per_side = 0;
    } else {
      int order = (v.space == DPG_SPACE_HGRAD) ? v.poly_order : v.poly_order - 1;
      L.basis = make_basis(side_topo, DPG_SPACE_HGRAD, order);
      if (P.d == 2) { L.basis.d = 1; L.basis.card = L.basis.closed.size(); }
      L.per_side = L.basis.card;
      L.ndofs = L.per_side * P.topo.nsides;
    }
    L.offset = off;
    off += L.ndofs;
    for (int i = 0; i < L.ndofs; i++) P.is_field.push_back(v.kind == DPG_VAR_FIELD ? 1 : 0);
    P.rv.push_back(L);
  }
  P.M = off;
  P.nf = 0;
  for (int x : P.is_field) P.nf += x;
  P.nt = P.M - P.nf;
  const bool tri = desc->topology == DPG_TOPO_TRI;
  P.rG = tri ? tri_rule(desc->cub_degree_G) : tensor_gauss(P.d, desc->cub_degree_G);
  P.rB = tri ? tri_rule(desc->cub_degree_B) : tensor_gauss(P.d, desc->cub_degree_B);
  P.rS = tensor_gauss(P.d - 1, desc->cub_degree_side);
  // map side points to the volume reference cell
  P.side_pts.resize(P.topo.nsides);
  for (int s = 0; s < P.topo.nsides; s++) {
    auto& sp = P.side_pts[s];
    sp.assign(P.rS.npts() * P.d, 0.0);
    for (int q = 0; q < P.rS.npts(); q++) {
      const real* t = &P.rS.pts[q * (P.d - 1)];
      if (P.d == 2) {
        const real* a = P.topo.v[P.topo.sv[s][0]];
        const real* b = P.topo.v[P.topo.sv[s][1]];
        for (int k = 0; k < 2; k++) sp[q * 2 + k] = 0.5 * (1 - t[0]) * a[k] + 0.5 * (1 + t[0]) * b[k];
      } else {
        real Nq[4] = {0.25 * (1 - t[0]) * (1 - t[1]), 0.25 * (1 + t[0]) * (1 - t[1]),
                        0.25 * (1 + t[0]) * (1 + t[1]), 0.25 * (1 - t[0]) * (1 + t[1])};
        for (int k = 0; k < 3; k++) {
          real x = 0;
          for (int a = 0; a < 4; a++) x += Nq[a] * P.topo.v[P.topo.sv[s][a]][k];
          sp[q * 3 + k] = x;
        }
      }
    }
  }
  P.nIPterms = 0;
  for (auto& e : P.ip) P.nIPterms = std::max(P.nIPterms, e.term + 1);
  P.ip_ncomp.assign(P.nIPterms, 0);
  for (auto& e : P.ip) P.ip_ncomp[e.term] = std::max(P.ip_ncomp[e.term], e.comp + 1);
  // reference tables
  auto sets = [&](const Basis& b) {
    vector<RefTab> v;
    v.push_back(tabulate(b, P.rG.pts.data(), P.rG.npts()));
    v.push_back(tabulate(b, P.rB.pts.data(), P.rB.npts()));
    for (int s = 0; s < P.topo.nsides; s++) v.push_back(tabulate(b, P.side_pts[s].data(), P.rS.npts()));
    return v;
  };
  for (auto& L : P.tv) P.test_tab.push_back(sets(L.basis));
  for (auto& L : P.rv) {
    if (L.kind == DPG_VAR_FIELD) { P.field_tab.push_back(sets(L.basis)); P.trace_tab.push_back(RefTab()); }
    else { P.field_tab.push_back({}); P.trace_tab.push_back(tabulate(L.basis, P.rS.pts.data(), P.rS.npts())); }
  }
  // validate ops
  for (auto& t : P.bf) {
    if (t.trial_var < 0 || t.trial_var >= (int)P.rv.size() || t.test_var < 0 || t.test_var >= (int)P.tv.size()) {
      g_err = "bf term var index out of range"; return false;
    }
    if (P.rv[t.trial_var].kind != DPG_VAR_FIELD && !t.boundary) { g_err = "trace/flux term must be a boundary term"; return false; }
  }
  return true;
}

// Geometry at a reference point.
struct Geo {
  real J[3][3], Ji[3][3], det;
};

static void geometry(const Plan& P, const real* nodes, const real* xi, Geo& g) {
  int d = P.d, nv = P.topo.nv;
  real Nv[8], dN[24];
  geom_shape(P.topo, xi, Nv, dN);
  for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) g.J[i][j] = (i == j && i >= d) ? 1.0 : 0.0;
  for (int i = 0; i < d; i++)
    for (int j = 0; j < d; j++) {
      real s = 0;
      for (int a = 0; a < nv; a++) s += nodes[a * d + i] * dN[a * d + j];
      g.J[i][j] = s;
    }
  if (d == 2) {
    g.det = g.J[0][0] * g.J[1][1] - g.J[0][1] * g.J[1][0];
    g.Ji[0][0] = g.J[1][1] / g.det; g.Ji[0][1] = -g.J[0][1] / g.det;
    g.Ji[1][0] = -g.J[1][0] / g.det; g.Ji[1][1] = g.J[0][0] / g.det;
  } else {
    real (*A)[3] = g.J;
    real c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    real c01 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
    real c02 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
    g.det = A[0][0] * c00 + A[0][1] * c01 + A[0][2] * c02;
    real id = 1.0 / g.det;
    g.Ji[0][0] = c00 * id;
    g.Ji[1][0] = c01 * id;
    g.Ji[2][0] = c02 * id;
    g.Ji[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * id;
    g.Ji[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id;
    g.Ji[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * id;
    g.Ji[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id;
    g.Ji[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * id;
    g.Ji[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id;
  }
}

// Side measure factor and outward unit normal at side point q of side s.
static void side_geometry(const Plan& P, const Geo& g, int s, int q, real& meas, real* n) {
  int d = P.d;
  if (d == 2) {
    const real* a = P.topo.v[P.topo.sv[s][0]];
    const real* b = P.topo.v[P.topo.sv[s][1]];
    real tr[2] = {0.5 * (b[0] - a[0]), 0.5 * (b[1] - a[1])};
    real T[2] = {g.J[0][0] * tr[0] + g.J[0][1] * tr[1], g.J[1][0] * tr[0] + g.J[1][1] * tr[1]};
    meas = r_sqrt(T[0] * T[0] + T[1] * T[1]);
    n[0] = T[1] / meas; n[1] = -T[0] / meas; n[2] = 0;
  } else {
    const real* t = &P.rS.pts[q * 2];
    real dNs[4] = {-0.25 * (1 - t[1]), 0.25 * (1 - t[1]), 0.25 * (1 + t[1]), -0.25 * (1 + t[1])};
    real dNt[4] = {-0.25 * (1 - t[0]), -0.25 * (1 + t[0]), 0.25 * (1 + t[0]), 0.25 * (1 - t[0])};
    real rs[3] = {0, 0, 0}, rt[3] = {0, 0, 0};
    for (int a = 0; a < 4; a++)
      for (int k = 0; k < 3; k++) {
        rs[k] += dNs[a] * P.topo.v[P.topo.sv[s][a]][k];
        rt[k] += dNt[a] * P.topo.v[P.topo.sv[s][a]][k];
      }
    real Ts[3], Tt[3];
    for (int i = 0; i < 3; i++) {
      Ts[i] = g.J[i][0] * rs[0] + g.J[i][1] * rs[1] + g.J[i][2] * rs[2];
      Tt[i] = g.J[i][0] * rt[0] + g.J[i][1] * rt[1] + g.J[i][2] * rt[2];
    }
    real c[3] = {Ts[1] * Tt[2] - Ts[2] * Tt[1], Ts[2] * Tt[0] - Ts[0] * Tt[2], Ts[0] * Tt[1] - Ts[1] * Tt[0]};
    meas = r_sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    for (int k = 0; k < 3; k++) n[k] = c[k] / meas;
  }
}

// Physical value of test op for all dofs of a test var at point q of a table.
// out[i] for i in [0, card)
static void test_op_values(const Plan& P, const RefTab& T, int q, int op, const Geo& g, const real* nrm,
                           real* out) {
  int d = P.d, card = T.card;
  bool vec = T.vdim > 1;
  const real* val = &T.val[(size_t)q * card * T.vdim];
  for (int i = 0; i < card; i++) {
    real r = 0;
    if (!vec) {
      if (op == DPG_OP_VALUE) r = val[i];
      else if (op >= DPG_OP_DX && op <= DPG_OP_DZ) {
        const real* grad = &T.grad[((size_t)q * card + i) * d];
        int c = op - DPG_OP_DX;
        for (int j = 0; j < d; j++) r += g.Ji[j][c] * grad[j];  // (J^-T grad)_c
      }
    } else {
      real pv[3] = {0, 0, 0};
      for (int c = 0; c < d; c++) {
        real s = 0;
        for (int j = 0; j < d; j++) s += g.J[c][j] * val[i * d + j];
        pv[c] = s / g.det;
      }
      if (op >= DPG_OP_X && op <= DPG_OP_Z) r = pv[op - DPG_OP_X];
      else if (op == DPG_OP_DIV) r = T.div[(size_t)q * card + i] / g.det;
      else if (op == DPG_OP_DOT_NORMAL) { for (int c = 0; c < d; c++) r += pv[c] * nrm[c]; }
    }
    out[i] = r;
  }
}

// Trial values of field var L (op VALUE or component) at point q of a table.
static void field_values(const VarLayout& L, const RefTab& T, int q, int op, real* out) {
  const Basis& b = L.basis;
  const real* val = &T.val[(size_t)q * T.card];
  int per = b.card / b.ncomp;
  int comp = (b.ncomp > 1) ? (op - DPG_OP_X) : 0;
  for (int i = 0; i < b.card; i++) out[i] = (i / per == comp) ? val[i] : 0.0;
}

static inline real slotval(const real* coeff_cell, int P_total, int slot, int p) {
  return slot < 0 ? 1.0 : coeff_cell[slot * P_total + p];
}

struct CellOut {
  vector<real> G, B, F;  // G NxN, B MxN (row = trial), F N
};

static void assemble_cell(const Plan& P, const real* nodes, const int8_t* parity, const real* coeff,
                          CellOut& o) {
  int N = P.N, M = P.M, d = P.d;
  int QG = P.rG.npts(), QB = P.rB.npts(), QS = P.rS.npts();
  int Ptot = QG + QB + P.topo.nsides * QS;
  o.G.assign((size_t)N * N, 0.0);
  o.B.assign((size_t)M * N, 0.0);
  o.F.assign(N, 0.0);
  real nrm0[3] = {0, 0, 0};
  // ---- G, in the reference's order (IP.cpp:238-244 -> LinearTerm.cpp:470-606):
  // for each graph-norm term, for each (u var, v var) pair of that term, the
  // weighted u values are contracted with the v values over (point, component) in
  // one product (FunctionSpaceTools::integrate, COMP_BLAS) and the block is then
  // added into G.  The order matters at h = 1/48: summing every term's products in
  // one running sum per entry is 3-4x further from the exact G's factorisation.
  {
    int nT = 0;
    vector<int> row0(P.nIPterms + 1, 0);
    for (int t = 0; t < P.nIPterms; t++) { row0[t] = nT; nT += P.ip_ncomp[t]; }
    row0[P.nIPterms] = nT;
    // L[q][row][N]: term-component rows of every point; wm[q] = w |J|
    vector<real> Lm((size_t)QG * nT * N, 0.0), wm(QG);
    vector<real> tmp(N);
    for (int q = 0; q < QG; q++) {
      const real* xi = &P.rG.pts[q * d];
      Geo g;
      geometry(P, nodes, xi, g);
      wm[q] = P.rG.wts[q] * g.det;
      real* Lq = &Lm[(size_t)q * nT * N];
      for (auto& e : P.ip) {
        const int row = row0[e.term] + e.comp;
        const VarLayout& L = P.tv[e.test_var];
        test_op_values(P, P.test_tab[e.test_var][0], q, e.test_op, g, nrm0, tmp.data());
        real cf = e.coef * slotval(coeff, Ptot, e.slot, q);
        for (int i = 0; i < L.ndofs; i++) Lq[(size_t)row * N + L.offset + i] += cf * tmp[i];
      }
    }
    vector<real> wu;
    for (int t = 0; t < P.nIPterms; t++) {
      vector<int> vars;
      for (auto& e : P.ip)
        if (e.term == t && std::find(vars.begin(), vars.end(), e.test_var) == vars.end()) vars.push_back(e.test_var);
      std::sort(vars.begin(), vars.end());
      const int nc = P.ip_ncomp[t];
      for (int u : vars) {
        const VarLayout& U = P.tv[u];
        // weighted u values (C, F, P, D) for this term: wu[i][q][c]
        wu.assign((size_t)U.ndofs * QG * nc, 0.0);
        for (int i = 0; i < U.ndofs; i++)
          for (int q = 0; q < QG; q++)
            for (int c = 0; c < nc; c++)
              wu[((size_t)i * QG + q) * nc + c] = wm[q] * Lm[((size_t)q * nT + row0[t] + c) * N + U.offset + i];
        for (int v : vars) {
          const VarLayout& V = P.tv[v];
          for (int i = 0; i < U.ndofs; i++)
            for (int j = 0; j < V.ndofs; j++) {
              real acc = 0.0;
              const real* a = &wu[(size_t)i * QG * nc];
              for (int q = 0; q < QG; q++)
                for (int c = 0; c < nc; c++)
                  acc += a[q * nc + c] * Lm[((size_t)q * nT + row0[t] + c) * N + V.offset + j];
              o.G[(size_t)(U.offset + i) * N + V.offset + j] += acc;
            }
        }
      }
    }
  }
  // ---- B and F volume ------------------------------------------------------
  {
    vector<real> tv(N), rvv(M);
    for (int q = 0; q < QB; q++) {
      const real* xi = &P.rB.pts[q * d];
      Geo g;
      geometry(P, nodes, xi, g);
      real wm = P.rB.wts[q] * g.det;
      int p = QG + q;
      for (auto& t : P.bf) {
        if (t.boundary) continue;
        const VarLayout& TL = P.tv[t.test_var];
        const VarLayout& RL = P.rv[t.trial_var];
        test_op_values(P, P.test_tab[t.test_var][1], q, t.test_op, g, nrm0, tv.data());
        field_values(RL, P.field_tab[t.trial_var][1], q, t.trial_op, rvv.data());
        real cf = wm * t.coef * slotval(coeff, Ptot, t.slot, p);
        for (int m = 0; m < RL.ndofs; m++) {
          real a = cf * rvv[m];
          if (a == 0.0) continue;
          real* Bm = &o.B[(size_t)(RL.offset + m) * N + TL.offset];
          for (int i = 0; i < TL.ndofs; i++) Bm[i] += a * tv[i];
        }
      }
      for (auto& r : P.rhs) {
        const VarLayout& TL = P.tv[r.test_var];
        test_op_values(P, P.test_tab[r.test_var][1], q, r.test_op, g, nrm0, tv.data());
        real cf = wm * r.coef * slotval(coeff, Ptot, r.slot, p);
        for (int i = 0; i < TL.ndofs; i++) o.F[TL.offset + i] += cf * tv[i];
      }
    }
  }
  // ---- B sides ---------------------------------------------------------------
  {
    vector<real> tv(N), rvv(M);
    for (int s = 0; s < P.topo.nsides; s++) {
      for (int q = 0; q < QS; q++) {
        const real* xi = &P.side_pts[s][q * d];
        Geo g;
        geometry(P, nodes, xi, g);
        real meas, nrm[3];
        side_geometry(P, g, s, q, meas, nrm);
        real wm = P.rS.wts[q] * meas;
        int p = QG + QB + s * QS + q;
        for (auto& t : P.bf) {
          if (!t.boundary) continue;
          const VarLayout& TL = P.tv[t.test_var];
          const VarLayout& RL = P.rv[t.trial_var];
          test_op_values(P, P.test_tab[t.test_var][2 + s], q, t.test_op, g, nrm, tv.data());
          real cf = wm * t.coef * slotval(coeff, Ptot, t.slot, p);
          if (t.normal_comp >= 0) cf *= nrm[t.normal_comp];
          int m0, mcount;
          if (RL.kind == DPG_VAR_FIELD) {
            field_values(RL, P.field_tab[t.trial_var][2 + s], q, t.trial_op, rvv.data());
            m0 = RL.offset; mcount = RL.ndofs;
          } else {
            const RefTab& TT = P.trace_tab[t.trial_var];
            for (int m = 0; m < RL.per_side; m++) rvv[m] = TT.val[(size_t)q * TT.card + m];
            if (RL.kind == DPG_VAR_FLUX) cf *= (real)parity[s];
            m0 = RL.offset + s * RL.per_side; mcount = RL.per_side;
          }
          for (int m = 0; m < mcount; m++) {
            real a = cf * rvv[m];
            if (a == 0.0) continue;
            real* Bm = &o.B[(size_t)(m0 + m) * N + TL.offset];
            for (int i = 0; i < TL.ndofs; i++) Bm[i] += a * tv[i];
          }
        }
      }
    }
  }
}

// The same quadrature as assemble_cell, returned as operator rows instead of sums
// (used by the tests that emulate reduced-precision contractions term by term):
//   G = sum_q wm[q] sum_rows L[q][row]^T L[q][row]   (row = graph-norm term component,
//       rterm[row] its term),
//   B = sum_r U[r]^T V[r]   (U: M trial values times weight, coefficient, normal
//       component and parity; V: N test-operator values), F = sum_r fw[r] FV[r].
// dims = {term-component rows, B rows, F rows}.
static void cell_operators(const Plan& P, const real* nodes, const int8_t* parity, const real* coeff,
                           vector<real>& L, vector<real>& wm, vector<int>& rterm, vector<real>& U,
                           vector<real>& V, vector<real>& fw, vector<real>& FV) {
  int N = P.N, M = P.M, d = P.d;
  int QG = P.rG.npts(), QB = P.rB.npts(), QS = P.rS.npts();
  int Ptot = QG + QB + P.topo.nsides * QS;
  int nT = 0;
  vector<int> row0(P.nIPterms + 1, 0);
  rterm.clear();
  for (int t = 0; t < P.nIPterms; t++) {
    row0[t] = nT;
    nT += P.ip_ncomp[t];
    for (int c = 0; c < P.ip_ncomp[t]; c++) rterm.push_back(t);
  }
  L.assign((size_t)QG * nT * N, 0.0);
  wm.assign(QG, 0.0);
  real nrm0[3] = {0, 0, 0};
  vector<real> tmp(N), rvv(M);
  for (int q = 0; q < QG; q++) {
    Geo g;
    geometry(P, nodes, &P.rG.pts[q * d], g);
    wm[q] = P.rG.wts[q] * g.det;
    for (auto& e : P.ip) {
      const VarLayout& TL = P.tv[e.test_var];
      test_op_values(P, P.test_tab[e.test_var][0], q, e.test_op, g, nrm0, tmp.data());
      real cf = e.coef * slotval(coeff, Ptot, e.slot, q);
      for (int i = 0; i < TL.ndofs; i++) L[((size_t)q * nT + row0[e.term] + e.comp) * N + TL.offset + i] += cf * tmp[i];
    }
  }
  U.clear(); V.clear(); fw.clear(); FV.clear();
  auto push_row = [&](vector<real>& dst, int n) { dst.resize(dst.size() + n, 0.0); return dst.size() - n; };
  for (int q = 0; q < QB; q++) {
    Geo g;
    geometry(P, nodes, &P.rB.pts[q * d], g);
    real w = P.rB.wts[q] * g.det;
    int p = QG + q;
    for (auto& t : P.bf) {
      if (t.boundary) continue;
      const VarLayout& TL = P.tv[t.test_var];
      const VarLayout& RL = P.rv[t.trial_var];
      size_t u0 = push_row(U, M), v0 = push_row(V, N);
      test_op_values(P, P.test_tab[t.test_var][1], q, t.test_op, g, nrm0, tmp.data());
      field_values(RL, P.field_tab[t.trial_var][1], q, t.trial_op, rvv.data());
      real cf = w * t.coef * slotval(coeff, Ptot, t.slot, p);
      for (int m = 0; m < RL.ndofs; m++) U[u0 + RL.offset + m] = cf * rvv[m];
      for (int i = 0; i < TL.ndofs; i++) V[v0 + TL.offset + i] = tmp[i];
    }
    for (auto& r : P.rhs) {
      const VarLayout& TL = P.tv[r.test_var];
      size_t v0 = push_row(FV, N);
      test_op_values(P, P.test_tab[r.test_var][1], q, r.test_op, g, nrm0, tmp.data());
      fw.push_back(w * r.coef * slotval(coeff, Ptot, r.slot, p));
      for (int i = 0; i < TL.ndofs; i++) FV[v0 + TL.offset + i] = tmp[i];
    }
  }
  for (int s = 0; s < P.topo.nsides; s++)
    for (int q = 0; q < QS; q++) {
      Geo g;
      geometry(P, nodes, &P.side_pts[s][q * d], g);
      real meas, nrm[3];
      side_geometry(P, g, s, q, meas, nrm);
      real w = P.rS.wts[q] * meas;
      int p = QG + QB + s * QS + q;
      for (auto& t : P.bf) {
        if (!t.boundary) continue;
        const VarLayout& TL = P.tv[t.test_var];
        const VarLayout& RL = P.rv[t.trial_var];
        size_t u0 = push_row(U, M), v0 = push_row(V, N);
        test_op_values(P, P.test_tab[t.test_var][2 + s], q, t.test_op, g, nrm, tmp.data());
        real cf = w * t.coef * slotval(coeff, Ptot, t.slot, p);
        if (t.normal_comp >= 0) cf *= nrm[t.normal_comp];
        if (RL.kind == DPG_VAR_FIELD) {
          field_values(RL, P.field_tab[t.trial_var][2 + s], q, t.trial_op, rvv.data());
          for (int m = 0; m < RL.ndofs; m++) U[u0 + RL.offset + m] = cf * rvv[m];
        } else {
          const RefTab& TT = P.trace_tab[t.trial_var];
          if (RL.kind == DPG_VAR_FLUX) cf *= (real)parity[s];
          for (int m = 0; m < RL.per_side; m++) U[u0 + RL.offset + s * RL.per_side + m] = cf * TT.val[(size_t)q * TT.card + m];
        }
        for (int i = 0; i < TL.ndofs; i++) V[v0 + TL.offset + i] = tmp[i];
      }
    }
}

// Reverse mode (no counterpart in the reference; the hand gradient that the GPU's
// dpg_assemble_adjoint is checked against).  For J = <Kbar, K> + <lbar, l> on one cell,
// with X = G^-1 B^T and y = G^-1 F (B stored trial x test, K = B G^-1 B^T, l = B G^-1 F):
//   Bbar = (Kbar + Kbar^T) X^T + lbar y^T,   Fbar = X lbar,
//   Gbar + Gbar^T = -(X (Kbar + Kbar^T) X^T + X lbar y^T + y lbar^T X^T),
// then dJ/dslot(p) = <Bbar, dB/dslot(p)> + <Gbar, dG/dslot(p)> + Fbar . dF/dslot(p) through
// the same quadrature as assemble_cell (every form is linear in each coefficient slot
// value of a term, the Gram matrix quadratic through its rows L_r).
static void adjoint_cell(const Plan& P, const real* nodes, const int8_t* parity, const real* coeff,
                         const real* Kbar, const real* lbar, real* cbar) {
  const int N = P.N, M = P.M, d = P.d;
  const int QG = P.rG.npts(), QB = P.rB.npts(), QS = P.rS.npts();
  const int Ptot = QG + QB + P.topo.nsides * QS;
  CellOut o;
  assemble_cell(P, nodes, parity, coeff, o);
  // Cholesky of the equilibrated G (as BF.cpp:944-982), then X = G^-1 B^T and y = G^-1 F
  vector<real> s(N), Lf((size_t)N * N, 0.0);
  for (int i = 0; i < N; i++) s[i] = 1.0 / r_sqrt(o.G[(size_t)i * N + i]);
  for (int j = 0; j < N; j++) {
    real ajj = o.G[(size_t)j * N + j] * s[j] * s[j];
    for (int k = 0; k < j; k++) ajj -= Lf[(size_t)j * N + k] * Lf[(size_t)j * N + k];
    ajj = r_sqrt(ajj);
    Lf[(size_t)j * N + j] = ajj;
    for (int i = j + 1; i < N; i++) {
      real v = o.G[(size_t)i * N + j] * s[i] * s[j];
      for (int k = 0; k < j; k++) v -= Lf[(size_t)i * N + k] * Lf[(size_t)j * N + k];
      Lf[(size_t)i * N + j] = v / ajj;
    }
  }
  auto solve = [&](real* b) {  // b <- G^-1 b = S (Ls Ls^T)^-1 S b
    for (int i = 0; i < N; i++) b[i] *= s[i];
    for (int i = 0; i < N; i++) {
      real v = b[i];
      for (int k = 0; k < i; k++) v -= Lf[(size_t)i * N + k] * b[k];
      b[i] = v / Lf[(size_t)i * N + i];
    }
    for (int i = N - 1; i >= 0; i--) {
      real v = b[i];
      for (int k = i + 1; k < N; k++) v -= Lf[(size_t)k * N + i] * b[k];
      b[i] = v / Lf[(size_t)i * N + i];
    }
    for (int i = 0; i < N; i++) b[i] *= s[i];
  };
  vector<real> X((size_t)M * N), y(o.F);  // X stored as rows m: (G^-1 B^T)[:, m]
  for (int m = 0; m < M; m++) {
    std::copy(&o.B[(size_t)m * N], &o.B[(size_t)m * N] + N, &X[(size_t)m * N]);
    solve(&X[(size_t)m * N]);
  }
  solve(y.data());
  vector<real> Ks((size_t)M * M);
  for (int a = 0; a < M; a++)
    for (int b = 0; b < M; b++) Ks[(size_t)a * M + b] = Kbar[(size_t)a * M + b] + Kbar[(size_t)b * M + a];
  // Bbar (M x N), Fbar (N), Gs = Gbar + Gbar^T (N x N)
  vector<real> Bb((size_t)M * N, 0.0), Fb(N, 0.0), Gs((size_t)N * N, 0.0), XK((size_t)M * N, 0.0), Xl(N, 0.0);
  for (int a = 0; a < M; a++)
    for (int b = 0; b < M; b++) {
      const real k = Ks[(size_t)a * M + b];
      if (k == 0.0) continue;
      for (int i = 0; i < N; i++) XK[(size_t)a * N + i] += k * X[(size_t)b * N + i];  // rows of Ks X^T
    }
  for (int m = 0; m < M; m++)
    for (int i = 0; i < N; i++) Xl[i] += X[(size_t)m * N + i] * lbar[m];
  for (int m = 0; m < M; m++)
    for (int i = 0; i < N; i++) Bb[(size_t)m * N + i] = XK[(size_t)m * N + i] + lbar[m] * y[i];
  for (int i = 0; i < N; i++) Fb[i] = Xl[i];
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) {
      real v = 0.0;
      for (int m = 0; m < M; m++) v += X[(size_t)m * N + i] * XK[(size_t)m * N + j];
      Gs[(size_t)i * N + j] = -(v + Xl[i] * y[j] + y[i] * Xl[j]);
    }
  std::fill(cbar, cbar + (size_t)P.desc.n_slots * Ptot, 0.0);
  real nrm0[3] = {0, 0, 0};
  vector<real> tmp(N), rvv(M);
  // Gram points: dJ/dslot = wm sum_r dL_r^T Gs L_r
  {
    int nT = 0;
    vector<int> row0(P.nIPterms + 1, 0);
    for (int t = 0; t < P.nIPterms; t++) { row0[t] = nT; nT += P.ip_ncomp[t]; }
    vector<real> Lq((size_t)nT * N), Y((size_t)nT * N);
    for (int q = 0; q < QG; q++) {
      Geo g;
      geometry(P, nodes, &P.rG.pts[q * d], g);
      const real wm = P.rG.wts[q] * g.det;
      std::fill(Lq.begin(), Lq.end(), 0.0);
      for (auto& e : P.ip) {
        const VarLayout& TL = P.tv[e.test_var];
        test_op_values(P, P.test_tab[e.test_var][0], q, e.test_op, g, nrm0, tmp.data());
        real cf = e.coef * slotval(coeff, Ptot, e.slot, q);
        for (int i = 0; i < TL.ndofs; i++) Lq[(size_t)(row0[e.term] + e.comp) * N + TL.offset + i] += cf * tmp[i];
      }
      for (int r = 0; r < nT; r++)
        for (int i = 0; i < N; i++) {
          real v = 0.0;
          for (int j = 0; j < N; j++) v += Gs[(size_t)i * N + j] * Lq[(size_t)r * N + j];
          Y[(size_t)r * N + i] = v;
        }
      for (auto& e : P.ip) {
        if (e.slot < 0) continue;
        const VarLayout& TL = P.tv[e.test_var];
        test_op_values(P, P.test_tab[e.test_var][0], q, e.test_op, g, nrm0, tmp.data());
        real v = 0.0;
        for (int i = 0; i < TL.ndofs; i++) v += tmp[i] * Y[(size_t)(row0[e.term] + e.comp) * N + TL.offset + i];
        cbar[(size_t)e.slot * Ptot + q] += wm * e.coef * v;
      }
    }
  }
  // B and F volume points
  for (int q = 0; q < QB; q++) {
    Geo g;
    geometry(P, nodes, &P.rB.pts[q * d], g);
    const real wm = P.rB.wts[q] * g.det;
    const int p = QG + q;
    for (auto& t : P.bf) {
      if (t.boundary || t.slot < 0) continue;
      const VarLayout& TL = P.tv[t.test_var];
      const VarLayout& RL = P.rv[t.trial_var];
      test_op_values(P, P.test_tab[t.test_var][1], q, t.test_op, g, nrm0, tmp.data());
      field_values(RL, P.field_tab[t.trial_var][1], q, t.trial_op, rvv.data());
      real v = 0.0;
      for (int m = 0; m < RL.ndofs; m++) {
        if (rvv[m] == 0.0) continue;
        real w = 0.0;
        for (int i = 0; i < TL.ndofs; i++) w += Bb[(size_t)(RL.offset + m) * N + TL.offset + i] * tmp[i];
        v += rvv[m] * w;
      }
      cbar[(size_t)t.slot * Ptot + p] += wm * t.coef * v;
    }
    for (auto& r : P.rhs) {
      if (r.slot < 0) continue;
      const VarLayout& TL = P.tv[r.test_var];
      test_op_values(P, P.test_tab[r.test_var][1], q, r.test_op, g, nrm0, tmp.data());
      real v = 0.0;
      for (int i = 0; i < TL.ndofs; i++) v += Fb[TL.offset + i] * tmp[i];
      cbar[(size_t)r.slot * Ptot + p] += wm * r.coef * v;
    }
  }
  // B side points
  for (int sd = 0; sd < P.topo.nsides; sd++)
    for (int q = 0; q < QS; q++) {
      Geo g;
      geometry(P, nodes, &P.side_pts[sd][q * d], g);
      real meas, nrm[3];
      side_geometry(P, g, sd, q, meas, nrm);
      const real wm = P.rS.wts[q] * meas;
      const int p = QG + QB + sd * QS + q;
      for (auto& t : P.bf) {
        if (!t.boundary || t.slot < 0) continue;
        const VarLayout& TL = P.tv[t.test_var];
        const VarLayout& RL = P.rv[t.trial_var];
        test_op_values(P, P.test_tab[t.test_var][2 + sd], q, t.test_op, g, nrm, tmp.data());
        real cf = wm * t.coef;
        if (t.normal_comp >= 0) cf *= nrm[t.normal_comp];
        int m0, mcount;
        if (RL.kind == DPG_VAR_FIELD) {
          field_values(RL, P.field_tab[t.trial_var][2 + sd], q, t.trial_op, rvv.data());
          m0 = RL.offset; mcount = RL.ndofs;
        } else {
          const RefTab& TT = P.trace_tab[t.trial_var];
          for (int m = 0; m < RL.per_side; m++) rvv[m] = TT.val[(size_t)q * TT.card + m];
          if (RL.kind == DPG_VAR_FLUX) cf *= (real)parity[sd];
          m0 = RL.offset + sd * RL.per_side; mcount = RL.per_side;
        }
        real v = 0.0;
        for (int m = 0; m < mcount; m++) {
          if (rvv[m] == 0.0) continue;
          real w = 0.0;
          for (int i = 0; i < TL.ndofs; i++) w += Bb[(size_t)(m0 + m) * N + TL.offset + i] * tmp[i];
          v += rvv[m] * w;
        }
        cbar[(size_t)t.slot * Ptot + p] += cf * v;
      }
    }
}

// ----------------------------------------------------------------------------
// Dense kernels, LAPACK semantics (column-major views)
// ----------------------------------------------------------------------------

// BF.cpp:924-1018.  G (N x N, symmetric; overwritten), B column-major N x M
// (overwritten with L^-1 B), F (N; overwritten).  K row-major M x M, l (M).
int factored_cholesky_solve(int N, int M, real* G, real* B, real* F, real* K, real* l) {
  int result = 0;
  // DPOEQU
  vector<real> s(N);
  int info = 0;
  {
    real smin = G[0], amax = G[0];
    for (int i = 0; i < N; i++) {
      s[i] = G[i * N + i];
      smin = std::min(smin, s[i]);
      amax = std::max(amax, s[i]);
    }
    if (smin <= 0) {
      for (int i = 0; i < N; i++) if (s[i] <= 0) { info = i + 1; break; }
    } else {
      for (int i = 0; i < N; i++) s[i] = 1.0 / r_sqrt(s[i]);
    }
  }
  (void)info;
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) G[i * N + j] *= s[i] * s[j];
  // DPOTRF('L'), column-major A(i,j) = G[j*N+i]
  auto A = [&](int i, int j) -> real& { return G[(size_t)j * N + i]; };
  for (int j = 0; j < N; j++) {
    real ajj = A(j, j);
    for (int k = 0; k < j; k++) ajj -= A(j, k) * A(j, k);
    if (ajj <= 0.0 || r_isnan(ajj)) { result = j + 1; break; }
    ajj = r_sqrt(ajj);
    A(j, j) = ajj;
    for (int i = j + 1; i < N; i++) {
      real v = A(i, j);
      for (int k = 0; k < j; k++) v -= A(i, k) * A(j, k);
      A(i, j) = v / ajj;
    }
  }
  if (result != 0) return result;
  // unequilibrate L(i,j) /= s_i
  for (int j = 0; j < N; j++)
    for (int i = j; i < N; i++) A(i, j) /= s[i];
  // DTRSM L X = B  (B column-major N x M, ld N)
  for (int c = 0; c < M; c++) {
    real* b = &B[(size_t)c * N];
    for (int j = 0; j < N; j++) {
      if (b[j] != 0.0) {
        b[j] /= A(j, j);
        real bj = b[j];
        for (int i = j + 1; i < N; i++) b[i] -= bj * A(i, j);
      }
    }
  }
  // DSYRK lower: K = W^T W, then mirror
  for (int i = 0; i < M; i++)
    for (int j = 0; j <= i; j++) {
      real acc = 0;
      const real* wi = &B[(size_t)i * N];
      const real* wj = &B[(size_t)j * N];
      for (int k = 0; k < N; k++) acc += wi[k] * wj[k];
      K[(size_t)i * M + j] = acc;
      K[(size_t)j * M + i] = acc;
    }
  // DTRSM on F
  for (int j = 0; j < N; j++) {
    if (F[j] != 0.0) {
      F[j] /= A(j, j);
      real fj = F[j];
      for (int i = j + 1; i < N; i++) F[i] -= fj * A(i, j);
    }
  }
  // l = W^T y
  for (int m = 0; m < M; m++) {
    real acc = 0;
    const real* w = &B[(size_t)m * N];
    for (int k = 0; k < N; k++) acc += w[k] * F[k];
    l[m] = acc;
  }
  return result;
}

// Epetra_SerialDenseSolver-style solve of D X = R (n x n, nrhs columns),
// optional DGEEQU equilibration (threshold 0.1), LU with partial pivoting.
// D row-major n x n (copied), R row-major n x nrhs (overwritten by X).
static int lu_solve_equilibrated(int n, const real* Din, real* R, int nrhs) {
  vector<real> A(Din, Din + (size_t)n * n);
  vector<real> r(n, 0.0), c(n, 0.0);
  const real smlnum = 2.2250738585072014e-308 / 2.220446049250313e-16;
  const real bignum = 1.0 / smlnum;
  real rcmin = bignum, rcmax = 0.0;
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < n; j++) r[i] = std::max(r[i], r_fabs(A[(size_t)i * n + j]));
    rcmin = std::min(rcmin, r[i]);
    rcmax = std::max(rcmax, r[i]);
  }
  bool equil = false;
  real rowcnd = 0, colcnd = 0;
  if (rcmin > 0.0) {
    for (int i = 0; i < n; i++) r[i] = 1.0 / std::min(std::max(r[i], smlnum), bignum);
    rowcnd = std::max(rcmin, smlnum) / std::min(rcmax, bignum);
    real ccmin = bignum, ccmax = 0.0;
    for (int j = 0; j < n; j++) {
      for (int i = 0; i < n; i++) c[j] = std::max(c[j], r_fabs(A[(size_t)i * n + j]) * r[i]);
      ccmin = std::min(ccmin, c[j]);
      ccmax = std::max(ccmax, c[j]);
    }
    if (ccmin > 0.0) {
      for (int j = 0; j < n; j++) c[j] = 1.0 / std::min(std::max(c[j], smlnum), bignum);
      colcnd = std::max(ccmin, smlnum) / std::min(ccmax, bignum);
      equil = (rowcnd <= 0.1) || (colcnd <= 0.1);
    }
  }
  if (equil) {
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) A[(size_t)i * n + j] *= r[i] * c[j];
    for (int i = 0; i < n; i++)
      for (int k = 0; k < nrhs; k++) R[(size_t)i * nrhs + k] *= r[i];
  }
  // LU with partial pivoting
  vector<int> piv(n);
  for (int k = 0; k < n; k++) {
    int p = k;
    real best = r_fabs(A[(size_t)k * n + k]);
    for (int i = k + 1; i < n; i++)
      if (r_fabs(A[(size_t)i * n + k]) > best) { best = r_fabs(A[(size_t)i * n + k]); p = i; }
    piv[k] = p;
    if (best == 0.0) return k + 1;
    if (p != k) {
      for (int j = 0; j < n; j++) std::swap(A[(size_t)k * n + j], A[(size_t)p * n + j]);
      for (int j = 0; j < nrhs; j++) std::swap(R[(size_t)k * nrhs + j], R[(size_t)p * nrhs + j]);
    }
    real inv = 1.0 / A[(size_t)k * n + k];
    for (int i = k + 1; i < n; i++) {
      real f = A[(size_t)i * n + k] * inv;
      A[(size_t)i * n + k] = f;
      if (f == 0.0) continue;
      for (int j = k + 1; j < n; j++) A[(size_t)i * n + j] -= f * A[(size_t)k * n + j];
      for (int j = 0; j < nrhs; j++) R[(size_t)i * nrhs + j] -= f * R[(size_t)k * nrhs + j];
    }
  }
  for (int k = n - 1; k >= 0; k--) {
    for (int j = 0; j < nrhs; j++) {
      real v = R[(size_t)k * nrhs + j];
      for (int i = k + 1; i < n; i++) v -= A[(size_t)k * n + i] * R[(size_t)i * nrhs + j];
      R[(size_t)k * nrhs + j] = v / A[(size_t)k * n + k];
    }
  }
  if (equil) {
    for (int i = 0; i < n; i++)
      for (int k = 0; k < nrhs; k++) R[(size_t)i * nrhs + k] *= c[i];
  }
  return 0;
}

// CondensedDofInterpreter.cpp:1138-1192 on the local K (fields = is_field).
int condense(int M, const int* is_field, const real* K, const real* l, real* S, real* s) {
  vector<int> fi, ti;
  for (int i = 0; i < M; i++) (is_field[i] ? fi : ti).push_back(i);
  int nf = (int)fi.size(), nt = (int)ti.size();
  vector<real> D((size_t)nf * nf), Bc((size_t)nf * nt), X, y(nf);
  for (int a = 0; a < nf; a++) {
    for (int b = 0; b < nf; b++) D[(size_t)a * nf + b] = K[(size_t)fi[a] * M + fi[b]];
    for (int b = 0; b < nt; b++) Bc[(size_t)a * nt + b] = K[(size_t)fi[a] * M + ti[b]];
    y[a] = l[fi[a]];
  }
  X = Bc;
  int err = 0;
  if (nf > 0) {
    err = lu_solve_equilibrated(nf, D.data(), X.data(), nt);
    int err2 = lu_solve_equilibrated(nf, D.data(), y.data(), 1);
    if (!err) err = err2;
  }
  for (int a = 0; a < nt; a++) {
    for (int b = 0; b < nt; b++) {
      real v = K[(size_t)ti[a] * M + ti[b]];
      for (int k = 0; k < nf; k++) v -= Bc[(size_t)k * nt + a] * X[(size_t)k * nt + b];
      S[(size_t)a * nt + b] = v;
    }
    real v = l[ti[a]];
    for (int k = 0; k < nf; k++) v -= Bc[(size_t)k * nt + a] * y[k];
    s[a] = v;
  }
  return err ? -err : 0;
}

#ifndef ORC_QUAD
// ----------------------------------------------------------------------------
// Fast mode: the CPU baseline.  The same algorithm with Camellia's cost structure:
// every quadrature contraction is one DGEMM per block, as Intrepid's
// FunctionSpaceTools::integrate(COMP_BLAS) does per (trial var, test var) pair
// (LinearTerm.cpp:574-576) -- G per graph-norm term and var pair, B per bilinear term
// (and side), F by DGEMV -- then DPOTRF, DTRSM, DSYRK and DGEMV as in
// BF.cpp:944-1016.  The BLAS/LAPACK routines are the caller's (the tests and the bench
// hand over scipy's OpenBLAS through scipy.linalg.cython_blas / cython_lapack, one
// thread per call).
// ----------------------------------------------------------------------------
typedef void (*DgemmFn)(const char*, const char*, const int*, const int*, const int*, const double*, const double*,
                        const int*, const double*, const int*, const double*, double*, const int*);
typedef void (*DgemvFn)(const char*, const int*, const int*, const double*, const double*, const int*, const double*,
                        const int*, const double*, double*, const int*);
typedef void (*DsyrkFn)(const char*, const char*, const int*, const int*, const double*, const double*, const int*,
                        const double*, double*, const int*);
typedef void (*DtrsmFn)(const char*, const char*, const char*, const char*, const int*, const int*, const double*,
                        const double*, const int*, double*, const int*);
typedef void (*DpotrfFn)(const char*, const int*, double*, const int*, int*);
struct BlasFns {
  DgemmFn dgemm = nullptr;
  DgemvFn dgemv = nullptr;
  DsyrkFn dsyrk = nullptr;
  DtrsmFn dtrsm = nullptr;
  DpotrfFn dpotrf = nullptr;
};
static BlasFns g_blas;

// One cell: K (M x M row-major), l (M), S, s (nullable), returns INFO.
static int assemble_cell_blas(const Plan& P, const double* nodes, const int8_t* parity, const double* coeff,
                              double* K, double* l, double* S, double* s) {
  const BlasFns& b = g_blas;
  const int N = P.N, M = P.M, d = P.d;
  const int QG = P.rG.npts(), QB = P.rB.npts(), QS = P.rS.npts(), ns = P.topo.nsides;
  const int Ptot = QG + QB + ns * QS;
  const double one = 1.0, zero = 0.0;
  const int ione = 1;
  double nrm0[3] = {0, 0, 0};
  vector<double> G((size_t)N * N, 0.0), B((size_t)M * N, 0.0), F(N, 0.0), tmp(N), rvv(M);
  // geometry at the Gram points
  vector<Geo> gG(QG);
  vector<double> wG(QG);
  for (int q = 0; q < QG; q++) {
    geometry(P, nodes, &P.rG.pts[q * d], gG[q]);
    wG[q] = P.rG.wts[q] * gG[q].det;
  }
  // G: per term, values of each of its vars over (point, component), k fastest
  for (int t = 0; t < P.nIPterms; t++) {
    const int nc = P.ip_ncomp[t], Kt = QG * nc;
    vector<int> vars;
    for (auto& e : P.ip)
      if (e.term == t && std::find(vars.begin(), vars.end(), e.test_var) == vars.end()) vars.push_back(e.test_var);
    std::sort(vars.begin(), vars.end());
    vector<vector<double>> val(vars.size()), wval(vars.size());
    for (size_t a = 0; a < vars.size(); a++) {
      const VarLayout& TL = P.tv[vars[a]];
      val[a].assign((size_t)TL.ndofs * Kt, 0.0);
      for (auto& e : P.ip) {
        if (e.term != t || e.test_var != vars[a]) continue;
        for (int q = 0; q < QG; q++) {
          test_op_values(P, P.test_tab[e.test_var][0], q, e.test_op, gG[q], nrm0, tmp.data());
          const double cf = e.coef * slotval(coeff, Ptot, e.slot, q);
          for (int i = 0; i < TL.ndofs; i++) val[a][(size_t)i * Kt + q * nc + e.comp] += cf * tmp[i];
        }
      }
      wval[a] = val[a];
      for (int i = 0; i < TL.ndofs; i++)
        for (int q = 0; q < QG; q++)
          for (int c = 0; c < nc; c++) wval[a][(size_t)i * Kt + q * nc + c] *= wG[q];
    }
    vector<double> mini;
    for (size_t a = 0; a < vars.size(); a++)
      for (size_t c2 = 0; c2 < vars.size(); c2++) {
        const VarLayout& U = P.tv[vars[a]];
        const VarLayout& V = P.tv[vars[c2]];
        const int nu = U.ndofs, nv = V.ndofs;
        mini.assign((size_t)nu * nv, 0.0);
        b.dgemm("T", "N", &nu, &nv, &Kt, &one, wval[a].data(), &Kt, val[c2].data(), &Kt, &zero, mini.data(), &nu);
        for (int j = 0; j < nv; j++)
          for (int i = 0; i < nu; i++) G[(size_t)(U.offset + i) * N + V.offset + j] += mini[(size_t)j * nu + i];
      }
  }
  // B and F: volume terms, one DGEMM per term over the B points
  {
    vector<Geo> gB(QB);
    vector<double> wB(QB);
    for (int q = 0; q < QB; q++) {
      geometry(P, nodes, &P.rB.pts[q * d], gB[q]);
      wB[q] = P.rB.wts[q] * gB[q].det;
    }
    for (auto& t : P.bf) {
      if (t.boundary) continue;
      const VarLayout& TL = P.tv[t.test_var];
      const VarLayout& RL = P.rv[t.trial_var];
      const int mu = RL.ndofs, nv = TL.ndofs;
      vector<double> Uw((size_t)mu * QB), Vt((size_t)nv * QB), blk((size_t)mu * nv);
      for (int q = 0; q < QB; q++) {
        test_op_values(P, P.test_tab[t.test_var][1], q, t.test_op, gB[q], nrm0, tmp.data());
        field_values(RL, P.field_tab[t.trial_var][1], q, t.trial_op, rvv.data());
        const double cf = wB[q] * t.coef * slotval(coeff, Ptot, t.slot, QG + q);
        for (int m = 0; m < mu; m++) Uw[(size_t)m * QB + q] = cf * rvv[m];
        for (int i = 0; i < nv; i++) Vt[(size_t)i * QB + q] = tmp[i];
      }
      b.dgemm("T", "N", &mu, &nv, &QB, &one, Uw.data(), &QB, Vt.data(), &QB, &zero, blk.data(), &mu);
      for (int i = 0; i < nv; i++)
        for (int m = 0; m < mu; m++) B[(size_t)(RL.offset + m) * N + TL.offset + i] += blk[(size_t)i * mu + m];
    }
    for (auto& r : P.rhs) {
      const VarLayout& TL = P.tv[r.test_var];
      const int nv = TL.ndofs;
      vector<double> Vt((size_t)QB * nv), fw(QB), out(nv);
      for (int q = 0; q < QB; q++) {
        test_op_values(P, P.test_tab[r.test_var][1], q, r.test_op, gB[q], nrm0, tmp.data());
        fw[q] = wB[q] * r.coef * slotval(coeff, Ptot, r.slot, QG + q);
        for (int i = 0; i < nv; i++) Vt[(size_t)i * QB + q] = tmp[i];
      }
      b.dgemv("T", &QB, &nv, &one, Vt.data(), &QB, fw.data(), &ione, &zero, out.data(), &ione);
      for (int i = 0; i < nv; i++) F[TL.offset + i] += out[i];
    }
  }
  // B: side terms, one DGEMM per (term, side) over the side points
  for (int sd = 0; sd < ns; sd++) {
    vector<Geo> gS(QS);
    vector<double> wS(QS), nS((size_t)QS * 3);
    for (int q = 0; q < QS; q++) {
      geometry(P, nodes, &P.side_pts[sd][q * d], gS[q]);
      double meas;
      side_geometry(P, gS[q], sd, q, meas, &nS[(size_t)q * 3]);
      wS[q] = P.rS.wts[q] * meas;
    }
    for (auto& t : P.bf) {
      if (!t.boundary) continue;
      const VarLayout& TL = P.tv[t.test_var];
      const VarLayout& RL = P.rv[t.trial_var];
      const bool field = RL.kind == DPG_VAR_FIELD;
      const int mu = field ? RL.ndofs : RL.per_side, m0 = field ? RL.offset : RL.offset + sd * RL.per_side;
      const int nv = TL.ndofs;
      vector<double> Uw((size_t)mu * QS), Vt((size_t)nv * QS), blk((size_t)mu * nv);
      for (int q = 0; q < QS; q++) {
        test_op_values(P, P.test_tab[t.test_var][2 + sd], q, t.test_op, gS[q], &nS[(size_t)q * 3], tmp.data());
        double cf = wS[q] * t.coef * slotval(coeff, Ptot, t.slot, QG + QB + sd * QS + q);
        if (t.normal_comp >= 0) cf *= nS[(size_t)q * 3 + t.normal_comp];
        if (field) {
          field_values(RL, P.field_tab[t.trial_var][2 + sd], q, t.trial_op, rvv.data());
        } else {
          const RefTab& TT = P.trace_tab[t.trial_var];
          for (int m = 0; m < mu; m++) rvv[m] = TT.val[(size_t)q * TT.card + m];
          if (RL.kind == DPG_VAR_FLUX) cf *= (double)parity[sd];
        }
        for (int m = 0; m < mu; m++) Uw[(size_t)m * QS + q] = cf * rvv[m];
        for (int i = 0; i < nv; i++) Vt[(size_t)i * QS + q] = tmp[i];
      }
      b.dgemm("T", "N", &mu, &nv, &QS, &one, Uw.data(), &QS, Vt.data(), &QS, &zero, blk.data(), &mu);
      for (int i = 0; i < nv; i++)
        for (int m = 0; m < mu; m++) B[(size_t)(m0 + m) * N + TL.offset + i] += blk[(size_t)i * mu + m];
    }
  }
  // factored Cholesky solve (BF.cpp:944-1016); G row-major = column-major transpose, symmetric
  vector<double> sc(N);
  for (int i = 0; i < N; i++) {
    const double gii = G[(size_t)i * N + i];
    if (!(gii > 0.0)) return i + 1;
    sc[i] = 1.0 / std::sqrt(gii);
  }
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) G[(size_t)i * N + j] *= sc[i] * sc[j];
  int info = 0;
  b.dpotrf("U", &N, G.data(), &N, &info);  // row-major lower = column-major upper
  if (info != 0) return info;
  // L (column-major lower) = transpose of the row-major upper factor: unscale L(i,j) /= s_i
  vector<double> L((size_t)N * N, 0.0);
  for (int j = 0; j < N; j++)
    for (int i = j; i < N; i++) L[(size_t)j * N + i] = G[(size_t)i * N + j] / sc[i];
  b.dtrsm("L", "L", "N", "N", &N, &M, &one, L.data(), &N, B.data(), &N);  // W = L^-1 B^T (N x M, ld N)
  vector<double> Kc((size_t)M * M, 0.0);
  b.dsyrk("L", "T", &M, &N, &one, B.data(), &N, &zero, Kc.data(), &M);   // K = W^T W (lower, column-major)
  for (int j = 0; j < M; j++)
    for (int i = j; i < M; i++) {
      K[(size_t)i * M + j] = Kc[(size_t)j * M + i];
      K[(size_t)j * M + i] = Kc[(size_t)j * M + i];
    }
  b.dtrsm("L", "L", "N", "N", &N, &ione, &one, L.data(), &N, F.data(), &N);  // y = L^-1 F
  b.dgemv("T", &N, &M, &one, B.data(), &N, F.data(), &ione, &zero, l, &ione);  // l = W^T y
  if (S || s) {
    vector<double> S_((size_t)P.nt * P.nt), s_(P.nt);
    int r = condense(M, P.is_field.data(), K, l, S_.data(), s_.data());
    if (S) std::copy(S_.begin(), S_.end(), S);
    if (s) std::copy(s_.begin(), s_.end(), s);
    if (r != 0) return r;
  }
  return 0;
}
#endif  // ORC_QUAD

}  // namespace ORC_NS

// ----------------------------------------------------------------------------
// C interface for the test harness (double in, double out)
// ----------------------------------------------------------------------------

using namespace ORC_NS;

static vector<real> widen(const double* x, size_t n) {
  vector<real> v(n);
  for (size_t i = 0; i < n; i++) v[i] = (real)x[i];
  return v;
}

template <class V>
static void narrow(const V& v, double* out) {
  for (size_t i = 0; i < v.size(); i++) out[i] = (double)v[i];
}

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

// 0 for the FP64 build, 1 for the extended-precision (__float128) build.
int orc_precision(void) {
#ifdef ORC_QUAD
  return 1;
#else
  return 0;
#endif
}

void* orc_plan_create(const dpg_bucket_desc* desc) {
  Plan* p = new Plan();
  if (!build_plan(*p, desc)) { delete p; return nullptr; }
  return p;
}

void orc_plan_destroy(void* p) { delete (Plan*)p; }

int orc_plan_query(void* pp, dpg_plan_info* info) {
  Plan* p = (Plan*)pp;
  info->N = p->N; info->M = p->M; info->n_field = p->nf; info->n_trace = p->nt;
  info->space_dim = p->d; info->n_vertices = p->topo.nv; info->n_sides = p->topo.nsides;
  info->Q_G = p->rG.npts(); info->Q_B = p->rB.npts(); info->Q_side = p->rS.npts();
  info->n_points_total = info->Q_G + info->Q_B + info->n_sides * info->Q_side;
  info->n_slots = p->desc.n_slots;
  info->precision = DPG_PREC_FP64;
  return 0;
}

// Assemble C cells on nthreads CPU threads.  Any output pointer may be NULL.
int orc_assemble(void* pp, int C, const double* nodes, const int8_t* parity, const double* coeff,
                 double* G, double* B, double* F, double* K, double* l, double* S, double* s,
                 int32_t* info, int nthreads) {
  Plan* p = (Plan*)pp;
  int N = p->N, M = p->M, nt = p->nt;
  int nv = p->topo.nv, d = p->d, ns = p->topo.nsides;
  dpg_plan_info pi;
  orc_plan_query(pp, &pi);
  size_t cstride = (size_t)p->desc.n_slots * pi.n_points_total;
  auto work = [&](int c0, int c1) {
    CellOut o;
    vector<real> Kc((size_t)M * M), lc(M);
    for (int c = c0; c < c1; c++) {
      vector<real> xn = widen(nodes + (size_t)c * nv * d, (size_t)nv * d);
      vector<real> xc = coeff ? widen(coeff + c * cstride, cstride) : vector<real>();
      assemble_cell(*p, xn.data(), parity + (size_t)c * ns, coeff ? xc.data() : nullptr, o);
      if (G) narrow(o.G, G + (size_t)c * N * N);
      if (B) narrow(o.B, B + (size_t)c * M * N);
      if (F) narrow(o.F, F + (size_t)c * N);
      if (!K && !l && !S && !s && !info) continue;
      int r = factored_cholesky_solve(N, M, o.G.data(), o.B.data(), o.F.data(), Kc.data(), lc.data());
      if (r == 0 && (S || s)) {
        vector<real> Sc((size_t)nt * nt), sc(nt);
        r = condense(M, p->is_field.data(), Kc.data(), lc.data(), Sc.data(), sc.data());
        if (S) narrow(Sc, S + (size_t)c * nt * nt);
        if (s) narrow(sc, s + (size_t)c * nt);
      }
      if (K) narrow(Kc, K + (size_t)c * M * M);
      if (l) narrow(lc, l + (size_t)c * M);
      if (info) info[c] = r;
    }
  };
  if (nthreads <= 1 || C < 2) {
    work(0, C);
  } else {
    std::vector<std::thread> th;
    int per = (C + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; t++) {
      int c0 = t * per, c1 = std::min(C, c0 + per);
      if (c0 >= c1) break;
      th.emplace_back(work, c0, c1);
    }
    for (auto& x : th) x.join();
  }
  return 0;
}

// Operator rows of one cell (see cell_operators).  With L == NULL only dims
// {term-component rows, B rows, F rows} are written.  L (QG, rows, N), wm (QG),
// rterm (rows), U (B rows, M), V (B rows, N), fw (F rows), FV (F rows, N).
int orc_cell_operators(void* pp, const double* nodes, const int8_t* parity, const double* coeff, int* dims,
                       double* L, double* wm, int* rterm, double* U, double* V, double* fw, double* FV) {
  Plan* p = (Plan*)pp;
  dpg_plan_info pi;
  orc_plan_query(pp, &pi);
  size_t cstride = (size_t)p->desc.n_slots * pi.n_points_total;
  vector<real> xn = widen(nodes, (size_t)p->topo.nv * p->d);
  vector<real> xc = coeff ? widen(coeff, cstride) : vector<real>();
  vector<real> L_, wm_, U_, V_, fw_, FV_;
  vector<int> rt;
  cell_operators(*p, xn.data(), parity, coeff ? xc.data() : nullptr, L_, wm_, rt, U_, V_, fw_, FV_);
  dims[0] = (int)rt.size();
  dims[1] = (int)(U_.size() / p->M);
  dims[2] = (int)fw_.size();
  if (!L) return 0;
  narrow(L_, L); narrow(wm_, wm); narrow(U_, U); narrow(V_, V); narrow(fw_, fw); narrow(FV_, FV);
  for (size_t i = 0; i < rt.size(); i++) rterm[i] = rt[i];
  return 0;
}

// Hand gradient of J = sum_c <Kbar_c, K_c> + <lbar_c, l_c> with respect to the
// coefficient slots: coeff_bar (C, n_slots, n_points_total).  Kbar (C, M, M), lbar (C, M).
int orc_adjoint(void* pp, int C, const double* nodes, const int8_t* parity, const double* coeff, const double* Kbar,
                const double* lbar, double* coeff_bar, int nthreads) {
  Plan* p = (Plan*)pp;
  const int M = p->M, nv = p->topo.nv, d = p->d, ns = p->topo.nsides;
  dpg_plan_info pi;
  orc_plan_query(pp, &pi);
  const size_t cstride = (size_t)p->desc.n_slots * pi.n_points_total;
  auto work = [&](int c0, int c1) {
    for (int c = c0; c < c1; c++) {
      vector<real> xn = widen(nodes + (size_t)c * nv * d, (size_t)nv * d);
      vector<real> xc = coeff ? widen(coeff + c * cstride, cstride) : vector<real>();
      vector<real> kb = widen(Kbar + (size_t)c * M * M, (size_t)M * M), lb = widen(lbar + (size_t)c * M, M);
      vector<real> cb(cstride);
      adjoint_cell(*p, xn.data(), parity + (size_t)c * ns, coeff ? xc.data() : nullptr, kb.data(), lb.data(), cb.data());
      narrow(cb, coeff_bar + c * cstride);
    }
  };
  if (nthreads <= 1 || C < 2) {
    work(0, C);
  } else {
    std::vector<std::thread> th;
    int per = (C + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; t++) {
      int c0 = t * per, c1 = std::min(C, c0 + per);
      if (c0 >= c1) break;
      th.emplace_back(work, c0, c1);
    }
    for (auto& x : th) x.join();
  }
  return 0;
}

// J = sum_c <Kbar_c, K_c> + <lbar_c, l_c> computed in `real` and returned as the
// unevaluated sum out[0] + out[1] of two doubles (out[0] = J rounded, out[1] = the
// rest), so that differences of nearby losses keep the build's precision.
int orc_loss(void* pp, int C, const double* nodes, const int8_t* parity, const double* coeff, const double* Kbar,
             const double* lbar, double* out, int nthreads) {
  Plan* p = (Plan*)pp;
  const int N = p->N, M = p->M, nv = p->topo.nv, d = p->d, ns = p->topo.nsides;
  dpg_plan_info pi;
  orc_plan_query(pp, &pi);
  const size_t cstride = (size_t)p->desc.n_slots * pi.n_points_total;
  vector<real> part(std::max(1, nthreads), 0.0);
  auto work = [&](int t, int c0, int c1) {
    CellOut o;
    vector<real> Kc((size_t)M * M), lc(M);
    real acc = 0.0;
    for (int c = c0; c < c1; c++) {
      vector<real> xn = widen(nodes + (size_t)c * nv * d, (size_t)nv * d);
      vector<real> xc = coeff ? widen(coeff + c * cstride, cstride) : vector<real>();
      assemble_cell(*p, xn.data(), parity + (size_t)c * ns, coeff ? xc.data() : nullptr, o);
      factored_cholesky_solve(N, M, o.G.data(), o.B.data(), o.F.data(), Kc.data(), lc.data());
      for (size_t k = 0; k < (size_t)M * M; k++) acc += (real)Kbar[(size_t)c * M * M + k] * Kc[k];
      for (int k = 0; k < M; k++) acc += (real)lbar[(size_t)c * M + k] * lc[k];
    }
    part[t] = acc;
  };
  if (nthreads <= 1 || C < 2) {
    work(0, 0, C);
  } else {
    std::vector<std::thread> th;
    int per = (C + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; t++) {
      int c0 = t * per, c1 = std::min(C, c0 + per);
      if (c0 >= c1) break;
      th.emplace_back(work, t, c0, c1);
    }
    for (auto& x : th) x.join();
  }
  real tot = 0.0;
  for (auto v : part) tot += v;
  out[0] = (double)tot;
  out[1] = (double)(tot - (real)out[0]);
  return 0;
}

// Central difference (J(coeff + h dir) - J(coeff - h dir)) / (2 h) of
// J = sum_c <Kbar_c, K_c> + <lbar_c, l_c>, computed entirely in `real` (the perturbed
// coefficients, both assemblies and the difference), so that in the __float128 build the
// result carries the difference's truncation error only.
double orc_fd_directional(void* pp, int C, const double* nodes, const int8_t* parity, const double* coeff,
                          const double* dir, double h, const double* Kbar, const double* lbar, int nthreads) {
  Plan* p = (Plan*)pp;
  const int N = p->N, M = p->M, nv = p->topo.nv, d = p->d, ns = p->topo.nsides;
  dpg_plan_info pi;
  orc_plan_query(pp, &pi);
  const size_t cstride = (size_t)p->desc.n_slots * pi.n_points_total;
  vector<real> part(std::max(1, nthreads), 0.0);
  auto work = [&](int t, int c0, int c1) {
    CellOut o;
    vector<real> Kc((size_t)M * M), lc(M);
    real acc = 0.0;
    for (int c = c0; c < c1; c++) {
      vector<real> xn = widen(nodes + (size_t)c * nv * d, (size_t)nv * d);
      for (int sg = -1; sg <= 1; sg += 2) {
        vector<real> xc(cstride);
        for (size_t k = 0; k < cstride; k++) xc[k] = (real)coeff[c * cstride + k] + sg * (real)h * (real)dir[c * cstride + k];
        assemble_cell(*p, xn.data(), parity + (size_t)c * ns, xc.data(), o);
        factored_cholesky_solve(N, M, o.G.data(), o.B.data(), o.F.data(), Kc.data(), lc.data());
        real J = 0.0;
        for (size_t k = 0; k < (size_t)M * M; k++) J += (real)Kbar[(size_t)c * M * M + k] * Kc[k];
        for (int k = 0; k < M; k++) J += (real)lbar[(size_t)c * M + k] * lc[k];
        acc += sg * J;
      }
    }
    part[t] = acc;
  };
  if (nthreads <= 1 || C < 2) {
    work(0, 0, C);
  } else {
    std::vector<std::thread> th;
    int per = (C + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; t++) {
      int c0 = t * per, c1 = std::min(C, c0 + per);
      if (c0 >= c1) break;
      th.emplace_back(work, t, c0, c1);
    }
    for (auto& x : th) x.join();
  }
  real tot = 0.0;
  for (auto v : part) tot += v;
  return (double)(tot / (2 * (real)h));
}

#ifndef ORC_QUAD
// BLAS/LAPACK entry points for the fast mode (Fortran LP64 interface; any NULL
// disables it).  Returns 0 when the fast mode is available.
int orc_set_blas(void* dgemm, void* dgemv, void* dsyrk, void* dtrsm, void* dpotrf) {
  g_blas.dgemm = (DgemmFn)dgemm;
  g_blas.dgemv = (DgemvFn)dgemv;
  g_blas.dsyrk = (DsyrkFn)dsyrk;
  g_blas.dtrsm = (DtrsmFn)dtrsm;
  g_blas.dpotrf = (DpotrfFn)dpotrf;
  return (dgemm && dgemv && dsyrk && dtrsm && dpotrf) ? 0 : 1;
}

// Fast mode (the CPU baseline): K, l, S, s, info of C cells on nthreads threads.
int orc_assemble_blas(void* pp, int C, const double* nodes, const int8_t* parity, const double* coeff, double* K,
                      double* l, double* S, double* s, int32_t* info, int nthreads) {
  if (!g_blas.dgemm || !g_blas.dgemv || !g_blas.dsyrk || !g_blas.dtrsm || !g_blas.dpotrf) {
    g_err = "orc_assemble_blas: BLAS entry points not set (orc_set_blas)";
    return 1;
  }
  Plan* p = (Plan*)pp;
  const int M = p->M, nt = p->nt, nv = p->topo.nv, d = p->d, ns = p->topo.nsides;
  dpg_plan_info pi;
  orc_plan_query(pp, &pi);
  const size_t cstride = (size_t)p->desc.n_slots * pi.n_points_total;
  auto work = [&](int c0, int c1) {
    vector<double> Kc((size_t)M * M), lc(M);
    for (int c = c0; c < c1; c++) {
      int r = assemble_cell_blas(*p, nodes + (size_t)c * nv * d, parity + (size_t)c * ns,
                                 coeff ? coeff + c * cstride : nullptr, K ? K + (size_t)c * M * M : Kc.data(),
                                 l ? l + (size_t)c * M : lc.data(), S ? S + (size_t)c * nt * nt : nullptr,
                                 s ? s + (size_t)c * nt : nullptr);
      if (info) info[c] = r;
    }
  };
  if (nthreads <= 1 || C < 2) {
    work(0, C);
  } else {
    std::vector<std::thread> th;
    int per = (C + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; t++) {
      int c0 = t * per, c1 = std::min(C, c0 + per);
      if (c0 >= c1) break;
      th.emplace_back(work, c0, c1);
    }
    for (auto& x : th) x.join();
  }
  return 0;
}
#endif  // ORC_QUAD

// Single-cell factored Cholesky (inputs copied): G row-major NxN, B (M,N), F (N).
int orc_factored_cholesky_solve(int N, int M, const double* G, const double* B, const double* F, double* K,
                                double* l) {
  vector<real> g = widen(G, (size_t)N * N), b = widen(B, (size_t)M * N), f = widen(F, N);
  vector<real> k((size_t)M * M), ll(M);
  int r = factored_cholesky_solve(N, M, g.data(), b.data(), f.data(), k.data(), ll.data());
  narrow(k, K);
  narrow(ll, l);
  return r;
}

int orc_condense(int M, const int* is_field, const double* K, const double* l, double* S, double* s) {
  int nt = 0;
  for (int i = 0; i < M; i++) nt += is_field[i] ? 0 : 1;
  vector<real> k = widen(K, (size_t)M * M), ll = widen(l, M), S_((size_t)nt * nt), s_(nt);
  int r = condense(M, is_field, k.data(), ll.data(), S_.data(), s_.data());
  narrow(S_, S);
  narrow(s_, s);
  return r;
}

int orc_trial_is_field(void* pp, int* out) {
  Plan* p = (Plan*)pp;
  for (int i = 0; i < p->M; i++) out[i] = p->is_field[i];
  return p->M;
}

// Tabulate a reference basis at npts points: val (npts, card, vdim),
// grad (npts, card, d) for scalar bases, div (npts, card) for HDIV.
// topo 0 = line.  Returns card.
int orc_basis_tabulate(int topo, int space, int n, int npts, const double* pts, double* val, double* grad,
                       double* div) {
  Basis b = make_basis(topo, space, n);
  if (topo == 0) { b.d = 1; b.card = b.closed.size(); }
  int d = b.d, vdim = b.rank ? d : 1;
  vector<real> v(b.card * vdim), g(b.card * d), dv(b.card);
  for (int q = 0; q < npts; q++) {
    vector<real> x = widen(pts + q * d, d);
    b.eval(x.data(), v.data(), b.rank ? nullptr : g.data(), b.rank ? dv.data() : nullptr);
    if (val) narrow(v, val + (size_t)q * b.card * vdim);
    if (grad && !b.rank) narrow(g, grad + (size_t)q * b.card * d);
    if (div && b.rank) narrow(dv, div + (size_t)q * b.card);
  }
  return b.card;
}

// Tensor Gauss rule of a degree on the line (dim 1), quad (2) or hex (3).
int orc_cubature(int dim, int degree, double* pts, double* wts) {
  Rule r = tensor_gauss(dim, degree);
  if (pts) narrow(r.pts, pts);
  if (wts) narrow(r.wts, wts);
  return r.npts();
}

// Triangle rule exact to `degree` on the reference triangle.
int orc_tri_cubature(int degree, double* pts, double* wts) {
  Rule r = tri_rule(degree);
  if (pts) narrow(r.pts, pts);
  if (wts) narrow(r.wts, wts);
  return r.npts();
}

// Warp & blend lattice of degree n (the nodes of the triangle HGRAD basis).
int orc_tri_nodes(int n, double* pts) {
  vector<real> x = warp_blend_tri(n);
  if (pts) narrow(x, pts);
  return (int)x.size() / 2;
}

}  // extern "C"
