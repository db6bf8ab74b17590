// dpg_host.cu — plan construction and the C ABI of the DPG assembly library.
//
// The plan reproduces, for one bucket (Camellia ElementType), what
// BasisCache/BasisFactory/DofOrdering set up on the CPU in the reference:
//   - tensor Gauss rules, n = degree/2 + 1 points per direction
//     (src/Basis/CubatureFactory.cpp:25-53, degrees src/Basis/BasisCache.cpp:68-84,236-267,198-222);
//   - reference bases (src/Basis/BasisFactory.cpp:122-420): HGRAD Cn nodal at
//     Gauss-Lobatto points (x fastest), HDIV In = tensor Raviart-Thomas
//     (component-major), HVOL of H1Order k = HGRAD C(k-1), VECTOR_HVOL =
//     component-major copies; traces: HGRAD C(k) / HVOL C(k-1) on each side in
//     the side's own parametrisation (shards side node order);
//   - dof numbering var by var, traces side by side
//     (src/DofOrdering/DofOrderingFactory.cpp:53-211, DofOrdering.cpp:27-60).
// The tables are uploaded once; the kernels apply the Piola transforms per cell.
#include "../../include/dpg_b200.h"
#include "dpg_plan.h"
#include "dpg_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <set>
#include <mutex>

#define DPG_CHA_HOST 4  // points per reverse-mode pull-back chunk (DPG_CHA in the kernel)
#include <string>
#include <vector>

namespace dpg {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

// ----------------------------------------------------------------------------
// 1D point families
// ----------------------------------------------------------------------------

// P_n(x) and P_n'(x)
static void legendre_pd(int n, double x, double* p, double* dp) {
  double a = 1.0, b = x;  // P_0, P_1
  if (n == 0) { *p = 1.0; *dp = 0.0; return; }
  for (int m = 1; m < n; m++) {
    double c = ((2 * m + 1) * x * b - m * a) / (m + 1);
    a = b;
    b = c;
  }
  *p = b;
  *dp = n * (x * b - a) / (x * x - 1.0);
}

// n-point Gauss-Legendre rule, nodes ascending.
static void gauss_rule(int n, std::vector<double>& x, std::vector<double>& w) {
  x.resize(n);
  w.resize(n);
  for (int i = 0; i < n; i++) {
    // Tricomi initial guess, refined by Newton
    double z = std::cos(M_PI * (n - i - 0.25) / (n + 0.5));
    for (int it = 0; it < 60; it++) {
      double p, dp;
      legendre_pd(n, z, &p, &dp);
      double step = p / dp;
      z -= step;
      if (std::fabs(step) <= 1e-17) break;
    }
    double p, dp;
    legendre_pd(n, z, &p, &dp);
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

// Gauss-Lobatto-Legendre nodes of degree p (p+1 nodes).
static std::vector<double> gll_nodes(int p) {
  std::vector<double> x(p + 1, 0.0);
  if (p == 0) return x;
  x[0] = -1.0;
  x[p] = 1.0;
  for (int i = 1; i < p; i++) {
    double z = -std::cos(M_PI * i / p);
    for (int it = 0; it < 60; it++) {
      double P, dP;
      legendre_pd(p, z, &P, &dP);
      // Newton on (1 - z^2) P'(z): derivative = -p(p+1) P(z) by Legendre's equation
      double f = (1.0 - z * z) * dP;
      double df = -p * (p + 1.0) * P;
      double step = f / df;
      z -= step;
      if (std::fabs(step) <= 1e-17) break;
    }
    x[i] = z;
  }
  return x;
}

struct Lagrange1D {
  std::vector<double> x;
  int n() const { return (int)x.size(); }
  // values and derivatives of all polynomials at s
  void eval(double s, double* v, double* dv) const {
    int m = n();
    if (m == 1) { v[0] = 1.0; dv[0] = 0.0; return; }
    for (int j = 0; j < m; j++) {
      double num = 1.0, den = 1.0, der = 0.0;
      for (int k = 0; k < m; k++) {
        if (k == j) continue;
        den *= (x[j] - x[k]);
        // derivative of prod_k (s - x_k): sum over the factor left out
        double term = 1.0;
        for (int q = 0; q < m; q++)
          if (q != j && q != k) term *= (s - x[q]);
        der += term;
        num *= (s - x[k]);
      }
      v[j] = num / den;
      dv[j] = der / den;
    }
  }
};

static Lagrange1D closed_family(int p) { return Lagrange1D{gll_nodes(p)}; }
static Lagrange1D open_family(int p) {  // degree p: p+1 Gauss points
  std::vector<double> x, w;
  gauss_rule(p + 1, x, w);
  return Lagrange1D{x};
}

// ----------------------------------------------------------------------------
// Reference bases: tabulate at points
// ----------------------------------------------------------------------------

// Scalar tensor Lagrange basis of degree p on [-1,1]^dim: per point, per dof,
// out[(dof)*(1+dim) + 0] = value, + 1 + k = d/dxi_k.  Returns card.
static int tab_hgrad(int dim, int p, const double* xi, double* out) {
  Lagrange1D L = closed_family(p);
  int m = L.n();
  double v[3][32], dv[3][32];
  for (int k = 0; k < dim; k++) L.eval(xi[k], v[k], dv[k]);
  int card = 1;
  for (int k = 0; k < dim; k++) card *= m;
  for (int idx = 0; idx < card; idx++) {
    int ii[3] = {idx % m, (idx / m) % m, idx / (m * m)};
    double val = 1.0;
    for (int k = 0; k < dim; k++) val *= v[k][ii[k]];
    out[idx * (1 + dim)] = val;
    for (int k = 0; k < dim; k++) {
      double g = 1.0;
      for (int j = 0; j < dim; j++) g *= (j == k) ? dv[j][ii[j]] : v[j][ii[j]];
      out[idx * (1 + dim) + 1 + k] = g;
    }
  }
  return card;
}

// Tensor Raviart-Thomas In: out[dof*(dim+1) + c] = value comp c, + dim = div.
static int tab_hdiv(int dim, int n, const double* xi, double* out) {
  Lagrange1D C = closed_family(n), O = open_family(n - 1);
  double cv[3][32], cd[3][32], ov[3][32], od[3][32];
  for (int k = 0; k < dim; k++) {
    C.eval(xi[k], cv[k], cd[k]);
    O.eval(xi[k], ov[k], od[k]);
  }
  int dof = 0;
  for (int comp = 0; comp < dim; comp++) {
    int ext[3];
    for (int k = 0; k < dim; k++) ext[k] = (k == comp) ? C.n() : O.n();
    int cnt = 1;
    for (int k = 0; k < dim; k++) cnt *= ext[k];
    for (int idx = 0; idx < cnt; idx++) {
      int ii[3], r = idx;
      for (int k = 0; k < dim; k++) { ii[k] = r % ext[k]; r /= ext[k]; }
      double f = 1.0, df = 1.0;
      for (int k = 0; k < dim; k++) {
        double a = (k == comp) ? cv[k][ii[k]] : ov[k][ii[k]];
        f *= a;
        df *= (k == comp) ? cd[k][ii[k]] : a;
      }
      for (int c = 0; c < dim; c++) out[dof * (dim + 1) + c] = (c == comp) ? f : 0.0;
      out[dof * (dim + 1) + dim] = df;
      dof++;
    }
  }
  return dof;
}

static int card_hgrad(int dim, int p) {
  int m = p + 1, c = 1;
  for (int k = 0; k < dim; k++) c *= m;
  return c;
}
static int card_hdiv(int dim, int n) { return dim == 2 ? 2 * n * (n + 1) : 3 * n * n * (n + 1); }

// ----------------------------------------------------------------------------
// Triangle bases (Intrepid Basis_HGRAD_TRI_Cn_FEM on the warp & blend lattice,
// Basis_HDIV_TRI_In_FEM = Raviart-Thomas RT_n; BasisFactory.cpp:198-350).  The
// lattice follows the published warp & blend construction (Warburton 2006,
// optimized alpha table); the Lagrange functions are built through the
// orthonormal PKD (Dubiner) polynomials, whose Vandermonde matrix on the lattice
// is well conditioned.  RT_n uses the modal basis (p,0), (0,p) for p in P_{n-1}
// and x psi for the orthonormal PKD polynomials psi of exact degree n-1 (a
// well-conditioned choice): only the span of a test space enters K, l and S.
// ----------------------------------------------------------------------------

// Orthonormal Jacobi polynomial P_n^{(a,b)} on [-1,1].
static double jacobi_p(double x, double a, double b, int n) {
  const double g0 =
      std::pow(2.0, a + b + 1) / (a + b + 1) * std::tgamma(a + 1) * std::tgamma(b + 1) / std::tgamma(a + b + 1);
  double pm = 1.0 / std::sqrt(g0);
  if (n == 0) return pm;
  const double g1 = (a + 1) * (b + 1) / (a + b + 3) * g0;
  double pc = ((a + b + 2) * x / 2 + (a - b) / 2) / std::sqrt(g1);
  double an = 2.0 / (2 + a + b) * std::sqrt((a + 1) * (b + 1) / (a + b + 3));
  for (int i = 1; i < n; i++) {
    const double h = 2.0 * i + a + b;
    const double an1 = 2.0 / (h + 2) * std::sqrt((i + 1) * (i + 1 + a + b) * (i + 1 + a) * (i + 1 + b) / (h + 1) / (h + 3));
    const double bn1 = -(a * a - b * b) / h / (h + 2);
    const double pn = (-an * pm + (x - bn1) * pc) / an1;
    pm = pc;
    pc = pn;
    an = an1;
  }
  return pc;
}
static double jacobi_dp(double x, double a, double b, int n) {
  return n == 0 ? 0.0 : std::sqrt(n * (n + a + b + 1)) * jacobi_p(x, a + 1, b + 1, n - 1);
}

// PKD polynomial (i, j) at (r, s) of the biunit triangle, with d/dr and d/ds.
static void pkd(int i, int j, double r, double s, double& v, double& dr, double& ds) {
  const double a = (std::fabs(s - 1.0) > 1e-14) ? 2.0 * (1.0 + r) / (1.0 - s) - 1.0 : -1.0, b = s;
  const double fa = jacobi_p(a, 0, 0, i), dfa = jacobi_dp(a, 0, 0, i);
  const double gb = jacobi_p(b, 2 * i + 1, 0, j), dgb = jacobi_dp(b, 2 * i + 1, 0, j);
  const double hb = 0.5 * (1.0 - b), sc = std::pow(2.0, i + 0.5);
  v = sc * fa * gb * std::pow(hb, i);
  double er = dfa * gb, es = dfa * gb * 0.5 * (1.0 + a);
  if (i > 0) { er *= std::pow(hb, i - 1); es *= std::pow(hb, i - 1); }
  double t = dgb * std::pow(hb, i);
  if (i > 0) t -= 0.5 * i * gb * std::pow(hb, i - 1);
  es += fa * t;
  dr = sc * er;
  ds = sc * es;
}

// Warp & blend lattice of degree N >= 1 on (0,0),(1,0),(0,1); rows of constant eta.
static std::vector<double> tri_lattice(int N) {
  static const double alpopt[15] = {0.0000, 0.0000, 1.4152, 0.1001, 0.2751, 0.9800, 1.0999, 1.2832,
                                    1.3648, 1.4773, 1.4959, 1.5743, 1.5770, 1.6223, 1.6258};
  const double alpha = N < 16 ? alpopt[N - 1] : 5.0 / 3.0;
  const std::vector<double> gll = gll_nodes(N);
  auto warp = [&](double r) {
    double w = 0.0;
    for (int i = 0; i <= N; i++) {
      const double ei = -1.0 + 2.0 * i / N;
      double l = 1.0;
      for (int j = 0; j <= N; j++)
        if (j != i) {
          const double ej = -1.0 + 2.0 * j / N;
          l *= (r - ej) / (ei - ej);
        }
      w += (gll[i] - ei) * l;
    }
    return std::fabs(r) < 1.0 - 1e-10 ? w / (1.0 - r * r) : 0.0;
  };
  const double s3 = std::sqrt(3.0);
  std::vector<double> out;
  for (int n = 0; n <= N; n++)
    for (int m = 0; m <= N - n; m++) {
      const double L1 = (double)n / N, L3 = (double)m / N, L2 = 1.0 - L1 - L3;
      double x = -L2 + L3, y = (-L2 - L3 + 2 * L1) / s3;
      const double w1 = 4 * L2 * L3 * warp(L3 - L2) * (1 + (alpha * L1) * (alpha * L1));
      const double w2 = 4 * L1 * L3 * warp(L1 - L3) * (1 + (alpha * L2) * (alpha * L2));
      const double w3 = 4 * L1 * L2 * warp(L2 - L1) * (1 + (alpha * L3) * (alpha * L3));
      x += w1 + std::cos(2 * M_PI / 3) * w2 + std::cos(4 * M_PI / 3) * w3;
      y += std::sin(2 * M_PI / 3) * w2 + std::sin(4 * M_PI / 3) * w3;
      const double b1 = (s3 * y + 1) / 3, b2 = (-3 * x - s3 * y + 2) / 6, b3 = (3 * x - s3 * y + 2) / 6;
      out.push_back(0.5 * (1 + (-b2 + b3 - b1)));
      out.push_back(0.5 * (1 + (-b2 - b3 + b1)));
    }
  return out;
}

// Coefficients of the degree-n Lagrange functions in the PKD basis (inverse
// Vandermonde), cached per degree.
static const std::vector<double>& tri_vinv(int n) {
  static std::mutex mu;
  static std::map<int, std::vector<double>> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(n);
  if (it != cache.end()) return it->second;
  const int c = (n + 1) * (n + 2) / 2;
  std::vector<double> X = tri_lattice(n), A((size_t)c * c), Xi((size_t)c * c, 0.0);
  for (int p = 0; p < c; p++) {
    int m = 0;
    for (int i = 0; i <= n; i++)
      for (int j = 0; j <= n - i; j++, m++) {
        double v, dr, ds;
        pkd(i, j, 2 * X[2 * p] - 1, 2 * X[2 * p + 1] - 1, v, dr, ds);
        A[(size_t)p * c + m] = v;
      }
  }
  for (int i = 0; i < c; i++) Xi[(size_t)i * c + i] = 1.0;
  for (int col = 0; col < c; col++) {  // Gauss-Jordan with partial pivoting
    int piv = col;
    for (int r = col + 1; r < c; r++)
      if (std::fabs(A[(size_t)r * c + col]) > std::fabs(A[(size_t)piv * c + col])) piv = r;
    for (int k = 0; k < c; k++) {
      std::swap(A[(size_t)col * c + k], A[(size_t)piv * c + k]);
      std::swap(Xi[(size_t)col * c + k], Xi[(size_t)piv * c + k]);
    }
    const double inv = 1.0 / A[(size_t)col * c + col];
    for (int k = 0; k < c; k++) { A[(size_t)col * c + k] *= inv; Xi[(size_t)col * c + k] *= inv; }
    for (int r = 0; r < c; r++) {
      if (r == col) continue;
      const double f = A[(size_t)r * c + col];
      if (f == 0.0) continue;
      for (int k = 0; k < c; k++) {
        A[(size_t)r * c + k] -= f * A[(size_t)col * c + k];
        Xi[(size_t)r * c + k] -= f * Xi[(size_t)col * c + k];
      }
    }
  }
  return cache.emplace(n, std::move(Xi)).first->second;
}

// HGRAD_TRI_Cn: out[dof*3 + 0] = value, + 1 + k = d/dxi_k.  Returns card.
static int tab_hgrad_tri(int n, const double* xi, double* out) {
  const int c = (n + 1) * (n + 2) / 2;
  if (n == 0) { out[0] = 1.0; out[1] = 0.0; out[2] = 0.0; return 1; }
  const std::vector<double>& Vi = tri_vinv(n);
  std::vector<double> pv(c), pr(c), ps(c);
  int m = 0;
  for (int i = 0; i <= n; i++)
    for (int j = 0; j <= n - i; j++, m++) pkd(i, j, 2 * xi[0] - 1, 2 * xi[1] - 1, pv[m], pr[m], ps[m]);
  for (int k = 0; k < c; k++) {
    double v = 0, gx = 0, gy = 0;
    for (int mm = 0; mm < c; mm++) {
      const double w = Vi[(size_t)mm * c + k];
      v += pv[mm] * w;
      gx += pr[mm] * w;
      gy += ps[mm] * w;
    }
    out[k * 3] = v;
    out[k * 3 + 1] = 2 * gx;
    out[k * 3 + 2] = 2 * gy;
  }
  return c;
}

// HDIV_TRI_In (RT_n): out[dof*3 + c] = value comp c, + 2 = div.  Returns card n (n + 2).
static int tab_hdiv_tri(int n, const double* xi, double* out) {
  const int np = n * (n + 1) / 2;
  std::vector<double> pv(np), pr(np), ps(np);
  int m = 0;
  for (int i = 0; i <= n - 1; i++)
    for (int j = 0; j <= n - 1 - i; j++, m++) pkd(i, j, 2 * xi[0] - 1, 2 * xi[1] - 1, pv[m], pr[m], ps[m]);
  int dof = 0;
  for (int c = 0; c < 2; c++)
    for (int k = 0; k < np; k++, dof++) {
      out[dof * 3] = c == 0 ? pv[k] : 0.0;
      out[dof * 3 + 1] = c == 1 ? pv[k] : 0.0;
      out[dof * 3 + 2] = 2 * (c == 0 ? pr[k] : ps[k]);
    }
  // x psi for the PKD polynomials psi of exact degree n-1: their leading homogeneous parts span
  // the homogeneous polynomials of degree n-1, and unlike monomials they stay well conditioned
  for (int j = 0; j < n; j++, dof++) {
    double v, dr, ds;
    pkd(n - 1 - j, j, 2 * xi[0] - 1, 2 * xi[1] - 1, v, dr, ds);
    out[dof * 3] = xi[0] * v;
    out[dof * 3 + 1] = xi[1] * v;
    out[dof * 3 + 2] = 2 * v + 2 * (xi[0] * dr + xi[1] * ds);  // div(x psi) = 2 psi + x . grad psi
  }
  return dof;
}

// Reference-cell bases by topology (tensor cells on [-1,1]^dim, or the triangle).
static int tab_hgrad_t(int topo, int dim, int p, const double* xi, double* out) {
  return topo == DPG_TOPO_TRI ? tab_hgrad_tri(p, xi, out) : tab_hgrad(dim, p, xi, out);
}
static int tab_hdiv_t(int topo, int dim, int n, const double* xi, double* out) {
  return topo == DPG_TOPO_TRI ? tab_hdiv_tri(n, xi, out) : tab_hdiv(dim, n, xi, out);
}
static int card_hgrad_t(int topo, int dim, int p) {
  return topo == DPG_TOPO_TRI ? (p + 1) * (p + 2) / 2 : card_hgrad(dim, p);
}
static int card_hdiv_t(int topo, int dim, int n) { return topo == DPG_TOPO_TRI ? n * (n + 2) : card_hdiv(dim, n); }

// ----------------------------------------------------------------------------
// Topology data (shards)
// ----------------------------------------------------------------------------

struct TopoData {
  int key, d, nv, ns;
  double v[8][3];
  int sv[6][4];
};

static bool topo_data(int key, TopoData& t) {
  std::memset(&t, 0, sizeof(t));
  t.key = key;
  if (key == DPG_TOPO_QUAD) {
    t.d = 2; t.nv = 4; t.ns = 4;
    const double v[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
    for (int a = 0; a < 4; a++) { t.v[a][0] = v[a][0]; t.v[a][1] = v[a][1]; }
    for (int s = 0; s < 4; s++) { t.sv[s][0] = s; t.sv[s][1] = (s + 1) & 3; }
    return true;
  }
  if (key == DPG_TOPO_TRI) {
    t.d = 2; t.nv = 3; t.ns = 3;
    const double v[3][2] = {{0, 0}, {1, 0}, {0, 1}};
    for (int a = 0; a < 3; a++) { t.v[a][0] = v[a][0]; t.v[a][1] = v[a][1]; }
    for (int s = 0; s < 3; s++) { t.sv[s][0] = s; t.sv[s][1] = (s + 1) % 3; }
    t.key = key;
    return true;
  }
  if (key == DPG_TOPO_HEX) {
    t.d = 3; t.nv = 8; t.ns = 6;
    for (int a = 0; a < 8; a++) {
      int lo = a & 3;
      t.v[a][0] = (lo == 1 || lo == 2) ? 1 : -1;
      t.v[a][1] = (lo >= 2) ? 1 : -1;
      t.v[a][2] = (a >= 4) ? 1 : -1;
    }
    const int f[6][4] = {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {0, 4, 7, 3}, {0, 3, 2, 1}, {4, 5, 6, 7}};
    std::memcpy(t.sv, f, sizeof(f));
    return true;
  }
  return false;
}

// d(vertex shape)/d(xi) of the (bi/tri)linear geometric map
static void geom_dshape(const TopoData& t, const double* xi, double* dN) {
  if (t.key == DPG_TOPO_TRI) {  // affine: N = (1 - xi - eta, xi, eta)
    dN[0] = -1; dN[1] = -1; dN[2] = 1; dN[3] = 0; dN[4] = 0; dN[5] = 1;
    return;
  }
  for (int a = 0; a < t.nv; a++)
    for (int k = 0; k < t.d; k++) {
      double g = 0.5 * t.v[a][k];
      for (int j = 0; j < t.d; j++)
        if (j != k) g *= 0.5 * (1.0 + xi[j] * t.v[a][j]);
      dN[a * t.d + k] = g;
    }
}

// ----------------------------------------------------------------------------
// Plan
// ----------------------------------------------------------------------------

static int pad8(int n) { return (n + 7) & ~7; }
static int ld_pad(int n) {  // >= n, == 4 (mod 16): conflict-free fragment loads
  int x = n;
  while ((x & 15) != 4) x++;
  return x;
}

struct HostPlan;

static double* upload(HostPlan* P, const std::vector<double>& v);
static int* upload_i(HostPlan* P, const std::vector<int>& v);

struct HostPlan {
  dpg_bucket_desc desc;
  dpg_plan_info info;
  DpgPlanDev dev;           // host copy with device pointers inside
  DpgPlanDev* d_dev = nullptr;
  std::vector<void*> allocs;
  int device = 0;
  // host staging for dpg_assemble_host
  void* h_ws = nullptr;
  size_t ws_bytes = 0;
  void* d_ws = nullptr;
  cudaStream_t streams[2] = {nullptr, nullptr};
  bool adj_terms_ok = false;  // every coefficient use of the bucket is one the reverse mode covers
};

static double* upload(HostPlan* P, const std::vector<double>& v) {
  void* p = nullptr;
  size_t bytes = std::max<size_t>(8, v.size() * sizeof(double));
  if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
  if (!v.empty()) cudaMemcpy(p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice);
  P->allocs.push_back(p);
  return (double*)p;
}
static int* upload_i(HostPlan* P, const std::vector<int>& v) {
  void* p = nullptr;
  size_t bytes = std::max<size_t>(8, v.size() * sizeof(int));
  if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
  if (!v.empty()) cudaMemcpy(p, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice);
  P->allocs.push_back(p);
  return (int*)p;
}

struct Rule {
  std::vector<double> x, w;  // x: npts*dim
  int n = 0;
};

static Rule tensor_rule(int dim, int degree) {
  int n1 = degree / 2 + 1;
  std::vector<double> x, w;
  gauss_rule(n1, x, w);
  Rule r;
  r.n = 1;
  for (int k = 0; k < dim; k++) r.n *= n1;
  r.x.resize(r.n * dim);
  r.w.resize(r.n);
  for (int q = 0; q < r.n; q++) {
    int rem = q;
    double wt = 1.0;
    for (int k = 0; k < dim; k++) {
      int i = rem % n1;
      rem /= n1;
      r.x[q * dim + k] = x[i];
      wt *= w[i];
    }
    r.w[q] = wt;
  }
  return r;
}

// Triangle rule exact to `degree` (any exact rule integrates the polynomial
// integrands of an affine triangle identically): collapsed Gauss-Legendre,
// xi = u (1 - v), eta = v on [0,1]^2, weight w_u w_v (1 - v) / 4, u fastest.
static Rule tri_rule(int degree) {
  const int nu = degree / 2 + 1, nv = (degree + 1) / 2 + 1;
  std::vector<double> xu, wu, xv, wv;
  gauss_rule(nu, xu, wu);
  gauss_rule(nv, xv, wv);
  Rule r;
  r.n = nu * nv;
  for (int j = 0; j < nv; j++)
    for (int i = 0; i < nu; i++) {
      const double u = 0.5 * (1 + xu[i]), v = 0.5 * (1 + xv[j]);
      r.x.push_back(u * (1 - v));
      r.x.push_back(v);
      r.w.push_back(0.25 * wu[i] * wv[j] * (1 - v));
    }
  return r;
}

// Tables and memory layout of the large-bucket kernel (dpg_big_kernel): the formation
// entries of E (one per segment and term), the test vars of each IP row, the user -> device
// trial map, the per-CTA workspace (Z, then the per-point factors) and shared memory.
static int big_layout(HostPlan* P) {
  DpgPlanDev& g = P->dev;
  g.adj_ok = 0;
  g.Zn = g.Np + g.Mp;
  if (g.Np > 4096 || g.Zn > 6144) return fail(DPG_ERR_UNSUPPORTED, "bucket too large for the large-bucket kernel");
  g.ldz = (g.Zn + 7) & ~7;
  for (int r = 0; r < g.niprows; r++) {
    g.ipmask[r] = 0;
    for (int e = g.rowstart[r]; e < g.rowstart[r + 1]; e++) g.ipmask[r] |= 1 << (g.ipent[e].gslot >> 2);
  }
  int vrow = 0;
  g.nbe = 0;
  for (int sg = 0; sg < g.nseg; sg++)
    for (int lt = 0; lt < g.seg[sg].nterm; lt++) {
      g.be[g.nbe++] = make_int4(sg, lt, vrow, g.seg[sg].npts);
      vrow += g.seg[sg].npts;
    }
  std::vector<int> u2d(g.M, 0);
  for (int b = 0; b < g.ntrial; b++) {
    const DpgTrialVar& tr = g.trial[b];
    const int cnt = (tr.kind == DPG_VAR_FIELD) ? tr.ncomp * tr.card_comp : tr.per_side * g.ns;
    for (int i = 0; i < cnt; i++) u2d[tr.user_off + i] = tr.dev_off + i;
  }
  g.u2d_trial = upload_i(P, u2d);
  std::vector<int> u2dt(g.N, 0);
  for (int a = 0; a < g.ntest; a++)
    for (int i = 0; i < g.test[a].card; i++) u2dt[g.test[a].user_off + i] = g.test[a].dev_off + i;
  g.u2d_test = upload_i(P, u2dt);
  auto al = [](size_t x) { return (x + 31) & ~(size_t)31; };  // 256-byte aligned regions
  size_t o = al((size_t)g.Zn * g.ldz);
  g.bz_wq = (int)o; o += al(g.QGpad);
  g.bz_bh = (int)o; o += al((size_t)g.QGpad * g.niprows * g.ntest * 4);
  g.bz_vt = (int)o; o += al((size_t)vrow * 4);
  g.bz_per_cta = o;
  g.big_zk = 32;
  int s = 5 * 64 * 68;  // diagonal block, its inverse, three panel blocks (formation buffers alias them)
  g.bs_sc = s; s += (g.Np + 15) & ~15;
  g.bs_col = s; s += ((g.Np + 1) / 2 + 15) & ~15;
  g.bs_int = s; s += 256;  // 512 ints: flags, chunk point maps, relevance lists
  g.bs_nodes = s; s += 32;
  g.bs_total = s;
  if ((size_t)s * 8 > 232448) return fail(DPG_ERR_UNSUPPORTED, "large-bucket kernel: shared memory exceeded");
  g.sm_total = s;
  return DPG_OK;
}

// Shared-memory layout (doubles) of the single-CTA kernels for Gram chunks of chg points:
// DPG_OK, -1 when it needs more shared memory than one CTA has, or a failure code.
static int smem_layout(DpgPlanDev& g, int chg, bool adj_terms_ok) {
  g.chg = chg;
  auto al = [](int x) { return (x + 15) & ~15; };  // 128-byte aligned regions
  int o = 0;
  // Gram phase
  g.g_fref0 = o; o += al(g.chg * g.featstride);
  g.g_fref1 = o; o += al(g.chg * g.featstride);
  g.g_h = o;
  g.g_beta = o;  // per-point IP rows in reference slots; dead before the first h chunk
  o += al(std::max(g.chg * g.hstride, g.QGpad * g.niprows * 4 * g.ntest));
  g.g_geo = o; o += al(g.QGpad * 24);
  g.g_D = o; o += al(g.QGpad * g.npairs * 16);
  int gphase = o;
  // factor
  o = 0;
  g.sm_gt = o; o += al(g.ngt * 64);
  g.sm_linv = o; o += al(g.NBT * 64);
  g.sm_scale = o; o += al(g.Np);
  int fphase = o;
  // B phase (runs first; whole body available)
  o = 0;
  g.b_rec0 = o; o += al(g.max_chunk * g.max_rec);
  g.b_rec1 = o; o += al(g.max_chunk * g.max_rec);
  g.b_u = o; o += al(g.max_chunk * g.max_ustride);
  g.b_geo = o; o += al(g.nbpts * 24);
  g.b_fac = o; o += al(g.nse * g.QS);
  int bphase = o;
  g.sm_w = 0;
  int wsz = g.MBT * g.NBT * 64;
  g.sm_k = 0;
  int ksz = g.MBT * (g.MBT + 1) / 2 * 64;
  if (g.sm_linv < ksz || g.sm_linv + g.MBT * 64 > g.sm_linv + al(g.NBT * 64))
    return fail(DPG_ERR_UNSUPPORTED, "trial tiles outnumber test tiles: condensation workspace overlaps K");
  int body = std::max(std::max(gphase, bphase), std::max(std::max(wsz, ksz), fphase));
  // reverse mode: S_A, then the pull-back staging (both reuse the body after the factor)
  {
    const int Mx = g.MBT * 8;
    g.a_ldS = ((Mx + 15) & ~15) + 4;  // == 4 mod 16: conflict-free B-fragments
    g.a_sa = 0;
    const int sa_end = Mx * g.a_ldS;
    int fsl = g.featstride;
    if (g.seg[0].nterm > 0) fsl = std::max(fsl, g.seg[0].rec_len);
    int q = 0;
    g.a_fs = q; q += al(DPG_CHA_HOST * fsl);
    g.a_ldx = 2 * Mx;
    g.a_xpf = q; q += al(DPG_CHA_HOST * g.ntest * 4 * g.a_ldx);
    g.a_geo = q; q += al(std::max(DPG_CHA_HOST, g.ns * g.QS) * 24);
    g.a_beta = q; q += al(DPG_CHA_HOST * g.niprows * 4 * g.ntest);
    g.a_cbar = q; q += al(std::max(1, g.nslots * g.Ptot));
    g.adj_ok = adj_terms_ok && std::max(sa_end, q) <= body && g.QB > 0;
  }
  g.sm_coef = al(body);
  g.sm_tiles = g.sm_coef + al(std::max(1, g.nslots * g.Ptot));
  g.sm_nodes = g.sm_tiles + al((g.ngb * (int)sizeof(DpgGTile) + 7) / 8);
  g.sm_invd = g.sm_nodes + 192;
  g.sm_total = g.sm_invd + al(std::max(g.Np, g.Mp));
  if ((size_t)g.sm_total * 8 > 232448) {
    return -1;
  }
  // Gram sums in two levels: after every 32 points the warps' DMMA accumulators of the
  // blocks that several graph-norm terms feed are added into FP64 running sums in the
  // CTA's scratch slot and restart from zero.  A single running sum over all points and
  // terms puts 1.4x more rounding error into K at h = 1/48 (the reference sums each term
  // on its own, IP.cpp:238-244); one flush at half way costs ~2 % of the kernel's time,
  // one every 8 points 17 % (the running sums then cross L2 seven times per cell).
  g.gflush = std::max(1, 32 / g.chg);
  g.gsum_off = (size_t)g.MBT * g.NBT * 64;
  g.scratch_per_cta = g.gsum_off + (size_t)g.ngb * 128;
  return DPG_OK;
}

static int build(HostPlan* P, const dpg_bucket_desc* D) {
  DpgPlanDev& g = P->dev;
  std::memset(&g, 0, sizeof(g));
  TopoData T;
  if (!topo_data(D->topology, T)) return fail(DPG_ERR_INVALID_ARGUMENT, "unknown topology");
  // Only the FP64 form is built.  The split-precision recipes with FP32 accumulation
  // (3-term BF16 or TF32) leave the condensed matrix 1e-3..1 away from the FP64 result at
  // h = 1/48, and the integer-slicing recipe that reaches 1e-10 (six int8 slices, 36 exact
  // slice products) replaces only the Gram quadrature, a third of the kernel's time.
  if (D->precision == DPG_PREC_MIXED)
    return fail(DPG_ERR_UNSUPPORTED, "DPG_PREC_MIXED: no mixed-precision form is built; use DPG_PREC_FP64");
  if (D->precision != DPG_PREC_FP64) return fail(DPG_ERR_INVALID_ARGUMENT, "unknown precision mode");
  const int topo = D->topology;
  if (D->n_test < 1 || D->n_test > DPG_MAXV || D->n_trial < 1 || D->n_trial > DPG_MAXV)
    return fail(DPG_ERR_UNSUPPORTED, "number of test/trial vars out of range (1..16)");
  const int d = T.d;
  g.d = d; g.nv = T.nv; g.ns = T.ns;
  g.nslots = D->n_slots;
  const bool tri = topo == DPG_TOPO_TRI;
  Rule rG = tri ? tri_rule(D->cub_degree_G) : tensor_rule(d, D->cub_degree_G),
       rB = tri ? tri_rule(D->cub_degree_B) : tensor_rule(d, D->cub_degree_B),
       rS = tensor_rule(d - 1, D->cub_degree_side);
  g.QG = rG.n; g.QB = rB.n; g.QS = rS.n;
  if (g.QG > DPG_MAX_QG) return fail(DPG_ERR_UNSUPPORTED, "Gram cubature rule too large");
  auto padc = [](int n, int c) { return (n + c - 1) / c * c; };
  g.QGpad = padc(g.QG, DPG_CHG);
  g.QBpad = padc(g.QB, 8);
  g.QSpad = padc(g.QS, 8);
  g.Ptot = g.QG + g.QB + g.ns * g.QS;
  // side points in the volume reference cell and reference tangents (padded per side)
  std::vector<double> sidepts((size_t)g.ns * g.QSpad * d), sideT((size_t)g.ns * g.QSpad * 6, 0.0);
  for (int s = 0; s < g.ns; s++)
    for (int qq = 0; qq < g.QSpad; qq++) {
      const int q = qq < g.QS ? qq : 0;  // padding repeats point 0 (weight 0)
      double* X = &sidepts[((size_t)s * g.QSpad + qq) * d];
      double* Tq = &sideT[((size_t)s * g.QSpad + qq) * 6];
      if (d == 2) {
        double t = rS.x[q];
        const double* a = T.v[T.sv[s][0]];
        const double* b = T.v[T.sv[s][1]];
        for (int k = 0; k < 2; k++) {
          X[k] = 0.5 * (1 - t) * a[k] + 0.5 * (1 + t) * b[k];
          Tq[k] = 0.5 * (b[k] - a[k]);
        }
      } else {
        double u = rS.x[q * 2], w = rS.x[q * 2 + 1];
        double Nq[4] = {0.25 * (1 - u) * (1 - w), 0.25 * (1 + u) * (1 - w), 0.25 * (1 + u) * (1 + w),
                        0.25 * (1 - u) * (1 + w)};
        double Nu[4] = {-0.25 * (1 - w), 0.25 * (1 - w), 0.25 * (1 + w), -0.25 * (1 + w)};
        double Nw[4] = {-0.25 * (1 - u), -0.25 * (1 + u), 0.25 * (1 + u), 0.25 * (1 - u)};
        for (int k = 0; k < 3; k++) {
          X[k] = 0; Tq[k] = 0; Tq[3 + k] = 0;
          for (int a = 0; a < 4; a++) {
            const double* V = T.v[T.sv[s][a]];
            X[k] += Nq[a] * V[k];
            Tq[k] += Nu[a] * V[k];
            Tq[3 + k] += Nw[a] * V[k];
          }
        }
      }
    }
  // padded volume point lists (padding repeats point 0 with weight 0)
  auto pad_pts = [&](const Rule& r, int npad, std::vector<double>& x, std::vector<double>& w) {
    x.assign((size_t)npad * d, 0.0);
    w.assign(npad, 0.0);
    for (int q = 0; q < npad; q++) {
      int src = q < r.n ? q : 0;
      for (int k = 0; k < d; k++) x[(size_t)q * d + k] = r.x[(size_t)src * d + k];
      w[q] = q < r.n ? r.w[q] : 0.0;
    }
  };
  std::vector<double> xG, wG, xB, wB;
  pad_pts(rG, g.QGpad, xG, wG);
  pad_pts(rB, g.QBpad, xB, wB);
  std::vector<double> wS(g.QSpad, 0.0);
  for (int q = 0; q < g.QS; q++) wS[q] = rS.w[q];
  auto dshape = [&](const std::vector<double>& x, int n) {
    std::vector<double> out((size_t)n * T.nv * d);
    for (int q = 0; q < n; q++) geom_dshape(T, &x[(size_t)q * d], &out[(size_t)q * T.nv * d]);
    return out;
  };

  // ---- test vars ----------------------------------------------------------
  // Large buckets (more than 192 test rows or 120 trial columns after padding) run on the
  // large-bucket kernel, whose tiles need test vars padded to 8 rows only (the single-CTA
  // kernel's 16 x 8 blocks need 16).
  bool big_pre = false;
  {
    int np16 = 0, nf = 0, nt = 0;
    for (int a = 0; a < D->n_test; a++) {
      const dpg_var_desc& V = D->test[a];
      const int c = V.space == DPG_SPACE_HGRAD ? card_hgrad_t(topo, d, V.poly_order)
                                               : card_hdiv_t(topo, d, std::max(V.poly_order, 1));
      np16 += (c + 15) & ~15;
    }
    for (int b = 0; b < D->n_trial; b++) {
      const dpg_var_desc& V = D->trial[b];
      if (V.kind == DPG_VAR_FIELD)
        nf += (V.space == DPG_SPACE_VECTOR_HVOL ? d : 1) * card_hgrad_t(topo, d, std::max(V.poly_order - 1, 0));
      else
        nt += card_hgrad(d - 1, std::max(V.space == DPG_SPACE_HGRAD ? V.poly_order : V.poly_order - 1, 0)) * T.ns;
    }
    big_pre = np16 / 8 > DPG_MAX_NBT || (pad8(nf) + pad8(nt) + 8) / 8 > DPG_MAX_MBT;
  }
  if (big_pre) g.big = 1;
  int dev_row = 0, user_row = 0, foff = 0;
  std::vector<int> test_n(D->n_test);
  for (int a = 0; a < D->n_test; a++) {
    const dpg_var_desc& V = D->test[a];
    DpgTestVar& tv = g.test[a];
    tv.space = V.space;
    int n = V.poly_order;
    test_n[a] = n;
    if (V.space == DPG_SPACE_HGRAD) tv.card = card_hgrad_t(topo, d, n);
    else if (V.space == DPG_SPACE_HDIV) {
      if (n < 1) return fail(DPG_ERR_INVALID_ARGUMENT, "HDIV test order must be >= 1");
      tv.card = card_hdiv_t(topo, d, n);
    } else return fail(DPG_ERR_INVALID_ARGUMENT, "test vars must be HGRAD or HDIV");
    // rows padded to pairs of 8-row tiles (16x8 mma blocks never straddle two vars)
    const int rows = big_pre ? (tv.card + 7) & ~7 : (tv.card + 15) & ~15;
    tv.dev_off = dev_row;
    tv.user_off = user_row;
    tv.ntile0 = dev_row / 8;
    tv.ntiles = rows / 8;
    tv.ldA = ld_pad(rows);
    tv.foff = foff;
    foff += 4 * tv.ldA;
    dev_row += rows;
    user_row += tv.card;
  }
  g.ntest = D->n_test;
  g.featstride = foff;
  g.N = user_row;
  g.Np = dev_row;
  g.NBT = g.Np / 8;
  if (g.NBT > DPG_MAX_NBT) g.big = 1;  // the large-bucket kernel
  // staged reference slots of all test vars at a list of volume-reference points
  auto fref_table = [&](const double* pts, int npts) {
    std::vector<double> out((size_t)npts * g.featstride, 0.0);
    for (int q = 0; q < npts; q++)
      for (int a = 0; a < g.ntest; a++) {
        const DpgTestVar& tv = g.test[a];
        std::vector<double> tmp((size_t)tv.card * (d + 1));
        if (tv.space == DPG_SPACE_HGRAD) tab_hgrad_t(topo, d, test_n[a], pts + (size_t)q * d, tmp.data());
        else tab_hdiv_t(topo, d, test_n[a], pts + (size_t)q * d, tmp.data());
        double* dst = &out[(size_t)q * g.featstride + tv.foff];
        for (int i = 0; i < tv.card; i++)
          for (int m = 0; m <= d; m++) dst[(size_t)m * tv.ldA + i] = tmp[(size_t)i * (d + 1) + m];
      }
    return out;
  };
  g.frefG = upload(P, fref_table(xG.data(), g.QGpad));
  g.wG = upload(P, wG);
  g.dNG = upload(P, dshape(xG, g.QGpad));

  // ---- trial vars -----------------------------------------------------------
  bool seen_trace = false;
  for (int b = 0; b < D->n_trial; b++) {
    if (D->trial[b].kind == DPG_VAR_FIELD) {
      if (seen_trace) return fail(DPG_ERR_UNSUPPORTED, "field vars must precede trace/flux vars");
    } else seen_trace = true;
  }
  int fcount = 0, user_col = 0;
  std::vector<std::vector<double>> host_tabB(D->n_trial), host_tabS(D->n_trial);
  for (int b = 0; b < D->n_trial; b++) {
    const dpg_var_desc& V = D->trial[b];
    DpgTrialVar& tr = g.trial[b];
    tr.kind = V.kind;
    tr.space = V.space;
    if (V.kind == DPG_VAR_FIELD) {
      if (V.space != DPG_SPACE_HVOL && V.space != DPG_SPACE_VECTOR_HVOL)
        return fail(DPG_ERR_INVALID_ARGUMENT, "field vars must be HVOL or VECTOR_HVOL");
      int p = V.poly_order - 1;
      if (p < 0) return fail(DPG_ERR_INVALID_ARGUMENT, "field H1Order must be >= 1");
      tr.ncomp = (V.space == DPG_SPACE_VECTOR_HVOL) ? d : 1;
      tr.card_comp = card_hgrad_t(topo, d, p);
      tr.user_off = user_col;
      tr.dev_off = fcount;
      fcount += tr.ncomp * tr.card_comp;
      user_col += tr.ncomp * tr.card_comp;
      std::vector<double> tb((size_t)g.QBpad * tr.card_comp), ts((size_t)g.ns * g.QSpad * tr.card_comp);
      std::vector<double> tmp((size_t)tr.card_comp * (1 + d));
      for (int q = 0; q < g.QBpad; q++) {
        tab_hgrad_t(topo, d, p, &xB[(size_t)q * d], tmp.data());
        for (int i = 0; i < tr.card_comp; i++) tb[(size_t)q * tr.card_comp + i] = tmp[(size_t)i * (1 + d)];
      }
      for (int q = 0; q < g.ns * g.QSpad; q++) {
        tab_hgrad_t(topo, d, p, &sidepts[(size_t)q * d], tmp.data());
        for (int i = 0; i < tr.card_comp; i++) ts[(size_t)q * tr.card_comp + i] = tmp[(size_t)i * (1 + d)];
      }
      tr.tabB = upload(P, tb);
      tr.tabS = upload(P, ts);
      host_tabB[b] = tb;
      host_tabS[b] = ts;
    } else if (V.kind == DPG_VAR_TRACE || V.kind == DPG_VAR_FLUX) {
      int p = (V.space == DPG_SPACE_HGRAD) ? V.poly_order : V.poly_order - 1;
      if (p < 0) return fail(DPG_ERR_INVALID_ARGUMENT, "trace order must be >= 0");
      tr.ncomp = 1;
      tr.per_side = card_hgrad(d - 1, p);
      tr.card_comp = tr.per_side;
      tr.user_off = user_col;
      user_col += tr.per_side * g.ns;
      std::vector<double> ts((size_t)g.QSpad * tr.per_side), tmp((size_t)tr.per_side * d);
      for (int qq = 0; qq < g.QSpad; qq++) {
        int q = qq < g.QS ? qq : 0;
        tab_hgrad(d - 1, p, &rS.x[(size_t)q * (d - 1)], tmp.data());
        for (int i = 0; i < tr.per_side; i++) ts[(size_t)qq * tr.per_side + i] = tmp[(size_t)i * d];
      }
      tr.tabS = upload(P, ts);
      tr.tabB = nullptr;
      host_tabS[b] = ts;
    } else {
      return fail(DPG_ERR_INVALID_ARGUMENT, "trial var kind must be FIELD, TRACE or FLUX");
    }
  }
  g.ntrial = D->n_trial;
  g.M = user_col;
  g.nf = fcount;
  g.nt = g.M - fcount;
  g.nfp = pad8(g.nf);
  g.ntp = pad8(g.nt);
  g.nfb = g.nfp / 8;
  g.fcol = g.nfp + g.ntp;
  g.Mp = g.fcol + 8;
  g.MBT = g.Mp / 8;
  if (g.MBT > DPG_MAX_MBT) g.big = 1;
  {
    int off = g.nfp;
    for (int b = 0; b < D->n_trial; b++) {
      DpgTrialVar& tr = g.trial[b];
      if (tr.kind == DPG_VAR_FIELD) continue;
      tr.dev_off = off;
      off += tr.per_side * g.ns;
    }
  }
  std::vector<int> d2u_trial(g.Mp, -1), d2u_test(g.Np, -1);
  for (int b = 0; b < D->n_trial; b++) {
    const DpgTrialVar& tr = g.trial[b];
    int cnt = (tr.kind == DPG_VAR_FIELD) ? tr.ncomp * tr.card_comp : tr.per_side * g.ns;
    for (int i = 0; i < cnt; i++) d2u_trial[tr.dev_off + i] = tr.user_off + i;
  }
  for (int a = 0; a < g.ntest; a++)
    for (int i = 0; i < g.test[a].card; i++) d2u_test[g.test[a].dev_off + i] = g.test[a].user_off + i;
  g.dev2user_trial = upload_i(P, d2u_trial);
  g.dev2user_test = upload_i(P, d2u_test);

  // ---- Gram: IP entries on physical slots ----------------------------------
  if (D->n_ip > DPG_MAX_IP) return fail(DPG_ERR_UNSUPPORTED, "too many IP entries");
  std::map<std::pair<int, int>, int> rowid;
  auto phys_slot = [&](int a, int op) -> int {
    const DpgTestVar& tv = g.test[a];
    if (tv.space == DPG_SPACE_HGRAD) {
      if (op == DPG_OP_VALUE) return 0;
      if (op >= DPG_OP_DX && op < DPG_OP_DX + d) return 1 + (op - DPG_OP_DX);
      return -1;
    }
    if (op >= DPG_OP_X && op < DPG_OP_X + d) return op - DPG_OP_X;
    if (op == DPG_OP_DIV) return d;
    return -1;
  };
  for (int e = 0; e < D->n_ip; e++) {
    const dpg_ip_entry& E = D->ip[e];
    if (E.test_var < 0 || E.test_var >= g.ntest) return fail(DPG_ERR_INVALID_ARGUMENT, "IP entry test var out of range");
    int sl = phys_slot(E.test_var, E.test_op);
    if (sl < 0) return fail(DPG_ERR_INVALID_ARGUMENT, "IP op not valid for the test var's space");
    if (E.slot >= D->n_slots) return fail(DPG_ERR_INVALID_ARGUMENT, "IP slot out of range");
    auto key = std::make_pair(E.term, E.comp);
    if (!rowid.count(key)) {
      int r = (int)rowid.size();
      rowid[key] = r;
    }
    DpgIPEnt& I = g.ipent[e];
    I.row = rowid[key];
    I.gslot = E.test_var * 4 + sl;
    I.coef = E.coef;
    I.slot = E.slot;
  }
  g.nipent = D->n_ip;
  std::stable_sort(g.ipent, g.ipent + g.nipent, [](const DpgIPEnt& x, const DpgIPEnt& y) { return x.row < y.row; });
  g.niprows = (int)rowid.size();
  if (g.niprows > DPG_MAX_IPROWS) return fail(DPG_ERR_UNSUPPORTED, "too many IP rows");
  for (int r = 0, e = 0; r <= g.niprows; r++) {
    while (e < g.nipent && g.ipent[e].row < r) e++;
    g.rowstart[r] = e;
  }
  // var pairs (a >= b) that some IP row couples (the others' G blocks are zero), h block offsets
  {
    std::vector<int> coupled(g.ntest * g.ntest, 0);
    for (int r = 0; r < g.niprows; r++)
      for (int e = g.rowstart[r]; e < g.rowstart[r + 1]; e++)
        for (int e2 = g.rowstart[r]; e2 < g.rowstart[r + 1]; e2++)
          coupled[(g.ipent[e].gslot >> 2) * g.ntest + (g.ipent[e2].gslot >> 2)] = 1;
    std::vector<int> pidx(g.ntest * g.ntest, -1);
    // var pairs that two or more graph-norm terms couple (their blocks sum products of
    // very different scales: the ones whose partial sums are flushed)
    std::vector<std::set<int>> terms_of(g.ntest);
    for (int e = 0; e < D->n_ip; e++) terms_of[D->ip[e].test_var].insert(D->ip[e].term);
    auto multi_term = [&](int a, int b) {
      int n = 0;
      for (int t : terms_of[a]) n += (int)terms_of[b].count(t);
      return n >= 2;
    };
    std::vector<char> tile_multi;
    int off = 0, np = 0;
    for (int a = 0; a < g.ntest; a++)
      for (int b = 0; b <= a; b++) {
        if (!coupled[a * g.ntest + b]) continue;
        if (np >= DPG_MAX_PAIRS) return fail(DPG_ERR_UNSUPPORTED, "too many test var pairs");
        g.pair_a[np] = a;
        g.pair_b[np] = b;
        g.hoff[np] = off;
        pidx[a * g.ntest + b] = np;
        off += 4 * g.test[b].ldA;
        np++;
      }
    g.npairs = np;
    g.hstride = off;
    std::vector<DpgGTile> tiles;
    std::vector<char> covered(g.NBT * (g.NBT + 1) / 2, 0);
    // 16 x 8 blocks of the single-CTA kernel (large plans have none: their test vars may
    // have an odd number of 8-row tiles)
    for (int a = 0; a < g.ntest && !g.big; a++)
      for (int rp = 0; rp < g.test[a].ntiles; rp += 2) {
        const int I = g.test[a].ntile0 + rp;
        for (int b = 0; b <= a; b++)
          for (int jj = 0; jj < g.test[b].ntiles; jj++) {
            const int J = g.test[b].ntile0 + jj;
            if (J > I + 1) continue;
            if (pidx[a * g.ntest + b] < 0) continue;
            if (J <= I) covered[I * (I + 1) / 2 + J] = 1;
            covered[(I + 1) * (I + 2) / 2 + J] = 1;
            DpgGTile t;
            t.I = (int16_t)I; t.J = (int16_t)J;
            t.aoff = g.test[a].foff + rp * 8;
            t.lda = (int16_t)g.test[a].ldA;
            t.boff = g.hoff[pidx[a * g.ntest + b]] + jj * 8;
            t.ldb = (int16_t)g.test[b].ldA;
            tiles.push_back(t);
            tile_multi.push_back(multi_term(a, b) ? 1 : 0);
          }
      }
    g.ngb = (int)tiles.size();
    g.ngt = g.NBT * (g.NBT + 1) / 2;
    {  // the kernel's balanced block ownership: warp w owns blocks [tau0, tau0 + ntw)
      const int gbase = g.ngb / DPG_NWARPS, gextra = g.ngb % DPG_NWARPS;
      for (int w = 0; w < DPG_NWARPS; w++) {
        const int ntw = gbase + (w < gextra ? 1 : 0), tau0 = w * gbase + std::min(w, gextra);
        uint32_t bits = 0;
        for (int u = 0; u < ntw && u < 32; u++)
          if (tile_multi[tau0 + u]) bits |= 1u << u;
        g.gflushbits[w] = bits;
      }
    }
    std::vector<int> gz;  // lower tiles no block writes (uncoupled var pairs)
    for (int u = 0; u < g.ngt && !g.big; u++)
      if (!covered[u]) gz.push_back(u);
    g.ngz = (int)gz.size();
    g.gzero = upload_i(P, gz);
    if (!g.big && (g.ngb + DPG_NWARPS - 1) / DPG_NWARPS > DPG_MAX_GT)
      return fail(DPG_ERR_UNSUPPORTED, "too many G blocks");
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(1, tiles.size()) * sizeof(DpgGTile)) != cudaSuccess)
      return fail(DPG_ERR_OUT_OF_MEMORY, "cudaMalloc");
    if (!tiles.empty()) cudaMemcpy(p, tiles.data(), tiles.size() * sizeof(DpgGTile), cudaMemcpyHostToDevice);
    P->allocs.push_back(p);
    g.gtiles = (const DpgGTile*)p;
  }

  // ---- B terms, segments, RHS ----------------------------------------------
  if (D->n_rhs > DPG_MAX_RHS) return fail(DPG_ERR_UNSUPPORTED, "too many RHS terms");
  std::vector<std::pair<int, DpgBTerm>> terms;  // (segment, term)
  std::vector<std::pair<int, DpgBTerm>> sterms; // (side, term): separable boundary terms
  auto separable = [&](int a, int op) {
    if (g.big) return false;  // the large-bucket kernel integrates every side term by quadrature
    const int sp = g.test[a].space;
    return (sp == DPG_SPACE_HGRAD && op == DPG_OP_VALUE) || (sp == DPG_SPACE_HDIV && op == DPG_OP_DOT_NORMAL);
  };
  auto test_op_ok = [&](int a, int op, bool side) {
    if (phys_slot(a, op) >= 0) return true;
    return side && g.test[a].space == DPG_SPACE_HDIV && op == DPG_OP_DOT_NORMAL;
  };
  for (int e = 0; e < D->n_bf; e++) {
    const dpg_bf_term& B = D->bf[e];
    if (B.trial_var < 0 || B.trial_var >= g.ntrial || B.test_var < 0 || B.test_var >= g.ntest)
      return fail(DPG_ERR_INVALID_ARGUMENT, "bf term var index out of range");
    if (B.slot >= D->n_slots) return fail(DPG_ERR_INVALID_ARGUMENT, "bf slot out of range");
    const DpgTrialVar& tr = g.trial[B.trial_var];
    if (!test_op_ok(B.test_var, B.test_op, B.boundary)) return fail(DPG_ERR_INVALID_ARGUMENT, "bf test op invalid");
    if (tr.kind != DPG_VAR_FIELD && !B.boundary) return fail(DPG_ERR_INVALID_ARGUMENT, "trace/flux terms must be boundary terms");
    if (B.normal_comp >= d) return fail(DPG_ERR_INVALID_ARGUMENT, "normal component out of range");
    if ((B.normal_comp >= 0 || B.test_op == DPG_OP_DOT_NORMAL) && !B.boundary)
      return fail(DPG_ERR_INVALID_ARGUMENT, "normal-dependent terms must be boundary terms");
    int comp = 0;
    if (tr.kind == DPG_VAR_FIELD) {
      if (tr.ncomp > 1) {
        if (B.trial_op < DPG_OP_X || B.trial_op >= DPG_OP_X + d) return fail(DPG_ERR_INVALID_ARGUMENT, "vector field needs op X/Y/Z");
        comp = B.trial_op - DPG_OP_X;
      } else if (B.trial_op != DPG_OP_VALUE) return fail(DPG_ERR_INVALID_ARGUMENT, "scalar field needs op VALUE");
    }
    int nseg = B.boundary ? g.ns : 1;
    for (int sg = 0; sg < nseg; sg++) {
      DpgBTerm t;
      std::memset(&t, 0, sizeof(t));
      t.trial_var = B.trial_var; t.test_var = B.test_var; t.test_op = B.test_op;
      t.coef = B.coef; t.slot = B.slot; t.normal_comp = B.normal_comp;
      t.kind = tr.kind;
      if (tr.kind == DPG_VAR_FIELD) { t.col0 = tr.dev_off + comp * tr.card_comp; t.ncol = tr.card_comp; }
      else { t.col0 = tr.dev_off + sg * tr.per_side; t.ncol = tr.per_side; }
      if (B.boundary && separable(B.test_var, B.test_op)) sterms.push_back({sg, t});
      else terms.push_back({B.boundary ? 1 + sg : 0, t});
    }
  }
  for (int e = 0; e < D->n_rhs; e++) {
    const dpg_rhs_term& R = D->rhs[e];
    if (R.test_var < 0 || R.test_var >= g.ntest || !test_op_ok(R.test_var, R.test_op, false))
      return fail(DPG_ERR_INVALID_ARGUMENT, "rhs term invalid");
    if (R.slot >= D->n_slots) return fail(DPG_ERR_INVALID_ARGUMENT, "rhs slot out of range");
    DpgBTerm t;
    std::memset(&t, 0, sizeof(t));
    t.trial_var = -1; t.test_var = R.test_var; t.test_op = R.test_op;
    t.coef = R.coef; t.slot = R.slot; t.normal_comp = -1; t.kind = -1;
    t.col0 = g.fcol; t.ncol = 1;
    terms.push_back({0, t});
  }
  std::stable_sort(terms.begin(), terms.end(),
                   [](const std::pair<int, DpgBTerm>& x, const std::pair<int, DpgBTerm>& y) { return x.first < y.first; });
  if ((int)terms.size() > DPG_MAX_BF) return fail(DPG_ERR_UNSUPPORTED, "too many expanded bilinear terms");
  g.nbterm = (int)terms.size();
  for (int i = 0; i < g.nbterm; i++) g.bterm[i] = terms[i].second;
  g.nseg = 1 + g.ns;
  // all B points: volume (QB) then each side (QS); geometry tables for them
  g.nbpts = g.QB + g.ns * g.QS;
  {
    std::vector<double> xall((size_t)g.nbpts * d), wall(g.nbpts), tall((size_t)g.nbpts * 6, 0.0);
    for (int q = 0; q < g.QB; q++) {
      for (int k = 0; k < d; k++) xall[(size_t)q * d + k] = rB.x[(size_t)q * d + k];
      wall[q] = rB.w[q];
    }
    for (int s2 = 0; s2 < g.ns; s2++)
      for (int q = 0; q < g.QS; q++) {
        int o = g.QB + s2 * g.QS + q;
        for (int k = 0; k < d; k++) xall[(size_t)o * d + k] = sidepts[((size_t)s2 * g.QSpad + q) * d + k];
        for (int k = 0; k < 6; k++) tall[(size_t)o * 6 + k] = sideT[((size_t)s2 * g.QSpad + q) * 6 + k];
        wall[o] = rS.w[q];
      }
    g.dNB = upload(P, dshape(xall, g.nbpts));
    g.wB = upload(P, wall);
    g.tangB = upload(P, tall);
  }
  // shared-memory budget for the B phase: two record buffers, U, geometry of all
  // B points, per-point term rows R, coefficients
  const int budget = 232448 / 8 - 192 - 2 * ((g.ngb * (int)sizeof(DpgGTile) + 7) / 8) - 64 - g.Np - g.Mp - 64;
  g.max_rec = 0; g.max_chunk = 0; g.max_ustride = 0; g.max_nterm = 0;
  std::vector<int4> btiles;
  for (int sg = 0; sg < g.nseg; sg++) {
    DpgSeg& S = g.seg[sg];
    S.side = sg - 1;
    S.npts = sg == 0 ? g.QB : g.QS;
    S.pbase = sg == 0 ? g.QG : g.QG + g.QB + (sg - 1) * g.QS;
    S.geo0 = sg == 0 ? 0 : g.QB + (sg - 1) * g.QS;
    S.term0 = -1;
    S.nterm = 0;
    S.nblk = 0;
    int off = 0, tv = g.featstride;
    for (int i = 0; i < g.nbterm; i++) {
      if (terms[i].first != sg) continue;
      if (S.term0 < 0) S.term0 = i;
      int lt = S.nterm++;
      if (lt >= DPG_MAX_BF / 4) return fail(DPG_ERR_UNSUPPORTED, "too many terms in one segment");
      const DpgBTerm& t = g.bterm[i];
      S.tvoff[lt] = tv;
      tv += t.ncol;
      for (int J = t.col0 / 8; !g.big && J <= (t.col0 + t.ncol - 1) / 8; J++) {
        int k = -1;
        for (int kk = 0; kk < S.nblk; kk++)
          if (S.blk[kk].var == t.test_var && S.blk[kk].J == J) k = kk;
        if (k < 0) {
          if (S.nblk >= DPG_MAX_BLK) return fail(DPG_ERR_UNSUPPORTED, "too many active B blocks in a segment");
          k = S.nblk++;
          S.blk[k].var = t.test_var;
          S.blk[k].J = J;
          S.blk[k].off = off;
          S.blk[k].nt = 0;
          off += 4 * DPG_ULD;
        }
        if (S.blk[k].nt >= DPG_MAX_BT) return fail(DPG_ERR_UNSUPPORTED, "too many terms feeding one B block");
        S.blk[k].terms[S.blk[k].nt++] = lt;
      }
    }
    if (S.term0 < 0) S.term0 = 0;
    S.ustride = off;
    S.rec_len = (tv + 1) & ~1;
    S.tile0 = (int)btiles.size();
    // 16x8 blocks (row-tile pairs of the block's test var) of the active (var, column tile) blocks
    for (int kb = 0; kb < S.nblk; kb++) {
      const DpgTestVar& V = g.test[S.blk[kb].var];
      for (int I = V.ntile0; I < V.ntile0 + V.ntiles; I += 2) btiles.push_back(make_int4(I, S.blk[kb].J, kb, 0));
    }
    S.ntile = (int)btiles.size() - S.tile0;
    if (!g.big && (S.ntile + DPG_NWARPS - 1) / DPG_NWARPS > DPG_MAX_BTW)
      return fail(DPG_ERR_UNSUPPORTED, "too many active B blocks in a segment");
    if (S.nterm == 0) continue;
    g.max_rec = std::max(g.max_rec, S.rec_len);
    g.max_ustride = std::max(g.max_ustride, S.ustride);
    g.max_nterm = std::max(g.max_nterm, S.nterm);
  }
  {
    void* p = nullptr;
    size_t nb = std::max<size_t>(1, btiles.size()) * sizeof(int4);
    if (cudaMalloc(&p, nb) != cudaSuccess) return fail(DPG_ERR_OUT_OF_MEMORY, "cudaMalloc");
    if (!btiles.empty()) cudaMemcpy(p, btiles.data(), btiles.size() * sizeof(int4), cudaMemcpyHostToDevice);
    P->allocs.push_back(p);
    g.btiles = (const int4*)p;
  }
  // chunk size: all points of a side in one chunk when it fits; the volume in equal chunks
  {
    auto fits = [&](int ch) {
      int need = 2 * ch * g.max_rec + ch * g.max_ustride + g.nbpts * 24 + g.nslots * g.Ptot + 64 +
                 (int)sterms.size() * g.QS + 16;
      return need <= budget;
    };
    // chunks are multiples of 4 points (one m16n8k16 k-step = 4 points x 4 slots)
    int ch = DPG_MAX_CHB;
    while (ch > 4 && !fits(ch)) ch -= 4;
    if (g.big) ch = 1 << 20;  // no staging: one chunk per segment
    else if (!fits(ch)) return fail(DPG_ERR_UNSUPPORTED, "B-phase staging does not fit in shared memory");
    for (int sg = 0; sg < g.nseg; sg++) {
      DpgSeg& S = g.seg[sg];
      if (S.nterm == 0) continue;
      S.chunk = std::min(ch, (S.npts + 3) & ~3);
      S.nchunk = (S.npts + S.chunk - 1) / S.chunk;  // the last chunk may be short
      g.max_chunk = std::max(g.max_chunk, S.chunk);
    }
  }
  // per-segment point records: reference slots of every test var, then each term's trial values
  for (int sg = 0; sg < g.nseg; sg++) {
    DpgSeg& S = g.seg[sg];
    if (S.nterm == 0) continue;
    const int npad = S.nchunk * S.chunk;
    std::vector<double> xs((size_t)npad * d, 0.0);
    for (int q = 0; q < npad; q++) {
      int src = q < S.npts ? q : 0;
      for (int k = 0; k < d; k++)
        xs[(size_t)q * d + k] = (sg == 0) ? rB.x[(size_t)src * d + k]
                                          : sidepts[((size_t)(sg - 1) * g.QSpad + src) * d + k];
    }
    std::vector<double> slots = fref_table(xs.data(), npad);
    std::vector<double> rec((size_t)npad * S.rec_len, 0.0);
    for (int q = 0; q < npad; q++) {
      std::copy(slots.begin() + (size_t)q * g.featstride, slots.begin() + (size_t)(q + 1) * g.featstride,
                rec.begin() + (size_t)q * S.rec_len);
      if (q >= S.npts) continue;
      for (int lt = 0; lt < S.nterm; lt++) {
        const DpgBTerm& t = g.bterm[S.term0 + lt];
        double* dst = &rec[(size_t)q * S.rec_len + S.tvoff[lt]];
        if (t.kind < 0) { dst[0] = 1.0; continue; }
        const DpgTrialVar& tr = g.trial[t.trial_var];
        for (int m = 0; m < t.ncol; m++) {
          if (t.kind == DPG_VAR_FIELD)
            dst[m] = (sg == 0) ? host_tabB[t.trial_var][(size_t)q * tr.card_comp + m]
                               : host_tabS[t.trial_var][((size_t)(sg - 1) * g.QSpad + q) * tr.card_comp + m];
          else
            dst[m] = host_tabS[t.trial_var][(size_t)q * tr.per_side + m];
        }
      }
    }
    S.rec = upload(P, rec);
  }

  // separable side terms -> entries (row, col) with per-point weights
  if (sterms.size() > 0) {
    std::vector<double> sidex((size_t)g.QS * d);
    std::vector<DpgSideTerm> ses;
    std::map<std::pair<int, int>, std::vector<std::pair<int, std::vector<double>>>> ent;  // (row, col) -> (se, W[q])
    for (size_t e = 0; e < sterms.size(); e++) {
      const int sd = sterms[e].first;
      const DpgBTerm& t = sterms[e].second;
      const DpgTestVar& V = g.test[t.test_var];
      const bool normal_trace = V.space == DPG_SPACE_HDIV && t.test_op == DPG_OP_DOT_NORMAL;
      DpgSideTerm st;
      st.side = sd;
      st.pbase = g.QG + g.QB + sd * g.QS;
      st.slot = t.slot;
      st.normal_comp = t.normal_comp;
      st.flux = t.kind == DPG_VAR_FLUX;
      st.use_meas = normal_trace ? 0 : 1;
      st.coef = t.coef;
      const int se = (int)ses.size();
      ses.push_back(st);
      for (int q = 0; q < g.QS; q++)
        for (int k = 0; k < d; k++) sidex[(size_t)q * d + k] = sidepts[((size_t)sd * g.QSpad + q) * d + k];
      std::vector<double> sl = fref_table(sidex.data(), g.QS);
      // reference side values of the test operator: T[q][r]
      std::vector<double> T((size_t)g.QS * V.card, 0.0);
      double tmax = 0.0;
      for (int q = 0; q < g.QS; q++) {
        const double* f = &sl[(size_t)q * g.featstride + V.foff];
        double c[3] = {0.0, 0.0, 0.0};
        if (normal_trace) {
          const double* tq = &sideT[((size_t)sd * g.QSpad + q) * 6];
          if (d == 2) { c[0] = tq[1]; c[1] = -tq[0]; }
          else {
            c[0] = tq[1] * tq[5] - tq[2] * tq[4];
            c[1] = tq[2] * tq[3] - tq[0] * tq[5];
            c[2] = tq[0] * tq[4] - tq[1] * tq[3];
          }
        }
        for (int r = 0; r < V.card; r++) {
          double v;
          if (normal_trace) {
            v = 0.0;
            for (int k = 0; k < d; k++) v += c[k] * f[k * V.ldA + r];
            v *= rS.w[q];
          } else {
            v = f[r];
          }
          T[(size_t)q * V.card + r] = v;
          tmax = std::max(tmax, std::fabs(v));
        }
      }
      const DpgTrialVar& tr = g.trial[t.trial_var];
      for (int r = 0; r < V.card; r++) {
        double rmax = 0.0;
        for (int q = 0; q < g.QS; q++) rmax = std::max(rmax, std::fabs(T[(size_t)q * V.card + r]));
        if (!(rmax > 1e-14 * tmax)) continue;  // zero on this side (to roundoff)
        for (int m = 0; m < t.ncol; m++) {
          std::vector<double> W(g.QS);
          for (int q = 0; q < g.QS; q++) {
            double tv = (t.kind == DPG_VAR_FIELD) ? host_tabS[t.trial_var][((size_t)sd * g.QSpad + q) * tr.card_comp + m]
                                                  : host_tabS[t.trial_var][(size_t)q * tr.per_side + m];
            W[q] = T[(size_t)q * V.card + r] * tv;
          }
          ent[{V.dev_off + r, t.col0 + m}].push_back({se, W});
        }
      }
    }
    // entries: (scratch element, first contribution, count, side term of the first |
    // 1 << 16 when no bilinear block writes the element's column tile, so a store suffices)
    std::vector<char> blk_col(g.MBT + 1, 0);
    for (int sg = 0; sg < g.nseg; sg++)
      for (int kb = 0; kb < g.seg[sg].nblk; kb++) blk_col[g.seg[sg].blk[kb].J] = 1;
    std::vector<int4> sent;
    std::vector<int> scon_se;
    std::vector<int2> rc;
    std::vector<std::vector<double>> wl;
    for (auto& kv : ent) {
      const int row = kv.first.first, col = kv.first.second;
      const int idx = (((col >> 3) * g.NBT + (row >> 3)) * 32 + (row & 7) * 4 + ((col & 7) >> 1)) * 2 + (col & 1);
      const int store = blk_col[col >> 3] ? 0 : 1;
      sent.push_back(make_int4(idx, (int)scon_se.size(), (int)kv.second.size(), kv.second[0].first | (store << 16)));
      for (auto& c : kv.second) {
        scon_se.push_back(c.first);
        wl.push_back(c.second);
        rc.push_back(make_int2(row, col));
      }
    }
    g.nse = (int)ses.size();
    g.nsent = (int)sent.size();
    g.ncon = (int)scon_se.size();
    std::vector<double> wq((size_t)g.QS * g.ncon);
    for (int c = 0; c < g.ncon; c++)
      for (int q = 0; q < g.QS; q++) wq[(size_t)q * g.ncon + c] = wl[c][q];
    void* p = nullptr;
    if (cudaMalloc(&p, ses.size() * sizeof(DpgSideTerm)) != cudaSuccess) return fail(DPG_ERR_OUT_OF_MEMORY, "cudaMalloc");
    cudaMemcpy(p, ses.data(), ses.size() * sizeof(DpgSideTerm), cudaMemcpyHostToDevice);
    P->allocs.push_back(p);
    g.se = (const DpgSideTerm*)p;
    p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(1, sent.size()) * sizeof(int4)) != cudaSuccess)
      return fail(DPG_ERR_OUT_OF_MEMORY, "cudaMalloc");
    if (!sent.empty()) cudaMemcpy(p, sent.data(), sent.size() * sizeof(int4), cudaMemcpyHostToDevice);
    P->allocs.push_back(p);
    g.sent = (const int4*)p;
    g.scon_se = upload_i(P, scon_se);
    g.scon_w = upload(P, wq);
    // reverse mode: contributions grouped by side term, with their (row, col)
    std::vector<int> sstart(g.nse + 1, 0), scon;
    for (int se = 0; se < g.nse; se++) {
      sstart[se] = (int)scon.size();
      for (int c = 0; c < g.ncon; c++)
        if (scon_se[c] == se) scon.push_back(c);
    }
    sstart[g.nse] = (int)scon.size();
    g.sadj_start = upload_i(P, sstart);
    g.sadj_con = upload_i(P, scon);
    p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(1, rc.size()) * sizeof(int2)) != cudaSuccess)
      return fail(DPG_ERR_OUT_OF_MEMORY, "cudaMalloc");
    if (!rc.empty()) cudaMemcpy(p, rc.data(), rc.size() * sizeof(int2), cudaMemcpyHostToDevice);
    P->allocs.push_back(p);
    g.scon_rc = (const int2*)p;
    for (const DpgSideTerm& st : ses) g.se_slots |= st.slot >= 0;
  }
  // coefficient uses the reverse mode covers: IP entries, volume B and load terms,
  // separable side terms
  for (int e = 0; e < g.nipent; e++) g.ip_slots |= g.ipent[e].slot >= 0;
  bool adj_terms_ok = true;
  for (int sg = 0; sg < g.nseg; sg++)
    for (int lt = 0; lt < g.seg[sg].nterm; lt++) {
      const DpgBTerm& t = g.bterm[g.seg[sg].term0 + lt];
      if (t.slot < 0) continue;
      if (sg == 0) g.b_slots = 1;
      else adj_terms_ok = false;  // a non-separable side term with a coefficient
    }

  if (g.big) {
    int rc = big_layout(P);
    if (rc != DPG_OK) return rc;
  }
  // ---- shared memory layout (doubles) ----------------------------------------
  if (!g.big) {
    int rc = smem_layout(g, DPG_CHG, adj_terms_ok);
    if (rc == -1) rc = smem_layout(g, DPG_CHG / 2, adj_terms_ok);  // half-size Gram chunks
    if (rc == -1) return fail(DPG_ERR_UNSUPPORTED, "bucket needs more shared memory than one CTA has");
    if (rc != DPG_OK) return rc;
  }
  P->adj_terms_ok = adj_terms_ok;
  // info
  dpg_plan_info& I = P->info;
  I.N = g.N; I.M = g.M; I.n_field = g.nf; I.n_trace = g.nt;
  I.space_dim = d; I.n_vertices = T.nv; I.n_sides = T.ns;
  I.Q_G = g.QG; I.Q_B = g.QB; I.Q_side = g.QS; I.n_points_total = g.Ptot;
  I.n_slots = g.nslots; I.precision = D->precision;
  void* p = nullptr;
  if (cudaMalloc(&p, sizeof(DpgPlanDev)) != cudaSuccess) return fail(DPG_ERR_OUT_OF_MEMORY, "cudaMalloc plan");
  cudaMemcpy(p, &g, sizeof(DpgPlanDev), cudaMemcpyHostToDevice);
  P->allocs.push_back(p);
  P->d_dev = (DpgPlanDev*)p;
  for (void* a : P->allocs)
    if (!a) return fail(DPG_ERR_OUT_OF_MEMORY, "device table allocation failed");
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return fail(DPG_ERR_CUDA, std::string("plan upload: ") + cudaGetErrorString(err));
  return DPG_OK;
}

}  // namespace dpg

// Plan of the bare optimal-test solve (TBF::factoredCholeskySolve): one test
// block of N rows, M trial columns treated as fields (no condensation).
int dpg_make_solve_plan(int N, int M, DpgPlanDev* out) {
  DpgPlanDev& g = *out;
  std::memset(&g, 0, sizeof(g));
  auto pad8 = [](int n) { return (n + 7) & ~7; };
  auto al = [](int x) { return (x + 15) & ~15; };
  g.d = 2; g.nv = 0; g.ns = 0;
  g.N = N; g.M = M; g.nf = M; g.nt = 0;
  g.Np = pad8(N); g.NBT = g.Np / 8;
  g.nfp = pad8(M); g.ntp = 0; g.nfb = g.nfp / 8; g.fcol = g.nfp; g.Mp = g.nfp + 8; g.MBT = g.Mp / 8;
  if (g.NBT > DPG_MAX_NBT) return dpg::fail(DPG_ERR_UNSUPPORTED, "N too large for the single-CTA solve (N <= 192)");
  if (g.MBT > DPG_MAX_MBT) return dpg::fail(DPG_ERR_UNSUPPORTED, "M too large for the single-CTA solve (M <= 120)");
  g.ntest = 1;
  g.test[0].card = N; g.test[0].ntiles = g.NBT;
  g.ntrial = 1;
  g.trial[0].kind = DPG_VAR_FIELD; g.trial[0].ncomp = 1; g.trial[0].card_comp = M;
  g.ngt = g.NBT * (g.NBT + 1) / 2;
  g.sm_gt = 0;
  g.sm_linv = al(g.ngt * 64);
  g.sm_scale = g.sm_linv + al(g.NBT * 64);
  int a = g.sm_scale + al(g.Np);
  int w = g.MBT * g.NBT * 64, k = g.MBT * (g.MBT + 1) / 2 * 64;
  g.sm_w = 0; g.sm_k = 0;
  g.sm_coef = al(std::max(a, std::max(w, k)));
  g.sm_tiles = g.sm_coef;
  g.sm_nodes = g.sm_tiles;
  g.scratch_per_cta = 0;
  g.chg = DPG_CHG;  // no Gram phase; selects the standard kernel instances
  g.sm_invd = g.sm_nodes + 192;
  g.sm_total = g.sm_invd + al(std::max(g.Np, g.Mp));
  return DPG_OK;
}

// Host-buffer pipeline: cells go through device memory in chunks on two
// streams so that the copies of one chunk overlap the kernel of the other.
int dpg_host_pipeline(const DpgPlanDev* plan, const DpgPlanDev* d_plan, void** d_ws, size_t* ws_bytes,
                      cudaStream_t* streams, int C, const double* nodes, const int8_t* parity, const double* coeff,
                      double* K, double* l, double* S, double* s, int32_t* info, int flags) {
  const DpgPlanDev& g = *plan;
  if (C < 0) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "negative cell count");
  if (C == 0) return DPG_OK;
  if (!nodes || !parity || !info) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "nodes, parity and info are required");
  if (g.nslots > 0 && !coeff) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "coefficients required by this plan");
  bool wantK = !(flags & DPG_FLAG_NO_K), wantS = !(flags & DPG_FLAG_NO_CONDENSE);
  if (wantK && (!K || !l)) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "K and l required");
  if (wantS && (!S || !s)) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "S and s required");
  const size_t nb_nodes = (size_t)g.nv * g.d * 8, nb_par = (size_t)g.ns, nb_co = (size_t)g.nslots * g.Ptot * 8;
  const size_t nb_K = wantK ? (size_t)g.M * g.M * 8 : 0, nb_l = wantK ? (size_t)g.M * 8 : 0;
  const size_t nb_S = wantS ? (size_t)g.nt * g.nt * 8 : 0, nb_s = wantS ? (size_t)g.nt * 8 : 0;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const int chunk = std::min(C, 4096);
  const size_t per_buf = al(chunk * nb_nodes) + al(chunk * nb_par) + al(chunk * nb_co) + al(chunk * nb_K) +
                         al(chunk * nb_l) + al(chunk * nb_S) + al(chunk * nb_s) + al(chunk * 4);
  if (*ws_bytes < 2 * per_buf) {
    if (*d_ws) cudaFree(*d_ws);
    *d_ws = nullptr;
    *ws_bytes = 0;
    if (cudaMalloc(d_ws, 2 * per_buf) != cudaSuccess) {
      cudaGetLastError();
      return dpg::fail(DPG_ERR_OUT_OF_MEMORY, "workspace allocation failed");
    }
    *ws_bytes = 2 * per_buf;
  }
  for (int i = 0; i < 2; i++)
    if (!streams[i] && cudaStreamCreateWithFlags(&streams[i], cudaStreamNonBlocking) != cudaSuccess)
      return dpg::fail(DPG_ERR_CUDA, "stream creation failed");
  for (int c0 = 0, it = 0; c0 < C; c0 += chunk, it++) {
    const int n = std::min(chunk, C - c0);
    const int b = it & 1;
    cudaStream_t st = streams[b];
    char* base = (char*)*d_ws + b * per_buf;
    double* dn = (double*)base; base += al(chunk * nb_nodes);
    int8_t* dp = (int8_t*)base; base += al(chunk * nb_par);
    double* dc = (double*)base; base += al(chunk * nb_co);
    double* dK = (double*)base; base += al(chunk * nb_K);
    double* dl = (double*)base; base += al(chunk * nb_l);
    double* dS = (double*)base; base += al(chunk * nb_S);
    double* ds = (double*)base; base += al(chunk * nb_s);
    int32_t* di = (int32_t*)base;
    cudaMemcpyAsync(dn, (const char*)nodes + c0 * nb_nodes, n * nb_nodes, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dp, parity + (size_t)c0 * g.ns, n * nb_par, cudaMemcpyHostToDevice, st);
    if (nb_co) cudaMemcpyAsync(dc, (const char*)coeff + c0 * nb_co, n * nb_co, cudaMemcpyHostToDevice, st);
    DpgLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.C = n; L.nodes = dn; L.parity = dp; L.coeff = nb_co ? dc : nullptr;
    L.K = wantK ? dK : nullptr; L.l = wantK ? dl : nullptr;
    L.S = wantS ? dS : nullptr; L.s = wantS ? ds : nullptr;
    L.info = di;
    int rc = dpg_launch_assemble(plan, d_plan, &L, st);
    if (rc != DPG_OK) return rc;
    if (wantK) {
      cudaMemcpyAsync((char*)K + c0 * nb_K, dK, n * nb_K, cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync((char*)l + c0 * nb_l, dl, n * nb_l, cudaMemcpyDeviceToHost, st);
    }
    if (wantS) {
      cudaMemcpyAsync((char*)S + c0 * nb_S, dS, n * nb_S, cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync((char*)s + c0 * nb_s, ds, n * nb_s, cudaMemcpyDeviceToHost, st);
    }
    cudaMemcpyAsync(info + c0, di, n * 4, cudaMemcpyDeviceToHost, st);
  }
  cudaError_t e1 = cudaStreamSynchronize(streams[0]);
  cudaError_t e2 = cudaStreamSynchronize(streams[1]);
  if (e1 != cudaSuccess || e2 != cudaSuccess)
    return dpg::fail(DPG_ERR_CUDA, std::string("host pipeline: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
  return DPG_OK;
}

// ============================================================================
// C ABI
// ============================================================================

using namespace dpg;

struct dpg_plan {
  HostPlan hp;
};

extern "C" {

const char* dpg_last_error_string(void) { return g_last_error.c_str(); }

const char* dpg_version(void) { return "camellia2_b200 dpg 1 (sm_100a, FP64 DMMA)"; }

int dpg_basis_tabulate(int topology, int space, int n, int npts, const double* pts, double* out) {
  TopoData T;
  if (!topo_data(topology, T)) return -fail(DPG_ERR_INVALID_ARGUMENT, "unknown topology");
  if (npts < 0 || (npts > 0 && (!pts || !out))) return -fail(DPG_ERR_INVALID_ARGUMENT, "null argument");
  const int dim = T.d;
  int card;
  if (space == DPG_SPACE_HGRAD) {
    if (n < 0) return -fail(DPG_ERR_INVALID_ARGUMENT, "HGRAD order must be >= 0");
    card = card_hgrad_t(topology, dim, n);
  } else if (space == DPG_SPACE_HDIV) {
    if (n < 1) return -fail(DPG_ERR_INVALID_ARGUMENT, "HDIV order must be >= 1");
    card = card_hdiv_t(topology, dim, n);
  } else {
    return -fail(DPG_ERR_INVALID_ARGUMENT, "space must be HGRAD or HDIV");
  }
  std::vector<double> buf((size_t)card * (dim + 1));
  for (int q = 0; q < npts; q++) {
    if (space == DPG_SPACE_HGRAD) tab_hgrad_t(topology, dim, n, pts + (size_t)q * dim, buf.data());
    else tab_hdiv_t(topology, dim, n, pts + (size_t)q * dim, buf.data());
    std::copy(buf.begin(), buf.end(), out + (size_t)q * card * (dim + 1));
  }
  return card;
}

int dpg_cubature(int topology, int degree, double* pts, double* wts) {
  TopoData T;
  if (!topo_data(topology, T)) return -fail(DPG_ERR_INVALID_ARGUMENT, "unknown topology");
  if (degree < 0) return -fail(DPG_ERR_INVALID_ARGUMENT, "degree must be >= 0");
  const Rule r = topology == DPG_TOPO_TRI ? tri_rule(degree) : tensor_rule(T.d, degree);
  if (pts) std::copy(r.x.begin(), r.x.end(), pts);
  if (wts) std::copy(r.w.begin(), r.w.end(), wts);
  return r.n;
}

int dpg_plan_create(const dpg_bucket_desc* desc, dpg_plan** out) {
  if (!desc || !out) return fail(DPG_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (desc->abi_version != DPG_ABI_VERSION) return fail(DPG_ERR_INVALID_ARGUMENT, "ABI version mismatch");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(DPG_ERR_CUDA, "no CUDA device available");
  }
  dpg_plan* p = new dpg_plan();
  p->hp.desc = *desc;
  cudaGetDevice(&p->hp.device);
  int rc = build(&p->hp, desc);
  if (rc != DPG_OK) {
    std::string msg = g_last_error;
    dpg_plan_destroy(p);
    g_last_error = msg;
    return rc;
  }
  rc = dpg_configure_kernels(&p->hp.dev);
  if (rc != DPG_OK) {
    std::string msg = g_last_error;
    dpg_plan_destroy(p);
    g_last_error = msg;
    return rc;
  }
  *out = p;
  return DPG_OK;
}

int dpg_plan_destroy(dpg_plan* p) {
  if (!p) return DPG_OK;
  for (void* a : p->hp.allocs)
    if (a) cudaFree(a);
  if (p->hp.d_ws) cudaFree(p->hp.d_ws);
  for (auto& s : p->hp.streams)
    if (s) cudaStreamDestroy(s);
  delete p;
  return DPG_OK;
}

int dpg_plan_query(const dpg_plan* p, dpg_plan_info* info) {
  if (!p || !info) return fail(DPG_ERR_INVALID_ARGUMENT, "null argument");
  *info = p->hp.info;
  return DPG_OK;
}

int dpg_assemble(dpg_plan* p, int C, const double* nodes, const int8_t* parity, const double* coeff, double* K,
                 double* l, double* S, double* s, int32_t* info, void* stream, int flags) {
  if (!p) return fail(DPG_ERR_BAD_PLAN, "null plan");
  if (C < 0) return fail(DPG_ERR_INVALID_ARGUMENT, "negative cell count");
  if (C == 0) return DPG_OK;
  if (!nodes || !parity || !info) return fail(DPG_ERR_INVALID_ARGUMENT, "nodes, parity and info are required");
  if (p->hp.dev.nslots > 0 && !coeff) return fail(DPG_ERR_INVALID_ARGUMENT, "coefficients required by this plan");
  if (!(flags & DPG_FLAG_NO_K) && (!K || !l)) return fail(DPG_ERR_INVALID_ARGUMENT, "K and l required");
  if (!(flags & DPG_FLAG_NO_CONDENSE) && (!S || !s)) return fail(DPG_ERR_INVALID_ARGUMENT, "S and s required");
  DpgLaunch L;
  std::memset(&L, 0, sizeof(L));
  L.C = C; L.nodes = nodes; L.parity = parity; L.coeff = coeff;
  L.K = (flags & DPG_FLAG_NO_K) ? nullptr : K;
  L.l = (flags & DPG_FLAG_NO_K) ? nullptr : l;
  L.S = (flags & DPG_FLAG_NO_CONDENSE) ? nullptr : S;
  L.s = (flags & DPG_FLAG_NO_CONDENSE) ? nullptr : s;
  L.info = info;
  return dpg_launch_assemble(&p->hp.dev, p->hp.d_dev, &L, (cudaStream_t)stream);
}

int dpg_plan_autotune(dpg_plan* p, int C, const double* nodes, const int8_t* parity, const double* coeff, void* stream,
                      int* chosen) {
  if (!p) return fail(DPG_ERR_BAD_PLAN, "null plan");
  if (!chosen) return fail(DPG_ERR_INVALID_ARGUMENT, "null output");
  *chosen = 0;
  if (C <= 0 || !nodes || !parity) return fail(DPG_ERR_INVALID_ARGUMENT, "cells, nodes and parity are required");
  if (p->hp.dev.nslots > 0 && !coeff) return fail(DPG_ERR_INVALID_ARGUMENT, "coefficients required by this plan");
  cudaStream_t st = (cudaStream_t)stream;
  const DpgPlanDev& g0 = p->hp.dev;
  const size_t nK = (size_t)C * g0.M * g0.M, nl = (size_t)C * g0.M, nS = (size_t)C * g0.nt * g0.nt, ns = (size_t)C * g0.nt;
  void* out = nullptr;
  if (dpg::ws_alloc(&out, (nK + nl + nS + ns) * sizeof(double) + (size_t)C * 4, st) != cudaSuccess) {
    cudaGetLastError();
    return fail(DPG_ERR_OUT_OF_MEMORY, "autotune outputs");
  }
  DpgLaunch L;
  std::memset(&L, 0, sizeof(L));
  L.C = C; L.nodes = nodes; L.parity = parity; L.coeff = coeff;
  L.K = (double*)out; L.l = L.K + nK; L.S = L.l + nl; L.s = L.S + nS; L.info = (int32_t*)(L.s + ns);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = -1.0f;
  DpgPlanDev best_plan = g0;
  int rc = DPG_OK;
  // candidates: single-CTA plans, the Gram staging chunk (8 or 4 points: the shared-memory
  // layout and the kernel instance); large plans, the formation k-chunk (32 or 16 points)
  for (int cnd = 0; cnd < 2 && rc == DPG_OK; cnd++) {
    DpgPlanDev cand = g0;
    if (g0.big) cand.big_zk = cnd == 0 ? 32 : 16;
    else if (smem_layout(cand, cnd == 0 ? DPG_CHG : DPG_CHG / 2, p->hp.adj_terms_ok) != DPG_OK) continue;
    if ((rc = dpg_configure_kernels(&cand)) != DPG_OK) break;
    if ((rc = dpg_launch_assemble(&cand, nullptr, &L, st)) != DPG_OK) break;  // warm-up
    cudaEventRecord(e0, st);
    for (int r = 0; r < 2 && rc == DPG_OK; r++) rc = dpg_launch_assemble(&cand, nullptr, &L, st);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) rc = fail(DPG_ERR_CUDA, "autotune timing");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rc == DPG_OK && (best < 0.0f || ms < best)) {
      best = ms;
      best_plan = cand;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(out, st);
  if (rc != DPG_OK) return rc;
  if (best < 0.0f) return fail(DPG_ERR_UNSUPPORTED, "no Gram chunk size fits this bucket");
  p->hp.dev = best_plan;
  if (cudaMemcpy(p->hp.d_dev, &p->hp.dev, sizeof(DpgPlanDev), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(DPG_ERR_CUDA, "plan upload");
  rc = dpg_configure_kernels(&p->hp.dev);
  if (rc != DPG_OK) return rc;
  *chosen = p->hp.dev.big ? p->hp.dev.big_zk : p->hp.dev.chg;
  return DPG_OK;
}

int dpg_assemble_noalloc(dpg_plan* p, int C, const double* nodes, const int8_t* parity, const double* coeff,
                         double* K, double* l, double* S, double* s, int32_t* info, void* stream, int flags) {
  if (!p) return fail(DPG_ERR_BAD_PLAN, "null plan");
  if (C < 0) return fail(DPG_ERR_INVALID_ARGUMENT, "negative cell count");
  if (C == 0) return DPG_OK;
  if (!nodes || !parity || !info) return fail(DPG_ERR_INVALID_ARGUMENT, "nodes, parity and info are required");
  if (p->hp.dev.nslots > 0 && !coeff) return fail(DPG_ERR_INVALID_ARGUMENT, "coefficients required by this plan");
  if (!(flags & DPG_FLAG_NO_K) && (!K || !l)) return fail(DPG_ERR_INVALID_ARGUMENT, "K and l required");
  if (!(flags & DPG_FLAG_NO_CONDENSE) && (!S || !s)) return fail(DPG_ERR_INVALID_ARGUMENT, "S and s required");
  DpgLaunch L;
  std::memset(&L, 0, sizeof(L));
  L.C = C; L.nodes = nodes; L.parity = parity; L.coeff = coeff;
  L.K = (flags & DPG_FLAG_NO_K) ? nullptr : K;
  L.l = (flags & DPG_FLAG_NO_K) ? nullptr : l;
  L.S = (flags & DPG_FLAG_NO_CONDENSE) ? nullptr : S;
  L.s = (flags & DPG_FLAG_NO_CONDENSE) ? nullptr : s;
  L.info = info;
  return dpg_launch_assemble_noalloc(&p->hp.dev, &L, (cudaStream_t)stream);
}

int dpg_assemble_parts(dpg_plan* p, int C, const double* nodes, const int8_t* parity, const double* coeff, double* G,
                       double* B, double* F, void* stream) {
  if (!p) return fail(DPG_ERR_BAD_PLAN, "null plan");
  if (C < 0) return fail(DPG_ERR_INVALID_ARGUMENT, "negative cell count");
  if (C == 0) return DPG_OK;
  if (!nodes || !parity) return fail(DPG_ERR_INVALID_ARGUMENT, "nodes and parity are required");
  if (p->hp.dev.nslots > 0 && !coeff) return fail(DPG_ERR_INVALID_ARGUMENT, "coefficients required by this plan");
  DpgLaunch L;
  std::memset(&L, 0, sizeof(L));
  L.C = C; L.nodes = nodes; L.parity = parity; L.coeff = coeff;
  L.G = G; L.B = B; L.F = F;
  L.parts = 1;
  return dpg_launch_assemble(&p->hp.dev, p->hp.d_dev, &L, (cudaStream_t)stream);
}

int dpg_assemble_host(dpg_plan* p, int C, const double* nodes, const int8_t* parity, const double* coeff, double* K,
                      double* l, double* S, double* s, int32_t* info, int flags) {
  if (!p) return fail(DPG_ERR_BAD_PLAN, "null plan");
  return dpg_host_pipeline(&p->hp.dev, p->hp.d_dev, &p->hp.d_ws, &p->hp.ws_bytes, p->hp.streams, C, nodes, parity,
                           coeff, K, l, S, s, info, flags);
}

int dpg_factored_cholesky_solve(int C, int N, int M, const double* G, const double* B, const double* F, double* K,
                                double* l, int32_t* info, void* stream) {
  if (C < 0 || N <= 0 || M <= 0) return fail(DPG_ERR_INVALID_ARGUMENT, "bad sizes");
  if (C == 0) return DPG_OK;
  if (!G || !B || !F || !K || !l || !info) return fail(DPG_ERR_INVALID_ARGUMENT, "null argument");
  DpgPlanDev P;
  int rc = dpg_make_solve_plan(N, M, &P);
  if (rc != DPG_OK) return rc;
  rc = dpg_configure_kernels(&P);
  if (rc != DPG_OK) return rc;
  DpgLaunch L;
  std::memset(&L, 0, sizeof(L));
  L.C = C; L.solve_only = 1; L.Gin = G; L.Bin = B; L.Fin = F; L.K = K; L.l = l; L.info = info;
  return dpg_launch_assemble(&P, nullptr, &L, (cudaStream_t)stream);
}

int dpg_assemble_adjoint(dpg_plan* p, int C, const double* nodes, const int8_t* parity, const double* coeff,
                         const double* Kbar, const double* lbar, double* coeff_bar, int32_t* info, void* stream) {
  if (!p) return fail(DPG_ERR_BAD_PLAN, "null plan");
  if (C < 0) return fail(DPG_ERR_INVALID_ARGUMENT, "negative cell count");
  if (C == 0) return DPG_OK;
  if (!nodes || !parity || !info || !Kbar) return fail(DPG_ERR_INVALID_ARGUMENT, "nodes, parity, Kbar and info are required");
  const DpgPlanDev& g = p->hp.dev;
  if (g.nslots > 0 && (!coeff || !coeff_bar))
    return fail(DPG_ERR_INVALID_ARGUMENT, "coefficients and their gradient buffer are required by this plan");
  if (g.nslots == 0) return DPG_OK;  // nothing to differentiate
  DpgLaunch L;
  std::memset(&L, 0, sizeof(L));
  L.C = C; L.nodes = nodes; L.parity = parity; L.coeff = coeff;
  L.info = info;
  L.Kbar = Kbar; L.lbar = lbar; L.coeff_bar = coeff_bar;
  return dpg_launch_adjoint(&g, &L, (cudaStream_t)stream);
}

// Validated per-bucket launch arguments of a multi-bucket call.
static int multi_args(int n_buckets, const dpg_bucket_batch* buckets, int flags, std::vector<DpgPlanDev>& plans,
                      std::vector<DpgLaunch>& ls) {
  if (n_buckets < 0 || (n_buckets > 0 && !buckets)) return fail(DPG_ERR_INVALID_ARGUMENT, "bad bucket list");
  for (int i = 0; i < n_buckets; i++) {
    const dpg_bucket_batch& b = buckets[i];
    if (!b.plan) return fail(DPG_ERR_BAD_PLAN, "null plan in bucket list");
    if (b.C < 0) return fail(DPG_ERR_INVALID_ARGUMENT, "negative cell count");
    if (b.C == 0) continue;
    const DpgPlanDev& g = b.plan->hp.dev;
    if (!b.nodes || !b.parity || !b.info) return fail(DPG_ERR_INVALID_ARGUMENT, "nodes, parity and info are required");
    if (g.nslots > 0 && !b.coeff) return fail(DPG_ERR_INVALID_ARGUMENT, "coefficients required by this plan");
    if (!(flags & DPG_FLAG_NO_K) && (!b.K || !b.l)) return fail(DPG_ERR_INVALID_ARGUMENT, "K and l required");
    if (!(flags & DPG_FLAG_NO_CONDENSE) && (!b.S || !b.s)) return fail(DPG_ERR_INVALID_ARGUMENT, "S and s required");
    DpgLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.C = b.C; L.nodes = b.nodes; L.parity = b.parity; L.coeff = b.coeff;
    L.K = (flags & DPG_FLAG_NO_K) ? nullptr : b.K;
    L.l = (flags & DPG_FLAG_NO_K) ? nullptr : b.l;
    L.S = (flags & DPG_FLAG_NO_CONDENSE) ? nullptr : b.S;
    L.s = (flags & DPG_FLAG_NO_CONDENSE) ? nullptr : b.s;
    L.info = b.info;
    plans.push_back(g);
    ls.push_back(L);
  }
  return DPG_OK;
}

int dpg_scatter_global(int C, int t, const int64_t* map_ptr, const int64_t* map_gid, const double* map_w,
                       int64_t n_global, const int64_t* row_ptr, const int64_t* col_idx, const double* S,
                       const double* s, double* values, double* rhs, int* missing, void* stream) {
  if (C < 0 || t < 0) return fail(DPG_ERR_INVALID_ARGUMENT, "negative size");
  if (C == 0 || t == 0) return DPG_OK;
  if (!map_ptr || !map_gid || !row_ptr || !col_idx || !S || !values || !missing)
    return fail(DPG_ERR_INVALID_ARGUMENT, "map, graph, S, values and the missing counter are required");
  if (n_global <= 0) return fail(DPG_ERR_INVALID_ARGUMENT, "empty global system");
  return dpg_launch_scatter_global(C, t, map_ptr, map_gid, map_w, n_global, row_ptr, col_idx, S, s, values, rhs,
                                   missing, (cudaStream_t)stream);
}

int dpg_energy_error(dpg_plan* p, int C, const double* nodes, const int8_t* parity, const double* coeff,
                     const double* local_coeff, double* energy, int32_t* info, void* stream) {
  if (!p) return fail(DPG_ERR_BAD_PLAN, "null plan");
  if (C < 0) return fail(DPG_ERR_INVALID_ARGUMENT, "negative cell count");
  if (C == 0) return DPG_OK;
  if (!nodes || !parity || !local_coeff || !energy || !info)
    return fail(DPG_ERR_INVALID_ARGUMENT, "nodes, parity, local coefficients, energy and info are required");
  if (p->hp.dev.nslots > 0 && !coeff) return fail(DPG_ERR_INVALID_ARGUMENT, "coefficients required by this plan");
  DpgLaunch L;
  std::memset(&L, 0, sizeof(L));
  L.C = C; L.nodes = nodes; L.parity = parity; L.coeff = coeff;
  L.info = info;
  L.xsol = local_coeff;
  L.energy = energy;
  return dpg_launch_energy(&p->hp.dev, &L, (cudaStream_t)stream);
}

int dpg_assemble_dls(dpg_plan* p, int C, const double* nodes, const int8_t* parity, const double* coeff, double* W,
                     double* y, int32_t* info, void* stream) {
  if (!p) return fail(DPG_ERR_BAD_PLAN, "null plan");
  if (C < 0) return fail(DPG_ERR_INVALID_ARGUMENT, "negative cell count");
  if (C == 0) return DPG_OK;
  if (!nodes || !parity || !W || !y || !info) return fail(DPG_ERR_INVALID_ARGUMENT, "nodes, parity, W, y and info are required");
  if (p->hp.dev.nslots > 0 && !coeff) return fail(DPG_ERR_INVALID_ARGUMENT, "coefficients required by this plan");
  DpgLaunch L;
  std::memset(&L, 0, sizeof(L));
  L.C = C; L.nodes = nodes; L.parity = parity; L.coeff = coeff;
  L.info = info;
  L.B = W;
  L.F = y;
  return dpg_launch_energy(&p->hp.dev, &L, (cudaStream_t)stream);  // no trial solution: the DLS kernel
}

int dpg_recover_fields(dpg_plan* p, int C, const double* K, const double* l, const double* trace_coeff,
                       double* local_coeff, int32_t* info, void* stream) {
  if (!p) return fail(DPG_ERR_BAD_PLAN, "null plan");
  if (C < 0) return fail(DPG_ERR_INVALID_ARGUMENT, "negative cell count");
  if (C == 0) return DPG_OK;
  if (!K || !l || !local_coeff || !info || (p->hp.dev.nt > 0 && !trace_coeff))
    return fail(DPG_ERR_INVALID_ARGUMENT, "K, l, trace coefficients, output and info are required");
  const DpgPlanDev& g = p->hp.dev;
  return dpg_launch_recover_fields(C, g.M, g.nf, K, l, trace_coeff, local_coeff, info, (cudaStream_t)stream);
}

// The buckets of a multi-bucket call: the single-CTA ones stay in (plans, ls) for one
// persistent launch; the large ones move to (bp, bl) and follow on the same stream, one
// launch of the large-bucket kernel each.
// Work items a CTA of the multi-bucket launch claims at a time (flags bits 8-15; 0 -> 1).
static int claim_of(int flags) { return std::max(1, (flags >> 8) & 0xff); }

// The large buckets go to their own launches (the specialized kernel, whose plan lives in
// kernel parameters: a work queue holding them ran their cells 11-28 % slower), in
// decreasing order of per-cell cost; the single-CTA buckets share one work-queue launch.
static void split_big(std::vector<DpgPlanDev>& plans, std::vector<DpgLaunch>& ls, std::vector<DpgPlanDev>& bp,
                      std::vector<DpgLaunch>& bl) {
  std::vector<DpgPlanDev> sp;
  std::vector<DpgLaunch> sl;
  std::vector<size_t> big;
  for (size_t i = 0; i < plans.size(); i++) {
    if (plans[i].big) {
      big.push_back(i);
    } else {
      sp.push_back(plans[i]);
      sl.push_back(ls[i]);
    }
  }
  std::stable_sort(big.begin(), big.end(), [&](size_t x, size_t y) { return plans[x].Zn > plans[y].Zn; });
  for (size_t i : big) {
    bp.push_back(plans[i]);
    bl.push_back(ls[i]);
  }
  plans.swap(sp);
  ls.swap(sl);
}

int dpg_assemble_multi(int n_buckets, const dpg_bucket_batch* buckets, void* stream, int flags) {
  std::vector<DpgPlanDev> plans, bp;
  std::vector<DpgLaunch> ls, bl;
  int rc = multi_args(n_buckets, buckets, flags, plans, ls);
  if (rc != DPG_OK) return rc;
  split_big(plans, ls, bp, bl);
  for (size_t i = 0; rc == DPG_OK && i < bp.size(); i++)
    rc = dpg_launch_assemble(&bp[i], nullptr, &bl[i], (cudaStream_t)stream);
  if (rc == DPG_OK && !plans.empty())
    rc = dpg_launch_multi(plans.data(), ls.data(), (int)plans.size(), (cudaStream_t)stream, nullptr, claim_of(flags));
  return rc;
}

int dpg_multi_autotune(int n_buckets, const dpg_bucket_batch* buckets, void* stream, int flags, int* chosen) {
  if (!chosen) return fail(DPG_ERR_INVALID_ARGUMENT, "null output");
  *chosen = 0;
  std::vector<DpgPlanDev> plans, bp;
  std::vector<DpgLaunch> ls, bl;
  int rc = multi_args(n_buckets, buckets, flags, plans, ls);
  if (rc != DPG_OK) return rc;
  split_big(plans, ls, bp, bl);  // the claim size concerns the work queue of the single-CTA buckets
  if (plans.empty()) {
    *chosen = 1;
    return DPG_OK;
  }
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = -1.0f;
  int best_claim = 1;
  for (int claim : {1, 2, 4, 8}) {
    if ((rc = dpg_launch_multi(plans.data(), ls.data(), (int)plans.size(), st, nullptr, claim)) != DPG_OK) break;
    cudaEventRecord(e0, st);
    rc = dpg_launch_multi(plans.data(), ls.data(), (int)plans.size(), st, nullptr, claim);
    cudaEventRecord(e1, st);
    if (rc != DPG_OK) break;
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      rc = fail(DPG_ERR_CUDA, "multi autotune timing");
      break;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (best < 0.0f || ms < best) {
      best = ms;
      best_claim = claim;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != DPG_OK) return rc;
  *chosen = best_claim;
  return DPG_OK;
}

struct dpg_graph {
  DpgMultiDev dev;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
  void* big_ws = nullptr;  // workspace of the large-bucket launches (they run one after another)
};

int dpg_graph_capture(int n_buckets, const dpg_bucket_batch* buckets, int flags, dpg_graph** out) {
  if (!out) return fail(DPG_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  std::vector<DpgPlanDev> plans, bp;
  std::vector<DpgLaunch> ls, bl;
  int rc = multi_args(n_buckets, buckets, flags, plans, ls);
  if (rc != DPG_OK) return rc;
  split_big(plans, ls, bp, bl);
  size_t big_bytes = 0;
  for (size_t i = 0; i < bp.size(); i++) big_bytes = std::max(big_bytes, dpg_big_workspace_bytes(&bp[i], bl[i].C));
  if (plans.empty() && bp.empty()) return fail(DPG_ERR_INVALID_ARGUMENT, "no cells to capture");
  dpg_graph* G = new dpg_graph();
  std::memset(&G->dev, 0, sizeof(G->dev));
  cudaGetDevice(&G->device);
  if (!plans.empty()) {
    G->dev.bytes = dpg_multi_bytes(plans.data(), ls.data(), (int)plans.size());
    if (cudaMalloc(&G->dev.base, G->dev.bytes) != cudaSuccess) {
      cudaGetLastError();
      G->dev.base = nullptr;
      dpg_graph_destroy(G);
      return fail(DPG_ERR_OUT_OF_MEMORY, "graph workspace");
    }
    rc = dpg_launch_multi(plans.data(), ls.data(), (int)plans.size(), nullptr, &G->dev, claim_of(flags));
  }
  if (rc == DPG_OK && big_bytes > 0 && cudaMalloc(&G->big_ws, big_bytes) != cudaSuccess) {
    cudaGetLastError();
    G->big_ws = nullptr;
    rc = fail(DPG_ERR_OUT_OF_MEMORY, "graph workspace of the large buckets");
  }
  // one stream: the large buckets' launches in decreasing order of cost, then the work queue
  // of the single-CTA buckets (run beside them on a second branch, the queue's CTAs took SMs
  // before the long large cells had started and lengthened the whole: 1.19 s against 1.17 s
  // on the uneven-cell workload)
  cudaStream_t cs0 = nullptr;
  if (rc == DPG_OK && cudaStreamCreateWithFlags(&cs0, cudaStreamNonBlocking) != cudaSuccess)
    rc = fail(DPG_ERR_CUDA, "stream creation");
  if (rc == DPG_OK) {
    cudaError_t e = cudaStreamBeginCapture(cs0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      for (size_t i = 0; rc == DPG_OK && i < bp.size(); i++) {
        bl[i].scratch = (double*)G->big_ws;
        rc = dpg_launch_assemble(&bp[i], nullptr, &bl[i], cs0);
      }
      if (rc == DPG_OK && !plans.empty()) rc = dpg_launch_multi_prepared(&G->dev, cs0);
      cudaError_t e2 = cudaStreamEndCapture(cs0, &G->graph);
      if (rc == DPG_OK && e2 != cudaSuccess) rc = fail(DPG_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e2));
    } else {
      rc = fail(DPG_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    }
  }
  if (rc == DPG_OK && cudaGraphInstantiate(&G->exec, G->graph, 0) != cudaSuccess)
    rc = fail(DPG_ERR_CUDA, "graph instantiation");
  if (cs0) cudaStreamDestroy(cs0);
  if (rc != DPG_OK) {
    cudaGetLastError();
    dpg_graph_destroy(G);
    return rc;
  }
  *out = G;
  return DPG_OK;
}

int dpg_graph_launch(dpg_graph* G, void* stream) {
  if (!G || !G->exec) return fail(DPG_ERR_INVALID_ARGUMENT, "null graph");
  cudaError_t e = cudaGraphLaunch(G->exec, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(DPG_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}

int dpg_graph_destroy(dpg_graph* G) {
  if (!G) return DPG_OK;
  if (G->exec) cudaGraphExecDestroy(G->exec);
  if (G->graph) cudaGraphDestroy(G->graph);
  if (G->dev.base) cudaFree(G->dev.base);
  if (G->big_ws) cudaFree(G->big_ws);
  delete G;
  return DPG_OK;
}

}  // extern "C"
