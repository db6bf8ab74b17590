// dpg_kernel.cu — fused FP64 per-cell DPG assembly for sm_100a.
//
// One CTA (16 warps) assembles one cell end to end:
//   1. Gram matrix G (BasisCache + IP::computeInnerProductMatrix, IP.cpp:215-292):
//      physical test features are staged in shared memory four quadrature
//      points at a time; every warp owns a contiguous run of lower 8x8 tiles of
//      G and accumulates them in registers with mma.m8n8k4.f64 (DMMA).
//   2. Equilibrated Cholesky of G (BF.cpp:944-982: DPOEQU scaling, DPOTRF('L'),
//      unscaling), blocked right-looking on tiles held in shared memory.
//   3. B and F (TBF::stiffnessMatrix, BF.cpp:575-656; RHS.cpp:68-82): warp J owns
//      trial column tile J and accumulates all of B[:, J] in registers.
//   4. W = L^-1 [B | F] in registers (BF.cpp:987-988, 1013-1014): each warp runs
//      a blocked forward substitution on its own column tile; diagonal blocks use
//      precomputed inverses so every step is a DMMA.
//   5. K_ext = W^T W (DSYRK, BF.cpp:993-1005) including l = W^T y (BF.cpp:1016).
//   6. Static condensation (CondensedDofInterpreter.cpp:1138-1192): the first
//      field-tile steps of a blocked Cholesky of K_ext leave the Schur complement
//      [S s; s^T .] in the trailing block.
// Numerical failures are reported per cell in info (DPOTRF INFO semantics).
#include "../../include/dpg_b200.h"
#include "dpg_internal.h"
#include "dpg_plan.h"

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>

namespace {

constexpr int NT = DPG_NTHREADS;

__device__ __forceinline__ void dmma(double2& c, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c.x), "+d"(c.y)
               : "d"(a), "d"(b));
}

// AK layout index of element (r, c) of an 8x8 tile
__device__ __forceinline__ int ak(int r, int c) { return ((c >> 2) * 8 + r) * 4 + (c & 3); }

// Offset of the C-fragment pair (g, 2t..2t+1) in AK layout
__device__ __forceinline__ int ak_cfrag(int g, int t) { return ((t >> 1) * 8 + g) * 4 + (t & 1) * 2; }

__device__ __forceinline__ int tri_row(int tau) {
  int I = (int)((sqrt(8.0 * tau + 1.0) - 1.0) * 0.5);
  while ((I + 1) * (I + 2) / 2 <= tau) I++;
  while (I * (I + 1) / 2 > tau) I--;
  return I;
}

// Convert a C-fragment (rows g, cols 2t, 2t+1) into the two B-fragments of the
// same 8x8 matrix used as the k x n operand: B_h[t][g] = X[4h + t][g].
__device__ __forceinline__ void cfrag_to_bfrag(const double2 c, int lane, double& b0, double& b1) {
  const int g = lane >> 2, t = lane & 3;
  const int src0 = t * 4 + (g >> 1);
  const int src1 = 16 + t * 4 + (g >> 1);
  double x0 = __shfl_sync(0xffffffffu, c.x, src0);
  double y0 = __shfl_sync(0xffffffffu, c.y, src0);
  double x1 = __shfl_sync(0xffffffffu, c.x, src1);
  double y1 = __shfl_sync(0xffffffffu, c.y, src1);
  b0 = (g & 1) ? y0 : x0;
  b1 = (g & 1) ? y1 : x1;
}

struct Geo {
  double J[9], Ji[9], det;
};

// Jacobian, inverse and determinant from the vertex-shape derivatives at a point.
__device__ __forceinline__ void geometry(int d, int nv, const double* __restrict__ X, const double* __restrict__ dN,
                                         Geo& G) {
#pragma unroll
  for (int i = 0; i < 9; i++) G.J[i] = 0.0;
  for (int a = 0; a < nv; a++)
    for (int i = 0; i < d; i++) {
      double xa = X[a * d + i];
      for (int j = 0; j < d; j++) G.J[i * 3 + j] += xa * dN[a * d + j];
    }
  if (d == 2) {
    G.det = G.J[0] * G.J[4] - G.J[1] * G.J[3];
    double id = 1.0 / G.det;
    G.Ji[0] = G.J[4] * id; G.Ji[1] = -G.J[1] * id; G.Ji[2] = 0;
    G.Ji[3] = -G.J[3] * id; G.Ji[4] = G.J[0] * id; G.Ji[5] = 0;
    G.Ji[6] = 0; G.Ji[7] = 0; G.Ji[8] = 1;
  } else {
    const double* A = G.J;
    double c00 = A[4] * A[8] - A[5] * A[7];
    double c01 = A[5] * A[6] - A[3] * A[8];
    double c02 = A[3] * A[7] - A[4] * A[6];
    G.det = A[0] * c00 + A[1] * c01 + A[2] * c02;
    double id = 1.0 / G.det;
    G.Ji[0] = c00 * id;
    G.Ji[3] = c01 * id;
    G.Ji[6] = c02 * id;
    G.Ji[1] = (A[2] * A[7] - A[1] * A[8]) * id;
    G.Ji[4] = (A[0] * A[8] - A[2] * A[6]) * id;
    G.Ji[7] = (A[1] * A[6] - A[0] * A[7]) * id;
    G.Ji[2] = (A[1] * A[5] - A[2] * A[4]) * id;
    G.Ji[5] = (A[2] * A[3] - A[0] * A[5]) * id;
    G.Ji[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  }
}

// Physical value of a test operator from the reference record of one dof.
// geo: [J(9) Ji(9) det wdet meas n(3)]
__device__ __forceinline__ double test_op(int space, int d, int op, const double* __restrict__ ref,
                                          const double* __restrict__ geo) {
  if (space == DPG_SPACE_HGRAD) {
    if (op == DPG_OP_VALUE) return ref[0];
    int c = op - DPG_OP_DX;  // (J^-T grad)_c = sum_j Ji[j][c] grad_j
    double s = 0.0;
    for (int j = 0; j < d; j++) s += geo[9 + j * 3 + c] * ref[1 + j];
    return s;
  }
  double idet = 1.0 / geo[18];
  if (op == DPG_OP_DIV) return ref[d] * idet;
  if (op == DPG_OP_DOT_NORMAL) {
    double s = 0.0;
    for (int c = 0; c < d; c++) {
      double v = 0.0;
      for (int j = 0; j < d; j++) v += geo[c * 3 + j] * ref[j];
      s += v * geo[21 + c];
    }
    return s * idet;
  }
  int c = op - DPG_OP_X;
  double v = 0.0;
  for (int j = 0; j < d; j++) v += geo[c * 3 + j] * ref[j];
  return v * idet;
}

// Element (r, c) of the symmetric matrix stored as lower AK tiles at base.
__device__ __forceinline__ double sym_get(const double* base, int r, int c) {
  if (r < c) { int x = r; r = c; c = x; }
  int I = r >> 3, J = c >> 3;
  return base[(I * (I + 1) / 2 + J) * 64 + ak(r & 7, c & 7)];
}

// Blocked right-looking Cholesky of the leading nsteps tiles of a tile-lower
// matrix with nb tiles in shared memory.  Records the first failing global
// pivot (1-based) into *flag with sign `sgn` if *flag is still 0.
__device__ void tile_cholesky(double* __restrict__ T, int nb, int nsteps, int* flag, int sgn) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  for (int k = 0; k < nsteps; k++) {
    double* Tkk = T + (k * (k + 1) / 2 + k) * 64;
    if (warp == 0) {
      double row[8];
      const int r = lane & 7;
#pragma unroll
      for (int c = 0; c < 8; c++) row[c] = Tkk[ak(r, c)];
      bool failed = false;
      int fail_j = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        double piv = __shfl_sync(0xffffffffu, row[j], j);
        if (!(piv > 0.0) && !failed) { failed = true; fail_j = j; }
        double dj = sqrt(piv);
        double inv = 1.0 / dj;
        if (r == j) row[j] = dj;
        else if (r > j) row[j] *= inv;
#pragma unroll
        for (int c = j + 1; c < 8; c++) {
          double lcj = __shfl_sync(0xffffffffu, row[j], c);
          if (r >= c) row[c] -= row[j] * lcj;
        }
      }
      if (lane < 8) {
#pragma unroll
        for (int c = 0; c < 8; c++) Tkk[ak(r, c)] = (c <= r) ? row[c] : 0.0;
      }
      if (lane == 0 && failed && *flag == 0) *flag = sgn * (k * 8 + fail_j + 1);
    }
    __syncthreads();
    // panel: L_ik = A_ik L_kk^-T, one row per thread
    int nrows = (nb - 1 - k) * 8;
    for (int w = tid; w < nrows; w += NT) {
      int i = k + 1 + (w >> 3), r = w & 7;
      double* Tik = T + (i * (i + 1) / 2 + k) * 64;
      double x[8];
#pragma unroll
      for (int c = 0; c < 8; c++) x[c] = Tik[ak(r, c)];
#pragma unroll
      for (int c = 0; c < 8; c++) {
        double v = x[c];
#pragma unroll
        for (int m = 0; m < c; m++) v -= x[m] * Tkk[ak(c, m)];
        x[c] = v / Tkk[ak(c, c)];
      }
#pragma unroll
      for (int c = 0; c < 8; c++) Tik[ak(r, c)] = x[c];
    }
    __syncthreads();
    // trailing update: A_ij -= L_ik L_jk^T for k < j <= i < nb
    int m = nb - 1 - k;
    int ntr = m * (m + 1) / 2;
    for (int u = warp; u < ntr; u += DPG_NWARPS) {
      int ii = tri_row(u), jj = u - ii * (ii + 1) / 2;
      int i = k + 1 + ii, j = k + 1 + jj;
      double* Tij = T + (i * (i + 1) / 2 + j) * 64;
      const double* Lik = T + (i * (i + 1) / 2 + k) * 64;
      const double* Ljk = T + (j * (j + 1) / 2 + k) * 64;
      double2 c = *reinterpret_cast<const double2*>(Tij + ak_cfrag(g, t));
      dmma(c, -Lik[lane], Ljk[lane]);
      dmma(c, -Lik[32 + lane], Ljk[32 + lane]);
      *reinterpret_cast<double2*>(Tij + ak_cfrag(g, t)) = c;
    }
    __syncthreads();
  }
}

template <int NBTM>
__global__ void __launch_bounds__(NT, 1) dpg_cell_kernel(const __grid_constant__ DpgPlanDev P, const DpgLaunch L) {
  extern __shared__ __align__(16) double sm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int cell = blockIdx.x;
  const int d = P.d, nv = P.nv;
  double* nodes_s = sm + P.sm_total - 64;
  int* flag_s = reinterpret_cast<int*>(sm + P.sm_total - 8);
  if (!L.solve_only && tid < nv * d) nodes_s[tid] = L.nodes[(size_t)cell * nv * d + tid];
  if (tid == 0) { flag_s[0] = 0; flag_s[1] = 0; }
  const double* coef_c = L.coeff ? L.coeff + (size_t)cell * P.nslots * P.Ptot : nullptr;
  const int8_t* par_c = L.solve_only ? nullptr : L.parity + (size_t)cell * P.ns;
  __syncthreads();

  double* GT = sm + P.sm_gt;  // lower tiles of G, AK layout

  // ======================= 1. Gram matrix ===================================
  if (L.solve_only) {
    const double* Gc = L.Gin + (size_t)cell * P.N * P.N;
    for (int e = tid; e < P.ngt * 64; e += NT) {
      int tau = e >> 6, idx = e & 63;
      int I = tri_row(tau), J = tau - I * (I + 1) / 2;
      int r = (idx >> 2) & 7, c = (idx >> 5) * 4 + (idx & 3);
      int gr = I * 8 + r, gc = J * 8 + c;
      double v = 0.0;
      if (gr < P.N && gc < P.N) v = Gc[(size_t)gr * P.N + gc];
      else if (gr == gc) v = 1.0;
      GT[e] = v;
    }
    __syncthreads();
  } else {
    const int per = (P.ngt + DPG_NWARPS - 1) / DPG_NWARPS;
    const int tau0 = warp * per;
    const int ntw = max(0, min(per, P.ngt - tau0));
    double2 acc[DPG_MAX_GT];
#pragma unroll
    for (int u = 0; u < DPG_MAX_GT; u++) acc[u] = make_double2(0.0, 0.0);
    double* geo = sm + P.sm_geo;
    double* avec = sm + P.sm_cmat + DPG_CHUNK * P.Ftot * P.Ftot;  // [q][row][F]
    double* cm = sm + P.sm_cmat;                                   // [q][F][F]
    double* feat = sm + P.sm_feat;
    double* hb = sm + P.sm_h;
    const int F = P.Ftot;
    for (int q0 = 0; q0 < P.QG; q0 += DPG_CHUNK) {
      const int np = min(DPG_CHUNK, P.QG - q0);
      if (tid < DPG_CHUNK) {
        double* gq = geo + tid * 32;
        if (tid < np) {
          Geo G;
          geometry(d, nv, nodes_s, P.dNG + (size_t)(q0 + tid) * nv * d, G);
#pragma unroll
          for (int i = 0; i < 9; i++) { gq[i] = G.J[i]; gq[9 + i] = G.Ji[i]; }
          gq[18] = G.det;
          gq[19] = P.wG[q0 + tid] * G.det;
        } else {
#pragma unroll
          for (int i = 0; i < 9; i++) { gq[i] = (i % 4 == 0) ? 1.0 : 0.0; gq[9 + i] = gq[i]; }
          gq[18] = 1.0;
          gq[19] = 0.0;
        }
      }
      for (int i = tid; i < DPG_CHUNK * DPG_MAX_IPROWS * F; i += NT) avec[i] = 0.0;
      __syncthreads();
      if (tid < DPG_CHUNK) {
        const int q = tid;
        for (int e = 0; e < P.nipent; e++) {
          const DpgIPEnt& E = P.ipent[e];
          double v = E.coef;
          if (E.slot >= 0) v *= (q < np) ? coef_c[(size_t)E.slot * P.Ptot + q0 + q] : 0.0;
          avec[(q * DPG_MAX_IPROWS + E.row) * F + E.gfeat] += v;
        }
      }
      // physical features [q][var][4][ldA]
      for (int q = 0; q < DPG_CHUNK; q++) {
        const double* gq = geo + q * 32;
        int foff = 0;
        for (int a = 0; a < P.ntest; a++) {
          const DpgTestVar& V = P.test[a];
          const int n = 4 * V.ldA;
          double* dst = feat + q * P.featstride + foff;
          for (int i = tid; i < n; i += NT) {
            int k = i / V.ldA, row = i - k * V.ldA;
            double v = 0.0;
            if (q < np && k < V.nfeat && row < V.card)
              v = test_op(V.space, d, V.feat_op[k], V.tabG + ((size_t)(q0 + q) * V.card + row) * V.nref, gq);
            dst[i] = v;
          }
          foff += n;
        }
      }
      __syncthreads();
      // coefficient matrix C_q = wdet * sum_r a_r a_r^T
      for (int i = tid; i < DPG_CHUNK * F * F; i += NT) {
        int q = i / (F * F), rem = i - q * F * F, f1 = rem / F, f2 = rem - f1 * F;
        double s = 0.0;
        const double* aq = avec + q * DPG_MAX_IPROWS * F;
        for (int r = 0; r < P.niprows; r++) s += aq[r * F + f1] * aq[r * F + f2];
        cm[i] = s * geo[q * 32 + 19];
      }
      __syncthreads();
      // h_{b->a}[q][k][j] = sum_l C[4a+k][4b+l] f_b[q][l][j]
      for (int q = 0; q < DPG_CHUNK; q++) {
        const double* Cq = cm + q * F * F;
        for (int a = 0; a < P.ntest; a++) {
          int foff_b = 0;
          for (int b = 0; b <= a; b++) {
            const DpgTestVar& Vb = P.test[b];
            const int n = 4 * Vb.ldA;
            const double* fb = feat + q * P.featstride + foff_b;
            double* dst = hb + q * P.hstride + P.hoff[a][b];
            for (int i = tid; i < n; i += NT) {
              int k = i / Vb.ldA, j = i - k * Vb.ldA;
              const double* crow = Cq + (4 * a + k) * F + 4 * b;
              dst[i] = crow[0] * fb[j] + crow[1] * fb[Vb.ldA + j] + crow[2] * fb[2 * Vb.ldA + j] +
                       crow[3] * fb[3 * Vb.ldA + j];
            }
            foff_b += n;
          }
        }
      }
      __syncthreads();
      // DMMA accumulation of the owned tiles
      for (int q = 0; q < np; q++) {
        const double* fq = feat + q * P.featstride;
        const double* hq = hb + q * P.hstride;
        int lastI = -1;
        double afr = 0.0;
#pragma unroll
        for (int u = 0; u < DPG_MAX_GT; u++) {
          if (u < ntw) {
            const DpgGTile T = P.gtiles[tau0 + u];
            if (T.I != lastI) { afr = fq[T.aoff + t * T.lda + g]; lastI = T.I; }
            double bfr = hq[T.boff + t * T.ldb + g];
            dmma(acc[u], afr, bfr);
          }
        }
      }
      __syncthreads();
    }
    // accumulators -> tile-lower shared storage (overlaps the staging area)
#pragma unroll
    for (int u = 0; u < DPG_MAX_GT; u++)
      if (u < ntw) *reinterpret_cast<double2*>(GT + (tau0 + u) * 64 + ak_cfrag(g, t)) = acc[u];
    __syncthreads();
    // padded rows decouple: unit diagonal
    for (int r = tid; r < P.Np; r += NT)
      if (P.dev2user_test[r] < 0) GT[((r >> 3) * ((r >> 3) + 1) / 2 + (r >> 3)) * 64 + ak(r & 7, r & 7)] = 1.0;
    __syncthreads();
    if (L.parts && L.G) {
      double* Gc = L.G + (size_t)cell * P.N * P.N;
      for (int e = tid; e < P.Np * P.Np; e += NT) {
        int r = e / P.Np, c = e - r * P.Np;
        int ur = P.dev2user_test[r], uc = P.dev2user_test[c];
        if (ur >= 0 && uc >= 0) Gc[(size_t)ur * P.N + uc] = sym_get(GT, r, c);
      }
    }
  }

  // ======================= 2. equilibrated Cholesky ==========================
  double* scale = sm + P.sm_scale;
  double* LINV = sm + P.sm_linv;
  if (!L.parts) {
    for (int r = tid; r < P.Np; r += NT) {
      int I = r >> 3;
      double dg = GT[(I * (I + 1) / 2 + I) * 64 + ak(r & 7, r & 7)];
      scale[r] = (dg > 0.0) ? 1.0 / sqrt(dg) : 1.0;
    }
    __syncthreads();
    for (int e = tid; e < P.ngt * 64; e += NT) {
      int tau = e >> 6, idx = e & 63;
      int I = tri_row(tau), J = tau - I * (I + 1) / 2;
      int r = (idx >> 2) & 7, c = (idx >> 5) * 4 + (idx & 3);
      GT[e] *= scale[I * 8 + r] * scale[J * 8 + c];
    }
    __syncthreads();
    tile_cholesky(GT, P.NBT, P.NBT, flag_s, 1);
    // unscale rows: L(i, j) /= s_i
    for (int e = tid; e < P.ngt * 64; e += NT) {
      int tau = e >> 6, idx = e & 63;
      int I = tri_row(tau);
      int r = (idx >> 2) & 7;
      GT[e] /= scale[I * 8 + r];
    }
    __syncthreads();
    // inverses of the diagonal tiles (column per lane)
    for (int k = warp; k < P.NBT; k += DPG_NWARPS) {
      const double* Lkk = GT + (k * (k + 1) / 2 + k) * 64;
      double* X = LINV + k * 64;
      if (lane < 8) {
        const int c = lane;
        double x[8];
#pragma unroll
        for (int r = 0; r < 8; r++) {
          double v = (r == c) ? 1.0 : 0.0;
#pragma unroll
          for (int m = 0; m < r; m++) v -= Lkk[ak(r, m)] * x[m];
          x[r] = (r < c) ? 0.0 : v / Lkk[ak(r, r)];
        }
#pragma unroll
        for (int r = 0; r < 8; r++) X[ak(r, c)] = x[r];
      }
    }
    __syncthreads();
  }

  // ======================= 3. B and F, one trial tile column per warp ========
  const int J = warp;
  const bool has_col = J < P.MBT;
  double2 bacc[NBTM];
#pragma unroll
  for (int i = 0; i < NBTM; i++) bacc[i] = make_double2(0.0, 0.0);
  if (L.solve_only) {
    if (has_col) {
      const double* Bc = L.Bin + (size_t)cell * P.M * P.N;
      const double* Fc = L.Fin + (size_t)cell * P.N;
#pragma unroll
      for (int I = 0; I < NBTM; I++) {
        if (I < P.NBT) {
          int row = I * 8 + g;
          double v[2];
#pragma unroll
          for (int e = 0; e < 2; e++) {
            int col = J * 8 + 2 * t + e;
            double x = 0.0;
            if (row < P.N) {
              if (col < P.M) x = Bc[(size_t)col * P.N + row];
              else if (col == P.fcol) x = Fc[row];
            }
            v[e] = x;
          }
          bacc[I] = make_double2(v[0], v[1]);
        }
      }
    }
  } else {
    double* geo = sm + P.sm_misc;
    double* bops = sm + P.sm_bops;
    double* bval = sm + P.sm_bval;
    for (int sgi = 0; sgi < P.nseg; sgi++) {
      const DpgSeg& S = P.seg[sgi];
      if (S.nterm == 0) continue;
      const int side = sgi - 1;
      for (int q0 = 0; q0 < S.npts; q0 += DPG_CHUNK) {
        const int np = min(DPG_CHUNK, S.npts - q0);
        __syncthreads();
        if (tid < DPG_CHUNK) {
          double* gq = geo + tid * 32;
          if (tid < np) {
            Geo G;
            const double* dN = (side < 0) ? P.dNB + (size_t)(q0 + tid) * nv * d
                                          : P.dNS + ((size_t)side * P.QS + q0 + tid) * nv * d;
            geometry(d, nv, nodes_s, dN, G);
#pragma unroll
            for (int i = 0; i < 9; i++) { gq[i] = G.J[i]; gq[9 + i] = G.Ji[i]; }
            gq[18] = G.det;
            if (side < 0) {
              gq[19] = P.wB[q0 + tid] * G.det;
              gq[21] = gq[22] = gq[23] = 0.0;
            } else {
              const double* Tq = P.sideT + ((size_t)side * P.QS + q0 + tid) * 6;
              double T0[3] = {0, 0, 0}, T1[3] = {0, 0, 0};
              for (int i = 0; i < d; i++)
                for (int j = 0; j < d; j++) {
                  T0[i] += G.J[i * 3 + j] * Tq[j];
                  T1[i] += G.J[i * 3 + j] * Tq[3 + j];
                }
              double meas, n[3];
              if (d == 2) {
                meas = sqrt(T0[0] * T0[0] + T0[1] * T0[1]);
                n[0] = T0[1] / meas; n[1] = -T0[0] / meas; n[2] = 0.0;
              } else {
                double c0 = T0[1] * T1[2] - T0[2] * T1[1];
                double c1 = T0[2] * T1[0] - T0[0] * T1[2];
                double c2 = T0[0] * T1[1] - T0[1] * T1[0];
                meas = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
                n[0] = c0 / meas; n[1] = c1 / meas; n[2] = c2 / meas;
              }
              gq[19] = P.wS[q0 + tid] * meas;
              gq[21] = n[0]; gq[22] = n[1]; gq[23] = n[2];
            }
          } else {
#pragma unroll
            for (int i = 0; i < 9; i++) { gq[i] = (i % 4 == 0) ? 1.0 : 0.0; gq[9 + i] = gq[i]; }
            gq[18] = 1.0;
            gq[19] = 0.0;
            gq[21] = gq[22] = gq[23] = 0.0;
          }
        }
        __syncthreads();
        // stage test ops [op][q][ldA]
        for (int o = 0; o < S.nops; o++) {
          const DpgBOp& O = S.ops[o];
          const DpgTestVar& V = P.test[O.var];
          const int n = DPG_CHUNK * V.ldA;
          double* dst = bops + O.off;
          for (int i = tid; i < n; i += NT) {
            int q = i / V.ldA, row = i - q * V.ldA;
            double v = 0.0;
            if (q < np && row < V.card) {
              const double* ref = (side < 0)
                  ? V.tabB + ((size_t)(q0 + q) * V.card + row) * V.nref
                  : V.tabS + (((size_t)side * P.QS + q0 + q) * V.card + row) * V.nref;
              v = test_op(V.space, d, O.op, ref, geo + q * 32);
            }
            dst[i] = v;
          }
        }
        // stage weighted trial values [term][q][ldT]
        for (int tt = 0; tt < S.nterm; tt++) {
          const DpgBTerm& Tm = P.bterm[S.term0 + tt];
          double* dst = bval + tt * DPG_CHUNK * P.ldT;
          for (int i = tid; i < DPG_CHUNK * P.ldT; i += NT) {
            int q = i / P.ldT, m = i - q * P.ldT;
            double v = 0.0;
            int mm = m - Tm.col0;
            if (q < np && mm >= 0 && mm < Tm.ncol) {
              const double* gq = geo + q * 32;
              double w = gq[19] * Tm.coef;
              if (Tm.slot >= 0) {
                int pidx = (side < 0) ? P.QG + q0 + q : P.QG + P.QB + side * P.QS + q0 + q;
                w *= coef_c[(size_t)Tm.slot * P.Ptot + pidx];
              }
              if (Tm.normal_comp >= 0) w *= gq[21 + Tm.normal_comp];
              if (Tm.kind < 0) {
                v = w;  // RHS: the F column
              } else {
                const DpgTrialVar& TV = P.trial[Tm.trial_var];
                double val;
                if (Tm.kind == DPG_VAR_FIELD) {
                  val = (side < 0) ? TV.tabB[(size_t)(q0 + q) * TV.card_comp + mm]
                                   : TV.tabS[((size_t)side * P.QS + q0 + q) * TV.card_comp + mm];
                } else {
                  val = TV.tabS[(size_t)(q0 + q) * TV.per_side + mm];
                  if (Tm.kind == DPG_VAR_FLUX) w *= (double)par_c[side];
                }
                v = w * val;
              }
            }
            dst[i] = v;
          }
        }
        __syncthreads();
        if (has_col) {
          for (int tt = 0; tt < S.nterm; tt++) {
            const DpgBTerm& Tm = P.bterm[S.term0 + tt];
            if (Tm.col0 >= J * 8 + 8 || Tm.col0 + Tm.ncol <= J * 8) continue;
            const DpgBOp& O = S.ops[Tm.bop];
            const DpgTestVar& V = P.test[O.var];
            const double bfr = bval[(tt * DPG_CHUNK + t) * P.ldT + J * 8 + g];
            const double* abase = bops + O.off + t * V.ldA + g - V.ntile0 * 8;
            const int i0 = V.ntile0, i1 = V.ntile0 + V.ntiles;
#pragma unroll
            for (int I = 0; I < NBTM; I++)
              if (I >= i0 && I < i1) dmma(bacc[I], abase[I * 8], bfr);
          }
        }
      }
    }
    __syncthreads();
  }

  if (L.parts) {
    if (has_col) {
      double* Bc = L.B ? L.B + (size_t)cell * P.M * P.N : nullptr;
      double* Fc = L.F ? L.F + (size_t)cell * P.N : nullptr;
#pragma unroll
      for (int I = 0; I < NBTM; I++) {
        if (I < P.NBT) {
          int ur = P.dev2user_test[I * 8 + g];
          if (ur >= 0) {
#pragma unroll
            for (int e = 0; e < 2; e++) {
              int col = J * 8 + 2 * t + e;
              double v = e ? bacc[I].y : bacc[I].x;
              int uc = P.dev2user_trial[col];
              if (Bc && uc >= 0) Bc[(size_t)uc * P.N + ur] = v;
              if (Fc && col == P.fcol) Fc[ur] = v;
            }
          }
        }
      }
    }
    return;
  }

  // ======================= 4. W = L^-1 [B | F] in registers ===================
  if (has_col) {
#pragma unroll
    for (int k = 0; k < NBTM; k++) {
      if (k < P.NBT) {
        double y0, y1;
        cfrag_to_bfrag(bacc[k], lane, y0, y1);
        const double* Li = LINV + k * 64;
        double2 x = make_double2(0.0, 0.0);
        dmma(x, Li[lane], y0);
        dmma(x, Li[32 + lane], y1);
        bacc[k] = x;
        double x0, x1;
        cfrag_to_bfrag(x, lane, x0, x1);
        x0 = -x0;
        x1 = -x1;
#pragma unroll
        for (int i = k + 1; i < NBTM; i++) {
          if (i < P.NBT) {
            const double* Lik = GT + (i * (i + 1) / 2 + k) * 64;
            dmma(bacc[i], Lik[lane], x0);
            dmma(bacc[i], Lik[32 + lane], x1);
          }
        }
      }
    }
  }
  __syncthreads();
  // W^T tiles (trial J, test I) in AK layout
  double* WT = sm + P.sm_w;
  if (has_col) {
#pragma unroll
    for (int I = 0; I < NBTM; I++) {
      if (I < P.NBT) {
        double* tile = WT + (J * P.NBT + I) * 64;
        tile[((g >> 2) * 8 + 2 * t) * 4 + (g & 3)] = bacc[I].x;
        tile[((g >> 2) * 8 + 2 * t + 1) * 4 + (g & 3)] = bacc[I].y;
      }
    }
  }
  __syncthreads();

  // ======================= 5. K_ext = W^T W (lower tiles) =====================
  {
    const int nk = P.MBT * (P.MBT + 1) / 2;
    const int per = (nk + DPG_NWARPS - 1) / DPG_NWARPS;
    const int k0 = warp * per;
    const int nkw = max(0, min(per, nk - k0));
    double2 kacc[DPG_MAX_KT];
    int kI[DPG_MAX_KT], kJ[DPG_MAX_KT];
#pragma unroll
    for (int u = 0; u < DPG_MAX_KT; u++) {
      kacc[u] = make_double2(0.0, 0.0);
      int tau = k0 + u;
      int I = tri_row(tau);
      kI[u] = I;
      kJ[u] = tau - I * (I + 1) / 2;
    }
    for (int R = 0; R < P.NBT; R++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        int lastI = -1;
        double afr = 0.0;
#pragma unroll
        for (int u = 0; u < DPG_MAX_KT; u++) {
          if (u < nkw) {
            if (kI[u] != lastI) { afr = WT[(kI[u] * P.NBT + R) * 64 + h * 32 + lane]; lastI = kI[u]; }
            double bfr = WT[(kJ[u] * P.NBT + R) * 64 + h * 32 + lane];
            dmma(kacc[u], afr, bfr);
          }
        }
      }
    }
    __syncthreads();
    double* KT = sm + P.sm_k;
#pragma unroll
    for (int u = 0; u < DPG_MAX_KT; u++)
      if (u < nkw) *reinterpret_cast<double2*>(KT + (k0 + u) * 64 + ak_cfrag(g, t)) = kacc[u];
    __syncthreads();
  }
  double* KT = sm + P.sm_k;
  // K and l out (user numbering; fields first: dev = i for i < nf, nfp + (i - nf) otherwise)
  if (L.K) {
    double* Kc = L.K + (size_t)cell * P.M * P.M;
    for (int e = tid; e < P.M * P.M; e += NT) {
      int i = e / P.M, j = e - i * P.M;
      int di = i < P.nf ? i : P.nfp + (i - P.nf);
      int dj = j < P.nf ? j : P.nfp + (j - P.nf);
      Kc[e] = sym_get(KT, di, dj);
    }
    double* lc = L.l + (size_t)cell * P.M;
    for (int i = tid; i < P.M; i += NT) {
      int di = i < P.nf ? i : P.nfp + (i - P.nf);
      lc[i] = sym_get(KT, P.fcol, di);
    }
  }
  // ======================= 6. condensation ===================================
  if (L.S && P.nfb > 0 && P.nt > 0) {
    __syncthreads();
    for (int r = P.nf + tid; r < P.nfp; r += NT) {
      int I = r >> 3;
      KT[(I * (I + 1) / 2 + I) * 64 + ak(r & 7, r & 7)] = 1.0;
    }
    __syncthreads();
    tile_cholesky(KT, P.MBT, P.nfb, flag_s + 1, -1);
    double* Sc = L.S + (size_t)cell * P.nt * P.nt;
    for (int e = tid; e < P.nt * P.nt; e += NT) {
      int i = e / P.nt, j = e - i * P.nt;
      Sc[e] = sym_get(KT, P.nfp + i, P.nfp + j);
    }
    double* sc = L.s + (size_t)cell * P.nt;
    for (int i = tid; i < P.nt; i += NT) sc[i] = sym_get(KT, P.fcol, P.nfp + i);
  } else if (L.S && P.nt > 0) {
    double* Sc = L.S + (size_t)cell * P.nt * P.nt;
    for (int e = tid; e < P.nt * P.nt; e += NT) {
      int i = e / P.nt, j = e - i * P.nt;
      Sc[e] = sym_get(KT, P.nfp + i, P.nfp + j);
    }
    double* sc = L.s + (size_t)cell * P.nt;
    for (int i = tid; i < P.nt; i += NT) sc[i] = sym_get(KT, P.fcol, P.nfp + i);
  }
  __syncthreads();
  if (tid == 0 && L.info) {
    int f0 = flag_s[0], f1 = flag_s[1];
    int v = 0;
    if (f0 != 0) {
      // device test row -> user test index (1-based)
      int r = f0 - 1;
      int u = L.solve_only ? r : P.dev2user_test[r];
      v = (u >= 0 ? u : r) + 1;
    } else if (f1 != 0) {
      v = f1;
    }
    L.info[cell] = v;
  }
}

}  // namespace

int dpg_configure_kernels(const DpgPlanDev* plan) {
  size_t bytes = (size_t)plan->sm_total * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(dpg_cell_kernel<DPG_MAX_NBT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)bytes);
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  return DPG_OK;
}

int dpg_launch_assemble(const DpgPlanDev* plan, const DpgPlanDev* d_plan, const DpgLaunch* L, cudaStream_t stream) {
  (void)d_plan;
  if (L->C <= 0) return DPG_OK;
  size_t bytes = (size_t)plan->sm_total * sizeof(double);
  dpg_cell_kernel<DPG_MAX_NBT><<<L->C, NT, bytes, stream>>>(*plan, *L);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}
