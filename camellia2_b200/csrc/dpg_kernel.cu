// dpg_kernel.cu — fused FP64 per-cell DPG assembly for sm_100a.
//
// Persistent CTAs (16 warps, one per SM) walk the cells.  Per cell:
//   1. B and F (TBF::stiffnessMatrix, BF.cpp:575-656; RHS.cpp:68-82).  Volume: the
//      per-point records (reference slots of the test bases plus each term's trial
//      values) arrive by bulk (TMA) copy, double buffered; U = (weight x coefficient
//      x Piola row) x trial value per active (test var, column tile) block, and each
//      warp accumulates its 16x8 blocks with mma.m16n8k16.f64 over k-steps of 4
//      points x 4 slots.  Boundary terms with a cell-independent side transform
//      (HGRAD value; HDIV normal trace by the Piola identity) are separable: compact
//      per-entry sums over the test rows nonzero on the side.  The tiles wait in a
//      per-CTA scratch slot (L2-resident).
//   2. Gram matrix G (IP::computeInnerProductMatrix, IP.cpp:215-292): the same slot
//      form; per point and coupled test-var pair a 4x4 coupling D = T_a^T C T_b (C:
//      graph-norm coefficients, T: Piola maps), h = D x slots by DMMA per chunk, and
//      each warp accumulates its 16x8 blocks of the lower triangle (m16n8k16).
//   3. Equilibrated Cholesky of G (BF.cpp:944-982: DPOEQU scaling, DPOTRF('L'),
//      unscaling), blocked right-looking with look-ahead on 8x8 tiles in shared memory.
//   4. W = L^-1 [B | F] in registers (BF.cpp:987-988, 1013-1014): each warp runs a
//      blocked forward substitution on its own column tile; diagonal blocks use
//      precomputed inverses, row pairs update with mma.m16n8k8.f64.
//   5. K_ext = W^T W (DSYRK, BF.cpp:993-1005) including l = W^T y (BF.cpp:1016).
//   6. Static condensation (CondensedDofInterpreter.cpp:1138-1192): the first
//      field-tile steps of a blocked Cholesky of K_ext leave the Schur complement
//      [S s; s^T .] in the trailing block.
// Numerical failures are reported per cell in info (DPOTRF INFO semantics).  The
// reverse mode, the energy error and the multi-bucket launch reuse these phases.
#include "../../include/dpg_b200.h"
#include "dpg_internal.h"
#include "dpg_plan.h"

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

// The CTA's dynamic shared memory; every shared pointer below is derived from it
// so the compiler keeps shared-space (LDS/STS) addressing inside the phase functions.
extern __shared__ __align__(128) double dpg_smem[];

namespace {

constexpr int NT = DPG_NTHREADS;
constexpr int MBAR_SPIN_LIMIT = 1 << 22;
constexpr int ERR_TIMEOUT_FLAG = 0x7fff0000;
constexpr int GEO = 24;  // doubles per point geometry record: J(9) Ji(9) det w*|J| n(3) 1/det

__device__ __forceinline__ void dmma(double2& c, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c.x), "+d"(c.y)
               : "d"(a), "d"(b));
}

// D(16x8) += A(16x16) B(16x8), FP64.  Fragments: a[2i] = A[g][t+4i], a[2i+1] = A[g+8][t+4i],
// b[i] = B[t+4i][g]; c = {C[g][2t], C[g][2t+1], C[g+8][2t], C[g+8][2t+1]}.
__device__ __forceinline__ void dmma16(double* c, const double* a, const double* b) {
  asm("mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// D(16x8) += A(16x8) * B(8x8): a0 = A[g][t], a1 = A[g+8][t], a2 = A[g][t+4], a3 = A[g+8][t+4];
// b0 = B[t][g], b1 = B[t+4][g]; c_lo holds rows g, c_hi rows g+8 (columns 2t, 2t+1 each).
__device__ __forceinline__ void dmma16x8(double2& c_lo, double2& c_hi, double a0, double a1, double a2, double a3,
                                         double b0, double b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(c_lo.x), "+d"(c_lo.y), "+d"(c_hi.x), "+d"(c_hi.y)
      : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

// Global -> shared bulk copy completing on an mbarrier (16-byte aligned, bytes % 16 == 0).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(b))
               : "memory");
}

// Bounded wait on an mbarrier phase; false if the limit was reached.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, int limit = MBAR_SPIN_LIMIT) {
  for (int it = 0; it < limit; it++) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// AK layout index of element (r, c) of an 8x8 tile
__device__ __forceinline__ int ak(int r, int c) { return ((c >> 2) * 8 + r) * 4 + (c & 3); }

// Offset of the C-fragment pair (g, 2t..2t+1) in AK layout
__device__ __forceinline__ int ak_cfrag(int g, int t) { return ((t >> 1) * 8 + g) * 4 + (t & 1) * 2; }

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

// Geometry record of one point: Jacobian, inverse, determinant, weighted
// measure (w*detJ, or w*|side Jacobian| when tang != nullptr) and, on a side,
// the outward unit normal.  All vertex-shape derivatives are loaded up front.
__device__ __forceinline__ void point_geometry(int d, int nv, const double* __restrict__ X,
                                               const double* __restrict__ dN, double w,
                                               const double* __restrict__ tang, double* gq) {
  double dn[24];
#pragma unroll
  for (int i = 0; i < 24; i++) dn[i] = (i < nv * d) ? __ldg(dN + i) : 0.0;
  double tg[6];
  if (tang) {
#pragma unroll
    for (int i = 0; i < 6; i++) tg[i] = __ldg(tang + i);
  }
  double J[9];
#pragma unroll
  for (int i = 0; i < 9; i++) J[i] = 0.0;
  if (d == 3) {
#pragma unroll
    for (int a = 0; a < 8; a++) {
      if (a < nv) {
#pragma unroll
        for (int i = 0; i < 3; i++) {
          double xa = X[a * 3 + i];
#pragma unroll
          for (int j = 0; j < 3; j++) J[i * 3 + j] += xa * dn[a * 3 + j];
        }
      }
    }
  } else {
#pragma unroll
    for (int a = 0; a < 4; a++) {
      if (a < nv) {
#pragma unroll
        for (int i = 0; i < 2; i++) {
          double xa = X[a * 2 + i];
#pragma unroll
          for (int j = 0; j < 2; j++) J[i * 3 + j] += xa * dn[a * 2 + j];
        }
      }
    }
  }
  double Ji[9], det;
  if (d == 2) {
    det = J[0] * J[4] - J[1] * J[3];
    double id = 1.0 / det;
    Ji[0] = J[4] * id; Ji[1] = -J[1] * id; Ji[2] = 0;
    Ji[3] = -J[3] * id; Ji[4] = J[0] * id; Ji[5] = 0;
    Ji[6] = 0; Ji[7] = 0; Ji[8] = 1;
  } else {
    double c00 = J[4] * J[8] - J[5] * J[7];
    double c01 = J[5] * J[6] - J[3] * J[8];
    double c02 = J[3] * J[7] - J[4] * J[6];
    det = J[0] * c00 + J[1] * c01 + J[2] * c02;
    double id = 1.0 / det;
    Ji[0] = c00 * id;
    Ji[3] = c01 * id;
    Ji[6] = c02 * id;
    Ji[1] = (J[2] * J[7] - J[1] * J[8]) * id;
    Ji[4] = (J[0] * J[8] - J[2] * J[6]) * id;
    Ji[7] = (J[1] * J[6] - J[0] * J[7]) * id;
    Ji[2] = (J[1] * J[5] - J[2] * J[4]) * id;
    Ji[5] = (J[2] * J[3] - J[0] * J[5]) * id;
    Ji[8] = (J[0] * J[4] - J[1] * J[3]) * id;
  }
#pragma unroll
  for (int i = 0; i < 9; i++) { gq[i] = J[i]; gq[9 + i] = Ji[i]; }
  gq[18] = det;
  gq[23] = 1.0 / det;
  gq[20] = gq[21] = gq[22] = 0.0;
  if (!tang) {
    gq[19] = w * det;
    return;
  }
  double T0[3] = {0, 0, 0}, T1[3] = {0, 0, 0};
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      T0[i] += J[i * 3 + j] * tg[j];
      T1[i] += J[i * 3 + j] * tg[3 + j];
    }
  double meas;
  if (d == 2) {
    meas = sqrt(T0[0] * T0[0] + T0[1] * T0[1]);
    gq[20] = T0[1] / meas;
    gq[21] = -T0[0] / meas;
  } else {
    double c0 = T0[1] * T1[2] - T0[2] * T1[1];
    double c1 = T0[2] * T1[0] - T0[0] * T1[2];
    double c2 = T0[0] * T1[1] - T0[1] * T1[0];
    meas = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
    gq[20] = c0 / meas; gq[21] = c1 / meas; gq[22] = c2 / meas;
  }
  gq[19] = w * meas;
}

// Row `m` of the slot transform T of a test var at a point: physical value of
// the operator in physical slot m = sum_k T[m][k] * reference slot k.
//   HGRAD slots (value, d/dx_0..): T[0][0] = 1, T[1+c][1+j] = Ji[j][c]
//   HDIV  slots (v_0.., div):      T[c][j] = J[c][j]/det, T[d][d] = 1/det
__device__ __forceinline__ void trow_slot(int space, int d, int m, const double* gq, double* r) {
  r[0] = r[1] = r[2] = r[3] = 0.0;
  if (space == DPG_SPACE_HGRAD) {
    if (m == 0) r[0] = 1.0;
    else if (m <= d) {
      int c = m - 1;
      for (int j = 0; j < d; j++) r[1 + j] = gq[9 + j * 3 + c];
    }
  } else {
    const double id = gq[23];
    if (m < d) {
      for (int j = 0; j < d; j++) r[j] = gq[m * 3 + j] * id;
    } else if (m == d) {
      r[d] = id;
    }
  }
}

// Row of T for a physical operator (incl. tau . n on a side; normal at gq[20..22]).
__device__ __forceinline__ void trow_op(int space, int d, int op, const double* gq, double* r) {
  if (space == DPG_SPACE_HGRAD) {
    trow_slot(space, d, op == DPG_OP_VALUE ? 0 : 1 + (op - DPG_OP_DX), gq, r);
    return;
  }
  if (op == DPG_OP_DOT_NORMAL) {
    const double id = gq[23];
    r[0] = r[1] = r[2] = r[3] = 0.0;
    for (int c = 0; c < d; c++)
      for (int j = 0; j < d; j++) r[j] += gq[20 + c] * gq[c * 3 + j] * id;
    return;
  }
  trow_slot(space, d, op == DPG_OP_DIV ? d : op - DPG_OP_X, gq, r);
}

// Element (r, c) of the symmetric matrix stored as lower AK tiles at base.
__device__ __forceinline__ double sym_get(const double* base, int r, int c) {
  if (r < c) { int x = r; r = c; c = x; }
  int I = r >> 3, J = c >> 3;
  return base[(I * (I + 1) / 2 + J) * 64 + ak(r & 7, c & 7)];
}

struct Ctx {
  uint32_t* phase;     // mbarrier use counters [4]
};

// Shared-memory views of the persistent region (derived from dpg_smem).
#define DPG_SMEM_VIEWS(P)                                                              \
  double* const sm = dpg_smem;                                                         \
  int* const flag_s = reinterpret_cast<int*>(sm + (P).sm_nodes + 24);                  \
  uint64_t* const mbar_s = reinterpret_cast<uint64_t*>(sm + (P).sm_nodes + 26);        \
  const int* const tri_s = reinterpret_cast<const int*>(sm + (P).sm_nodes + 32);       \
  const double* const nodes_s = sm + (P).sm_nodes;                                     \
  const double* const coef_s = sm + (P).sm_coef;                                       \
  double* const invd_s = sm + (P).sm_invd;                                             \
  (void)flag_s; (void)mbar_s; (void)tri_s; (void)nodes_s; (void)coef_s; (void)invd_s;

// Factor the diagonal tile k in place (one warp).  Every lane loads the lower triangle and
// runs the whole factorisation in its own registers, so the pivot chain is eight reciprocal
// square roots, each followed by one multiply and one FMA, with no shuffle on it; then lane
// c < 8 forms column c of the inverse tile L_kk^-1 from the same registers.  Records
// 1 / L_jj in invd[8k + j] and the inverse tile (AK layout) in linv[64 k].  First failing
// pivot (1-based) -> *flag (sign sgn).
__device__ __forceinline__ void factor_diag(double* __restrict__ T, int k, int* flag, int sgn, double* invd,
                                            double* linv) {
  const int lane = threadIdx.x & 31;
  double* Tkk = T + (k * (k + 1) / 2 + k) * 64;
  double a[36];  // a[r (r + 1) / 2 + c], c <= r
#pragma unroll
  for (int r = 0; r < 8; r++)
#pragma unroll
    for (int c = 0; c <= r; c++) a[r * (r + 1) / 2 + c] = Tkk[ak(r, c)];
  double iv[8];
  bool failed = false;
  int fail_j = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const double piv = a[j * (j + 1) / 2 + j];
    if (!(piv > 0.0) && !failed) { failed = true; fail_j = j; }
    const double inv = rsqrt(piv);
    iv[j] = inv;
    a[j * (j + 1) / 2 + j] = piv * inv;
#pragma unroll
    for (int r = j + 1; r < 8; r++) a[r * (r + 1) / 2 + j] *= inv;
#pragma unroll
    for (int c = j + 1; c < 8; c++)
#pragma unroll
      for (int r = c; r < 8; r++) a[r * (r + 1) / 2 + c] -= a[r * (r + 1) / 2 + j] * a[c * (c + 1) / 2 + j];
  }
  __syncwarp();
  if (lane == 0) {
    // row r, columns 4q .. 4q+3 are contiguous in the AK layout
#pragma unroll
    for (int r = 0; r < 8; r++)
#pragma unroll
      for (int q = 0; q < 2; q++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int c0 = 4 * q + 2 * h;
          const double v0 = (c0 <= r) ? a[r * (r + 1) / 2 + c0] : 0.0;
          const double v1 = (c0 + 1 <= r) ? a[r * (r + 1) / 2 + c0 + 1] : 0.0;
          *reinterpret_cast<double2*>(Tkk + (q * 8 + r) * 4 + 2 * h) = make_double2(v0, v1);
        }
#pragma unroll
    for (int j = 0; j < 8; j += 2) *reinterpret_cast<double2*>(invd + k * 8 + j) = make_double2(iv[j], iv[j + 1]);
    if (failed && *flag == 0) *flag = sgn * (k * 8 + fail_j + 1);
  }
  // column c of L_kk^-1 by forward substitution (lane c)
  const int c = lane & 7;
  double x[8];
#pragma unroll
  for (int rr = 0; rr < 8; rr++) {
    double v = (rr == c) ? 1.0 : 0.0;
#pragma unroll
    for (int m = 0; m < rr; m++) v -= a[rr * (rr + 1) / 2 + m] * x[m];
    x[rr] = (rr < c) ? 0.0 : v * iv[rr];
  }
  if (lane < 8) {
#pragma unroll
    for (int rr = 0; rr < 8; rr++) linv[k * 64 + ak(rr, c)] = x[rr];
  }
  __syncwarp();
}

// Blocked right-looking Cholesky of the leading nsteps tiles of a tile-lower
// matrix with nb tiles in shared memory (AK tiles).  Look-ahead: while the warps
// of sub-partitions 1..3 apply the trailing update of step k, warp 0 updates diagonal
// tile k+1 first and factors it, so each step costs two barriers (warp 0 only arrives
// at the first).  The panel multiplies by
// the inverse diagonal tile (two DMMAs per tile).  linv (NBT x 64) receives the
// inverses of the factored diagonal tiles; invd the inverse pivots.
__device__ __noinline__ void tile_cholesky(int T_off, int nb, int nsteps, int flag_idx, int sgn, int tri_off,
                                           int invd_off, int linv_off) {
  double* const T = dpg_smem + T_off;
  int* const flag = reinterpret_cast<int*>(dpg_smem) + flag_idx;
  const int* const tri = reinterpret_cast<const int*>(dpg_smem + tri_off);
  double* const invd = dpg_smem + invd_off;
  double* const linv = dpg_smem + linv_off;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  if (nsteps <= 0) return;
  if (warp == 0) factor_diag(T, 0, flag, sgn, invd, linv);
  __syncthreads();
  for (int k = 0; k < nsteps; k++) {
    // panel: L_ik = A_ik L_kk^-T
    const double* Li = linv + k * 64;
    for (int i = k + 1 + warp; i < nb; i += DPG_NWARPS) {
      double* Tik = T + (i * (i + 1) / 2 + k) * 64;
      const double a0 = Tik[lane], a1 = Tik[32 + lane];
      double2 c = make_double2(0.0, 0.0);
      dmma(c, a0, Li[lane]);
      dmma(c, a1, Li[32 + lane]);
      __syncwarp();
      *reinterpret_cast<double2*>(Tik + ak_cfrag(g, t)) = c;
    }
    // warp 0 needs only its own panel tile (k+1, k) for what follows, so it signals the
    // barrier without waiting at it; the other warps wait for every panel tile
    if (warp == 0) {
      asm volatile("bar.arrive 1, %0;" ::"n"(NT) : "memory");
      __syncwarp();
    } else {
      asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
    }
    // trailing update: A_ij -= L_ik L_jk^T for k < j <= i < nb; warp 0 does (k+1, k+1) and factors it
    const int m = nb - 1 - k;
    const int ntr = m * (m + 1) / 2;
    if (warp == 0) {
      if (m > 0) {
        const int i = k + 1;
        double* Tii = T + (i * (i + 1) / 2 + i) * 64;
        const double* Lik = T + (i * (i + 1) / 2 + k) * 64;
        double2 c = *reinterpret_cast<const double2*>(Tii + ak_cfrag(g, t));
        dmma(c, -Lik[lane], Lik[lane]);
        dmma(c, -Lik[32 + lane], Lik[32 + lane]);
        *reinterpret_cast<double2*>(Tii + ak_cfrag(g, t)) = c;
        __syncwarp();
        if (k + 1 < nsteps) factor_diag(T, k + 1, flag, sgn, invd, linv);
      }
    } else if (warp & 3) {
      // the update runs on the other three sub-partitions' warps: warps 4, 8, 12 stay
      // idle so that warp 0's serial diagonal factorisation has its sub-partition (issue
      // slots) to itself; it is the critical path of every step
      // each warp takes a contiguous range of the row-major tile list, so consecutive
      // tiles share row i and L_ik stays in registers
      const int hidx = warp - (warp >> 2) - 1;
      const int nwt = DPG_NWARPS - DPG_NWARPS / 4;
      const int tb = (ntr - 1) / nwt, te = (ntr - 1) % nwt;
      const int u0 = 1 + hidx * tb + min(hidx, te), u1 = u0 + tb + (hidx < te ? 1 : 0);
      int lastI = -1;
      double a0 = 0.0, a1 = 0.0;
      for (int u = u0; u < u1; u++) {
        const int ij = tri[u];
        const int i = k + 1 + (ij & 255), j = k + 1 + (ij >> 8);
        double* Tij = T + (i * (i + 1) / 2 + j) * 64;
        if (i != lastI) {
          const double* Lik = T + (i * (i + 1) / 2 + k) * 64;
          a0 = -Lik[lane];
          a1 = -Lik[32 + lane];
          lastI = i;
        }
        const double* Ljk = T + (j * (j + 1) / 2 + k) * 64;
        double2 c = *reinterpret_cast<const double2*>(Tij + ak_cfrag(g, t));
        dmma(c, a0, Ljk[lane]);
        dmma(c, a1, Ljk[32 + lane]);
        *reinterpret_cast<double2*>(Tij + ak_cfrag(g, t)) = c;
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Phase 1: B and F -> per-CTA scratch (or the B/F outputs in parts mode)
// ---------------------------------------------------------------------------
template <int BTW>
__device__ __noinline__ void phase_b(const DpgPlanDev& P, const DpgLaunch& L, int cell, const Ctx& X) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int d = P.d, nv = P.nv;
  DPG_SMEM_VIEWS(P);
  double* geo = sm + P.b_geo;
  double* U = sm + P.b_u;
  const int8_t* par_c = L.parity + (size_t)cell * P.ns;
  double2* scr = reinterpret_cast<double2*>(L.scratch + (size_t)blockIdx.x * P.scratch_per_cta);
  // prologue: first chunk's records in flight while the geometry is computed
  int first_seg = 0;
  while (first_seg < P.nseg && P.seg[first_seg].nterm == 0) first_seg++;
  if (tid == 0 && first_seg < P.nseg) {
    const DpgSeg& S = P.seg[first_seg];
    const uint32_t bytes = (uint32_t)(((min(S.chunk, S.npts) + 3) & ~3) * S.rec_len * sizeof(double));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&mbar_s[2], bytes);
    bulk_g2s(sm + P.b_rec0, S.rec, bytes, &mbar_s[2]);
  }
  // [B | F] tiles accumulate in this CTA's scratch slot, C-fragment layout per tile
  for (int i = tid; i < P.MBT * P.NBT * 32; i += NT) scr[i] = make_double2(0.0, 0.0);
  for (int q = tid; q < P.nbpts; q += NT)
    point_geometry(d, nv, nodes_s, P.dNB + (size_t)q * nv * d, P.wB[q], q >= P.QB ? P.tangB + (size_t)q * 6 : nullptr,
                   geo + q * GEO);
  // separable side terms, while the first volume chunk is in flight: per-point factors,
  // then one thread per entry (scratch element); entries are unique, and an element
  // that a bilinear block also writes is read-modified-written (the blocks add to it
  // after the chunk loop's barriers)
  if (P.nse > 0) {
    double* fac = sm + P.b_fac;  // [nse][QS]
    __syncthreads();             // geometry complete, scratch zeroed
    for (int task = tid; task < P.nse * P.QS; task += NT) {
      const int se = task / P.QS, q = task - se * P.QS;
      const DpgSideTerm& E = P.se[se];
      const double* gq = geo + (P.QB + E.side * P.QS + q) * GEO;
      double v = E.coef;
      if (E.use_meas) v *= gq[19];
      if (E.slot >= 0) v *= coef_s[E.slot * P.Ptot + E.pbase + q];
      if (E.normal_comp >= 0) v *= gq[20 + E.normal_comp];
      if (E.flux) v *= (double)par_c[E.side];
      fac[task] = v;
    }
    __syncthreads();
    double* scd = reinterpret_cast<double*>(scr);
    for (int e = tid; e < P.nsent; e += NT) {
      const int4 en = __ldg(P.sent + e);
      double acc = 0.0;
      if (en.z == 1) {
        const double* f = fac + (en.w & 0xffff) * P.QS;
        const double* w = P.scon_w + en.y;
        for (int q = 0; q < P.QS; q++) acc += __ldg(w + (size_t)q * P.ncon) * f[q];
      } else {
        for (int c = en.y; c < en.y + en.z; c++) {
          const double* f = fac + __ldg(P.scon_se + c) * P.QS;
          for (int q = 0; q < P.QS; q++) acc += __ldg(P.scon_w + (size_t)q * P.ncon + c) * f[q];
        }
      }
      if (en.w >> 16) scd[en.x] = acc;
      else scd[en.x] += acc;
    }
  }
  int gc = 0;  // global chunk counter (buffer parity)
  for (int sgi = first_seg; sgi < P.nseg; sgi++) {
    const DpgSeg& S = P.seg[sgi];
    if (S.nterm == 0) continue;
    // this warp's active 16x8 blocks of the segment: operand offsets and accumulators
    const int bbase = S.ntile / DPG_NWARPS, bextra = S.ntile % DPG_NWARPS;
    const int my0 = S.tile0 + warp * bbase + min(warp, bextra);
    const int nmine = bbase + (warp < bextra ? 1 : 0);
    uint32_t pk[BTW];
    double acc[BTW][4];
#pragma unroll
    for (int u = 0; u < BTW; u++) {
      acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0;
      uint32_t v = 0;
      if (u < nmine) {
        const int4 td = P.btiles[my0 + u];
        const DpgBBlock& Bk = S.blk[td.z];
        const DpgTestVar& V = P.test[Bk.var];
        v = (uint32_t)(V.foff + t * V.ldA + (td.x - V.ntile0) * 8 + g) | ((uint32_t)(Bk.off + t * DPG_ULD + g) << 16);
      }
      pk[u] = v;
    }
    for (int c = 0; c < S.nchunk; c++, gc++) {
      const int buf = gc & 1;
      double* rec = sm + (buf ? P.b_rec1 : P.b_rec0);
      __syncthreads();  // the other buffer and U are free; geometry is complete
      if (tid == 0) {
        // prefetch the next chunk (this segment or the next one with terms)
        int ns = sgi, nc = c + 1;
        if (nc >= S.nchunk) {
          ns = sgi + 1;
          nc = 0;
          while (ns < P.nseg && P.seg[ns].nterm == 0) ns++;
        }
        if (ns < P.nseg) {
          const DpgSeg& S2 = P.seg[ns];
          // the records of the chunk's points, rounded up to a whole k-step (the table is padded)
          const uint32_t bytes =
              (uint32_t)(((min(S2.chunk, S2.npts - nc * S2.chunk) + 3) & ~3) * S2.rec_len * sizeof(double));
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_expect_tx(&mbar_s[2 + (buf ^ 1)], bytes);
          bulk_g2s(sm + (buf ? P.b_rec0 : P.b_rec1), S2.rec + (size_t)nc * S2.chunk * S2.rec_len, bytes,
                   &mbar_s[2 + (buf ^ 1)]);
        }
        if (!mbar_wait(&mbar_s[2 + buf], X.phase[2 + buf] & 1)) flag_s[2] = 1;
      }
      X.phase[2 + buf]++;
      const int q0 = c * S.chunk;
      const int nq = min(S.chunk, S.npts - q0);
      __syncthreads();
      // U blocks: U[lq][blk][m][col] = sum over the block's terms of
      //   (w*|J| * coef * slot * (n) * (parity) * T_op[m]) * trial value
      for (int task = tid; task < S.chunk * S.nblk * 8; task += NT) {
        const int lq = task / (S.nblk * 8);
        const int rem = task - lq * S.nblk * 8;
        const int kb = rem >> 3, cl = rem & 7;
        const DpgBBlock& Bk = S.blk[kb];
        const int col = Bk.J * 8 + cl;
        double u0 = 0.0, u1 = 0.0, u2 = 0.0, u3 = 0.0;
        if (lq < nq) {
          const int q = q0 + lq;
          const double* rq = rec + lq * S.rec_len;
          const double* gq = geo + (S.geo0 + q) * GEO;
          const int space = P.test[Bk.var].space;
          for (int i = 0; i < Bk.nt; i++) {
            const int lt = Bk.terms[i];
            const DpgBTerm& Tm = P.bterm[S.term0 + lt];
            const int mm = col - Tm.col0;
            if (mm < 0 || mm >= Tm.ncol) continue;
            double v = gq[19] * Tm.coef * rq[S.tvoff[lt] + mm];
            if (Tm.slot >= 0) v *= coef_s[Tm.slot * P.Ptot + S.pbase + q];
            if (Tm.normal_comp >= 0) v *= gq[20 + Tm.normal_comp];
            if (Tm.kind == DPG_VAR_FLUX) v *= (double)par_c[S.side];
            double tr[4];
            trow_op(space, d, Tm.test_op, gq, tr);
            u0 += tr[0] * v; u1 += tr[1] * v; u2 += tr[2] * v; u3 += tr[3] * v;
          }
        }
        double* uq = U + lq * S.ustride + Bk.off + cl;
        uq[0] = u0; uq[DPG_ULD] = u1; uq[2 * DPG_ULD] = u2; uq[3 * DPG_ULD] = u3;
      }
      __syncthreads();
      // DMMA over this warp's active blocks of the segment: m16n8k16, one k-step = 4 points x 4 slots
#pragma unroll 1
      for (int s4 = 0; s4 < nq; s4 += 4) {
        const double* ra = rec + s4 * S.rec_len;
        const double* ub = U + s4 * S.ustride;
        uint32_t prevA = 0xffffffffu;
        double av[8];
#pragma unroll
        for (int u = 0; u < BTW; u++) {
          if (u < nmine) {
            const uint32_t ao = pk[u] & 0xffffu, bo = pk[u] >> 16;
            if (ao != prevA) {
#pragma unroll
              for (int i = 0; i < 4; i++) {
                av[2 * i] = ra[i * S.rec_len + ao];
                av[2 * i + 1] = ra[i * S.rec_len + ao + 8];
              }
              prevA = ao;
            }
            double bv[4];
#pragma unroll
            for (int i = 0; i < 4; i++) bv[i] = ub[i * S.ustride + bo];
            dmma16(acc[u], av, bv);
          }
        }
      }
    }
    // segment contributions into the scratch tiles (each block has one owner per segment)
#pragma unroll
    for (int u = 0; u < BTW; u++) {
      if (u < nmine) {
        const int4 td = P.btiles[my0 + u];
        const int s0 = (td.y * P.NBT + td.x) * 32 + lane;
        double2 v0 = scr[s0], v1 = scr[s0 + 32];
        v0.x += acc[u][0]; v0.y += acc[u][1];
        v1.x += acc[u][2]; v1.y += acc[u][3];
        scr[s0] = v0;
        scr[s0 + 32] = v1;
      }
    }
  }
  if (!L.parts) return;
  __syncthreads();
  double* Bc = L.B ? L.B + (size_t)cell * P.M * P.N : nullptr;
  double* Fc = L.F ? L.F + (size_t)cell * P.N : nullptr;
  for (int tile = warp; tile < P.MBT * P.NBT; tile += DPG_NWARPS) {
    const int J = tile / P.NBT, I = tile - J * P.NBT;
    const double2 v = scr[tile * 32 + lane];
    const int ur = P.dev2user_test[I * 8 + g];
    if (ur < 0) continue;
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int col = J * 8 + 2 * t + e;
      const double x = e ? v.y : v.x;
      const int uc = P.dev2user_trial[col];
      if (Bc && uc >= 0) Bc[(size_t)uc * P.N + ur] = x;
      if (Fc && col == P.fcol) Fc[ur] = x;
    }
  }
}

// The Gram chunk loop for CH points per chunk (compile-time, so the h and DMMA loops
// unroll completely).
// Every P.gflush chunks (except after the last) each thread adds the accumulators of its
// flushed blocks (P.gflushbits) into its own running sums in gsum ([block][lane][4]; plain
// L2 loads and stores, one writer per element, so the order of additions is fixed) and
// restarts them from zero.
template <int GTM, int CH>
__device__ __forceinline__ void gram_chunks(const DpgPlanDev& P, const Ctx& X, const double* Dm, double* hb, int nunit,
                                            int ntw, const uint32_t (&pk)[GTM], double (&acc)[GTM][4],
                                            double* __restrict__ gsum) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  DPG_SMEM_VIEWS(P);
  const int nch = P.QGpad / CH;
  const uint32_t chunk_bytes = (uint32_t)(CH * P.featstride * sizeof(double));
  for (int c = 0; c < nch; c++) {
    const int buf = c & 1;
    const double* fref = sm + (buf ? P.g_fref1 : P.g_fref0);
    if (tid == 0) {
      if (c + 1 < nch) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&mbar_s[buf ^ 1], chunk_bytes);
        bulk_g2s(sm + (buf ? P.g_fref0 : P.g_fref1), P.frefG + (size_t)(c + 1) * CH * P.featstride,
                 chunk_bytes, &mbar_s[buf ^ 1]);
      }
      if (!mbar_wait(&mbar_s[buf], X.phase[buf] & 1)) flag_s[2] = 1;
    }
    X.phase[buf]++;
    __syncthreads();
    // h_{b->a}[q] = D_q (4x4, padded to 8 rows) * slots_b[q] (4 x 8 column tile): one DMMA per unit and point
    for (int un = warp; un < nunit; un += DPG_NWARPS) {
      int r = un, p = 0;
      while (r >= P.test[P.pair_b[p]].ntiles) { r -= P.test[P.pair_b[p]].ntiles; p++; }
      const int b = P.pair_b[p];
      const int ld = P.test[b].ldA;
      const double* dp = Dm + ((size_t)c * CH * P.npairs + p) * 16 + g * 4 + t;
      const double* fp = fref + P.test[b].foff + t * ld + r * 8 + g;
      double* hp = hb + P.hoff[p] + g * ld + r * 8 + 2 * t;
#pragma unroll
      for (int lq = 0; lq < CH; lq++) {
        const double av = (g < 4) ? dp[lq * P.npairs * 16] : 0.0;
        const double bv = fp[lq * P.featstride];
        double2 hc = make_double2(0.0, 0.0);
        dmma(hc, av, bv);
        if (g < 4) *reinterpret_cast<double2*>(hp + lq * P.hstride) = hc;
      }
    }
    __syncthreads();
    // m16n8k16 over the owned blocks: one k16 step = 4 points x 4 slots
#pragma unroll 1
    for (int s4 = 0; s4 < CH; s4 += 4) {
      const double* fa = fref + s4 * P.featstride;
      const double* hq = hb + s4 * P.hstride;
      uint32_t prevA = 0xffffffffu;
      double av[8];
#pragma unroll
      for (int u = 0; u < GTM; u++) {
        if (u < ntw) {
          const uint32_t ao = pk[u] & 0xffffu, bo = pk[u] >> 16;
          if (ao != prevA) {
#pragma unroll
            for (int i = 0; i < 4; i++) {
              av[2 * i] = fa[i * P.featstride + ao];
              av[2 * i + 1] = fa[i * P.featstride + ao + 8];
            }
            prevA = ao;
          }
          double bv[4];
#pragma unroll
          for (int i = 0; i < 4; i++) bv[i] = hq[i * P.hstride + bo];
          dmma16(acc[u], av, bv);
        }
      }
    }
    if (P.gflush > 0 && (c + 1) % P.gflush == 0 && c + 1 < nch) {
      const bool first = (c + 1) == P.gflush;
      const uint32_t fb = P.gflushbits[warp];
#pragma unroll
      for (int u = 0; u < GTM; u++) {
        if (u < ntw && ((fb >> u) & 1u)) {
          double2* sp = reinterpret_cast<double2*>(gsum + (u * 32 + lane) * 4);
          double2 lo = make_double2(acc[u][0], acc[u][1]), hi = make_double2(acc[u][2], acc[u][3]);
          if (!first) {
            const double2 a = __ldcg(sp), b = __ldcg(sp + 1);
            lo.x = a.x + lo.x; lo.y = a.y + lo.y; hi.x = b.x + hi.x; hi.y = b.y + hi.y;
          }
          __stcg(sp, lo);
          __stcg(sp + 1, hi);
          acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0;
        }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Phase 2: Gram matrix -> lower tiles in shared memory
// ---------------------------------------------------------------------------
template <int GTM, int CHG>
__device__ __forceinline__ void phase_gram(const DpgPlanDev& P, const DpgLaunch& L, int cell, const Ctx& X) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int d = P.d, nv = P.nv;
  DPG_SMEM_VIEWS(P);
  double* geo = sm + P.g_geo;
  double* Dm = sm + P.g_D;  // [q][pair][16]
  double* hb = sm + P.g_h;
  double* GT = sm + P.sm_gt;
  const uint32_t chunk_bytes = (uint32_t)(P.chg * P.featstride * sizeof(double));
  if (tid == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&mbar_s[0], chunk_bytes);
    bulk_g2s(sm + P.g_fref0, P.frefG, chunk_bytes, &mbar_s[0]);
  }
  for (int q = tid; q < P.QGpad; q += NT)
    point_geometry(d, nv, nodes_s, P.dNG + (size_t)q * nv * d, P.wG[q], nullptr, geo + q * GEO);
  __syncthreads();
  // beta_r,a[k] = sum over row-r entries on var a of coef * slot * T_a[slot_e][k]
  double* beta = sm + P.g_beta;  // [q][row][4 * ntest]
  const int F = 4 * P.ntest;
  for (int task = tid; task < P.QGpad * P.niprows * P.ntest; task += NT) {
    const int q = task / (P.niprows * P.ntest);
    const int rem = task - q * P.niprows * P.ntest;
    const int r = rem / P.ntest, a = rem - r * P.ntest;
    const double* gq = geo + q * GEO;
    double b0 = 0.0, b1 = 0.0, b2 = 0.0, b3 = 0.0;
    for (int e = P.rowstart[r]; e < P.rowstart[r + 1]; e++) {
      const DpgIPEnt& E = P.ipent[e];
      if ((E.gslot >> 2) != a) continue;
      double v = E.coef;
      if (E.slot >= 0) v *= (q < P.QG) ? coef_s[E.slot * P.Ptot + q] : 0.0;
      double tr[4];
      trow_slot(P.test[a].space, d, E.gslot & 3, gq, tr);
      b0 += v * tr[0]; b1 += v * tr[1]; b2 += v * tr[2]; b3 += v * tr[3];
    }
    double* dst = beta + (q * P.niprows + r) * F + 4 * a;
    dst[0] = b0; dst[1] = b1; dst[2] = b2; dst[3] = b3;
  }
  __syncthreads();
  // coupling D_ab[k][l] = wdet * sum_r beta_r,a[k] beta_r,b[l]
  for (int task = tid; task < P.QGpad * P.npairs * 16; task += NT) {
    const int q = task / (P.npairs * 16);
    const int rem = task - q * P.npairs * 16;
    const int p = rem >> 4, k = (rem >> 2) & 3, l = rem & 3;
    const double* bq = beta + q * P.niprows * F;
    const int ia = 4 * P.pair_a[p] + k, ib = 4 * P.pair_b[p] + l;
    double sacc = 0.0;
    for (int r = 0; r < P.niprows; r++) sacc += bq[r * F + ia] * bq[r * F + ib];
    Dm[task] = sacc * geo[q * GEO + 19];
  }
  // owned 16x8 blocks: packed per-thread operand offsets (A | B << 16)
  // balanced: warps 0 .. extra-1 take one block more, so the four SM sub-partitions
  // (warps w, w+4, w+8, w+12) carry equal tensor work
  const int gbase = P.ngb / DPG_NWARPS, gextra = P.ngb % DPG_NWARPS;
  const int ntw = gbase + (warp < gextra ? 1 : 0);
  const int tau0 = warp * gbase + min(warp, gextra);
  const int4* tdesc = reinterpret_cast<const int4*>(sm + P.sm_tiles) + tau0;
  uint32_t pk[GTM];
  double acc[GTM][4];
#pragma unroll
  for (int u = 0; u < GTM; u++) {
    acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0;
    uint32_t v = 0;
    if (u < ntw) {
      const int4 T = tdesc[u];
      v = (uint32_t)(T.z + t * (T.y & 0xffff) + g) | ((uint32_t)(T.w + t * (T.y >> 16) + g) << 16);
    }
    pk[u] = v;
  }
  // h work units per point: (pair, column tile of the pair's second var); warp w takes
  // units w, w + 16, ... for every point of the chunk
  int nunit = 0;
  for (int p = 0; p < P.npairs; p++) nunit += P.test[P.pair_b[p]].ntiles;
  __syncthreads();
  double* gsum = L.scratch + (size_t)blockIdx.x * P.scratch_per_cta + P.gsum_off + (size_t)tau0 * 128;
  if (CHG != 0) gram_chunks<GTM, CHG != 0 ? CHG : DPG_CHG>(P, X, Dm, hb, nunit, ntw, pk, acc, gsum);
  else if (P.chg == DPG_CHG) gram_chunks<GTM, DPG_CHG>(P, X, Dm, hb, nunit, ntw, pk, acc, gsum);
  else gram_chunks<GTM, DPG_CHG / 2>(P, X, Dm, hb, nunit, ntw, pk, acc, gsum);
  if (P.gflush > 0 && P.gflush < P.QGpad / P.chg) {  // the last group joins the running sums
    const uint32_t fb = P.gflushbits[warp];
#pragma unroll
    for (int u = 0; u < GTM; u++) {
      if (u < ntw && ((fb >> u) & 1u)) {
        const double2* sp = reinterpret_cast<const double2*>(gsum + (u * 32 + lane) * 4);
        const double2 a = __ldcg(sp), b = __ldcg(sp + 1);
        acc[u][0] = a.x + acc[u][0]; acc[u][1] = a.y + acc[u][1];
        acc[u][2] = b.x + acc[u][2]; acc[u][3] = b.y + acc[u][3];
      }
    }
  }
  // accumulators -> tile-lower shared storage (overlaps the staging area); tiles of
  // uncoupled var pairs are zero
  for (int e = tid; e < P.ngz * 64; e += NT) GT[P.gzero[e >> 6] * 64 + (e & 63)] = 0.0;
#pragma unroll
  for (int u = 0; u < GTM; u++) {
    if (u < ntw) {
      const int4 T = tdesc[u];
      const int I = T.x & 0xffff, J = T.x >> 16;
      if (J <= I)
        *reinterpret_cast<double2*>(GT + (I * (I + 1) / 2 + J) * 64 + ak_cfrag(g, t)) = make_double2(acc[u][0], acc[u][1]);
      *reinterpret_cast<double2*>(GT + ((I + 1) * (I + 2) / 2 + J) * 64 + ak_cfrag(g, t)) =
          make_double2(acc[u][2], acc[u][3]);
    }
  }
  __syncthreads();
  // padded rows decouple: unit diagonal
  for (int r = tid; r < P.Np; r += NT)
    if (P.dev2user_test[r] < 0) GT[((r >> 3) * ((r >> 3) + 1) / 2 + (r >> 3)) * 64 + ak(r & 7, r & 7)] = 1.0;
  __syncthreads();
  if (L.parts && L.G) {
    double* Gc = L.G + (size_t)cell * P.N * P.N;
    for (int e = tid; e < P.Np * P.Np; e += NT) {
      int r = e / P.Np, c2 = e - r * P.Np;
      int ur = P.dev2user_test[r], uc = P.dev2user_test[c2];
      if (ur >= 0 && uc >= 0) Gc[(size_t)ur * P.N + uc] = sym_get(GT, r, c2);
    }
  }
}

// ---------------------------------------------------------------------------
// Phase 3: equilibrated Cholesky of G and inverses of its diagonal tiles
// ---------------------------------------------------------------------------
__device__ __forceinline__ void phase_factor(const DpgPlanDev& P, const Ctx& X) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  DPG_SMEM_VIEWS(P);
  double* GT = sm + P.sm_gt;
  double* scale = sm + P.sm_scale;
  double* LINV = sm + P.sm_linv;
  for (int r = tid; r < P.Np; r += NT) {
    int I = r >> 3;
    double dg = GT[(I * (I + 1) / 2 + I) * 64 + ak(r & 7, r & 7)];
    scale[r] = (dg > 0.0) ? rsqrt(dg) : 1.0;
  }
  __syncthreads();
  for (int u = warp; u < P.ngt; u += DPG_NWARPS) {
    int ij = tri_s[u];
    int I = ij & 255, J = ij >> 8;
    double2* p = reinterpret_cast<double2*>(GT + u * 64 + ak_cfrag(g, t));
    double si = scale[I * 8 + g];
    double2 v = *p;
    v.x *= si * scale[J * 8 + 2 * t];
    v.y *= si * scale[J * 8 + 2 * t + 1];
    *p = v;
  }
  __syncthreads();
  tile_cholesky(P.sm_gt, P.NBT, P.NBT, 2 * (P.sm_nodes + 24), 1, P.sm_nodes + 32, P.sm_invd, P.sm_linv);
  // unscale: L = S^-1 Ls  (rows / s_i);  1 / L_ii = s_i / Ls_ii;  L_kk^-1 = Ls_kk^-1 S_k (columns * s_c)
  for (int u = warp; u < P.ngt; u += DPG_NWARPS) {
    int I = tri_s[u] & 255;
    double2* p = reinterpret_cast<double2*>(GT + u * 64 + ak_cfrag(g, t));
    double si = 1.0 / scale[I * 8 + g];
    double2 v = *p;
    v.x *= si;
    v.y *= si;
    *p = v;
  }
  for (int r = tid; r < P.Np; r += NT) invd_s[r] *= scale[r];
  for (int e = tid; e < P.NBT * 64; e += NT) {
    const int k = e >> 6, idx = e & 63;
    const int c = (idx >> 5) * 4 + (idx & 3);
    LINV[e] *= scale[k * 8 + c];
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Phase 4: W = L^-1 [B | F] per column tile in registers, W^T tiles to smem
// ---------------------------------------------------------------------------
template <int NBTM>
__device__ __forceinline__ void phase_trsm(const DpgPlanDev& P, const DpgLaunch& L, int cell, const Ctx& X) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  DPG_SMEM_VIEWS(P);
  const double* GT = sm + P.sm_gt;
  const double* LINV = sm + P.sm_linv;
  const int J = warp;
  const bool has_col = J < P.MBT;
  double2 bacc[NBTM];
#pragma unroll
  for (int i = 0; i < NBTM; i++) bacc[i] = make_double2(0.0, 0.0);
  if (has_col) {
    if (L.solve_only) {
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
    } else {
      const double2* scr = reinterpret_cast<const double2*>(L.scratch + (size_t)blockIdx.x * P.scratch_per_cta) +
                           (size_t)J * P.NBT * 32 + lane;
#pragma unroll
      for (int I = 0; I < NBTM; I++)
        if (I < P.NBT) bacc[I] = scr[I * 32];
    }
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
        // rows i, i+1 together: one m16n8k8 on the stacked tiles [L_ik; L_i+1,k]
#pragma unroll
        for (int i = k + 1; i < NBTM; i += 2) {
          const double* Lik = GT + (i * (i + 1) / 2 + k) * 64;
          if (i + 1 < NBTM && i + 1 < P.NBT) {
            const double* Li1k = GT + ((i + 1) * (i + 2) / 2 + k) * 64;
            dmma16x8(bacc[i], bacc[i + 1], Lik[lane], Li1k[lane], Lik[32 + lane], Li1k[32 + lane], x0, x1);
          } else if (i < P.NBT) {
            dmma(bacc[i], Lik[lane], x0);
            dmma(bacc[i], Lik[32 + lane], x1);
          }
        }
      }
    }
  }
  __syncthreads();
  // W^T tiles (trial J, test I) in AK layout (overlaps L: all warps are done with it)
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
}

// ---------------------------------------------------------------------------
// Phase 5/6: K_ext = W^T W, outputs, condensation
// ---------------------------------------------------------------------------
__device__ __forceinline__ void phase_syrk_out(const DpgPlanDev& P, const DpgLaunch& L, int cell, const Ctx& X) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  DPG_SMEM_VIEWS(P);
  const double* WT = sm + P.sm_w;
  double* KT = sm + P.sm_k;
  {
    const int nk = P.MBT * (P.MBT + 1) / 2;
    const int kbase = nk / DPG_NWARPS, kextra = nk % DPG_NWARPS;
    const int k0 = warp * kbase + min(warp, kextra);
    const int nkw = kbase + (warp < kextra ? 1 : 0);
    double2 kacc[DPG_MAX_KT];
    int kI[DPG_MAX_KT], kJ[DPG_MAX_KT];
#pragma unroll
    for (int u = 0; u < DPG_MAX_KT; u++) {
      kacc[u] = make_double2(0.0, 0.0);
      int ij = (u < nkw) ? tri_s[k0 + u] : 0;
      kI[u] = ij & 255;
      kJ[u] = ij >> 8;
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
#pragma unroll
    for (int u = 0; u < DPG_MAX_KT; u++)
      if (u < nkw) *reinterpret_cast<double2*>(KT + (k0 + u) * 64 + ak_cfrag(g, t)) = kacc[u];
    __syncthreads();
  }
  // K and l out (user numbering; fields first: dev = i for i < nf, nfp + (i - nf) otherwise);
  // streaming stores, so the outputs do not evict the CTA's scratch slot from L2
  if (L.K) {
    double* Kc = L.K + (size_t)cell * P.M * P.M;
    for (int i = warp; i < P.M; i += DPG_NWARPS) {
      const int di = i < P.nf ? i : P.nfp + (i - P.nf);
      for (int j = lane; j < P.M; j += 32) {
        const int dj = j < P.nf ? j : P.nfp + (j - P.nf);
        __stcs(&Kc[(size_t)i * P.M + j], sym_get(KT, di, dj));
      }
    }
    double* lc = L.l + (size_t)cell * P.M;
    for (int i = tid; i < P.M; i += NT) {
      int di = i < P.nf ? i : P.nfp + (i - P.nf);
      __stcs(&lc[i], sym_get(KT, P.fcol, di));
    }
  }
  if (L.S && P.nt > 0) {
    if (P.nfb > 0) {
      __syncthreads();
      for (int r = P.nf + tid; r < P.nfp; r += NT) {
        int I = r >> 3;
        KT[(I * (I + 1) / 2 + I) * 64 + ak(r & 7, r & 7)] = 1.0;
      }
      __syncthreads();
      tile_cholesky(P.sm_k, P.MBT, P.nfb, 2 * (P.sm_nodes + 24) + 1, -1, P.sm_nodes + 32, P.sm_invd, P.sm_linv);
    }
    double* Sc = L.S + (size_t)cell * P.nt * P.nt;
    for (int i = warp; i < P.nt; i += DPG_NWARPS)
      for (int j = lane; j < P.nt; j += 32) __stcs(&Sc[(size_t)i * P.nt + j], sym_get(KT, P.nfp + i, P.nfp + j));
    double* sc = L.s + (size_t)cell * P.nt;
    for (int i = tid; i < P.nt; i += NT) __stcs(&sc[i], sym_get(KT, P.fcol, P.nfp + i));
  }
}

template <int NBTM, int GTM, int BTW, int CHG>
__global__ void __launch_bounds__(NT, 1) dpg_cell_kernel(const __grid_constant__ DpgPlanDev P, const DpgLaunch L) {
  const int tid = threadIdx.x;
  Ctx X;
  double* const sm = dpg_smem;
  double* nodes_s = sm + P.sm_nodes;
  int* flag_s = reinterpret_cast<int*>(sm + P.sm_nodes + 24);
  uint64_t* mbar_s = reinterpret_cast<uint64_t*>(sm + P.sm_nodes + 26);
  int* tri_s = reinterpret_cast<int*>(sm + P.sm_nodes + 32);
  DpgGTile* tiles_s = reinterpret_cast<DpgGTile*>(sm + P.sm_tiles);
  double* coef_s = sm + P.sm_coef;
  uint32_t phase[4] = {0, 0, 0, 0};
  X.phase = phase;

  // per-CTA set-up: triangular index table, tile table, mbarriers
  const int ntri = DPG_MAX_NBT * (DPG_MAX_NBT + 1) / 2;
  for (int u = tid; u < ntri; u += NT) {
    int I = (int)((sqrt(8.0 * u + 1.0) - 1.0) * 0.5);
    while ((I + 1) * (I + 2) / 2 <= u) I++;
    while (I * (I + 1) / 2 > u) I--;
    tri_s[u] = I | ((u - I * (I + 1) / 2) << 8);
  }
  if (!L.solve_only)
    for (int u = tid; u < P.ngb; u += NT) tiles_s[u] = P.gtiles[u];
  if (tid == 0) {
    for (int i = 0; i < 4; i++) mbar_init(&mbar_s[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  for (int cell = blockIdx.x; cell < L.C; cell += gridDim.x) {
    if (tid == 0) { flag_s[0] = 0; flag_s[1] = 0; flag_s[2] = 0; }
    if (!L.solve_only) {
      if (tid < P.nv * P.d) nodes_s[tid] = L.nodes[(size_t)cell * P.nv * P.d + tid];
      const int nco = P.nslots * P.Ptot;
      if (L.coeff)
        for (int i = tid; i < nco; i += NT) coef_s[i] = L.coeff[(size_t)cell * nco + i];
    }
    __syncthreads();
    double* GT = sm + P.sm_gt;
    if (L.solve_only) {
      const double* Gc = L.Gin + (size_t)cell * P.N * P.N;
      for (int e = tid; e < P.ngt * 64; e += NT) {
        int tau = e >> 6, idx = e & 63;
        int ij = tri_s[tau];
        int I = ij & 255, J = ij >> 8;
        int r = (idx >> 2) & 7, c = (idx >> 5) * 4 + (idx & 3);
        int gr = I * 8 + r, gc = J * 8 + c;
        double v = 0.0;
        if (gr < P.N && gc < P.N) v = Gc[(size_t)gr * P.N + gc];
        else if (gr == gc) v = 1.0;
        GT[e] = v;
      }
      __syncthreads();
    } else {
      phase_b<BTW>(P, L, cell, X);
      __syncthreads();
      phase_gram<GTM, CHG>(P, L, cell, X);
      if (L.parts) {
        __syncthreads();
        continue;
      }
    }
    phase_factor(P, X);
    phase_trsm<NBTM>(P, L, cell, X);
    phase_syrk_out(P, L, cell, X);
    __syncthreads();
    if (tid == 0 && L.info) {
      int f0 = flag_s[0], f1 = flag_s[1];
      int v = 0;
      if (flag_s[2]) {
        v = ERR_TIMEOUT_FLAG;
      } else if (f0 != 0) {
        int r = f0 - 1;
        int u = L.solve_only ? r : P.dev2user_test[r];
        v = (u >= 0 ? u : r) + 1;
      } else if (f1 != 0) {
        v = f1;
      }
      L.info[cell] = v;
    }
    __syncthreads();
  }
}

// Instances: register arrays sized for the test-tile count of the bucket; the last
// argument is the Gram chunk size (plans short of shared memory use half chunks).
#define DPG_INSTANCES(X) \
  X(8, 3, 4, 8) X(12, 5, 4, 8) X(16, 6, 4, 8) X(18, 8, 4, 8) X(20, 8, 4, 8) X(22, 9, 3, 8) X(24, 12, 4, 8) \
  X(24, 12, 6, 8) X(24, 12, 6, 4)

typedef void (*KernelFn)(const DpgPlanDev, const DpgLaunch);

static KernelFn pick_kernel(const DpgPlanDev* plan) {
  const int per = (plan->ngb + DPG_NWARPS - 1) / DPG_NWARPS;
  int btw = 0;
  for (int s = 0; s < plan->nseg; s++) btw = std::max(btw, (plan->seg[s].ntile + DPG_NWARPS - 1) / DPG_NWARPS);
#define DPG_PICK(NB, GT, BT, CH) \
  if (plan->NBT <= NB && per <= GT && btw <= BT && plan->chg == CH) return dpg_cell_kernel<NB, GT, BT, CH>;
  DPG_INSTANCES(DPG_PICK)
#undef DPG_PICK
  return nullptr;
}

#include "dpg_adjoint.cuh"

__device__ __forceinline__ void mbar_inval(uint64_t* b) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(b)) : "memory");
}

// Per-CTA tables of one plan: triangular tile index, G block list, mbarriers.
__device__ __forceinline__ void cta_setup(const DpgPlanDev& P) {
  const int tid = threadIdx.x;
  double* const sm = dpg_smem;
  int* tri_s = reinterpret_cast<int*>(sm + P.sm_nodes + 32);
  DpgGTile* tiles_s = reinterpret_cast<DpgGTile*>(sm + P.sm_tiles);
  uint64_t* mbar_s = reinterpret_cast<uint64_t*>(sm + P.sm_nodes + 26);
  const int ntri = DPG_MAX_NBT * (DPG_MAX_NBT + 1) / 2;
  for (int u = tid; u < ntri; u += NT) {
    int I = (int)((sqrt(8.0 * u + 1.0) - 1.0) * 0.5);
    while ((I + 1) * (I + 2) / 2 <= u) I++;
    while (I * (I + 1) / 2 > u) I--;
    tri_s[u] = I | ((u - I * (I + 1) / 2) << 8);
  }
  for (int u = tid; u < P.ngb; u += NT) tiles_s[u] = P.gtiles[u];
  if (tid == 0) {
    for (int i = 0; i < 4; i++) mbar_init(&mbar_s[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

#include "dpg_energy.cuh"
#include "dpg_big.cuh"


// Claim `claim` work items from the queue counter; all threads see the same base.
__device__ __forceinline__ int queue_claim(int* counter, int claim, volatile int* slot) {
  if (threadIdx.x == 0) *slot = atomicAdd(counter, claim);
  __syncthreads();
  const int base = *slot;
  __syncthreads();  // every thread has its copy before the next claim overwrites it
  return base;
}

// The last CTA to leave the queue resets its counters, so the next launch (a graph
// replay) starts from zero; no CTA waits on another.
__device__ __forceinline__ void queue_leave(int* counters) {
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&counters[1], 1) == (int)gridDim.x - 1) {
      counters[0] = 0;
      counters[1] = 0;
      __threadfence();
    }
  }
}

// Multi-bucket work queue of the single-CTA plans: the buckets' cell ranges are
// concatenated in decreasing order of per-cell cost (the host orders them), and each CTA
// claims `claim` consecutive cells at a time from a device counter, so the long cells start
// first and the short ones fill the tail.  Switching buckets rebuilds the CTA's tables and
// mbarriers.  claim_slot: a shared-memory double beyond every plan's layout.
template <int NBTM, int GTM, int BTW>
__global__ void __launch_bounds__(NT, 1) dpg_queue_kernel(const DpgPlanDev* __restrict__ plans,
                                                          const DpgLaunch* __restrict__ launches,
                                                          const int* __restrict__ cstart, int nb,
                                                          int* __restrict__ counters, int claim, int claim_slot) {
  const int tid = threadIdx.x;
  Ctx X;
  uint32_t phase[4] = {0, 0, 0, 0};
  X.phase = phase;
  double* const sm = dpg_smem;
  volatile int* const claim_s = reinterpret_cast<volatile int*>(sm + claim_slot);
  int cur = -1;
  const int total = cstart[nb];
  for (;;) {
    const int base = queue_claim(&counters[0], claim, claim_s);
    if (base >= total) break;
    const int end = min(total, base + claim);
    for (int i = base; i < end; i++) {
      int b = cur < 0 ? 0 : cur;
      while (i >= cstart[b + 1]) b++;
      const DpgPlanDev& P = plans[b];
      const DpgLaunch& L = launches[b];
      if (b != cur) {
        __syncthreads();
        if (cur >= 0 && tid == 0) {
          uint64_t* old = reinterpret_cast<uint64_t*>(sm + plans[cur].sm_nodes + 26);
          for (int k = 0; k < 4; k++) mbar_inval(&old[k]);
        }
        __syncthreads();
        cta_setup(P);
        for (int k = 0; k < 4; k++) phase[k] = 0;
        cur = b;
      }
      const int cell = i - cstart[b];
      double* nodes_s = sm + P.sm_nodes;
      int* flag_s = reinterpret_cast<int*>(sm + P.sm_nodes + 24);
      double* coef_s = sm + P.sm_coef;
      if (tid == 0) { flag_s[0] = 0; flag_s[1] = 0; flag_s[2] = 0; }
      if (tid < P.nv * P.d) nodes_s[tid] = L.nodes[(size_t)cell * P.nv * P.d + tid];
      const int nco = P.nslots * P.Ptot;
      if (L.coeff)
        for (int k = tid; k < nco; k += NT) coef_s[k] = L.coeff[(size_t)cell * nco + k];
      __syncthreads();
      phase_b<BTW>(P, L, cell, X);
      __syncthreads();
      phase_gram<GTM, 0>(P, L, cell, X);
      phase_factor(P, X);
      phase_trsm<NBTM>(P, L, cell, X);
      phase_syrk_out(P, L, cell, X);
      __syncthreads();
      if (tid == 0 && L.info) {
        int v = 0;
        if (flag_s[2]) v = ERR_TIMEOUT_FLAG;
        else if (flag_s[0] != 0) {
          int r = flag_s[0] - 1;
          int u = P.dev2user_test[r];
          v = (u >= 0 ? u : r) + 1;
        } else if (flag_s[1] != 0) v = flag_s[1];
        L.info[cell] = v;
      }
      __syncthreads();
    }
  }
  queue_leave(counters);
}

typedef void (*QueueFn)(const DpgPlanDev*, const DpgLaunch*, const int*, int, int*, int, int);
#define DPG_QUEUE_INSTANCES(X) X(16, 6, 4) X(24, 12, 6)

// The smallest instance whose register arrays cover every single-CTA plan of the call.
static QueueFn pick_queue_kernel(const DpgPlanDev* plans, int nb) {
  int nbt = 0, per = 0, btw = 0;
  for (int b = 0; b < nb; b++) {
    const DpgPlanDev* p = &plans[b];
    nbt = std::max(nbt, p->NBT);
    per = std::max(per, (p->ngb + DPG_NWARPS - 1) / DPG_NWARPS);
    for (int s = 0; s < p->nseg; s++) btw = std::max(btw, (p->seg[s].ntile + DPG_NWARPS - 1) / DPG_NWARPS);
  }
#define DPG_PICK(NB, GT, BT) \
  if (nbt <= NB && per <= GT && btw <= BT) return dpg_queue_kernel<NB, GT, BT>;
  DPG_QUEUE_INSTANCES(DPG_PICK)
#undef DPG_PICK
  return nullptr;
}

}  // namespace

namespace dpg {
namespace {
constexpr int kMaxDevices = 64;
std::mutex g_dev_mu;
int g_dev_sms[kMaxDevices] = {0};
cudaMemPool_t g_dev_pool[kMaxDevices] = {nullptr};
bool g_dev_pool_tried[kMaxDevices] = {false};
}  // namespace

int num_sms() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kMaxDevices) return 148;
  std::lock_guard<std::mutex> g(g_dev_mu);
  if (g_dev_sms[dev] == 0) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    g_dev_sms[dev] = n > 0 ? n : 1;
    cudaGetLastError();
  }
  return g_dev_sms[dev];
}

cudaError_t ws_alloc(void** p, size_t bytes, cudaStream_t s) {
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
    cudaGetLastError();
    cap = cudaStreamCaptureStatusNone;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaMemPool_t pool = nullptr;
  if (cap == cudaStreamCaptureStatusNone && dev >= 0 && dev < kMaxDevices) {
    std::lock_guard<std::mutex> g(g_dev_mu);
    if (!g_dev_pool_tried[dev]) {
      g_dev_pool_tried[dev] = true;
      cudaMemPoolProps props;
      std::memset(&props, 0, sizeof(props));
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      cudaMemPool_t created = nullptr;
      if (cudaMemPoolCreate(&created, &props) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(created, cudaMemPoolAttrReleaseThreshold, &thr);
        g_dev_pool[dev] = created;
      }
      cudaGetLastError();
    }
    pool = g_dev_pool[dev];
  }
  if (pool) return cudaMallocFromPoolAsync(p, bytes, pool, s);
  return cudaMallocAsync(p, bytes, s);
}
}  // namespace dpg

static int configure_big(const DpgPlanDev* plan) {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  size_t bytes = (size_t)plan->bs_total * sizeof(double);
  if (optin > 0 && bytes > (size_t)optin) return dpg::fail(DPG_ERR_UNSUPPORTED, "bucket needs more shared memory than one CTA has");
  // every large plan shares the kernel: opt in to the device maximum so that configuring one
  // plan never lowers the limit another plan needs
  if (optin > 0) bytes = (size_t)optin;
  for (KernelFn k : {dpg_big_kernel<16>, dpg_big_kernel<32>}) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  }
  return DPG_OK;
}

// Large buckets: one CTA per SM, each with its own workspace (Z and the per-point factors).
static int launch_big(const DpgPlanDev* plan, const DpgLaunch* Lin, cudaStream_t stream) {
  if (Lin->solve_only)
    return dpg::fail(DPG_ERR_UNSUPPORTED, "large-bucket plans support the assembly entry points only");
  const int grid = std::min(Lin->C, dpg::num_sms());
  DpgLaunch L = *Lin;
  void* ws = nullptr;
  if (!L.scratch) {  // a caller-provided workspace holds dpg_big_workspace_bytes(plan, C)
    cudaError_t ea = dpg::ws_alloc(&ws, (size_t)grid * plan->bz_per_cta * sizeof(double), stream);
    if (ea != cudaSuccess) {
      cudaGetLastError();
      return dpg::fail(DPG_ERR_OUT_OF_MEMORY, std::string("workspace allocation: ") + cudaGetErrorString(ea));
    }
    L.scratch = (double*)ws;
  }
  KernelFn k = plan->big_zk == 16 ? dpg_big_kernel<16> : dpg_big_kernel<32>;
  k<<<grid, NT, (size_t)plan->bs_total * sizeof(double), stream>>>(*plan, L);
  cudaError_t e = cudaGetLastError();
  if (ws) cudaFreeAsync(ws, stream);
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}

size_t dpg_big_workspace_bytes(const DpgPlanDev* plan, int C) {
  const int grid = std::min(std::max(C, 1), dpg::num_sms());
  return (size_t)grid * plan->bz_per_cta * sizeof(double);
}

int dpg_configure_kernels(const DpgPlanDev* plan) {
  if (plan->big) return configure_big(plan);
  KernelFn k = pick_kernel(plan);
  if (!k) return dpg::fail(DPG_ERR_UNSUPPORTED, "no kernel instance for this bucket size");
  // Several plans may share a kernel instance: the opt-in limit is the device's
  // maximum, so configuring one plan never lowers another's.
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  size_t bytes = (size_t)plan->sm_total * sizeof(double);
  if (optin > 0 && bytes > (size_t)optin) return dpg::fail(DPG_ERR_UNSUPPORTED, "bucket needs more shared memory than one CTA has");
  if (optin > 0) bytes = (size_t)optin;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  if (plan->adj_ok) {
    KernelFn ka = pick_adjoint_kernel(plan);
    if (ka) {
      e = cudaFuncSetAttribute(ka, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
      if (e != cudaSuccess)
        return dpg::fail(DPG_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    }
  }
  return DPG_OK;
}

int dpg_launch_assemble(const DpgPlanDev* plan, const DpgPlanDev* d_plan, const DpgLaunch* Lin, cudaStream_t stream) {
  (void)d_plan;
  if (Lin->C <= 0) return DPG_OK;
  if (plan->big) return launch_big(plan, Lin, stream);
  KernelFn k = pick_kernel(plan);
  if (!k) return dpg::fail(DPG_ERR_UNSUPPORTED, "no kernel instance for this bucket size");
  const int grid = std::min(Lin->C, dpg::num_sms());
  DpgLaunch L = *Lin;
  void* scratch = nullptr;
  const bool need_scratch = !L.solve_only && plan->scratch_per_cta > 0 && !L.scratch;
  if (need_scratch) {
    cudaError_t ea = dpg::ws_alloc(&scratch, (size_t)grid * plan->scratch_per_cta * sizeof(double), stream);
    if (ea != cudaSuccess) {
      cudaGetLastError();
      return dpg::fail(DPG_ERR_OUT_OF_MEMORY, std::string("scratch allocation: ") + cudaGetErrorString(ea));
    }
    L.scratch = (double*)scratch;
  }
  size_t bytes = (size_t)plan->sm_total * sizeof(double);
  k<<<grid, NT, bytes, stream>>>(*plan, L);
  cudaError_t e = cudaGetLastError();
  if (scratch) cudaFreeAsync(scratch, stream);
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}

// Field recovery after the global solve (CondensedDofInterpreter::
// interpretGlobalCoefficients, CondensedDofInterpreter.cpp:1229-1346): per cell,
// K_ff u_f = l_f - K_ft t for the field dofs u_f given the cell's trace dofs t, with
// the local K, l of the assembly (user numbering: fields first).  One CTA per cell:
// K_ff is equilibrated (s_i = K_ii^-1/2) and Cholesky-factored in shared memory; the
// local coefficients [u_f | t] are written out.  info: 0, or the first non-positive
// pivot (1-based).
namespace {
__global__ void __launch_bounds__(256) recover_fields_kernel(int C, int M, int nf, const double* __restrict__ K,
                                                             const double* __restrict__ l,
                                                             const double* __restrict__ t_in, double* __restrict__ u,
                                                             int32_t* __restrict__ info) {
  extern __shared__ double rs[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const int nt = M - nf;
  double* A = rs;                 // nf x nf, row-major (lower triangle used)
  double* sc = A + nf * nf;       // scaling
  double* b = sc + nf;            // right-hand side, then the solution
  __shared__ int fail;
  for (int cell = blockIdx.x; cell < C; cell += gridDim.x) {
    const double* Kc = K + (size_t)cell * M * M;
    const double* lc = l + (size_t)cell * M;
    const double* tc = t_in + (size_t)cell * nt;
    if (tid == 0) fail = 0;
    for (int i = tid; i < nf; i += blockDim.x) {
      const double d = Kc[(size_t)i * M + i];
      sc[i] = d > 0.0 ? rsqrt(d) : 1.0;
    }
    __syncthreads();
    for (int e = tid; e < nf * nf; e += blockDim.x) {
      const int i = e / nf, j = e - i * nf;
      A[e] = sc[i] * Kc[(size_t)i * M + j] * sc[j];
    }
    // b = S (l_f - K_ft t): one warp per row
    for (int i = warp; i < nf; i += nw) {
      double acc = 0.0;
      for (int j = lane; j < nt; j += 32) acc += Kc[(size_t)i * M + nf + j] * tc[j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) b[i] = sc[i] * (lc[i] - acc);
    }
    __syncthreads();
    // right-looking Cholesky, column by column
    for (int k = 0; k < nf; k++) {
      const double piv = A[k * nf + k];
      if (!(piv > 0.0)) {
        if (tid == 0 && fail == 0) fail = k + 1;
      }
      const double inv = rsqrt(piv);
      __syncthreads();
      for (int i = k + tid; i < nf; i += blockDim.x) A[i * nf + k] = (i == k) ? piv * inv : A[i * nf + k] * inv;
      __syncthreads();
      const int m = nf - 1 - k;
      for (int e = tid; e < m * m; e += blockDim.x) {
        const int i = k + 1 + e / m, j = k + 1 + e % m;
        if (j <= i) A[i * nf + j] -= A[i * nf + k] * A[j * nf + k];
      }
      __syncthreads();
    }
    // L z = b, L^T y = z (warp 0; lanes split the dot products)
    if (warp == 0) {
      for (int i = 0; i < nf; i++) {
        double acc = 0.0;
        for (int j = lane; j < i; j += 32) acc += A[i * nf + j] * b[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) b[i] = (b[i] - acc) / A[i * nf + i];
        __syncwarp();
      }
      for (int i = nf - 1; i >= 0; i--) {
        double acc = 0.0;
        for (int j = i + 1 + lane; j < nf; j += 32) acc += A[j * nf + i] * b[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) b[i] = (b[i] - acc) / A[i * nf + i];
        __syncwarp();
      }
    }
    __syncthreads();
    double* uc = u + (size_t)cell * M;
    for (int i = tid; i < M; i += blockDim.x) uc[i] = i < nf ? sc[i] * b[i] : tc[i - nf];
    if (tid == 0 && info) info[cell] = fail;
    __syncthreads();
  }
}

// nf <= 32: one warp per cell.  K_ff goes to a per-warp shared tile by 8-byte
// asynchronous copies (all in flight at once); K_ft t is formed from coalesced reads of
// the K_ft rows, each lane holding partial sums of all rows, which one butterfly
// reduce-scatter (31 shuffles) turns into lane i's row sum.  Lane i then holds row i of
// the equilibrated K_ff in registers and the Cholesky factorisation, both triangular
// solves and the unscaling run on shuffles, without a block barrier.  Same results and
// info as the block kernel above.
constexpr int RF_MAXW = 1;  // warps per block

__global__ void __launch_bounds__(RF_MAXW * 32) recover_fields_warp_kernel(int C, int M, int nf,
                                                                         const double* __restrict__ K,
                                                                         const double* __restrict__ l,
                                                                         const double* __restrict__ t_in,
                                                                         double* __restrict__ u,
                                                                         int32_t* __restrict__ info) {
  extern __shared__ double rs[];
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  constexpr int ld = 33;                // odd row stride: conflict-free column reads
  double* st = rs + (size_t)warp * (32 * ld + M);
  double* ts = st + 32 * ld;            // trace values
  const int nt = M - nf;
  for (int cell = blockIdx.x * nwarps + warp; cell < C; cell += gridDim.x * nwarps) {
    const double* Kc = K + (size_t)cell * M * M;
    const double* tc = t_in + (size_t)cell * nt;
    for (int r = 0; r < nf; r++)
      if (lane < nf)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(st + r * ld + lane)),
                     "l"(Kc + (size_t)r * M + lane)
                     : "memory");
    for (int j = lane; j < nt; j += 32)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(ts + j)), "l"(tc + j) : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
    // partial sums of K_ft(i,:) t over this lane's columns, all rows
    double p[32];
#pragma unroll
    for (int i = 0; i < 32; i++) p[i] = 0.0;
    for (int c0 = 0; c0 < nt; c0 += 32) {
      const int c = c0 + lane;
      const double tv = c < nt ? tc[c] : 0.0;
#pragma unroll
      for (int i = 0; i < 32; i++)
        if (i < nf && c < nt) p[i] += Kc[(size_t)i * M + nf + c] * tv;
    }
    // reduce-scatter: after the step with offset o a lane keeps the rows whose bit o
    // matches its own; at the end lane i holds row i's sum in p[0]
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
      const bool hi = (lane & o) != 0;
#pragma unroll
      for (int r = 0; r < o; r++) {
        const double send = hi ? p[r] : p[r + o];
        const double keep = hi ? p[r + o] : p[r];
        p[r] = keep + __shfl_xor_sync(FULL, send, o);
      }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncwarp();
    const int i = lane;
    double bi = 0.0, sc = 1.0;  // lane i: l_i - K_ft(i,:) t and s_i = K_ii^-1/2
    if (i < nf) {
      bi = l[(size_t)cell * M + i] - p[0];
      const double d = st[i * ld + i];
      sc = d > 0.0 ? rsqrt(d) : 1.0;
    }
    // rows and columns nf..31 are padded with the identity, so every step below runs
    // unguarded on all 32 lanes and leaves the padding unchanged
    double a[32];
#pragma unroll
    for (int j = 0; j < 32; j++) {
      const double sj = __shfl_sync(FULL, sc, j);
      a[j] = (i < nf && j < nf) ? sc * st[i * ld + j] * sj : (i == j ? 1.0 : 0.0);
    }
    __syncwarp();
    bi = i < nf ? bi * sc : 0.0;
    // right-looking Cholesky: at step k lane k holds the pivot, lanes i > k column k;
    // entries above the diagonal are left unused
    int fail = 0;
    double dinv = 0.0;  // 1 / L_ii
#pragma unroll
    for (int k = 0; k < 32; k++) {
      const double piv = __shfl_sync(FULL, a[k], k);
      if (!(piv > 0.0) && fail == 0) fail = k + 1;
      const double inv = rsqrt(piv);
      const double lik = (i == k) ? piv * inv : a[k] * inv;
      a[k] = lik;
      if (i == k) dinv = inv;
#pragma unroll
      for (int j = k + 1; j < 32; j++) a[j] -= lik * __shfl_sync(FULL, lik, j);
    }
    // L z = b
#pragma unroll
    for (int k = 0; k < 32; k++) {
      const double zk = __shfl_sync(FULL, bi * dinv, k);
      if (i == k) bi = zk;
      else if (i > k) bi -= a[k] * zk;
    }
    // L^T y = z, column by column: L's rows go back to the (now free) shared tile, y_k is
    // broadcast and lanes j < k take L_kj y_k off their z_j
#pragma unroll
    for (int j = 0; j < 32; j++)
      if (i < nf && j <= i) st[i * ld + j] = a[j];
    __syncwarp();
    double y = bi;
    for (int k = nf - 1; k >= 0; k--) {
      const double yk = __shfl_sync(FULL, y * dinv, k);
      if (i == k) y = yk;
      else if (i < k) y -= st[k * ld + i] * yk;
    }
    __syncwarp();
    double* uc = u + (size_t)cell * M;
    if (i < nf) uc[i] = sc * y;
    for (int j = lane; j < nt; j += 32) uc[nf + j] = tc[j];
    if (lane == 0 && info) info[cell] = fail;
  }
}
}  // namespace

int dpg_launch_recover_fields(int C, int M, int nf, const double* K, const double* l, const double* t, double* u,
                              int32_t* info, cudaStream_t stream) {
  if (C <= 0) return DPG_OK;
  const size_t per_warp = ((size_t)32 * 33 + M) * sizeof(double);
  if (nf <= 32 && per_warp <= 100 * 1024) {
    // one-warp blocks: as many resident per SM as the staging tiles allow
    static int wconfigured = 0;
    if (!wconfigured) {
      cudaFuncSetAttribute(recover_fields_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
      wconfigured = 1;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, recover_fields_warp_kernel, 32, per_warp);
    const int sms = dpg::num_sms();
    const int grid = (int)std::min<long long>(C, (long long)sms * std::max(1, per_sm));
    recover_fields_warp_kernel<<<grid, 32, per_warp, stream>>>(C, M, nf, K, l, t, u, info);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return DPG_OK;
  }
  const size_t bytes = ((size_t)nf * nf + 2 * (size_t)nf) * sizeof(double);
  if (bytes > 200 * 1024) return dpg::fail(DPG_ERR_UNSUPPORTED, "too many field dofs for the recovery kernel");
  static int configured = 0;
  if (!configured) {
    cudaFuncSetAttribute(recover_fields_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    configured = 1;
  }
  const int grid = std::min(C, (dpg::num_sms()) * 4);
  recover_fields_kernel<<<grid, 256, bytes, stream>>>(C, M, nf, K, l, t, u, info);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}

// Bounded-wait probe: one thread waits, with the kernels' own wait routine, on an
// mbarrier whose transaction never arrives (a flag nothing sets), and reports the
// status the assembly kernels turn into info = 0x7fff0000.  Lets a test check that a
// stalled staging copy ends the wait with an error instead of hanging the GPU.
namespace {
__global__ void wait_probe_kernel(int limit, int* status) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_expect_tx(&bar, 16);  // no copy will deliver these bytes
    status[0] = mbar_wait(&bar, 0, limit) ? 0 : ERR_TIMEOUT_FLAG;
  }
}
}  // namespace

extern "C" int dpg_debug_wait_probe(int limit, int* status_dev, void* stream) {
  if (limit <= 0 || !status_dev) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "bad probe arguments");
  wait_probe_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(limit, status_dev);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}

int dpg_launch_adjoint(const DpgPlanDev* plan, const DpgLaunch* Lin, cudaStream_t stream) {
  if (Lin->C <= 0) return DPG_OK;
  if (!plan->adj_ok) return dpg::fail(DPG_ERR_UNSUPPORTED, "reverse mode is not available for this bucket");
  KernelFn k = pick_adjoint_kernel(plan);
  if (!k) return dpg::fail(DPG_ERR_UNSUPPORTED, "no adjoint kernel instance for this bucket size");
  const int grid = std::min(Lin->C, dpg::num_sms());
  DpgLaunch L = *Lin;
  void* scratch = nullptr;
  const size_t per = plan->scratch_per_cta;
  cudaError_t ea = dpg::ws_alloc(&scratch, (size_t)grid * per * 2 * sizeof(double), stream);
  if (ea != cudaSuccess) {
    cudaGetLastError();
    return dpg::fail(DPG_ERR_OUT_OF_MEMORY, std::string("scratch allocation: ") + cudaGetErrorString(ea));
  }
  L.scratch = (double*)scratch;
  L.scratch2 = L.scratch + (size_t)grid * per;
  size_t bytes = (size_t)plan->sm_total * sizeof(double);
  k<<<grid, NT, bytes, stream>>>(*plan, L);
  cudaError_t e = cudaGetLastError();
  cudaFreeAsync(scratch, stream);
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}

int dpg_launch_energy(const DpgPlanDev* plan, const DpgLaunch* Lin, cudaStream_t stream) {
  if (Lin->C <= 0) return DPG_OK;
  if (plan->big) return launch_big(plan, Lin, stream);  // energy error or DLS output
  KernelFn k = Lin->xsol ? pick_energy_kernel(plan) : pick_dls_kernel(plan);
  if (!k) return dpg::fail(DPG_ERR_UNSUPPORTED, "no kernel instance for this bucket size");
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       optin > 0 ? optin : (int)(plan->sm_total * sizeof(double)));
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  const int grid = std::min(Lin->C, dpg::num_sms());
  DpgLaunch L = *Lin;
  void* scratch = nullptr;
  cudaError_t ea = dpg::ws_alloc(&scratch, (size_t)grid * plan->scratch_per_cta * sizeof(double), stream);
  if (ea != cudaSuccess) {
    cudaGetLastError();
    return dpg::fail(DPG_ERR_OUT_OF_MEMORY, std::string("scratch allocation: ") + cudaGetErrorString(ea));
  }
  L.scratch = (double*)scratch;
  k<<<grid, NT, (size_t)plan->sm_total * sizeof(double), stream>>>(*plan, L);
  e = cudaGetLastError();
  cudaFreeAsync(scratch, stream);
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}

// The work queue of the single-CTA plans: the buckets that have cells, in decreasing order of
// per-cell cost (the cube of the order of the matrix a cell factors), their concatenated
// cell ranges, the common per-CTA scratch stride, the shared memory of the largest plan plus
// the claim slot, and the device bytes: tables, two counters, scratch slots.
struct QueuePart {
  std::vector<DpgPlanDev> plans;
  std::vector<DpgLaunch> ls;
  std::vector<int> cstart{0};
  size_t stride = 0;
  int smem_doubles = 0, claim_slot = 0;
  int total = 0, grid = 0;
  size_t bytes_tables = 0, bytes = 0;
};

static int queue_part(const DpgPlanDev* hplans, const DpgLaunch* hl, int nb, QueuePart& Q) {
  std::vector<int> order;
  for (int b = 0; b < nb; b++) {
    if (hl[b].C <= 0) continue;
    if (hplans[b].big) return dpg::fail(DPG_ERR_UNSUPPORTED, "large-bucket plans run on their own launches");
    if (hl[b].solve_only) return dpg::fail(DPG_ERR_UNSUPPORTED, "the multi-bucket launch assembles; no solve-only plans");
    order.push_back(b);
  }
  auto cost = [&](int b) {
    const double n = (double)(hplans[b].Np + hplans[b].Mp);
    return n * n * n;
  };
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(x) > cost(y); });
  for (int b : order) {
    Q.stride = std::max(Q.stride, hplans[b].scratch_per_cta);
    Q.smem_doubles = std::max(Q.smem_doubles, hplans[b].sm_total);
    Q.plans.push_back(hplans[b]);
    Q.ls.push_back(hl[b]);
    Q.cstart.push_back(Q.cstart.back() + hl[b].C);
  }
  Q.total = Q.cstart.back();
  Q.grid = std::min(std::max(Q.total, 1), dpg::num_sms());
  for (auto& p : Q.plans) p.scratch_per_cta = Q.stride;
  Q.claim_slot = (Q.smem_doubles + 1) & ~1;
  const int nq = (int)Q.plans.size();
  Q.bytes_tables = (nq * (sizeof(DpgPlanDev) + sizeof(DpgLaunch)) + (nq + 1) * sizeof(int) + 8 + 255) & ~(size_t)255;
  Q.bytes = Q.bytes_tables + (size_t)Q.grid * Q.stride * sizeof(double);
  return DPG_OK;
}

// hplans: host copies of the single-CTA buckets' plans; hl: per-bucket launch arguments;
// claim: cells a CTA claims at a time; dev: where the device copies of the tables go (null:
// stream-ordered temporaries freed after the launch).
int dpg_launch_multi(const DpgPlanDev* hplans, const DpgLaunch* hl, int nb, cudaStream_t stream, DpgMultiDev* dev,
                     int claim) {
  QueuePart Q;
  int rc = queue_part(hplans, hl, nb, Q);
  if (rc != DPG_OK) return rc;
  if (Q.total == 0) return DPG_OK;
  const int nq = (int)Q.plans.size();
  QueueFn k = pick_queue_kernel(Q.plans.data(), nq);
  if (!k) return dpg::fail(DPG_ERR_UNSUPPORTED, "no multi-bucket kernel instance covers these buckets");
  int dev_id = 0, optin = 0;
  cudaGetDevice(&dev_id);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev_id);
  const size_t smem = (size_t)(Q.claim_slot + 2) * sizeof(double);
  if (optin > 0 && smem > (size_t)optin)
    return dpg::fail(DPG_ERR_UNSUPPORTED, "multi-bucket launch: no room for the claim slot beside the largest plan");
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin > 0 ? optin : (int)smem);
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  claim = std::max(1, std::min(claim, 64));
  char* base = nullptr;
  if (dev) {
    if (dev->bytes < Q.bytes) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "multi workspace too small");
    base = (char*)dev->base;
  } else {
    e = dpg::ws_alloc((void**)&base, Q.bytes, stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return dpg::fail(DPG_ERR_OUT_OF_MEMORY, std::string("multi workspace: ") + cudaGetErrorString(e));
    }
  }
  double* scratch = (double*)(base + Q.bytes_tables);
  for (auto& l : Q.ls) l.scratch = scratch;
  DpgPlanDev* d_plans = (DpgPlanDev*)base;
  DpgLaunch* d_l = (DpgLaunch*)(base + nq * sizeof(DpgPlanDev));
  int* d_cs = (int*)(base + nq * (sizeof(DpgPlanDev) + sizeof(DpgLaunch)));
  int* d_ctr = d_cs + nq + 1;
  if (dev) {  // outside any capture: synchronous uploads; the kernel resets its counters itself
    cudaMemcpy(d_plans, Q.plans.data(), nq * sizeof(DpgPlanDev), cudaMemcpyHostToDevice);
    cudaMemcpy(d_l, Q.ls.data(), nq * sizeof(DpgLaunch), cudaMemcpyHostToDevice);
    cudaMemcpy(d_cs, Q.cstart.data(), (nq + 1) * sizeof(int), cudaMemcpyHostToDevice);
    e = cudaMemset(d_ctr, 0, 2 * sizeof(int));
    if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("counter reset: ") + cudaGetErrorString(e));
    dev->plans = d_plans; dev->launches = d_l; dev->cstart = d_cs; dev->nb = nq; dev->grid = Q.grid;
    dev->kernel = (void*)k; dev->smem = smem; dev->counters = d_ctr; dev->claim = claim; dev->claim_slot = Q.claim_slot;
    return DPG_OK;
  }
  cudaMemcpyAsync(d_plans, Q.plans.data(), nq * sizeof(DpgPlanDev), cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(d_l, Q.ls.data(), nq * sizeof(DpgLaunch), cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(d_cs, Q.cstart.data(), (nq + 1) * sizeof(int), cudaMemcpyHostToDevice, stream);
  cudaMemsetAsync(d_ctr, 0, 2 * sizeof(int), stream);
  k<<<Q.grid, NT, smem, stream>>>(d_plans, d_l, d_cs, nq, d_ctr, claim, Q.claim_slot);
  e = cudaGetLastError();
  cudaFreeAsync(base, stream);
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}

// Launch of the queue prepared by dpg_launch_multi(..., dev) (graph capture records this).
int dpg_launch_multi_prepared(const DpgMultiDev* dev, cudaStream_t stream) {
  QueueFn k = (QueueFn)dev->kernel;
  k<<<dev->grid, NT, dev->smem, stream>>>(dev->plans, dev->launches, dev->cstart, dev->nb, dev->counters, dev->claim,
                                          dev->claim_slot);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}

// Bytes a prepared multi-bucket launch needs (tables, counters, scratch slots).
size_t dpg_multi_bytes(const DpgPlanDev* hplans, const DpgLaunch* hl, int nb) {
  QueuePart Q;
  if (queue_part(hplans, hl, nb, Q) != DPG_OK) return 0;
  return Q.bytes;
}

// ---------------------------------------------------------------------------
// Allocation-free launch: the per-CTA scratch comes from a fixed device array
// instead of a stream-ordered allocation.  32 MiB (4 Mi doubles): the 3D hex k=2
// bucket needs 298 KiB per CTA (B tiles 165 KiB, Gram running sums 133 KiB), so
// 110 CTAs fit; smaller buckets run one CTA per SM.
// ---------------------------------------------------------------------------
#define DPG_NOALLOC_SCRATCH_DOUBLES ((size_t)4 << 20)

static __device__ __align__(256) double g_noalloc_scratch[DPG_NOALLOC_SCRATCH_DOUBLES];

namespace {
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[64] = {nullptr};           // device address of the array, per device ordinal
unsigned long long g_noalloc_ctx[64] = {0};      // id of the context that address belongs to

// Id of the current CUDA context (0 if the driver cannot tell).  A device reset
// followed by a new context changes it, and the array's address must then be looked
// up again.  The driver functions are reached through the runtime's entry-point query,
// so the library needs no link against the driver library.
unsigned long long current_context_id() {
  typedef int (*CtxGetCurrent)(void**);
  typedef int (*CtxGetId)(void*, unsigned long long*);
  static CtxGetCurrent get_current = nullptr;
  static CtxGetId get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {  // called with g_noalloc_mu held
    looked_up = true;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      get_current = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      get_id = nullptr;
    cudaGetLastError();
  }
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&ctx) == 0 && ctx && get_id(ctx, &id) == 0) return id;
  return 0;
}
}  // namespace

int dpg_launch_assemble_noalloc(const DpgPlanDev* plan, const DpgLaunch* Lin, cudaStream_t stream) {
  if (Lin->C <= 0) return DPG_OK;
  if (plan->big) return dpg::fail(DPG_ERR_UNSUPPORTED, "dpg_assemble_noalloc: large-bucket plans need dpg_assemble");
  KernelFn k = pick_kernel(plan);
  if (!k) return dpg::fail(DPG_ERR_UNSUPPORTED, "no kernel instance for this bucket size");
  if (plan->scratch_per_cta > DPG_NOALLOC_SCRATCH_DOUBLES)
    return dpg::fail(DPG_ERR_UNSUPPORTED,
                     "dpg_assemble_noalloc: the bucket needs more per-CTA scratch than the fixed 32 MiB array holds");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return dpg::fail(DPG_ERR_CUDA, "dpg_assemble_noalloc: no current CUDA device");
  }
  double* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    const unsigned long long ctx = current_context_id();
    if (!g_noalloc_ptr[dev] || (ctx != 0 && ctx != g_noalloc_ctx[dev])) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return dpg::fail(DPG_ERR_CUDA, std::string("dpg_assemble_noalloc: cudaGetSymbolAddress: ") +
                                           cudaGetErrorString(e));
      }
      g_noalloc_ptr[dev] = (double*)p;
      g_noalloc_ctx[dev] = current_context_id();  // the lookup made the context current if none was
    }
    base = g_noalloc_ptr[dev];
  }
  const size_t fit = plan->scratch_per_cta > 0 ? DPG_NOALLOC_SCRATCH_DOUBLES / plan->scratch_per_cta : (size_t)Lin->C;
  int grid = std::min(Lin->C, dpg::num_sms());
  grid = (int)std::min<size_t>((size_t)grid, fit);
  DpgLaunch L = *Lin;
  L.scratch = base;
  size_t bytes = (size_t)plan->sm_total * sizeof(double);
  k<<<grid, NT, bytes, stream>>>(*plan, L);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}
