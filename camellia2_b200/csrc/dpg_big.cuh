// dpg_big.cuh — large buckets (N > 192 or M > 120 after padding), included by dpg_kernel.cu.
//
// One persistent CTA (16 warps) per SM walks the cells.  A cell's matrices do not fit in
// shared memory, so each CTA owns a workspace in global memory (L2-resident for the
// smaller buckets) holding the lower triangle of
//
//     Z = [[ S G S , S E ],        E = [B^T | F]  (N x (M + 1), device trial order),
//          [ E^T S ,  0  ]]        S = diag(G_ii^-1/2)  (DPOEQU scaling, BF.cpp:944-960)
//
// rows/columns: device test rows, then device trial columns (fields, traces, F).
//   1. Per-point factors: w|J| and the IP rows' Piola-mapped coefficients at the Gram points,
//      the terms' (w|J| or side measure) x coefficient x normal x parity x Piola row at the
//      B points (LinearTerm::integrate, LinearTerm.cpp:427-627; BasisEvaluation.cpp:182-390).
//   2. Formation by 64 x 64 tiles on the FP64 tensor cores (mma.m16n8k16.f64): a G tile sums
//      w|J| L_r(v_i) L_r(v_j) over the points and the IP rows r touching both tiles'
//      test vars (IP::computeInnerProductMatrix, IP.cpp:215-292); an E tile sums trial value x
//      test-operator value over the points of every segment and term touching the tile
//      (TBF::stiffnessMatrix, BF.cpp:575-656; RHS.cpp:68-82).  The diagonal G tiles come
//      first and give the scales S.
//   3. Np steps of a blocked right-looking Cholesky: the 64 x 64 diagonal block is factored in
//      shared memory as 8 x 8 tiles (the single-CTA kernel's tile Cholesky) and inverted by block
//      forward substitution, the rows below it become L panels (the rows of
//      W^T = (L^-1 E)^T, BF.cpp:987-988) and the trailing update subtracts L_I L_J^T
//      (DSYRK, BF.cpp:993-1005).  The trailing block is then -E^T G^-1 E = -[[K, l], [l^T, .]].
//   4. K, l are written out, the trailing block is negated, and nfp more steps over the field
//      columns leave [S s] = the Schur complement (CondensedDofInterpreter.cpp:1138-1192).
// No step waits on another CTA or on an asynchronous copy.

constexpr int ZT = 64;  // tile edge
constexpr int ZL = 68;  // shared row stride, == 4 (mod 16) doubles: conflict-free DMMA fragments
// ZK (template parameter below): k-chunk of a formation tile, 16 or 32 points (one or two
// m16n8k16 steps per chunk); the plan's big_zk, chosen by dpg_plan_autotune
constexpr int BIG_NOFAIL = 0x7fffffff;

struct BigSm {
  double* D;   // [64][ZL] diagonal block, factored in place
  double* Xi;  // [64][ZL] inverse of its factor
  double* LI;  // [64][ZL] L panel rows of the current row block
  double* LJ;  // [64][ZL] panel rows of the column block / staging of the raw panel
  double* LJ1; // [64][ZL] second panel buffer (double buffering of the column blocks)
  double* fa;  // [2][2][ZK][ZL] formation operands (rows, columns) x two chunks (aliases D..LJ1)
  double* sc;  // [Np] equilibration scales
  int* col;    // [Np] test row record: var << 16 | local dof, or -1 (padding row)
  int* ints;   // [0] first failing G column, [1] first failing field column, [64..] relevance lists
  double* nodes;
};

__device__ __forceinline__ BigSm big_views(const DpgPlanDev& P) {
  double* const sm = dpg_smem;
  BigSm S;
  S.D = sm;
  S.Xi = sm + ZT * ZL;
  S.LI = sm + 2 * ZT * ZL;
  S.LJ = sm + 3 * ZT * ZL;
  S.LJ1 = sm + 4 * ZT * ZL;
  S.fa = sm;
  S.sc = sm + P.bs_sc;
  S.col = reinterpret_cast<int*>(sm + P.bs_col);
  S.ints = reinterpret_cast<int*>(sm + P.bs_int);
  S.nodes = sm + P.bs_nodes;
  return S;
}

// acc (a 16 x 16 warp tile: rows wr.., columns wc..) += A B over one ZK chunk, operands stored
// k-major: A[r][k] = fa[k][r], B[k][c] = fb[k][c].  The k16 steps alternate between acc and
// acc2, so four independent DMMA chains are in flight.
template <int ZK>
__device__ __forceinline__ void big_mma_kmajor(const double* fa, const double* fb, int wr, int wc, int g, int t,
                                               double (&acc)[2][4], double (&acc2)[2][4]) {
#pragma unroll
  for (int s16 = 0; s16 < ZK / 16; s16++) {
    const double* fa_s = fa + s16 * 16 * ZL;
    const double* fb_s = fb + s16 * 16 * ZL;
    double a[8];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      a[2 * i] = fa_s[(t + 4 * i) * ZL + wr + g];
      a[2 * i + 1] = fa_s[(t + 4 * i) * ZL + wr + g + 8];
    }
#pragma unroll
    for (int nb = 0; nb < 2; nb++) {
      double b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) b[i] = fb_s[(t + 4 * i) * ZL + wc + nb * 8 + g];
      dmma16((s16 & 1) ? acc2[nb] : acc[nb], a, b);
    }
  }
}

// acc += A B^T over k in [0, kn) (kn a multiple of 16), both stored row-major [row][k].  Odd
// k-steps go to a second set of accumulators, so four independent DMMA chains are in flight.
__device__ __forceinline__ void big_mma_rows(const double* A, const double* B, int kn, int wr, int wc, int g, int t,
                                             double (&acc)[2][4]) {
  double acc2[2][4];
#pragma unroll
  for (int nb = 0; nb < 2; nb++) acc2[nb][0] = acc2[nb][1] = acc2[nb][2] = acc2[nb][3] = 0.0;
  for (int k0 = 0; k0 < kn; k0 += 32) {
#pragma unroll
    for (int half = 0; half < 2; half++) {
      const int kk = k0 + 16 * half;
      if (kk < kn) {
        double a[8];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          a[2 * i] = A[(wr + g) * ZL + kk + t + 4 * i];
          a[2 * i + 1] = A[(wr + g + 8) * ZL + kk + t + 4 * i];
        }
#pragma unroll
        for (int nb = 0; nb < 2; nb++) {
          double b[4];
#pragma unroll
          for (int i = 0; i < 4; i++) b[i] = B[(wc + nb * 8 + g) * ZL + kk + t + 4 * i];
          dmma16(half ? acc2[nb] : acc[nb], a, b);
        }
      }
    }
  }
#pragma unroll
  for (int nb = 0; nb < 2; nb++)
#pragma unroll
    for (int e = 0; e < 4; e++) acc[nb][e] += acc2[nb][e];
}

// Test vars whose (padded) rows meet [r0, r0 + 64).
__device__ __forceinline__ int big_var_mask(const DpgPlanDev& P, int r0) {
  int m = 0;
  for (int a = 0; a < P.ntest; a++) {
    const int lo = P.test[a].dev_off, hi = lo + P.test[a].ntiles * 8;
    if (lo < r0 + ZT && hi > r0) m |= 1 << a;
  }
  return m;
}

// Per-point factors of one cell (workspace): wq[q] = w|J| at the Gram points;
// bh[q][r][a][k] = sum over IP entries of row r on var a of coef x slot x T_a[slot_e][k];
// vt[row][k] = (w|J| or side measure) x coef x slot x (n_c) x (parity) x T_op[k] per term and point.
__device__ void big_prep(const DpgPlanDev& P, const DpgLaunch& L, int cell, const BigSm& S, double* wq, double* bh,
                         double* vt) {
  const int tid = threadIdx.x;
  const int d = P.d, nv = P.nv;
  const double* co = L.coeff ? L.coeff + (size_t)cell * P.nslots * P.Ptot : nullptr;
  for (int task = tid; task < P.QGpad * P.niprows; task += NT) {
    const int q = task / P.niprows, r = task - q * P.niprows;
    double gq[GEO];
    point_geometry(d, nv, S.nodes, P.dNG + (size_t)q * nv * d, P.wG[q], nullptr, gq);
    if (r == 0) wq[q] = gq[19];
    for (int a = 0; a < P.ntest; a++) {
      double b0 = 0.0, b1 = 0.0, b2 = 0.0, b3 = 0.0;
      for (int e = P.rowstart[r]; e < P.rowstart[r + 1]; e++) {
        const DpgIPEnt& E = P.ipent[e];
        if ((E.gslot >> 2) != a) continue;
        double v = E.coef;
        if (E.slot >= 0) v *= (q < P.QG && co) ? co[E.slot * P.Ptot + q] : 0.0;
        double tr[4];
        trow_slot(P.test[a].space, d, E.gslot & 3, gq, tr);
        b0 += v * tr[0]; b1 += v * tr[1]; b2 += v * tr[2]; b3 += v * tr[3];
      }
      double* dst = bh + ((size_t)(q * P.niprows + r) * P.ntest + a) * 4;
      dst[0] = b0; dst[1] = b1; dst[2] = b2; dst[3] = b3;
    }
  }
  const int nvt = P.nbe > 0 ? P.be[P.nbe - 1].z + P.be[P.nbe - 1].w : 0;
  const int8_t* par = L.parity + (size_t)cell * P.ns;
  for (int task = tid; task < nvt; task += NT) {
    int e = 0;
    while (task >= P.be[e].z + P.be[e].w) e++;
    const int4 be = P.be[e];
    const int q = task - be.z;
    const DpgSeg& Sg = P.seg[be.x];
    const DpgBTerm& Tm = P.bterm[Sg.term0 + be.y];
    const int pt = Sg.geo0 + q;
    double gq[GEO];
    point_geometry(d, nv, S.nodes, P.dNB + (size_t)pt * nv * d, P.wB[pt], Sg.side >= 0 ? P.tangB + (size_t)pt * 6 : nullptr,
                   gq);
    double v = gq[19] * Tm.coef;
    if (Tm.slot >= 0) v *= co ? co[Tm.slot * P.Ptot + Sg.pbase + q] : 0.0;
    if (Tm.normal_comp >= 0) v *= gq[20 + Tm.normal_comp];
    if (Tm.kind == DPG_VAR_FLUX) v *= (double)par[Sg.side];
    double tr[4];
    trow_op(P.test[Tm.test_var].space, d, Tm.test_op, gq, tr);
    double* dst = vt + (size_t)task * 4;
    dst[0] = v * tr[0]; dst[1] = v * tr[1]; dst[2] = v * tr[2]; dst[3] = v * tr[3];
  }
}

// One formation tile.  kind 0: G rows r0.., columns c0.. (test rows); kind 1: E^T rows
// (device trial columns) r0.., columns c0.. (test rows).
template <int ZK>
__device__ void big_form_tile(const DpgPlanDev& P, const DpgLaunch& L, int kind, int r0, int c0, bool diag, double* Z,
                              const BigSm& S, const double* wq, const double* bh, const double* vt) {
  (void)L;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wr = (warp >> 2) * 16, wc = (warp & 3) * 16;
  int* rel = S.ints + 64;    // relevant IP rows (kind 0) or E entries (kind 1)
  int* relk = S.ints + 192;  // kind 1: first k of each relevant entry, then the total
  __syncthreads();           // lists and operand buffers free
  if (tid == 0) {
    int n = 0, k = 0;
    if (kind == 0) {
      const int mr = big_var_mask(P, r0), mc = big_var_mask(P, c0);
      for (int r = 0; r < P.niprows; r++)
        if ((P.ipmask[r] & mr) && (P.ipmask[r] & mc)) rel[n++] = r;
      k = n * P.QG;
    } else {
      const int mc = big_var_mask(P, c0);
      for (int e = 0; e < P.nbe; e++) {
        const int4 be = P.be[e];
        const DpgBTerm& Tm = P.bterm[P.seg[be.x].term0 + be.y];
        if (!((mc >> Tm.test_var) & 1)) continue;
        if (Tm.col0 >= r0 + ZT || Tm.col0 + Tm.ncol <= r0) continue;
        rel[n] = e;
        relk[n] = k;
        k += be.w;
        n++;
      }
    }
    relk[120] = n;
    relk[121] = k;
  }
  __syncthreads();
  const int nrel = relk[120], nk = relk[121];
  double acc[2][4], acc2[2][4];
#pragma unroll
  for (int nb = 0; nb < 2; nb++)
#pragma unroll
    for (int e = 0; e < 4; e++) acc[nb][e] = acc2[nb][e] = 0.0;
  // operands of k-chunk k0 (2 sides x ZK x 64 values) into buffer pair buf; chunk c + 1 is
  // formed while the MMAs of chunk c run on the other pair, one barrier per chunk.  A thread's
  // column is the same for every value it forms (NT is a multiple of 64), so its column records
  // are read once per tile; all of a thread's values are computed before any is stored, so
  // their loads overlap instead of waiting behind the shared-memory stores.
  constexpr int NU = 2 * ZK * ZT / NT;
  const int cc = tid & (ZT - 1);
  int crec[2];
#pragma unroll
  for (int side = 0; side < 2; side++) {
    const int i = (side ? c0 : r0) + cc;
    crec[side] = (kind == 1 && side == 0) ? -1 : (i < P.Np ? S.col[i] : -1);
  }
  // kind 1: each thread's k index only grows (chunk by chunk, and with u inside a chunk), so the
  // entry holding it is found by a forward cursor per side instead of a scan from the start
  int ecur[2] = {0, 0};
  // A thread forms KPT consecutive k of each side.  G tiles number k point-major (k = q nrel +
  // row), so a thread's run mostly stays on one point and reads its column's four reference slot
  // values once for all the IP rows.
  constexpr int KPT = ZK / (NT / ZT);
  auto operands = [&](int k0, int buf) {
    double* const fa = S.fa + buf * 2 * ZK * ZL;
    double vals[NU];
    int lastq = -1;
    double fv[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int u = 0; u < NU; u++) {
      const int side = u / KPT, kl = (tid >> 6) * KPT + (u % KPT);
      if (u % KPT == 0) lastq = -1;
      const int kk = k0 + kl;
      double val = 0.0;
      if (kk < nk) {
        if (kind == 0) {
          const int rec = crec[side];
          if (rec >= 0) {
            const int q = kk / nrel, r = rel[kk - q * nrel];
            const int a = rec >> 16;
            if (q != lastq) {
              const int ld = P.test[a].ldA;
              const double* f = P.frefG + (size_t)q * P.featstride + P.test[a].foff + (rec & 0xffff);
              fv[0] = __ldg(f); fv[1] = __ldg(f + ld); fv[2] = __ldg(f + 2 * ld); fv[3] = __ldg(f + 3 * ld);
              lastq = q;
            }
            const double* b = bh + ((size_t)(q * P.niprows + r) * P.ntest + a) * 4;
            val = b[0] * fv[0] + b[1] * fv[1] + b[2] * fv[2] + b[3] * fv[3];
            if (side == 0) val *= wq[q];
          }
        } else {
          int ei = ecur[side];
          while (ei + 1 < nrel && kk >= relk[ei + 1]) ei++;
          ecur[side] = ei;
          const int4 be = P.be[rel[ei]];
          const int q = kk - relk[ei];
          const DpgSeg& Sg = P.seg[be.x];
          const DpgBTerm& Tm = P.bterm[Sg.term0 + be.y];
          const double* rq = Sg.rec + (size_t)q * Sg.rec_len;
          if (side == 0) {
            const int j = r0 + cc;
            if (j >= Tm.col0 && j < Tm.col0 + Tm.ncol) val = __ldg(rq + Sg.tvoff[be.y] + (j - Tm.col0));
          } else {
            const int rec = crec[1];
            if (rec >= 0 && (rec >> 16) == Tm.test_var) {
              const int ld = P.test[Tm.test_var].ldA;
              const double* f = rq + P.test[Tm.test_var].foff + (rec & 0xffff);
              const double* v4 = vt + (size_t)(be.z + q) * 4;
              val = v4[0] * __ldg(f) + v4[1] * __ldg(f + ld) + v4[2] * __ldg(f + 2 * ld) + v4[3] * __ldg(f + 3 * ld);
            }
          }
        }
      }
      vals[u] = val;
    }
#pragma unroll
    for (int u = 0; u < NU; u++) {
      const int side = u / KPT, kl = (tid >> 6) * KPT + (u % KPT);
      fa[side * ZK * ZL + kl * ZL + cc] = vals[u];
    }
  };
  if (nk > 0) operands(0, 0);
  __syncthreads();
  for (int k0 = 0, c = 0; k0 < nk; k0 += ZK, c++) {
    // the products of chunk c are issued first, so they run while chunk c + 1's loads are in flight
    const double* fa = S.fa + (c & 1) * 2 * ZK * ZL;
    big_mma_kmajor<ZK>(fa, fa + ZK * ZL, wr, wc, g, t, acc, acc2);
    if (k0 + ZK < nk) operands(k0 + ZK, (c + 1) & 1);
    __syncthreads();
  }
#pragma unroll
  for (int nb = 0; nb < 2; nb++)
#pragma unroll
    for (int e = 0; e < 4; e++) acc[nb][e] += acc2[nb][e];
  const int ld = P.ldz;
  if (kind == 0) {
    if (diag) {
      // the diagonal of G gives the scales of these rows
#pragma unroll
      for (int nb = 0; nb < 2; nb++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int row = wr + g + (e >> 1) * 8, cl = wc + nb * 8 + 2 * t + (e & 1);
          const int i = r0 + row;
          if (row == cl && i < P.Np) {
            double s = 1.0;
            if (S.col[i] >= 0) {
              const double gii = acc[nb][e];
              if (gii > 0.0) s = 1.0 / sqrt(gii);
              else atomicMin(&S.ints[0], i);
            }
            S.sc[i] = s;
          }
        }
      __syncthreads();
    }
#pragma unroll
    for (int nb = 0; nb < 2; nb++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int i = r0 + wr + g + h * 8, j = c0 + wc + nb * 8 + 2 * t;
        if (i < P.Np && j < P.Np) {
          const double si = S.sc[i];
          double2 v = make_double2(acc[nb][2 * h] * si * S.sc[j], acc[nb][2 * h + 1] * si * S.sc[j + 1]);
          if (diag && S.col[i] < 0) {
            if (i == j) v.x = 1.0;
            if (i == j + 1) v.y = 1.0;
          }
          *reinterpret_cast<double2*>(Z + (size_t)i * ld + j) = v;
        }
      }
  } else {
#pragma unroll
    for (int nb = 0; nb < 2; nb++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int j = r0 + wr + g + h * 8, i = c0 + wc + nb * 8 + 2 * t;
        if (j < P.Mp && i < P.Np)
          *reinterpret_cast<double2*>(Z + (size_t)(P.Np + j) * ld + i) =
              make_double2(acc[nb][2 * h] * S.sc[i], acc[nb][2 * h + 1] * S.sc[i + 1]);
      }
  }
}

// The diagonal block Z[k0 .. k0+w) (w <= 64, padded to 64 with a unit diagonal): factored as
// 8 x 8 tiles in AK layout (in D) by the single-CTA kernel's blocked Cholesky (tile_cholesky:
// look-ahead, diagonal tiles factored in registers), then X = L_kk^-1 by block forward
// substitution, one warp per 8-column block (X_cc = L_cc^-1, X_ic = -L_ii^-1 sum_k L_ik X_kc),
// into Xi (row-major, zero above the diagonal).  The first column whose pivot is not positive
// goes to *fail (atomicMin).
__device__ __forceinline__ void big_diag_block(const double* Z, int ld, int k0, int w, const BigSm& S, int* fail) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  constexpr int NBD = ZT / 8;                 // 8 tiles
  constexpr int NTD = NBD * (NBD + 1) / 2;    // 36 lower tiles
  double* const T = S.D;
  double* const linv = S.LI;                  // [8][64] inverse diagonal tiles
  double* const invd = S.LI + NBD * 64;       // [64]
  int* const tri = reinterpret_cast<int*>(S.LI + NBD * 64 + ZT);
  int* const flag = tri + 64;
  __syncthreads();
  for (int e = tid; e < NTD * 64; e += NT) {
    const int tau = e >> 6, idx = e & 63;
    int I = 0;
    while ((I + 1) * (I + 2) / 2 <= tau) I++;
    const int J = tau - I * (I + 1) / 2;
    const int r = 8 * I + ((idx >> 2) & 7), c = 8 * J + (idx >> 5) * 4 + (idx & 3);
    double v = (r == c) ? 1.0 : 0.0;
    if (r < w && c <= r) v = Z[(size_t)(k0 + r) * ld + k0 + c];
    T[e] = v;
    if (idx == 0) tri[tau] = I | (J << 8);
  }
  if (tid == 0) *flag = 0;
  __syncthreads();
  tile_cholesky((int)(T - dpg_smem), NBD, NBD, (int)(flag - reinterpret_cast<int*>(dpg_smem)), 1,
                (int)(reinterpret_cast<double*>(tri) - dpg_smem), (int)(invd - dpg_smem), (int)(linv - dpg_smem));
  if (tid == 0 && *flag > 0) atomicMin(fail, k0 + *flag - 1);
  if (warp < NBD) {
    const int cb = warp;
    double2 acc[NBD];
#pragma unroll
    for (int i = 0; i < NBD; i++)
      acc[i] = (i == cb) ? make_double2(g == 2 * t ? 1.0 : 0.0, g == 2 * t + 1 ? 1.0 : 0.0) : make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < NBD; k++) {
      if (k >= cb) {
        double y0, y1;
        cfrag_to_bfrag(acc[k], lane, y0, y1);
        const double* Li = linv + k * 64;
        double2 x = make_double2(0.0, 0.0);
        dmma(x, Li[lane], y0);
        dmma(x, Li[32 + lane], y1);
        acc[k] = x;
        double x0, x1;
        cfrag_to_bfrag(x, lane, x0, x1);
        x0 = -x0;
        x1 = -x1;
#pragma unroll
        for (int i = k + 1; i < NBD; i += 2) {
          const double* Lik = T + (i * (i + 1) / 2 + k) * 64;
          if (i + 1 < NBD) {
            const double* Li1k = T + ((i + 1) * (i + 2) / 2 + k) * 64;
            dmma16x8(acc[i], acc[i + 1], Lik[lane], Li1k[lane], Lik[32 + lane], Li1k[32 + lane], x0, x1);
          } else {
            dmma(acc[i], Lik[lane], x0);
            dmma(acc[i], Lik[32 + lane], x1);
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < NBD; i++)
      *reinterpret_cast<double2*>(S.Xi + (8 * i + g) * ZL + 8 * cb + 2 * t) = acc[i];
  }
  __syncthreads();
}

// Steps kb .. ke-1 of a right-looking Cholesky of the lower triangle of Z (order Zn).  The
// first column whose pivot is not positive goes to *fail (atomicMin); the cell's outputs are
// then undefined (info reports the column).
__device__ void big_cholesky(const DpgPlanDev& P, double* Z, int kb, int ke, const BigSm& S, int* fail) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wr = (warp >> 2) * 16, wc = (warp & 3) * 16;
  const int ld = P.ldz, Zn = P.Zn;
  for (int k0 = kb; k0 < ke; k0 += ZT) {
    const int w = min(ZT, ke - k0);
    const int wk = (w + 15) & ~15;
    big_diag_block(Z, ld, k0, w, S, fail);
    // rows below the block: panel L_I = Z_I,k L_kk^-T (stored back), then Z_IJ -= L_I L_J^T
    const int rbeg = k0 + w;
    const int nrb = (Zn - rbeg + ZT - 1) / ZT;
    for (int bi = 0; bi < nrb; bi++) {
      const int ri0 = rbeg + bi * ZT, nri = min(ZT, Zn - ri0);
      for (int e = tid; e < ZT * ZT; e += NT) {
        const int r = e >> 6, c = e & (ZT - 1);
        S.LJ[r * ZL + c] = (r < nri && c < w) ? Z[(size_t)(ri0 + r) * ld + k0 + c] : 0.0;
      }
      __syncthreads();
      double acc[2][4];
#pragma unroll
      for (int nb = 0; nb < 2; nb++) acc[nb][0] = acc[nb][1] = acc[nb][2] = acc[nb][3] = 0.0;
      big_mma_rows(S.LJ, S.Xi, wk, wr, wc, g, t, acc);
#pragma unroll
      for (int nb = 0; nb < 2; nb++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int r = wr + g + h * 8, c = wc + nb * 8 + 2 * t;
          const double2 v = make_double2(acc[nb][2 * h], acc[nb][2 * h + 1]);
          *reinterpret_cast<double2*>(S.LI + r * ZL + c) = v;
          if (r < nri && c < w) *reinterpret_cast<double2*>(Z + (size_t)(ri0 + r) * ld + k0 + c) = v;
        }
      // column blocks bj < bi come from the stored panel, double buffered through registers:
      // tile bj + 1 is loaded while the MMAs of tile bj run; one barrier per tile
      double pre[ZT * ZT / NT];
      auto load_panel = [&](int bj) {
        const int rj0 = rbeg + bj * ZT, nrj = min(ZT, Zn - rj0);
#pragma unroll
        for (int u = 0; u < ZT * ZT / NT; u++) {
          const int e = tid + u * NT, r = e >> 6, c = e & (ZT - 1);
          pre[u] = (r < nrj && c < w) ? Z[(size_t)(rj0 + r) * ld + k0 + c] : 0.0;
        }
      };
      auto store_panel = [&](double* dst) {
#pragma unroll
        for (int u = 0; u < ZT * ZT / NT; u++) {
          const int e = tid + u * NT;
          dst[(e >> 6) * ZL + (e & (ZT - 1))] = pre[u];
        }
      };
      if (bi > 0) {
        load_panel(0);
        store_panel(S.LJ1);
      }
      __syncthreads();
      for (int bj = 0; bj <= bi; bj++) {
        const int rj0 = rbeg + bj * ZT, nrj = min(ZT, Zn - rj0);
        const double* Lj = bj == bi ? S.LI : ((bj & 1) ? S.LJ : S.LJ1);
        if (bj + 1 < bi) load_panel(bj + 1);
        double2 zo[2][2];
#pragma unroll
        for (int nb = 0; nb < 2; nb++)
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int r = wr + g + h * 8, c = wc + nb * 8 + 2 * t;
            zo[nb][h] = (r < nri && c < nrj) ? *reinterpret_cast<const double2*>(Z + (size_t)(ri0 + r) * ld + rj0 + c)
                                             : make_double2(0.0, 0.0);
          }
#pragma unroll
        for (int nb = 0; nb < 2; nb++) acc[nb][0] = acc[nb][1] = acc[nb][2] = acc[nb][3] = 0.0;
        // on the diagonal tile, warp tiles wholly above the diagonal are not needed
        const bool upper = bj == bi && wc >= wr + 16;
        if (!upper) big_mma_rows(S.LI, Lj, wk, wr, wc, g, t, acc);
#pragma unroll
        for (int nb = 0; nb < 2; nb++)
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int r = wr + g + h * 8, c = wc + nb * 8 + 2 * t;
            if (!upper && r < nri && c < nrj)
              *reinterpret_cast<double2*>(Z + (size_t)(ri0 + r) * ld + rj0 + c) =
                  make_double2(zo[nb][h].x - acc[nb][2 * h], zo[nb][h].y - acc[nb][2 * h + 1]);
          }
        if (bj + 1 < bi) store_panel(((bj + 1) & 1) ? S.LJ : S.LJ1);
        __syncthreads();
      }
    }
  }
  __syncthreads();
}

// Per-CTA table of a large plan: the test var and local dof of every device test row.
__device__ __forceinline__ void big_cta_setup(const DpgPlanDev& P, const BigSm& S) {
  for (int i = threadIdx.x; i < P.Np; i += NT) {
    int rec = -1;
    for (int a = 0; a < P.ntest; a++) {
      const int il = i - P.test[a].dev_off;
      if (il >= 0 && il < P.test[a].card) rec = (a << 16) | il;
    }
    S.col[i] = rec;
  }
}

// One cell of a large plan; Z is this CTA's workspace (bz_per_cta doubles).
template <int ZK>
__device__ __forceinline__ void big_cell_body(const DpgPlanDev& P, const DpgLaunch& L, int cell, const BigSm& S, double* const Z) {
  const int tid = threadIdx.x;
  double* const wq = Z + P.bz_wq;
  double* const bh = Z + P.bz_bh;
  double* const vt = Z + P.bz_vt;
  const int Np = P.Np, Mp = P.Mp, M = P.M, ld = P.ldz;
  {
    __syncthreads();
    if (tid == 0) { S.ints[0] = BIG_NOFAIL; S.ints[1] = BIG_NOFAIL; }
    if (tid < P.nv * P.d) S.nodes[tid] = L.nodes[(size_t)cell * P.nv * P.d + tid];
    __syncthreads();
    big_prep(P, L, cell, S, wq, bh, vt);
    for (size_t e = tid; e < (size_t)Mp * Mp; e += NT) {
      const int r = (int)(e / Mp), c = (int)(e - (size_t)r * Mp);
      if (c <= r) Z[(size_t)(Np + r) * ld + Np + c] = 0.0;
    }
    __syncthreads();
    const int nbg = (Np + ZT - 1) / ZT, nbm = (Mp + ZT - 1) / ZT;
    for (int I = 0; I < nbg; I++) big_form_tile<ZK>(P, L, 0, I * ZT, I * ZT, true, Z, S, wq, bh, vt);
    for (int I = 1; I < nbg; I++)
      for (int J = 0; J < I; J++) big_form_tile<ZK>(P, L, 0, I * ZT, J * ZT, false, Z, S, wq, bh, vt);
    for (int J = 0; J < nbm; J++)
      for (int I = 0; I < nbg; I++) big_form_tile<ZK>(P, L, 1, J * ZT, I * ZT, false, Z, S, wq, bh, vt);
    if (L.parts) {
      // G (N, N), B (M, N) and F (N) in user numbering: Z unscaled (dpg_assemble_parts)
      __syncthreads();
      const int N = P.N;
      if (L.G)
        for (int e = tid; e < N * N; e += NT) {
          const int ur = e / N, uc = e - ur * N;
          const int dr = __ldg(P.u2d_test + ur), dc = __ldg(P.u2d_test + uc);
          L.G[(size_t)cell * N * N + e] = Z[(size_t)max(dr, dc) * ld + min(dr, dc)] / (S.sc[dr] * S.sc[dc]);
        }
      if (L.B)
        for (int e = tid; e < M * N; e += NT) {
          const int ut = e / N, us = e - ut * N;
          const int ds = __ldg(P.u2d_test + us);
          L.B[(size_t)cell * M * N + e] = Z[(size_t)(Np + __ldg(P.u2d_trial + ut)) * ld + ds] / S.sc[ds];
        }
      if (L.F)
        for (int us = tid; us < N; us += NT) {
          const int ds = __ldg(P.u2d_test + us);
          L.F[(size_t)cell * N + us] = Z[(size_t)(Np + P.fcol) * ld + ds] / S.sc[ds];
        }
      __syncthreads();
      return;
    }
    big_cholesky(P, Z, 0, Np, S, &S.ints[0]);
    if (L.energy) {
      // energy error (dpg_energy_error): the rows below the test block now hold W = L^-1 E, so
      // e^2 = || L^-1 F - L^-1 B^T x ||^2 is a sum over the test rows, with no cancellation
      const double* x = L.xsol + (size_t)cell * M;
      double part = 0.0;
      for (int k = tid; k < Np; k += NT) {
        double r = Z[(size_t)(Np + P.fcol) * ld + k];
        for (int ut = 0; ut < M; ut++) r -= Z[(size_t)(Np + __ldg(P.u2d_trial + ut)) * ld + k] * x[ut];
        part += r * r;
      }
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
      double* red = S.LI;  // free after the factorisation
      if ((tid & 31) == 0) red[tid >> 5] = part;
      __syncthreads();
      if (tid == 0) {
        double e2 = 0.0;
        for (int w = 0; w < NT / 32; w++) e2 += red[w];
        // a failed factorisation of the test block leaves no energy to report
        L.energy[cell] = S.ints[0] == BIG_NOFAIL ? sqrt(e2) : __longlong_as_double(0x7ff8000000000000ll);
      }
    } else if (L.B) {
      // DLS local matrices (dpg_assemble_dls): the rows below the test block hold
      // W^T = (L^-1 E)^T, so W = L^-1 B^T and y = L^-1 F are read out in user numbering
      const int N = P.N;
      double* Wc = L.B + (size_t)cell * M * N;
      for (size_t e = tid; e < (size_t)M * N; e += NT) {
        const int ut = (int)(e / N), us = (int)(e - (size_t)ut * N);
        Wc[e] = Z[(size_t)(Np + __ldg(P.u2d_trial + ut)) * ld + __ldg(P.u2d_test + us)];
      }
      if (L.F)
        for (int us = tid; us < N; us += NT) L.F[(size_t)cell * N + us] = Z[(size_t)(Np + P.fcol) * ld + __ldg(P.u2d_test + us)];
    } else {
    // trailing block = -[K_ext]: K, l out, then negate (padded field columns get a unit pivot)
    const double* T = Z + (size_t)Np * ld + Np;
    if (L.K)
      for (size_t e = tid; e < (size_t)M * M; e += NT) {
        const int ur = (int)(e / M), uc = (int)(e - (size_t)ur * M);
        const int dr = __ldg(P.u2d_trial + ur), dc = __ldg(P.u2d_trial + uc);
        L.K[(size_t)cell * M * M + e] = -T[(size_t)max(dr, dc) * ld + min(dr, dc)];
      }
    if (L.l)
      for (int u = tid; u < M; u += NT) L.l[(size_t)cell * M + u] = -T[(size_t)P.fcol * ld + __ldg(P.u2d_trial + u)];
    if (L.S || L.s) {
      __syncthreads();
      for (size_t e = tid; e < (size_t)Mp * Mp; e += NT) {
        const int r = (int)(e / Mp), c = (int)(e - (size_t)r * Mp);
        if (c <= r) {
          double* p = Z + (size_t)(Np + r) * ld + Np + c;
          *p = (r == c && r < P.nfp && __ldg(P.dev2user_trial + r) < 0) ? 1.0 : -*p;
        }
      }
      big_cholesky(P, Z, Np, Np + P.nfp, S, &S.ints[1]);
      const int nt = P.nt, nf = P.nf;
      if (L.S)
        for (size_t e = tid; e < (size_t)nt * nt; e += NT) {
          const int ur = (int)(e / nt), uc = (int)(e - (size_t)ur * nt);
          const int dr = __ldg(P.u2d_trial + nf + ur), dc = __ldg(P.u2d_trial + nf + uc);
          L.S[(size_t)cell * nt * nt + e] = T[(size_t)max(dr, dc) * ld + min(dr, dc)];
        }
      if (L.s)
        for (int u = tid; u < nt; u += NT) L.s[(size_t)cell * nt + u] = T[(size_t)P.fcol * ld + __ldg(P.u2d_trial + nf + u)];
    }
    }
    __syncthreads();
    if (tid == 0 && L.info) {
      int v = 0;
      if (S.ints[0] != BIG_NOFAIL) {
        const int u = P.dev2user_test[S.ints[0]];
        v = (u >= 0 ? u : S.ints[0]) + 1;
      } else if (S.ints[1] != BIG_NOFAIL) {
        const int u = P.dev2user_trial[S.ints[1] - Np];
        v = -((u >= 0 ? u : S.ints[1] - Np) + 1);
      }
      L.info[cell] = v;
    }
  }
}

template <int ZK>
__global__ void __launch_bounds__(NT, 1) dpg_big_kernel(const __grid_constant__ DpgPlanDev P, const DpgLaunch L) {
  const BigSm S = big_views(P);
  big_cta_setup(P, S);
  for (int cell = blockIdx.x; cell < L.C; cell += gridDim.x)
    big_cell_body<ZK>(P, L, cell, S, L.scratch + (size_t)blockIdx.x * P.bz_per_cta);
}
