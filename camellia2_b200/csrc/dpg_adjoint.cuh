// dpg_adjoint.cuh — reverse mode of the per-cell assembly (included by dpg_kernel.cu
// inside its anonymous namespace; it reuses the forward phases defined there).
//
// For a loss J(K, l) with Kbar = dJ/dK and lbar = dJ/dl (no counterpart in the
// reference; the forward is TBF::localStiffnessMatrixAndRHS, BF.cpp:1385-1449):
//   X = G^-1 B, y = G^-1 F, Xe = [X | y]                  (N x (M+1), F rides as a column)
//   S_A = sym([[Kbar, lbar], [0, 0]])                     ((M+1) x (M+1))
//   P = Xe S_A,  [Bbar | Fbar] = 2 P,  Gbar = -P Xe^T      (Gbar symmetric, never formed)
// and the pull-back to the per-point coefficient slots:
//   G:   dJ/dslot_s(q) = -2 w|J| sum_{e: slot_e = s} coef_e (T_e f(q))^T P  .  Xe^T l_r(q)
//        with l_r(q) = sum_a beta_{r,a}(q) f_a(q) the IP row r at q (f: reference slots)
//   B,F: dJ/dslot_s(q) = 2 w|J| sum_{terms t: slot_t = s} coef_t (T_t f(q))^T P[:, cols_t] psi_t(q)
//   sides (separable terms): dJ/dslot_s(q) = 2 sum_c P[row_c, col_c] W[q][c] factor_t(q) / slot_s(q)
// The per-point products f(q)^T Xe and f(q)^T P are small GEMMs on the tensor
// cores over chunks of DPG_CHA points.

#define DPG_CHA 4  // quadrature points per pull-back chunk (two 8-row tiles of (point, slot))

// Element (r, c) of a C-fragment tiled N x (M+1) matrix in a scratch slot
// (tile (I, J) at ((J * NBT + I) * 32 + lane) double2, lane = r * 4 + c / 2).
__device__ __forceinline__ size_t cfrag_index(int NBT, int r, int c) {
  return ((size_t)((c >> 3) * NBT + (r >> 3)) * 32 + (r & 7) * 4 + ((c & 7) >> 1)) * 2 + (c & 1);
}

// Xe = G^-1 [B | F] per column tile: forward W = L^-1 Y, then backward X = L^-T W,
// in registers; the result replaces Y in the scratch slot.
template <int NBTM>
__device__ __forceinline__ void phase_adj_solve(const DpgPlanDev& P, const DpgLaunch& L) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const double* GT = dpg_smem + P.sm_gt;
  const double* LINV = dpg_smem + P.sm_linv;
  const int J = warp;
  if (J < P.MBT) {
    double2* scr = reinterpret_cast<double2*>(L.scratch + (size_t)blockIdx.x * P.scratch_per_cta) +
                   (size_t)J * P.NBT * 32 + lane;
    double2 acc[NBTM];
#pragma unroll
    for (int I = 0; I < NBTM; I++) acc[I] = (I < P.NBT) ? scr[I * 32] : make_double2(0.0, 0.0);
    // forward: X_k = L_kk^-1 Y_k; Y_i -= L_ik X_k
#pragma unroll
    for (int k = 0; k < NBTM; k++) {
      if (k < P.NBT) {
        double y0, y1;
        cfrag_to_bfrag(acc[k], lane, y0, y1);
        const double* Li = LINV + k * 64;
        double2 x = make_double2(0.0, 0.0);
        dmma(x, Li[lane], y0);
        dmma(x, Li[32 + lane], y1);
        acc[k] = x;
        double x0, x1;
        cfrag_to_bfrag(x, lane, x0, x1);
        x0 = -x0;
        x1 = -x1;
#pragma unroll
        for (int i = k + 1; i < NBTM; i += 2) {
          const double* Lik = GT + (i * (i + 1) / 2 + k) * 64;
          if (i + 1 < NBTM && i + 1 < P.NBT) {
            const double* Li1k = GT + ((i + 1) * (i + 2) / 2 + k) * 64;
            dmma16x8(acc[i], acc[i + 1], Lik[lane], Li1k[lane], Lik[32 + lane], Li1k[32 + lane], x0, x1);
          } else if (i < P.NBT) {
            dmma(acc[i], Lik[lane], x0);
            dmma(acc[i], Lik[32 + lane], x1);
          }
        }
      }
    }
    // backward: X_k = L_kk^-T W_k; W_i -= L_ki^T X_k for i < k.  A-fragments of a
    // transposed AK tile: element (t + 4h, g) at ((g >> 2) * 8 + t + 4h) * 4 + (g & 3).
    const int o0 = ((g >> 2) * 8 + t) * 4 + (g & 3), o1 = o0 + 16;
#pragma unroll
    for (int k = NBTM - 1; k >= 0; k--) {
      if (k < P.NBT) {
        double y0, y1;
        cfrag_to_bfrag(acc[k], lane, y0, y1);
        const double* Li = LINV + k * 64;
        double2 x = make_double2(0.0, 0.0);
        dmma(x, Li[o0], y0);
        dmma(x, Li[o1], y1);
        acc[k] = x;
        double x0, x1;
        cfrag_to_bfrag(x, lane, x0, x1);
        x0 = -x0;
        x1 = -x1;
        const double* Lk = GT + (k * (k + 1) / 2) * 64;  // tiles (k, i), i < k
#pragma unroll
        for (int i = 0; i < k; i += 2) {
          if (i + 1 < k) {
            dmma16x8(acc[i], acc[i + 1], Lk[i * 64 + o0], Lk[(i + 1) * 64 + o0], Lk[i * 64 + o1],
                     Lk[(i + 1) * 64 + o1], x0, x1);
          } else {
            dmma(acc[i], Lk[i * 64 + o0], x0);
            dmma(acc[i], Lk[i * 64 + o1], x1);
          }
        }
      }
    }
#pragma unroll
    for (int I = 0; I < NBTM; I++)
      if (I < P.NBT) scr[I * 32] = acc[I];
  }
  __syncthreads();
}

// P = Xe S_A with S_A built in shared memory from Kbar and lbar (user numbering).
template <int NBTM>
__device__ __forceinline__ void phase_adj_p(const DpgPlanDev& P, const DpgLaunch& L, int cell) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  double* SA = dpg_smem + P.a_sa;
  const int Mx = P.MBT * 8, ld = P.a_ldS;
  const double* Kb = L.Kbar + (size_t)cell * P.M * P.M;
  const double* lb = L.lbar ? L.lbar + (size_t)cell * P.M : nullptr;
  for (int e = tid; e < Mx * Mx; e += NT) {
    const int c = e / Mx, c2 = e - c * Mx;
    const int u = c < P.Mp ? P.dev2user_trial[c] : -1;
    const int u2 = c2 < P.Mp ? P.dev2user_trial[c2] : -1;
    double v = 0.0;
    if (u >= 0 && u2 >= 0) v = 0.5 * (Kb[(size_t)u * P.M + u2] + Kb[(size_t)u2 * P.M + u]);
    else if (c == P.fcol && u2 >= 0) v = lb ? 0.5 * lb[u2] : 0.0;
    else if (c2 == P.fcol && u >= 0) v = lb ? 0.5 * lb[u] : 0.0;
    SA[c * ld + c2] = v;
  }
  __syncthreads();
  const int J = warp;
  if (J < P.MBT) {
    const double* xe = L.scratch + (size_t)blockIdx.x * P.scratch_per_cta;
    double2 acc[NBTM];
#pragma unroll
    for (int I = 0; I < NBTM; I++) acc[I] = make_double2(0.0, 0.0);
    for (int K = 0; K < P.MBT; K++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const double b = SA[(K * 8 + 4 * h + t) * ld + J * 8 + g];
        // A[g][t] = Xe[I*8 + g][K*8 + 4h + t]
        const double* xk = xe + ((size_t)K * P.NBT * 32 + g * 4 + 2 * h + (t >> 1)) * 2 + (t & 1);
#pragma unroll
        for (int I = 0; I < NBTM; I++)
          if (I < P.NBT) dmma(acc[I], xk[I * 64], b);
      }
    }
    double2* p2 = reinterpret_cast<double2*>(L.scratch2 + (size_t)blockIdx.x * P.scratch_per_cta) +
                  (size_t)J * P.NBT * 32 + lane;
#pragma unroll
    for (int I = 0; I < NBTM; I++)
      if (I < P.NBT) p2[I * 32] = acc[I];
  }
  __syncthreads();
}

// out[q][a][k][c] = sum_i f[q][a][k][i] X[i][c] for the chunk's nq points, the
// column tiles ct < nct of [Xe | P] (ct < ncx from Xe, the rest from P).
__device__ __forceinline__ void adj_feature_gemm(const DpgPlanDev& P, const DpgLaunch& L, const double* fs, int fsl,
                                                 int nq, int nct, int ncx, double* out) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const double* xe = L.scratch + (size_t)blockIdx.x * P.scratch_per_cta;
  const double* pm = L.scratch2 + (size_t)blockIdx.x * P.scratch_per_cta;
  const int q0 = g >> 2, q1 = 2 + (g >> 2), k = g & 3;
  for (int ct = warp; ct < nct; ct += DPG_NWARPS) {
    const bool from_xe = ct < ncx;
    const int J = from_xe ? ct : ct - ncx;
    const double* src = from_xe ? xe : pm;
    for (int a = 0; a < P.ntest; a++) {
      const DpgTestVar& V = P.test[a];
      double2 acc0 = make_double2(0.0, 0.0), acc1 = make_double2(0.0, 0.0);
      const double* f0 = fs + q0 * fsl + V.foff + k * V.ldA + t;
      const double* f1 = fs + q1 * fsl + V.foff + k * V.ldA + t;
      const bool ok0 = q0 < nq, ok1 = q1 < nq;
      // 16 test rows per m16n8k16: A rows g = (point q0, slot k), rows g + 8 = (point q1, slot k)
      // (the vars' rows are padded to multiples of 16); the same accumulation order as four
      // m8n8k4 steps per point pair
      double c4[4] = {0.0, 0.0, 0.0, 0.0};
      for (int i = 0; i < V.ntiles * 8; i += 16) {
        double av[8], bv[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
          av[2 * j] = ok0 ? f0[i + 4 * j] : 0.0;
          av[2 * j + 1] = ok1 ? f1[i + 4 * j] : 0.0;
          bv[j] = src[cfrag_index(P.NBT, V.ntile0 * 8 + i + 4 * j + t, J * 8 + g)];
        }
        dmma16(c4, av, bv);
      }
      acc0 = make_double2(c4[0], c4[1]);
      acc1 = make_double2(c4[2], c4[3]);
      // C-fragment rows g -> (point 2R + g / 4, slot g % 4), columns 2t, 2t + 1
      if (ok0) *reinterpret_cast<double2*>(out + ((q0 * P.ntest + a) * 4 + k) * P.a_ldx + ct * 8 + 2 * t) = acc0;
      if (ok1) *reinterpret_cast<double2*>(out + ((q1 * P.ntest + a) * 4 + k) * P.a_ldx + ct * 8 + 2 * t) = acc1;
    }
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void phase_adj_pull(const DpgPlanDev& P, const DpgLaunch& L, int cell) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int d = P.d, nv = P.nv;
  DPG_SMEM_VIEWS(P);
  double* fs = sm + P.a_fs;
  double* xpf = sm + P.a_xpf;
  double* geo = sm + P.a_geo;
  double* beta = sm + P.a_beta;
  double* cbar = sm + P.a_cbar;
  const int Mx = P.MBT * 8;
  const int ncb = P.nslots * P.Ptot;
  for (int i = tid; i < ncb; i += NT) cbar[i] = 0.0;
  const int8_t* par_c = L.parity + (size_t)cell * P.ns;
  const double* pm = L.scratch2 + (size_t)blockIdx.x * P.scratch_per_cta;
  __syncthreads();
  // ---- Gram points ----
  if (P.ip_slots) {
    const int F = 4 * P.ntest;
    for (int q0 = 0; q0 < P.QG; q0 += DPG_CHA) {
      const int nq = min(DPG_CHA, P.QG - q0);
      for (int i = tid; i < nq * P.featstride; i += NT) fs[i] = P.frefG[(size_t)q0 * P.featstride + i];
      for (int q = tid; q < nq; q += NT)
        point_geometry(d, nv, nodes_s, P.dNG + (size_t)(q0 + q) * nv * d, P.wG[q0 + q], nullptr, geo + q * GEO);
      __syncthreads();
      for (int task = tid; task < nq * P.niprows * P.ntest; task += NT) {
        const int q = task / (P.niprows * P.ntest);
        const int rem = task - q * P.niprows * P.ntest;
        const int r = rem / P.ntest, a = rem - r * P.ntest;
        const double* gq = geo + q * GEO;
        double b0 = 0.0, b1 = 0.0, b2 = 0.0, b3 = 0.0;
        for (int e = P.rowstart[r]; e < P.rowstart[r + 1]; e++) {
          const DpgIPEnt& E = P.ipent[e];
          if ((E.gslot >> 2) != a) continue;
          double v = E.coef;
          if (E.slot >= 0) v *= coef_s[E.slot * P.Ptot + q0 + q];
          double tr[4];
          trow_slot(P.test[a].space, d, E.gslot & 3, gq, tr);
          b0 += v * tr[0]; b1 += v * tr[1]; b2 += v * tr[2]; b3 += v * tr[3];
        }
        double* dst = beta + (q * P.niprows + r) * F + 4 * a;
        dst[0] = b0; dst[1] = b1; dst[2] = b2; dst[3] = b3;
      }
      adj_feature_gemm(P, L, fs, P.featstride, nq, 2 * P.MBT, P.MBT, xpf);
      __syncthreads();
      // one warp per (point, slot): sum over the IP entries carrying the slot
      for (int task = warp; task < nq * P.nslots; task += DPG_NWARPS) {
        const int q = task / P.nslots, s = task - q * P.nslots;
        const double* gq = geo + q * GEO;
        double val = 0.0;
        for (int e = 0; e < P.nipent; e++) {
          const DpgIPEnt& E = P.ipent[e];
          if (E.slot != s) continue;
          const int ae = E.gslot >> 2;
          double te[4];
          trow_slot(P.test[ae].space, d, E.gslot & 3, gq, te);
          const double* br = beta + (q * P.niprows + E.row) * F;
          const double* pf = xpf + (q * P.ntest + ae) * 4 * P.a_ldx + Mx;
          double part = 0.0;
          for (int c = lane; c < Mx; c += 32) {
            double pe = 0.0, xl = 0.0;
#pragma unroll
            for (int kk = 0; kk < 4; kk++) pe += te[kk] * pf[kk * P.a_ldx + c];
            for (int a = 0; a < P.ntest; a++) {
              const double* xf = xpf + (q * P.ntest + a) * 4 * P.a_ldx;
#pragma unroll
              for (int kk = 0; kk < 4; kk++) xl += br[4 * a + kk] * xf[kk * P.a_ldx + c];
            }
            part += pe * xl;
          }
          val += E.coef * part;
        }
        val = warp_sum(val);
        if (lane == 0) cbar[s * P.Ptot + q0 + q] += -2.0 * gq[19] * val;
      }
      __syncthreads();
    }
  }
  // ---- volume B points (bilinear and load terms) ----
  if (P.b_slots) {
    const DpgSeg& S = P.seg[0];
    for (int q0 = 0; q0 < S.npts; q0 += DPG_CHA) {
      const int nq = min(DPG_CHA, S.npts - q0);
      for (int i = tid; i < nq * S.rec_len; i += NT) fs[i] = S.rec[(size_t)q0 * S.rec_len + i];
      for (int q = tid; q < nq; q += NT)
        point_geometry(d, nv, nodes_s, P.dNB + (size_t)(q0 + q) * nv * d, P.wB[q0 + q], nullptr, geo + q * GEO);
      __syncthreads();
      adj_feature_gemm(P, L, fs, S.rec_len, nq, P.MBT, 0, xpf);
      __syncthreads();
      for (int task = warp; task < nq * P.nslots; task += DPG_NWARPS) {
        const int q = task / P.nslots, s = task - q * P.nslots;
        const double* gq = geo + q * GEO;
        double val = 0.0;
        for (int lt = 0; lt < S.nterm; lt++) {
          const DpgBTerm& Tm = P.bterm[S.term0 + lt];
          if (Tm.slot != s) continue;
          const int a = Tm.test_var;
          double tr[4];
          trow_op(P.test[a].space, d, Tm.test_op, gq, tr);
          const double* pf = xpf + (q * P.ntest + a) * 4 * P.a_ldx;
          const double* psi = fs + q * S.rec_len + S.tvoff[lt];
          double part = 0.0;
          for (int m = lane; m < Tm.ncol; m += 32) {
            const int c = Tm.col0 + m;
            double pe = 0.0;
#pragma unroll
            for (int kk = 0; kk < 4; kk++) pe += tr[kk] * pf[kk * P.a_ldx + c];
            part += pe * psi[m];
          }
          val += Tm.coef * part;
        }
        val = warp_sum(val);
        if (lane == 0) cbar[s * P.Ptot + S.pbase + q0 + q] += 2.0 * gq[19] * val;
      }
      __syncthreads();
    }
  }
  // ---- side points of separable boundary terms ----
  if (P.se_slots) {
    const int nsp = P.ns * P.QS;
    for (int i = tid; i < nsp; i += NT)
      point_geometry(d, nv, nodes_s, P.dNB + (size_t)(P.QB + i) * nv * d, P.wB[P.QB + i], P.tangB + (size_t)(P.QB + i) * 6,
                     geo + i * GEO);
    __syncthreads();
    for (int task = warp; task < nsp * P.nslots; task += DPG_NWARPS) {
      const int sp = task / P.nslots, s = task - sp * P.nslots;
      const int sd = sp / P.QS, q = sp - sd * P.QS;
      const double* gq = geo + sp * GEO;
      double val = 0.0;
      for (int se = 0; se < P.nse; se++) {
        const DpgSideTerm& E = P.se[se];
        if (E.side != sd || E.slot != s) continue;
        double f = E.coef;
        if (E.use_meas) f *= gq[19];
        if (E.normal_comp >= 0) f *= gq[20 + E.normal_comp];
        if (E.flux) f *= (double)par_c[sd];
        double part = 0.0;
        for (int i = P.sadj_start[se] + lane; i < P.sadj_start[se + 1]; i += 32) {
          const int c = P.sadj_con[i];
          const int2 rc = P.scon_rc[c];
          part += pm[cfrag_index(P.NBT, rc.x, rc.y)] * P.scon_w[(size_t)q * P.ncon + c];
        }
        val += f * part;
      }
      val = warp_sum(val);
      if (lane == 0) cbar[s * P.Ptot + P.QG + P.QB + sp] += 2.0 * val;
    }
    __syncthreads();
  }
  __syncthreads();
  double* cb = L.coeff_bar + (size_t)cell * ncb;
  for (int i = tid; i < ncb; i += NT) cb[i] = cbar[i];
  __syncthreads();
}

template <int NBTM, int GTM, int BTW, int CH>
__global__ void __launch_bounds__(NT, 1) dpg_adjoint_kernel(const __grid_constant__ DpgPlanDev P, const DpgLaunch L) {
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
  for (int cell = blockIdx.x; cell < L.C; cell += gridDim.x) {
    if (tid == 0) { flag_s[0] = 0; flag_s[1] = 0; flag_s[2] = 0; }
    if (tid < P.nv * P.d) nodes_s[tid] = L.nodes[(size_t)cell * P.nv * P.d + tid];
    const int nco = P.nslots * P.Ptot;
    if (L.coeff)
      for (int i = tid; i < nco; i += NT) coef_s[i] = L.coeff[(size_t)cell * nco + i];
    __syncthreads();
    phase_b<BTW>(P, L, cell, X);
    __syncthreads();
    phase_gram<GTM, CH>(P, L, cell, X);
    phase_factor(P, X);
    phase_adj_solve<NBTM>(P, L);
    phase_adj_p<NBTM>(P, L, cell);
    phase_adj_pull(P, L, cell);
    if (tid == 0 && L.info) {
      int v = 0;
      if (flag_s[2]) v = ERR_TIMEOUT_FLAG;
      else if (flag_s[0] != 0) {
        int r = flag_s[0] - 1;
        int u = P.dev2user_test[r];
        v = (u >= 0 ? u : r) + 1;
      }
      L.info[cell] = v;
    }
    __syncthreads();
  }
}

#define DPG_ADJ_INSTANCES(X) X(12, 5, 4, 8) X(16, 6, 4, 8) X(20, 8, 4, 8) X(24, 12, 6, 8) X(24, 12, 6, 4)

static KernelFn pick_adjoint_kernel(const DpgPlanDev* plan) {
  const int per = (plan->ngb + DPG_NWARPS - 1) / DPG_NWARPS;
  int btw = 0;
  for (int s = 0; s < plan->nseg; s++) btw = std::max(btw, (plan->seg[s].ntile + DPG_NWARPS - 1) / DPG_NWARPS);
#define DPG_PICK(NB, GT, BT, CH) \
  if (plan->NBT <= NB && per <= GT && btw <= BT && plan->chg == CH) return dpg_adjoint_kernel<NB, GT, BT, CH>;
  DPG_ADJ_INSTANCES(DPG_PICK)
#undef DPG_PICK
  return nullptr;
}
