// dpg_energy.cuh — per-cell energy error of a trial solution and the DLS local
// matrices (included by dpg_kernel.cu inside its anonymous namespace; both reuse
// the forward phases).
//
// TSolution::rankLocalEnergyError (Solution.cpp:2653-2684) with the error
// representation of computeErrorRepresentation (Solution.cpp:2688-2722): for the
// cell's local trial coefficients x, the residual r = F - B x on the test space,
// e = G^-1 r (the Riesz representation) and the energy error sqrt(r^T e).  Here r
// replaces F as the extra column of the triangular solve, so W's last column is
// L^-1 r and r^T G^-1 r = |L^-1 r|^2: no difference of large numbers is formed.

// r = F - B x into the F column of the cell's [B | F] scratch tiles.
__device__ __forceinline__ void energy_residual(const DpgPlanDev& P, const DpgLaunch& L, int cell) {
  double* scr = L.scratch + (size_t)blockIdx.x * P.scratch_per_cta;
  const double* xc = L.xsol + (size_t)cell * P.M;
  for (int i = threadIdx.x; i < P.Np; i += NT) {
    double r = scr[cfrag_index(P.NBT, i, P.fcol)];
    for (int j = 0; j < P.Mp; j++) {
      const int u = P.dev2user_trial[j];
      if (u >= 0) r -= scr[cfrag_index(P.NBT, i, j)] * xc[u];
    }
    scr[cfrag_index(P.NBT, i, P.fcol)] = r;
  }
}

template <int NBTM, int GTM, int BTW, int CH>
__global__ void __launch_bounds__(NT, 1) dpg_energy_kernel(const __grid_constant__ DpgPlanDev P, const DpgLaunch L) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  Ctx X;
  double* const sm = dpg_smem;
  double* nodes_s = sm + P.sm_nodes;
  int* flag_s = reinterpret_cast<int*>(sm + P.sm_nodes + 24);
  double* coef_s = sm + P.sm_coef;
  uint32_t phase[4] = {0, 0, 0, 0};
  X.phase = phase;
  cta_setup(P);
  for (int cell = blockIdx.x; cell < L.C; cell += gridDim.x) {
    if (tid == 0) { flag_s[0] = 0; flag_s[1] = 0; flag_s[2] = 0; }
    if (tid < P.nv * P.d) nodes_s[tid] = L.nodes[(size_t)cell * P.nv * P.d + tid];
    const int nco = P.nslots * P.Ptot;
    if (L.coeff)
      for (int i = tid; i < nco; i += NT) coef_s[i] = L.coeff[(size_t)cell * nco + i];
    __syncthreads();
    phase_b<BTW>(P, L, cell, X);
    __syncthreads();
    energy_residual(P, L, cell);
    __syncthreads();
    phase_gram<GTM, CH>(P, L, cell, X);
    phase_factor(P, X);
    phase_trsm<NBTM>(P, L, cell, X);
    // |L^-1 r|^2: row fcol of the W^T tiles of column tile fcol / 8
    const double* WT = sm + P.sm_w + (size_t)(P.fcol >> 3) * P.NBT * 64;
    const int fr = P.fcol & 7;
    double acc = 0.0;
    if (warp == 0)
      for (int e = lane; e < P.NBT * 8; e += 32) {
        const double w = WT[(e >> 3) * 64 + ak(fr, e & 7)];
        acc += w * w;
      }
    if (warp == 0) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) {
        int v = 0;
        if (flag_s[2]) v = ERR_TIMEOUT_FLAG;
        else if (flag_s[0] != 0) {
          const int r = flag_s[0] - 1, u = P.dev2user_test[r];
          v = (u >= 0 ? u : r) + 1;
        }
        // a failed factorisation leaves no energy to report
        L.energy[cell] = v == 0 ? sqrt(acc) : __longlong_as_double(0x7ff8000000000000ll);
        if (L.info) L.info[cell] = v;
      }
    }
    __syncthreads();
  }
}

// Gram points per chunk (CH) fixed at compile time, as in the assembly kernel; the
// picker takes the first instance whose sizes and chunk length fit the plan.
#define DPG_ENERGY_INSTANCES(X) \
  X(12, 5, 4, 8) X(16, 6, 4, 8) X(20, 8, 4, 8) X(22, 9, 3, 8) X(24, 12, 6, 8) X(24, 12, 6, 4)

static KernelFn pick_energy_kernel(const DpgPlanDev* plan) {
  const int per = (plan->ngb + DPG_NWARPS - 1) / DPG_NWARPS;
  int btw = 0;
  for (int s = 0; s < plan->nseg; s++) btw = std::max(btw, (plan->seg[s].ntile + DPG_NWARPS - 1) / DPG_NWARPS);
#define DPG_PICK(NB, GT, BT, CH) \
  if (plan->NBT <= NB && per <= GT && btw <= BT && plan->chg == CH) return dpg_energy_kernel<NB, GT, BT, CH>;
  DPG_ENERGY_INSTANCES(DPG_PICK)
#undef DPG_PICK
  return nullptr;
}

// DLS local matrices (TBF::localStiffnessMatrixAndRHS_DLS, BF.cpp:1169-1306: the
// factored solve overwrites B and F in place): W = L^-1 B as (C, M, N) "trial x
// test" and y = L^-1 F as (C, N), user numbering, L the unscaled Cholesky factor of G.
template <int NBTM, int GTM, int BTW, int CH>
__global__ void __launch_bounds__(NT, 1) dpg_dls_kernel(const __grid_constant__ DpgPlanDev P, const DpgLaunch L) {
  const int tid = threadIdx.x;
  Ctx X;
  double* const sm = dpg_smem;
  double* nodes_s = sm + P.sm_nodes;
  int* flag_s = reinterpret_cast<int*>(sm + P.sm_nodes + 24);
  double* coef_s = sm + P.sm_coef;
  uint32_t phase[4] = {0, 0, 0, 0};
  X.phase = phase;
  cta_setup(P);
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
    phase_trsm<NBTM>(P, L, cell, X);
    // W^T tile (J, I), element (r, c) = W[I*8 + c][J*8 + r]
    const double* WT = sm + P.sm_w;
    double* Wc = L.B + (size_t)cell * P.M * P.N;
    double* yc = L.F + (size_t)cell * P.N;
    for (int e = tid; e < P.Mp * P.Np; e += NT) {
      const int j = e / P.Np, i = e - j * P.Np;
      const int ui = P.dev2user_test[i];
      if (ui < 0) continue;
      const double v = WT[((j >> 3) * P.NBT + (i >> 3)) * 64 + ak(j & 7, i & 7)];
      const int uj = P.dev2user_trial[j];
      if (uj >= 0) Wc[(size_t)uj * P.N + ui] = v;
      else if (j == P.fcol) yc[ui] = v;
    }
    if (tid == 0 && L.info) {
      int v = 0;
      if (flag_s[2]) v = ERR_TIMEOUT_FLAG;
      else if (flag_s[0] != 0) {
        const int r = flag_s[0] - 1, u = P.dev2user_test[r];
        v = (u >= 0 ? u : r) + 1;
      }
      L.info[cell] = v;
    }
    __syncthreads();
  }
}

static KernelFn pick_dls_kernel(const DpgPlanDev* plan) {
  const int per = (plan->ngb + DPG_NWARPS - 1) / DPG_NWARPS;
  int btw = 0;
  for (int s = 0; s < plan->nseg; s++) btw = std::max(btw, (plan->seg[s].ntile + DPG_NWARPS - 1) / DPG_NWARPS);
#define DPG_PICK(NB, GT, BT, CH) \
  if (plan->NBT <= NB && per <= GT && btw <= BT && plan->chg == CH) return dpg_dls_kernel<NB, GT, BT, CH>;
  DPG_ENERGY_INSTANCES(DPG_PICK)
#undef DPG_PICK
  return nullptr;
}
