// dpg_internal.h — declarations shared by the host builder and the kernel launchers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "dpg_plan.h"

namespace dpg {
extern thread_local std::string g_last_error;
int fail(int code, const std::string& msg);
// Stream-ordered workspace allocation.  Outside stream capture it draws from a memory
// pool the library owns on the current device (created on first use, with a release
// threshold that keeps freed workspaces between calls); the caller's pools and the
// device's default pool are not modified.  Inside a capture it uses cudaMallocAsync,
// which the capture turns into a graph allocation.  Free with cudaFreeAsync.
cudaError_t ws_alloc(void** p, size_t bytes, cudaStream_t s);
// Number of SMs of the current device (cached per device).
int num_sms();
}  // namespace dpg

// Arguments of one assembly launch (device pointers).
struct DpgLaunch {
  int C;
  const double* nodes;
  const int8_t* parity;
  const double* coeff;
  double* K;
  double* l;
  double* S;
  double* s;
  int32_t* info;
  // dpg_assemble_parts outputs (parts = 1): G (C,N,N), B (C,M,N), F (C,N)
  int parts;
  double* G;
  double* B;
  double* F;
  // dpg_factored_cholesky_solve inputs (solve_only = 1)
  int solve_only;
  const double* Gin;
  const double* Bin;
  const double* Fin;
  // B tiles between the B phase and the triangular solve: scratch_per_cta doubles per CTA
  double* scratch;
  // dpg_assemble_adjoint: loss gradients in, coefficient gradients out; scratch2 holds P
  const double* Kbar;
  const double* lbar;
  double* coeff_bar;
  double* scratch2;
  // dpg_energy_error: local trial coefficients in (C, M), energy error out (C)
  const double* xsol;
  double* energy;
};

int dpg_configure_kernels(const DpgPlanDev* plan);
int dpg_launch_assemble(const DpgPlanDev* plan, const DpgPlanDev* d_plan, const DpgLaunch* L, cudaStream_t stream);
int dpg_host_pipeline(const DpgPlanDev* plan, const DpgPlanDev* d_plan, void** d_ws, size_t* ws_bytes,
                      cudaStream_t* streams, int C, const double* nodes, const int8_t* parity, const double* coeff,
                      double* K, double* l, double* S, double* s, int32_t* info, int flags);
int dpg_make_solve_plan(int N, int M, DpgPlanDev* out);
size_t dpg_big_workspace_bytes(const DpgPlanDev* plan, int C);  // large buckets: workspace of one launch
int dpg_launch_assemble_noalloc(const DpgPlanDev* plan, const DpgLaunch* L, cudaStream_t stream);
int dpg_launch_adjoint(const DpgPlanDev* plan, const DpgLaunch* L, cudaStream_t stream);
int dpg_launch_energy(const DpgPlanDev* plan, const DpgLaunch* L, cudaStream_t stream);
int dpg_launch_scatter_global(int C, int t, const int64_t* ptr, const int64_t* gid, const double* w,
                              int64_t n_global, const int64_t* row_ptr, const int64_t* col, const double* S,
                              const double* s, double* values, double* rhs, int* missing, cudaStream_t stream);
int dpg_launch_recover_fields(int C, int M, int nf, const double* K, const double* l, const double* t, double* u,
                              int32_t* info, cudaStream_t stream);

// Device tables of a prepared work-queue launch of single-CTA buckets (CUDA graph capture).
struct DpgMultiDev {
  void* base;          // caller-owned device block: tables, counters, then scratch slots
  size_t bytes;
  DpgPlanDev* plans;
  DpgLaunch* launches;
  int* cstart;
  int* counters;       // claim and leave counters (the kernel resets them at its end)
  int nb, grid;
  int claim, claim_slot;
  void* kernel;
  size_t smem;
};
int dpg_launch_multi(const DpgPlanDev* hplans, const DpgLaunch* hl, int nb, cudaStream_t stream, DpgMultiDev* dev,
                     int claim);
int dpg_launch_multi_prepared(const DpgMultiDev* dev, cudaStream_t stream);
size_t dpg_multi_bytes(const DpgPlanDev* hplans, const DpgLaunch* hl, int nb);
