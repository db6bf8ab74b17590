// dpg_maps.cu — local-to-global dof maps on the device.
//
// Galerkin coarse operators for geometric multigrid.  GMGOperator::
// computeCoarseStiffnessMatrix (src/Solution/GMGOperator.cpp:173-366) forms P^T A P with
// two sparse matrix products, A being the assembled fine matrix sum_c C_c^T S_c C_c and P
// the prolongation built from per-fine-cell LocalDofMappers (constructProlongationOperator,
// GMGOperator.cpp:420-773).  Since P^T A P = sum_c (C_c P)^T S_c (C_c P), composing each
// cell's local-to-fine map C_c with P gives a local-to-coarse map, and the global scatter
// of the cells' S with that map assembles the coarse operator directly: no fine matrix,
// no sparse triple product.  dpg_compose_map forms C_c P for all cells at once:
//   count   one thread per local dof row: the length of its composed row;
//   scan    inclusive scan of the lengths into row offsets (block scan + recursion);
//   fill    one thread per local dof row writes its coarse ids and weights w_k * P_kj.
// Coarse ids that repeat within a row are kept (the scatter adds them up).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/dpg_b200.h"
#include "dpg_internal.h"

namespace {

constexpr int SCAN_T = 1024;               // threads per scan block
constexpr int SCAN_V = 4;                  // values per thread
constexpr int SCAN_B = SCAN_T * SCAN_V;    // values per scan block

// Inclusive scan of x[0, n) within blocks of SCAN_B values; block totals to sums.
__global__ void __launch_bounds__(SCAN_T) scan_block_kernel(int64_t* __restrict__ x, long long n,
                                                            int64_t* __restrict__ sums) {
  __shared__ int64_t warp_tot[32];
  const long long base = (long long)blockIdx.x * SCAN_B + (long long)threadIdx.x * SCAN_V;
  int64_t v[SCAN_V];
  int64_t run = 0;
#pragma unroll
  for (int i = 0; i < SCAN_V; i++) {
    run += (base + i < n) ? x[base + i] : 0;
    v[i] = run;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t incl = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int64_t wt = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, wt, o);
      if (lane >= o) wt += y;
    }
    warp_tot[lane] = wt;
  }
  __syncthreads();
  const int64_t before = (incl - run) + (warp > 0 ? warp_tot[warp - 1] : 0);
#pragma unroll
  for (int i = 0; i < SCAN_V; i++)
    if (base + i < n) x[base + i] = v[i] + before;
  if (sums && threadIdx.x == SCAN_T - 1) sums[blockIdx.x] = before + run;
}

// Adds the scanned total of blocks 0..b-1 to block b (b >= 1).
__global__ void __launch_bounds__(SCAN_T) scan_add_kernel(int64_t* __restrict__ x, long long n,
                                                          const int64_t* __restrict__ sums) {
  const long long b = (long long)blockIdx.x + 1;
  const int64_t add = sums[b - 1];
  const long long base = b * SCAN_B;
  for (int i = threadIdx.x; i < SCAN_B; i += SCAN_T)
    if (base + i < n) x[base + i] += add;
}

int inclusive_scan(int64_t* x, long long n, cudaStream_t st) {
  if (n <= 0) return DPG_OK;
  const long long nb = (n + SCAN_B - 1) / SCAN_B;
  if (nb == 1) {
    scan_block_kernel<<<1, SCAN_T, 0, st>>>(x, n, nullptr);
    return DPG_OK;
  }
  int64_t* sums = nullptr;
  if (cudaMallocAsync((void**)&sums, (size_t)nb * sizeof(int64_t), st) != cudaSuccess) {
    cudaGetLastError();
    return dpg::fail(DPG_ERR_OUT_OF_MEMORY, "scan workspace allocation failed");
  }
  scan_block_kernel<<<(unsigned)nb, SCAN_T, 0, st>>>(x, n, sums);
  int rc = inclusive_scan(sums, nb, st);
  if (rc == DPG_OK) scan_add_kernel<<<(unsigned)(nb - 1), SCAN_T, 0, st>>>(x, n, sums);
  cudaFreeAsync(sums, st);
  return rc;
}

__global__ void compose_count_kernel(long long rows, const int64_t* __restrict__ ptr,
                                     const int64_t* __restrict__ gid, int64_t n_fine,
                                     const int64_t* __restrict__ prow, int64_t* __restrict__ out_ptr,
                                     int* __restrict__ missing) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < rows;
       r += (long long)gridDim.x * blockDim.x) {
    int64_t n = 0;
    for (int64_t k = ptr[r]; k < ptr[r + 1]; k++) {
      const int64_t g = gid[k];
      if (g < 0 || g >= n_fine) {
        if (missing) atomicAdd(missing, 1);
        continue;
      }
      n += prow[g + 1] - prow[g];
    }
    out_ptr[r + 1] = n;
    if (r == 0) out_ptr[0] = 0;
  }
}

__global__ void compose_fill_kernel(long long rows, const int64_t* __restrict__ ptr,
                                    const int64_t* __restrict__ gid, const double* __restrict__ w,
                                    int64_t n_fine, const int64_t* __restrict__ prow,
                                    const int64_t* __restrict__ pcol, const double* __restrict__ pval,
                                    const int64_t* __restrict__ out_ptr, int64_t cap,
                                    int64_t* __restrict__ out_gid, double* __restrict__ out_w) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < rows;
       r += (long long)gridDim.x * blockDim.x) {
    int64_t pos = out_ptr[r];
    const int64_t end = out_ptr[r + 1];
    for (int64_t k = ptr[r]; k < ptr[r + 1]; k++) {
      const int64_t g = gid[k];
      if (g < 0 || g >= n_fine) continue;
      const double wk = w ? w[k] : 1.0;
      for (int64_t j = prow[g]; j < prow[g + 1]; j++, pos++) {
        if (pos >= end || pos >= cap) continue;  // offsets and counts agree; guards only
        out_gid[pos] = pcol[j];
        out_w[pos] = wk * pval[j];
      }
    }
  }
}

int grid_for(long long rows) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return (int)std::max<long long>(1, std::min<long long>((rows + 255) / 256, (long long)sms * 8));
}

}  // namespace

extern "C" int dpg_compose_map(int C, int t, const int64_t* map_ptr, const int64_t* map_gid, const double* map_w,
                               int64_t n_fine, const int64_t* P_row_ptr, const int64_t* P_col,
                               const double* P_val, int64_t* out_ptr, int64_t* out_gid, double* out_w,
                               int64_t capacity, int64_t* out_count, int* missing, void* stream) {
  if (C < 0 || t < 0 || n_fine < 0 || capacity < 0) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "negative size");
  if (!out_count) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "out_count is required");
  *out_count = 0;
  const long long rows = (long long)C * t;
  if (rows == 0) return DPG_OK;
  if (!map_ptr || !map_gid || !P_row_ptr || !out_ptr)
    return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "map, prolongation rows and out_ptr are required");
  if (out_gid && (!out_w || !P_col || !P_val))
    return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "filling needs out_w and the prolongation's columns and values");
  cudaStream_t st = (cudaStream_t)stream;
  const int grid = grid_for(rows);
  compose_count_kernel<<<grid, 256, 0, st>>>(rows, map_ptr, map_gid, n_fine, P_row_ptr, out_ptr, missing);
  int rc = inclusive_scan(out_ptr + 1, rows, st);
  if (rc != DPG_OK) return rc;
  int64_t total = 0;
  cudaMemcpyAsync(&total, out_ptr + rows, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("compose map: ") + cudaGetErrorString(e));
  *out_count = total;
  if (!out_gid) return DPG_OK;
  if (total > capacity) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "composed map exceeds the given capacity");
  compose_fill_kernel<<<grid, 256, 0, st>>>(rows, map_ptr, map_gid, map_w, n_fine, P_row_ptr, P_col, P_val, out_ptr,
                                            capacity, out_gid, out_w);
  e = cudaGetLastError();
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}
