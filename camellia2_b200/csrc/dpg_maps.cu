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
//
// Global assembly of the condensed cell matrices (GDAMinimumRule::interpretLocalData,
// GDAMinimumRule.cpp:714-800, through LocalDofMapper's C, then the insertion into the
// global system, Solution.cpp:1263-1293): values += sum_c C_c^T S_c C_c and
// rhs += sum_c C_c^T s_c on a CSR graph the caller owns.  Local dof a of cell c stands
// for sum_k w_k x[gid_k], k in [ptr[c t + a], ptr[c t + a + 1]).  Each cell's map entries
// are ranked by global id, so C_c^T S_c C_c is formed on the cell's distinct global dofs
// (a trace point shared by three faces of a hex is one row, not three): a distinct
// (row, column) pair costs one atomic instead of one per pair of local dofs.  The targets
// come from each distinct row's CSR row, read once and matched against the cell's sorted
// ids.  Within a cell the sums have a fixed order; across cells the atomics make the last
// bits depend on the order of arrival.
//   dpg_scatter_global        does all of it per call (a cell with more map entries than
//                             the shared tables hold goes through a per-entry path);
//   dpg_scatter_plan_create   does the symbolic part once for a fixed mesh and graph: the
//                             distinct ids, the grouped entries and the CSR position of
//                             every distinct pair, into device arrays;
//   dpg_scatter_plan_apply    is then only the pair sums and the atomics.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

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
  if (dpg::ws_alloc((void**)&sums, (size_t)nb * sizeof(int64_t), st) != cudaSuccess) {
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

// ---------------------------------------------------------------------------
// Global scatter of S, s
// ---------------------------------------------------------------------------
__device__ __forceinline__ long long csr_find(const int64_t* __restrict__ row_ptr, const int64_t* __restrict__ col,
                                              int64_t r, int64_t c) {
  long long lo = row_ptr[r], hi = row_ptr[r + 1] - 1;
  while (lo <= hi) {
    const long long mid = (lo + hi) >> 1;
    const int64_t v = col[mid];
    if (v == c) return mid;
    if (v < c) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

constexpr int SG_T = 256;

// Shared tables of one cell: ecap map entries at most.
struct SgTables {
  int64_t* ug;     // distinct in-range global ids, ascending
  int64_t* rbeg;   // row_ptr[ug[u]]
  int64_t* eg;     // entry global id
  double* ew;      // entry weight
  int* erow;       // entry local row
  int* erank;      // entry's distinct index, -1 when out of range
  int* efirst;     // 1 for the first entry of each in-range id
  int* elist;      // entries grouped by distinct index: elist[ufirst[u] .. ufirst[u+1])
  int* ufirst;
  int* pos;        // (one-shot kernel) nu*nu: offset of (u, v) in CSR row ug[u], or -1
};

__host__ __device__ inline size_t sg_tables_bytes(int ecap) {
  return (size_t)ecap * (8 + 8 + 8 + 8) + (size_t)ecap * 4 * 4 + ((size_t)ecap + 1) * 4 + 4;
}

__device__ inline SgTables sg_tables(void* base, int ecap) {
  SgTables T;
  char* p = (char*)base;
  T.ug = (int64_t*)p; p += (size_t)ecap * 8;
  T.rbeg = (int64_t*)p; p += (size_t)ecap * 8;
  T.eg = (int64_t*)p; p += (size_t)ecap * 8;
  T.ew = (double*)p; p += (size_t)ecap * 8;
  T.erow = (int*)p; p += (size_t)ecap * 4;
  T.erank = (int*)p; p += (size_t)ecap * 4;
  T.efirst = (int*)p; p += (size_t)ecap * 4;
  T.elist = (int*)p; p += (size_t)ecap * 4;
  T.ufirst = (int*)p; p += ((size_t)ecap + 1) * 4 + 4;
  T.pos = (int*)p;
  return T;
}

// The distinct ids of cell c (ne <= ecap map entries, first entry e0), the entries grouped
// by them and the CSR row starts.  All threads of the block call it; it ends with a barrier.
// Returns nu (distinct in-range ids) and nin (in-range entries).
__device__ void sg_cell_tables(const SgTables& T, int c, int t, int64_t e0, int ne, const int64_t* __restrict__ ptr,
                               const int64_t* __restrict__ gid, const double* __restrict__ w, int64_t n,
                               const int64_t* __restrict__ row_ptr, int* s_cnt, int& nu, int& nin) {
  const int tid = threadIdx.x;
  if (tid == 0) { s_cnt[0] = 0; s_cnt[1] = 0; }
  for (int a = tid; a < t; a += blockDim.x)
    for (int64_t k = ptr[(size_t)c * t + a]; k < ptr[(size_t)c * t + a + 1]; k++) {
      const int e = (int)(k - e0);
      T.eg[e] = gid[k];
      T.ew[e] = w ? w[k] : 1.0;
      T.erow[e] = a;
    }
  __syncthreads();
  int my_first = 0, my_in = 0;
  for (int e = tid; e < ne; e += blockDim.x) {
    const int64_t g = T.eg[e];
    const int in = g >= 0 && g < n;
    int first = in;
    for (int q = 0; q < e && first; q++) first = T.eg[q] != g;
    T.efirst[e] = first;
    my_first += first;
    my_in += in;
  }
  if (my_first) atomicAdd(&s_cnt[0], my_first);
  if (my_in) atomicAdd(&s_cnt[1], my_in);
  __syncthreads();
  nu = s_cnt[0];
  nin = s_cnt[1];
  for (int e = tid; e < ne; e += blockDim.x) {
    const int64_t g = T.eg[e];
    int rank = -1;
    if (g >= 0 && g < n) {
      rank = 0;
      for (int f = 0; f < ne; f++) rank += T.efirst[f] && T.eg[f] < g;
      if (T.efirst[e]) {
        T.ug[rank] = g;
        T.rbeg[rank] = row_ptr[g];
      }
    }
    T.erank[e] = rank;
  }
  __syncthreads();
  for (int e = tid; e < ne; e += blockDim.x) {
    const int r = T.erank[e];
    if (r < 0) continue;
    int p = 0;
    for (int f = 0; f < ne; f++) {
      const int rf = T.erank[f];
      p += rf >= 0 && (rf < r || (rf == r && f < e));
    }
    T.elist[p] = e;
    if (T.efirst[e]) T.ufirst[r] = p;
  }
  if (tid == 0) T.ufirst[nu] = nin;
  __syncthreads();
}

// CSR positions of the cell's distinct pairs: pos[u * nu + v] = offset of column ug[v] in
// row ug[u], or -1.  One warp per distinct row reads the row once, coalesced, and finds each
// column among the sorted ids.  pos may be shared or global memory; ends with a barrier.
__device__ void sg_cell_targets(const SgTables& T, int nu, const int64_t* __restrict__ row_ptr,
                                const int64_t* __restrict__ col, int* pos) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  for (int e = tid; e < nu * nu; e += blockDim.x) pos[e] = -1;
  __syncthreads();
  for (int u = warp; u < nu; u += nwarp) {
    const int64_t beg = T.rbeg[u], end = row_ptr[T.ug[u] + 1];
    for (int64_t p = beg + lane; p < end; p += 32) {
      const int64_t cc = __ldg(col + p);
      int lo = 0, hi = nu - 1;
      while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int64_t x = T.ug[mid];
        if (x == cc) { pos[u * nu + mid] = (int)(p - beg); break; }
        if (x < cc) lo = mid + 1;
        else hi = mid - 1;
      }
    }
  }
  __syncthreads();
}

// The per-entry path of one cell (any number of map entries).
__device__ void scatter_cell_entries(int c, int t, const int64_t* __restrict__ ptr, const int64_t* __restrict__ gid,
                                     const double* __restrict__ w, int64_t n, const int64_t* __restrict__ row_ptr,
                                     const int64_t* __restrict__ col, const double* __restrict__ S,
                                     const double* __restrict__ sv, double* __restrict__ values,
                                     double* __restrict__ rhs, int* __restrict__ missing) {
  const int tt = t * t;
  for (int ab = threadIdx.x; ab < tt; ab += blockDim.x) {
    const int a = ab / t, b = ab - a * t;
    const double sab = S[(size_t)c * tt + ab];
    const long long ia = (long long)c * t + a, ib = (long long)c * t + b;
    for (int64_t ka = ptr[ia]; ka < ptr[ia + 1]; ka++) {
      const double wa = w ? w[ka] : 1.0;
      for (int64_t kb = ptr[ib]; kb < ptr[ib + 1]; kb++) {
        const int64_t r = gid[ka], cc = gid[kb];
        const long long pos = (r >= 0 && r < n && cc >= 0 && cc < n) ? csr_find(row_ptr, col, r, cc) : -1;
        if (pos < 0) { atomicAdd(missing, 1); continue; }
        atomicAdd(values + pos, wa * (w ? w[kb] : 1.0) * sab);
      }
    }
    if (b == 0 && sv && rhs)
      for (int64_t ka = ptr[ia]; ka < ptr[ia + 1]; ka++)
        if (gid[ka] >= 0 && gid[ka] < n) atomicAdd(rhs + gid[ka], (w ? w[ka] : 1.0) * sv[ia]);
  }
}

// The pair sum of distinct (u, v) of cell c: sum over the entries of u and of v of
// w_a w_b S[a][b], in entry order.
__device__ __forceinline__ double sg_pair_sum(const double* __restrict__ Sc, int t, const int* erow,
                                              const double* ew, int a0, int a1, int b0, int b1) {
  double acc = 0.0;
  for (int i = a0; i < a1; i++) {
    const double* Sa = Sc + (size_t)erow[i] * t;
    double racc = 0.0;
    for (int j = b0; j < b1; j++) racc += ew[j] * __ldg(Sa + erow[j]);
    acc += ew[i] * racc;
  }
  return acc;
}

__global__ void __launch_bounds__(SG_T) scatter_global_kernel(int C, int t, int ecap, const int64_t* __restrict__ ptr,
                                                              const int64_t* __restrict__ gid,
                                                              const double* __restrict__ w, int64_t n,
                                                              const int64_t* __restrict__ row_ptr,
                                                              const int64_t* __restrict__ col,
                                                              const double* __restrict__ S,
                                                              const double* __restrict__ sv,
                                                              double* __restrict__ values, double* __restrict__ rhs,
                                                              int* __restrict__ missing) {
  extern __shared__ __align__(16) double sg_smem[];
  const SgTables T = sg_tables(sg_smem, ecap);
  __shared__ int s_cnt[2], s_miss;
  const int tid = threadIdx.x;
  const int tt = t * t;
  for (int c = blockIdx.x; c < C; c += gridDim.x) {
    const int64_t e0 = ptr[(size_t)c * t], ne64 = ptr[(size_t)c * t + t] - e0;
    if (ne64 > ecap || ne64 < 0) {
      scatter_cell_entries(c, t, ptr, gid, w, n, row_ptr, col, S, sv, values, rhs, missing);
      continue;
    }
    const int ne = (int)ne64;
    if (tid == 0) s_miss = 0;
    int nu, nin;
    sg_cell_tables(T, c, t, e0, ne, ptr, gid, w, n, row_ptr, s_cnt, nu, nin);
    if ((long long)nu * nu > tt) {  // more distinct pairs than the position table holds
      scatter_cell_entries(c, t, ptr, gid, w, n, row_ptr, col, S, sv, values, rhs, missing);
      __syncthreads();
      continue;
    }
    // grouped rows and weights of the entries, in place of the raw ones (erank is free)
    int* grow = T.erank;
    double* gw = reinterpret_cast<double*>(T.eg);
    for (int i = tid; i < nin; i += SG_T) grow[i] = T.erow[T.elist[i]];
    __syncthreads();
    for (int i = tid; i < nin; i += SG_T) gw[i] = T.ew[T.elist[i]];
    sg_cell_targets(T, nu, row_ptr, col, T.pos);
    int my_miss = 0;
    const double* Sc = S + (size_t)c * tt;
    for (int e = tid; e < nu * nu; e += SG_T) {
      const int u = e / nu, v = e - u * nu;
      const int off = T.pos[e];
      if (off < 0) { my_miss++; continue; }
      atomicAdd(values + T.rbeg[u] + off,
                sg_pair_sum(Sc, t, grow, gw, T.ufirst[u], T.ufirst[u + 1], T.ufirst[v], T.ufirst[v + 1]));
    }
    if (sv && rhs)
      for (int u = tid; u < nu; u += SG_T) {
        double acc = 0.0;
        for (int i = T.ufirst[u]; i < T.ufirst[u + 1]; i++) acc += gw[i] * sv[(size_t)c * t + grow[i]];
        atomicAdd(rhs + T.ug[u], acc);
      }
    if (my_miss) atomicAdd(&s_miss, my_miss);
    __syncthreads();
    // out-of-range entries: every local pair they take part in is skipped
    if (tid == 0) {
      const int skipped = s_miss + (ne * ne - nin * nin);
      if (skipped) atomicAdd(missing, skipped);
    }
  }
}

// ---- plan: the symbolic part once, the numeric part per call ------------------------
__global__ void plan_max_entries_kernel(int C, int t, const int64_t* __restrict__ ptr, int* __restrict__ max_ne) {
  int m = 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
    const int64_t ne = ptr[(size_t)c * t + t] - ptr[(size_t)c * t];
    m = max(m, ne < (1 << 30) ? (int)ne : (1 << 30));
  }
  if (m) atomicMax(max_ne, m);
}

__global__ void __launch_bounds__(SG_T) plan_count_kernel(int C, int t, int ecap, const int64_t* __restrict__ ptr,
                                                          const int64_t* __restrict__ gid,
                                                          const double* __restrict__ w, int64_t n,
                                                          const int64_t* __restrict__ row_ptr,
                                                          int64_t* __restrict__ cnt_u, int64_t* __restrict__ cnt_e,
                                                          int64_t* __restrict__ cnt_p) {
  extern __shared__ __align__(16) double sg_smem[];
  const SgTables T = sg_tables(sg_smem, ecap);
  __shared__ int s_cnt[2];
  for (int c = blockIdx.x; c < C; c += gridDim.x) {
    const int64_t e0 = ptr[(size_t)c * t];
    const int ne = (int)(ptr[(size_t)c * t + t] - e0);
    int nu, nin;
    sg_cell_tables(T, c, t, e0, ne, ptr, gid, w, n, row_ptr, s_cnt, nu, nin);
    if (threadIdx.x == 0) {
      cnt_u[c + 1] = nu;
      cnt_e[c + 1] = nin;
      cnt_p[c + 1] = (int64_t)nu * nu;
      if (c == 0) cnt_u[0] = cnt_e[0] = cnt_p[0] = 0;
    }
  }
}

struct PlanArrays {
  const int64_t* offu;  // C+1: distinct ids before cell c
  const int64_t* offe;  // C+1: in-range entries before cell c
  const int64_t* offp;  // C+1: distinct pairs before cell c
  int64_t* u_rbeg;      // CSR row start of each distinct id
  int64_t* u_gid;       // the distinct ids
  int* u_first;         // per cell nu+1 starts of the grouped entries (at offu[c] + c)
  int* e_row;           // grouped entries: local row
  double* e_w;          //                  weight
  int* pos;             // per cell nu*nu CSR offsets within row u, or -1
};

__global__ void __launch_bounds__(SG_T) plan_fill_kernel(int C, int t, int ecap, const int64_t* __restrict__ ptr,
                                                         const int64_t* __restrict__ gid,
                                                         const double* __restrict__ w, int64_t n,
                                                         const int64_t* __restrict__ row_ptr,
                                                         const int64_t* __restrict__ col, PlanArrays A,
                                                         int* __restrict__ missing) {
  extern __shared__ __align__(16) double sg_smem[];
  const SgTables T = sg_tables(sg_smem, ecap);
  __shared__ int s_cnt[2], s_miss;
  const int tid = threadIdx.x;
  for (int c = blockIdx.x; c < C; c += gridDim.x) {
    const int64_t e0 = ptr[(size_t)c * t];
    const int ne = (int)(ptr[(size_t)c * t + t] - e0);
    if (tid == 0) s_miss = 0;
    int nu, nin;
    sg_cell_tables(T, c, t, e0, ne, ptr, gid, w, n, row_ptr, s_cnt, nu, nin);
    const int64_t ou = A.offu[c], oe = A.offe[c], op = A.offp[c];
    for (int u = tid; u < nu; u += SG_T) {
      A.u_rbeg[ou + u] = T.rbeg[u];
      A.u_gid[ou + u] = T.ug[u];
    }
    for (int u = tid; u <= nu; u += SG_T) A.u_first[ou + c + u] = T.ufirst[u];
    for (int i = tid; i < nin; i += SG_T) {
      A.e_row[oe + i] = T.erow[T.elist[i]];
      A.e_w[oe + i] = T.ew[T.elist[i]];
    }
    int* pc = A.pos + op;
    sg_cell_targets(T, nu, row_ptr, col, pc);
    int my_miss = 0;
    for (int e = tid; e < nu * nu; e += SG_T) my_miss += pc[e] < 0;
    if (my_miss) atomicAdd(&s_miss, my_miss);
    __syncthreads();
    if (tid == 0 && missing) {
      const int skipped = s_miss + (ne * ne - nin * nin);
      if (skipped) atomicAdd(missing, skipped);
    }
  }
}

__global__ void __launch_bounds__(SG_T) plan_apply_kernel(int C, int t, int ecap, PlanArrays A,
                                                          const double* __restrict__ S,
                                                          const double* __restrict__ sv,
                                                          double* __restrict__ values, double* __restrict__ rhs) {
  extern __shared__ __align__(16) double sg_smem[];
  double* ew = sg_smem;                                   // ecap
  int* er = reinterpret_cast<int*>(ew + ecap);            // ecap
  int* uf = er + ecap;                                    // ecap + 1
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = SG_T / 32;
  const int tt = t * t;
  for (int c = blockIdx.x; c < C; c += gridDim.x) {
    const int64_t ou = A.offu[c], oe = A.offe[c], op = A.offp[c];
    const int nu = (int)(A.offu[c + 1] - ou), nin = (int)(A.offe[c + 1] - oe);
    for (int i = tid; i < nin; i += SG_T) {
      ew[i] = A.e_w[oe + i];
      er[i] = A.e_row[oe + i];
    }
    for (int u = tid; u <= nu; u += SG_T) uf[u] = A.u_first[ou + c + u];
    __syncthreads();
    const double* Sc = S + (size_t)c * tt;
    const int* pc = A.pos + op;
    for (int u = warp; u < nu; u += nwarp) {
      const int64_t rb = A.u_rbeg[ou + u];
      const int a0 = uf[u], a1 = uf[u + 1];
      for (int v = lane; v < nu; v += 32) {
        const int off = pc[u * nu + v];
        if (off < 0) continue;
        atomicAdd(values + rb + off, sg_pair_sum(Sc, t, er, ew, a0, a1, uf[v], uf[v + 1]));
      }
    }
    if (sv && rhs)
      for (int u = tid; u < nu; u += SG_T) {
        double acc = 0.0;
        for (int i = uf[u]; i < uf[u + 1]; i++) acc += ew[i] * sv[(size_t)c * t + er[i]];
        atomicAdd(rhs + A.u_gid[ou + u], acc);
      }
    __syncthreads();
  }
}

int grid_for(long long rows) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return (int)std::max<long long>(1, std::min<long long>((rows + 255) / 256, (long long)sms * 8));
}

}  // namespace

int dpg_launch_scatter_global(int C, int t, const int64_t* ptr, const int64_t* gid, const double* w,
                              int64_t n_global, const int64_t* row_ptr, const int64_t* col, const double* S,
                              const double* s, double* values, double* rhs, int* missing, cudaStream_t stream) {
  if (C <= 0 || t <= 0) return DPG_OK;
  const int ecap = 2 * t;
  const size_t bytes = sg_tables_bytes(ecap) + (size_t)t * t * 4;
  if (bytes > 200 * 1024) return dpg::fail(DPG_ERR_UNSUPPORTED, "too many trace dofs per cell for the global scatter");
  cudaFuncSetAttribute(scatter_global_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  int per_sm = 0, dev = 0, sms = 148;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, scatter_global_kernel, SG_T, bytes);
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (int)std::min<long long>(C, (long long)sms * std::max(1, per_sm));
  scatter_global_kernel<<<grid, SG_T, bytes, stream>>>(C, t, ecap, ptr, gid, w, n_global, row_ptr, col, S, s, values,
                                                       rhs, missing);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}

struct dpg_scatter_plan {
  int C, t, ecap;
  int64_t n_global;
  void* base;
  PlanArrays A;
};

static int cell_grid(const void* kernel, size_t smem) {
  int per_sm = 0, dev = 0, sms = 148;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, SG_T, smem);
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms * std::max(1, per_sm);
}

extern "C" int dpg_scatter_plan_create(int C, int t, const int64_t* map_ptr, const int64_t* map_gid,
                                       const double* map_w, int64_t n_global, const int64_t* row_ptr,
                                       const int64_t* col_idx, int* missing, void* stream, dpg_scatter_plan** out) {
  if (!out) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "out is required");
  *out = nullptr;
  if (C < 0 || t < 0) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "negative size");
  if (C > 0 && t > 0 && (!map_ptr || !map_gid || !row_ptr || !col_idx))
    return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "map and graph are required");
  if (n_global <= 0) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "empty global system");
  cudaStream_t st = (cudaStream_t)stream;
  dpg_scatter_plan* P = new dpg_scatter_plan();
  P->C = (C > 0 && t > 0) ? C : 0;
  P->t = t;
  P->n_global = n_global;
  P->base = nullptr;
  P->ecap = 0;
  if (P->C == 0) {
    *out = P;
    return DPG_OK;
  }
  // the largest number of map entries of a cell sizes the shared tables
  void* tmp = nullptr;
  const size_t cnt_bytes = 3 * ((size_t)C + 1) * sizeof(int64_t);
  if (dpg::ws_alloc(&tmp, cnt_bytes + 16, st) != cudaSuccess) {
    cudaGetLastError();
    delete P;
    return dpg::fail(DPG_ERR_OUT_OF_MEMORY, "scatter plan workspace allocation failed");
  }
  int64_t* cnt = (int64_t*)tmp;
  int* d_max = (int*)((char*)tmp + cnt_bytes);
  cudaMemsetAsync(d_max, 0, sizeof(int), st);
  plan_max_entries_kernel<<<(C + 255) / 256 < 1184 ? (C + 255) / 256 : 1184, 256, 0, st>>>(C, t, map_ptr, d_max);
  int max_ne = 0;
  cudaMemcpyAsync(&max_ne, d_max, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  auto bail = [&](int code, const std::string& msg) {
    cudaFreeAsync(tmp, st);
    cudaStreamSynchronize(st);
    delete P;
    return dpg::fail(code, msg);
  };
  if (e != cudaSuccess) return bail(DPG_ERR_CUDA, std::string("scatter plan: ") + cudaGetErrorString(e));
  P->ecap = std::max(1, max_ne);
  const size_t tb = sg_tables_bytes(P->ecap);
  if (tb > 200 * 1024) return bail(DPG_ERR_UNSUPPORTED, "a cell has more map entries than the plan's shared tables hold");
  cudaFuncSetAttribute(plan_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(plan_fill_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(plan_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  int64_t *cu = cnt, *ce = cnt + (C + 1), *cp = cnt + 2 * ((size_t)C + 1);
  plan_count_kernel<<<std::min(C, cell_grid((const void*)plan_count_kernel, tb)), SG_T, tb, st>>>(
      C, t, P->ecap, map_ptr, map_gid, map_w, n_global, row_ptr, cu, ce, cp);
  int rc = DPG_OK;
  for (int64_t* x : {cu, ce, cp})
    if (rc == DPG_OK) rc = inclusive_scan(x + 1, C, st);
  if (rc != DPG_OK) return bail(rc, dpg::g_last_error);
  int64_t tot[3] = {0, 0, 0};
  cudaMemcpyAsync(&tot[0], cu + C, 8, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&tot[1], ce + C, 8, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&tot[2], cp + C, 8, cudaMemcpyDeviceToHost, st);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return bail(DPG_ERR_CUDA, std::string("scatter plan: ") + cudaGetErrorString(e));
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t b_off = al(3 * ((size_t)C + 1) * 8), b_u = al((size_t)tot[0] * 8), b_uf = al(((size_t)tot[0] + C) * 4),
               b_er = al((size_t)tot[1] * 4), b_ew = al((size_t)tot[1] * 8), b_pos = al((size_t)tot[2] * 4);
  const size_t bytes = b_off + 2 * b_u + b_uf + b_er + b_ew + b_pos;
  if (cudaMalloc(&P->base, bytes) != cudaSuccess) {
    cudaGetLastError();
    P->base = nullptr;
    return bail(DPG_ERR_OUT_OF_MEMORY, "scatter plan allocation failed");
  }
  char* b = (char*)P->base;
  cudaMemcpyAsync(b, cnt, 3 * ((size_t)C + 1) * 8, cudaMemcpyDeviceToDevice, st);
  P->A.offu = (const int64_t*)b;
  P->A.offe = P->A.offu + (C + 1);
  P->A.offp = P->A.offe + (C + 1);
  b += b_off;
  P->A.u_rbeg = (int64_t*)b; b += b_u;
  P->A.u_gid = (int64_t*)b; b += b_u;
  P->A.u_first = (int*)b; b += b_uf;
  P->A.e_row = (int*)b; b += b_er;
  P->A.e_w = (double*)b; b += b_ew;
  P->A.pos = (int*)b;
  plan_fill_kernel<<<std::min(C, cell_grid((const void*)plan_fill_kernel, tb)), SG_T, tb, st>>>(
      C, t, P->ecap, map_ptr, map_gid, map_w, n_global, row_ptr, col_idx, P->A, missing);
  e = cudaGetLastError();
  cudaFreeAsync(tmp, st);
  if (e != cudaSuccess) {
    cudaStreamSynchronize(st);
    cudaFree(P->base);
    delete P;
    return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  }
  *out = P;
  return DPG_OK;
}

extern "C" int dpg_scatter_plan_apply(const dpg_scatter_plan* P, const double* S, const double* s, double* values,
                                      double* rhs, void* stream) {
  if (!P) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "null plan");
  if (P->C == 0) return DPG_OK;
  if (!S || !values) return dpg::fail(DPG_ERR_INVALID_ARGUMENT, "S and values are required");
  const size_t smem = (size_t)P->ecap * 12 + ((size_t)P->ecap + 1) * 4;
  plan_apply_kernel<<<std::min(P->C, cell_grid((const void*)plan_apply_kernel, smem)), SG_T, smem,
                      (cudaStream_t)stream>>>(P->C, P->t, P->ecap, P->A, S, s, values, rhs);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return dpg::fail(DPG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DPG_OK;
}

extern "C" int dpg_scatter_plan_destroy(dpg_scatter_plan* P) {
  if (!P) return DPG_OK;
  if (P->base) cudaFree(P->base);
  delete P;
  return DPG_OK;
}

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
