/*
 * dpg_b200.h — C ABI of the B200-native DPG per-cell assembly library.
 *
 * One call assembles, for a batch of cells of ONE element type (Camellia's
 * ElementType: topology + trial ordering + test ordering), the optimal-test
 * local stiffness K = B^T G^-1 B, the load l = B^T G^-1 F, and the static
 * condensation of the field dofs S = K_tt - K_ft^T K_ff^-1 K_ft,
 * s = l_t - K_ft^T K_ff^-1 l_f.  Everything runs as hand-written sm_100a CUDA.
 *
 * Conventions shared by every entry point:
 *   - every function returns an int status (DPG_OK = 0); no exception crosses
 *     the boundary; dpg_last_error_string() describes the last failure on
 *     the calling thread;
 *   - all numbers are IEEE FP64, row-major, C-contiguous, one block per cell:
 *       K  (C, M, M)   l (C, M)   S (C, t, t)   s (C, t)
 *       G  (C, N, N)   B (C, M, N)  [Camellia's "stiffnessEnriched" layout]
 *       F  (C, N)
 *     N = test dofs, M = trial dofs, f = field dofs, t = M - f trace dofs;
 *   - trial dofs are numbered var by var in the order of the trial list
 *     (volume vars: all basis dofs; trace/flux vars: side 0 dofs, side 1
 *     dofs, ...), exactly like Camellia's DofOrderingFactory::trialOrdering;
 *     test dofs likewise in test-list order;
 *   - numerical failures (a Gram matrix that is not positive definite) are
 *     NOT errors: they are reported per cell in info[c] (0 = ok, k > 0 = the
 *     leading minor of order k is not positive, as LAPACK DPOTRF's INFO;
 *     -k = the condensation block failed at column k) and the call returns
 *     DPG_OK, mirroring BF.cpp's printed-and-returned INFO.
 *
 * Reference interfaces replaced (paths inside ApolloFramework/camellia2):
 *   dpg_plan_create           ElementType + BasisCache set-up for a bucket
 *                             (src/Solution/Solution.cpp:1162-1187,
 *                              src/Basis/BasisCache.cpp:236-267)
 *   dpg_assemble              TBF::localStiffnessMatrixAndRHS, FACTORED_CHOLESKY
 *                             (src/ScratchPad/BF.cpp:1309-1496) followed by
 *                             CondensedDofInterpreter::interpretLocalData
 *                             (src/Solution/CondensedDofInterpreter.cpp:1063-1225)
 *   dpg_assemble_host         the same, host buffers in and out
 *   dpg_assemble_parts        TIP::computeInnerProductMatrix (src/ScratchPad/IP.cpp:215-292),
 *                             TBF::stiffnessMatrix rowMajor=true (src/ScratchPad/BF.cpp:575-656),
 *                             TRHS::integrateAgainstStandardBasis (src/Problem/RHS.cpp:68-82)
 *   dpg_factored_cholesky_solve  TBF::factoredCholeskySolve (src/ScratchPad/BF.cpp:924-1018)
 *   dpg_assemble_adjoint      no counterpart in the reference (new capability)
 *   dpg_plan_autotune         no counterpart in the reference (GPU launch configuration)
 *   dpg_assemble_dls          TBF::localStiffnessMatrixAndRHS_DLS (src/ScratchPad/BF.cpp:1169-1306)
 *   dpg_scatter_global        GDAMinimumRule::interpretLocalData + global insertion
 *                             (src/Mesh/GDAMinimumRule.cpp:714-800, src/Solution/Solution.cpp:1263-1293)
 *   dpg_scatter_plan_*        the same, split into a symbolic part (once per mesh) and
 *                             a numeric part (per assembly)
 *   dpg_compose_map           GMGOperator::computeCoarseStiffnessMatrix's P^T A P, as
 *                             per-cell maps C_c P for dpg_scatter_global
 *                             (src/Solution/GMGOperator.cpp:173-366,420-773)
 *   dpg_energy_error          TSolution::rankLocalEnergyError, computeErrorRepresentation
 *                             (src/Solution/Solution.cpp:2653-2722)
 *   dpg_recover_fields        CondensedDofInterpreter::interpretGlobalCoefficients
 *                             (src/Solution/CondensedDofInterpreter.cpp:1229-1346)
 */
#ifndef DPG_B200_H
#define DPG_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DPG_ABI_VERSION 1

/* status codes */
#define DPG_OK 0
#define DPG_ERR_INVALID_ARGUMENT 1
#define DPG_ERR_UNSUPPORTED 2
#define DPG_ERR_CUDA 3
#define DPG_ERR_OUT_OF_MEMORY 4
#define DPG_ERR_TIMEOUT 5
#define DPG_ERR_BAD_PLAN 6

/* cell topologies (shards keys in the reference) */
#define DPG_TOPO_QUAD 1
#define DPG_TOPO_HEX 2
#define DPG_TOPO_TRI 3

/* function spaces (Camellia::Space / EFunctionSpace) */
#define DPG_SPACE_HGRAD 1
#define DPG_SPACE_HDIV 2
#define DPG_SPACE_HVOL 3        /* L2 */
#define DPG_SPACE_VECTOR_HVOL 4 /* VECTOR_L2, component-major dofs */

/* variable kinds (Camellia::VarType) */
#define DPG_VAR_FIELD 1
#define DPG_VAR_TRACE 2
#define DPG_VAR_FLUX 3 /* trace whose values are multiplied by the side parity */
#define DPG_VAR_TEST 4

/* operators (Camellia::EOperator subset) */
#define DPG_OP_VALUE 0
#define DPG_OP_X 1 /* vector component x (HDIV test, VECTOR_HVOL field) */
#define DPG_OP_Y 2
#define DPG_OP_Z 3
#define DPG_OP_DX 4 /* gradient components of an HGRAD test function */
#define DPG_OP_DY 5
#define DPG_OP_DZ 6
#define DPG_OP_DIV 7
#define DPG_OP_DOT_NORMAL 8 /* tau . n on a side */

/* precision of the quadrature contractions.  Only DPG_PREC_FP64 is built:
 * dpg_plan_create returns DPG_ERR_UNSUPPORTED for DPG_PREC_MIXED (split-precision
 * tensor-core contractions with an FP64 factor/solve), whose accuracy at the target
 * meshes is below the bar for the recipes with FP32 accumulation. */
#define DPG_PREC_FP64 0
#define DPG_PREC_MIXED 1

/* dpg_assemble flags */
#define DPG_FLAG_NO_K 1        /* do not write K / l (condensed outputs only) */
#define DPG_FLAG_NO_CONDENSE 2 /* do not write S / s */
/* multi-bucket calls: cells a CTA claims from the work queue at a time (1..255) */
#define DPG_FLAG_CLAIM(n) (((n) & 0xff) << 8)

typedef struct dpg_var_desc {
  int kind;       /* DPG_VAR_* */
  int space;      /* DPG_SPACE_* */
  int poly_order; /* Camellia H1Order of the variable (test: k + delta_k) */
} dpg_var_desc;

/* One scalar product in a bilinear term:
 *   coef * slot(x) * [n_{normal_comp}] * trialOp(u) * testOp(v)
 * integrated over the cell volume (boundary = 0) or over every side
 * (boundary = 1).  Vector dot products are expanded into components. */
typedef struct dpg_bf_term {
  int trial_var;   /* index into the trial list */
  int trial_op;    /* DPG_OP_VALUE, or DPG_OP_X/Y/Z for a VECTOR_HVOL field */
  int test_var;    /* index into the test list */
  int test_op;     /* DPG_OP_* */
  double coef;
  int slot;        /* coefficient slot, or -1 */
  int normal_comp; /* -1, or 0..2: also multiply by the outward unit normal's component */
  int boundary;    /* 0: volume integral, 1: sum of side integrals */
} dpg_bf_term;

/* One summand of the inner product (graph norm): term `term`, component
 * `comp` of the vector-valued linear term L_term gets coef*slot*op(v).
 * G = sum_term sum_comp  integral  L_{term,comp}(v_i) L_{term,comp}(v_j). */
typedef struct dpg_ip_entry {
  int term;
  int comp;
  int test_var;
  int test_op;
  double coef;
  int slot;
} dpg_ip_entry;

/* One summand of the load: F_i = integral coef * slot(x) * op(v_i) */
typedef struct dpg_rhs_term {
  int test_var;
  int test_op;
  double coef;
  int slot;
} dpg_rhs_term;

typedef struct dpg_bucket_desc {
  int abi_version; /* DPG_ABI_VERSION */
  int topology;    /* DPG_TOPO_* */
  int n_trial;
  const dpg_var_desc* trial;
  int n_test;
  const dpg_var_desc* test;
  int n_bf;
  const dpg_bf_term* bf;
  int n_ip;
  const dpg_ip_entry* ip;
  int n_rhs;
  const dpg_rhs_term* rhs;
  int cub_degree_G;    /* Gram (testVsTest) rule degree: 2 * max test degree */
  int cub_degree_B;    /* volume rule for B and F: max trial + max test degree */
  int cub_degree_side; /* side rule: max trace degree + max test degree */
  int n_slots;         /* number of per-point coefficient slots */
  int precision;       /* DPG_PREC_* */
} dpg_bucket_desc;

/* Sizes a caller needs to size its buffers. Coefficients are laid out
 * coeff[c][slot][p] with p over n_points_total = Q_G + Q_B + n_sides * Q_side
 * (Gram-rule volume points, then B-rule volume points, then side points
 * side-major).  Point order inside a tensor rule is x fastest. */
typedef struct dpg_plan_info {
  int N, M, n_field, n_trace;
  int space_dim, n_vertices, n_sides;
  int Q_G, Q_B, Q_side, n_points_total;
  int n_slots;
  int precision;
} dpg_plan_info;

typedef struct dpg_plan dpg_plan;

/* Build the per-bucket plan: basis and weight tables at the cubature points,
 * the compiled term lists and the launch configuration. Device tables are
 * created on the current CUDA device.  Buckets with more than 192 test or 120
 * trial dofs after padding get a plan for the large-bucket kernel (matrices in
 * a per-SM global workspace taken from the stream-ordered pool at each call);
 * such plans support dpg_assemble, dpg_assemble_host, dpg_assemble_parts,
 * dpg_energy_error, dpg_assemble_dls, dpg_assemble_multi and the graph calls,
 * and the other entry points return DPG_ERR_UNSUPPORTED. */
int dpg_plan_create(const dpg_bucket_desc* desc, dpg_plan** plan);
int dpg_plan_destroy(dpg_plan* plan);
int dpg_plan_query(const dpg_plan* plan, dpg_plan_info* info);

/* Per-bucket autotuner (no counterpart in the reference: Camellia has no GPU
 * launch shapes to choose).  Times dpg_assemble on the C given cells (DEVICE
 * pointers as for dpg_assemble) with each candidate shape, keeps the faster for
 * all later calls on this plan (dpg_assemble, the multi-bucket launch and its
 * graph) and returns it in *chosen: for single-CTA plans the Gram staging chunk
 * that fits the bucket's shared memory (8 or 4 quadrature points per chunk: it
 * sets the shared-memory layout and the kernel instance), for large-bucket plans
 * the formation k-chunk (32 or 16 points).  Results of the configurations agree
 * to rounding (sums are ordered differently).  Allocates its timing outputs from
 * the library's pool. */
int dpg_plan_autotune(dpg_plan* plan, int C, const double* nodes, const int8_t* parity, const double* coeff,
                      void* stream, int* chosen);

/* Assemble C cells; all pointers are DEVICE pointers.
 *   nodes  (C, n_vertices, space_dim)   physical vertex coordinates
 *   parity (C, n_sides) int8 +-1        Camellia cellSideParities
 *   coeff  (C, n_slots, n_points_total) may be NULL when n_slots == 0
 *   K, l, S, s as above (K/l may be NULL with DPG_FLAG_NO_K, S/s with
 *   DPG_FLAG_NO_CONDENSE); info (C) int32.
 * stream: a cudaStream_t (NULL = legacy default stream). Asynchronous. */
int dpg_assemble(dpg_plan* plan, int C, const double* nodes, const int8_t* parity,
                 const double* coeff, double* K, double* l, double* S, double* s,
                 int32_t* info, void* stream, int flags);

/* Same as dpg_assemble with HOST buffers (pinned memory is fastest). The
 * library stages the cells through device memory in chunks with copies
 * overlapped with compute; returns after the results are in host memory. */
int dpg_assemble_host(dpg_plan* plan, int C, const double* nodes, const int8_t* parity,
                      const double* coeff, double* K, double* l, double* S, double* s,
                      int32_t* info, int flags);

/* The quadrature products alone (device pointers; any output may be NULL). */
int dpg_assemble_parts(dpg_plan* plan, int C, const double* nodes, const int8_t* parity,
                       const double* coeff, double* G, double* B, double* F, void* stream);

/* Batched factored-Cholesky optimal-test solve on given matrices (device
 * pointers). G (C,N,N) symmetric, B (C,M,N) [column-major N x M per cell],
 * F (C,N). Outputs K (C,M,M), l (C,M), info (C). Inputs are not modified. */
int dpg_factored_cholesky_solve(int C, int N, int M, const double* G, const double* B,
                                const double* F, double* K, double* l, int32_t* info,
                                void* stream);

/* Adjoint of dpg_assemble (K and l outputs) for a loss J(K, l):
 * given Kbar (C,M,M) and lbar (C,M) = dJ/dK, dJ/dl (lbar may be NULL), writes
 * coeff_bar (C, n_slots, n_points_total) = dJ/dcoeff. Device pointers.
 * Covers coefficients in the inner product, in volume bilinear and load terms
 * and in boundary terms whose test operator is a value or a normal trace;
 * other plans return DPG_ERR_UNSUPPORTED. No counterpart in the reference. */
int dpg_assemble_adjoint(dpg_plan* plan, int C, const double* nodes, const int8_t* parity,
                         const double* coeff, const double* Kbar, const double* lbar,
                         double* coeff_bar, int32_t* info, void* stream);

/* Field back-substitution after the global (trace) solve: replaces
 * CondensedDofInterpreter::interpretGlobalCoefficients
 * (src/Solution/CondensedDofInterpreter.cpp:1229-1346).  For each cell solves
 * K_ff u_f = l_f - K_ft t with the cell's K (C,M,M) and l (C,M) from dpg_assemble
 * (user numbering, fields first) and its trace coefficients t (C, n_trace), and
 * writes the local coefficients [u_f | t] to local_coeff (C,M).  info[c] = first
 * non-positive pivot of the equilibrated K_ff (1-based) or 0.  Device pointers. */
int dpg_recover_fields(dpg_plan* plan, int C, const double* K, const double* l, const double* trace_coeff,
                       double* local_coeff, int32_t* info, void* stream);

/* DLS local matrices: replaces TBF::localStiffnessMatrixAndRHS_DLS
 * (src/ScratchPad/BF.cpp:1169-1306), whose factored solve leaves W = L^-1 B in the
 * "stiffnessEnriched" array and y = L^-1 F in the enriched load (G = L L^T).
 * W (C,M,N) trial x test and y (C,N), user numbering.  Device pointers. */
int dpg_assemble_dls(dpg_plan* plan, int C, const double* nodes, const int8_t* parity, const double* coeff,
                     double* W, double* y, int32_t* info, void* stream);

/* Energy error of a trial solution per cell: replaces TSolution::rankLocalEnergyError
 * with computeErrorRepresentation (src/Solution/Solution.cpp:2653-2722).  For the
 * cells' local trial coefficients x (C,M; user numbering, fields first) writes
 * energy[c] = sqrt(r^T G^-1 r), r = F - B x the residual on the test space.
 * info as for dpg_assemble; a cell whose Gram factorisation fails (info != 0)
 * gets energy[c] = NaN.  Device pointers. */
int dpg_energy_error(dpg_plan* plan, int C, const double* nodes, const int8_t* parity, const double* coeff,
                     const double* local_coeff, double* energy, int32_t* info, void* stream);

/* Global assembly of condensed cell systems: replaces the GDA interpretation
 * GDAMinimumRule::interpretLocalData (src/Mesh/GDAMinimumRule.cpp:714-800, C^T S C
 * through the LocalDofMapper) and the insertion into the global matrix
 * (src/Solution/Solution.cpp:1263-1293).  Local dof a of cell c stands for
 * sum_k map_w[k] x[map_gid[k]], k in [map_ptr[c t + a], map_ptr[c t + a + 1])
 * (map_w NULL: all weights 1).  Adds sum_c C_c^T S_c C_c into the values of the
 * caller's CSR graph (n_global rows; row_ptr, col_idx sorted within rows) and
 * sum_c C_c^T s_c into rhs (may be NULL); contributions whose target is absent from
 * the graph or whose global index is outside [0, n_global) are skipped and *missing
 * (device int) is raised by a positive count (0 when nothing was skipped).  S (C,t,t),
 * s (C,t) as from dpg_assemble.  Its per-cell tables take 4 t^2 + 104 t + 12 bytes of
 * shared memory, which must fit in 200 KB (t <= 213), else DPG_ERR_UNSUPPORTED.  Device pointers; the sum
 * over cells runs through atomics, so its last bits vary between runs. */
int dpg_scatter_global(int C, int t, const int64_t* map_ptr, const int64_t* map_gid, const double* map_w,
                       int64_t n_global, const int64_t* row_ptr, const int64_t* col_idx, const double* S,
                       const double* s, double* values, double* rhs, int* missing, void* stream);

/* The same global scatter split into a symbolic part, done once for a fixed mesh,
 * map and graph, and a numeric part per assembly (nonlinear iterations, time steps).
 * dpg_scatter_plan_create ranks every cell's map entries by global id, groups them and
 * finds the CSR position of each of the cell's distinct (row, column) pairs, into
 * device arrays the plan owns; contributions with no target in the graph or a global
 * id outside [0, n_global) raise *missing (device int, may be NULL) here, once, by a
 * positive count, and are skipped by every apply.  The call waits for the stream.
 * dpg_scatter_plan_apply adds sum_c C_c^T S_c C_c into values and sum_c C_c^T s_c
 * into rhs (s and rhs may be NULL), with the same arithmetic as dpg_scatter_global;
 * S, s and the plan's map and graph must describe the same cells.  A cell's map
 * entries must fit the plan's shared tables (48 bytes each, 200 KB in all), else
 * DPG_ERR_UNSUPPORTED.  Device pointers. */
typedef struct dpg_scatter_plan dpg_scatter_plan;
int dpg_scatter_plan_create(int C, int t, const int64_t* map_ptr, const int64_t* map_gid, const double* map_w,
                            int64_t n_global, const int64_t* row_ptr, const int64_t* col_idx, int* missing,
                            void* stream, dpg_scatter_plan** out);
int dpg_scatter_plan_apply(const dpg_scatter_plan* plan, const double* S, const double* s, double* values,
                           double* rhs, void* stream);
int dpg_scatter_plan_destroy(dpg_scatter_plan* plan);

/* Local-to-coarse maps for a Galerkin multigrid coarse operator.  Replaces the
 * sparse triple product P^T A P of GMGOperator::computeCoarseStiffnessMatrix
 * (src/Solution/GMGOperator.cpp:173-366), A the assembled fine matrix and P the
 * prolongation from the fine cells' LocalDofMappers (GMGOperator.cpp:420-773,
 * 959-1551): since P^T A P = sum_c (C_c P)^T S_c (C_c P), this call composes each
 * cell's local-to-fine map (map_ptr, map_gid, map_w as for dpg_scatter_global,
 * C*t rows, n_fine global dofs) with P (CSR: n_fine rows P_row_ptr, coarse column
 * ids P_col, values P_val), and dpg_scatter_global with the composed map and the
 * cells' S, s assembles the coarse operator and load.  Outputs: out_ptr (C*t+1
 * row offsets), and, when out_gid is not NULL, out_gid / out_w (coarse ids and
 * weights map_w[k] * P_val[j], in the order of k then j; repeated coarse ids are
 * kept).  *out_count (host) receives the number of composed entries; a call with
 * out_gid NULL is the size query.  Fails with DPG_ERR_INVALID_ARGUMENT when that
 * number exceeds capacity.  Map entries with a fine id outside [0, n_fine) are
 * skipped and added to *missing (device int, may be NULL) on every call.  Device
 * pointers except out_count; the call waits for the stream once (the count). */
int dpg_compose_map(int C, int t, const int64_t* map_ptr, const int64_t* map_gid, const double* map_w,
                    int64_t n_fine, const int64_t* P_row_ptr, const int64_t* P_col, const double* P_val,
                    int64_t* out_ptr, int64_t* out_gid, double* out_w, int64_t capacity,
                    int64_t* out_count, int* missing, void* stream);

/* Multi-bucket assembly (TSolution::populateStiffnessAndLoad's loop over
 * ElementType buckets, Solution.cpp:1131-1297).  The single-CTA buckets share one
 * persistent work-queue launch: their cell ranges are concatenated in decreasing
 * order of per-cell cost and each CTA claims DPG_FLAG_CLAIM(n) cells at a time
 * (default 1) from a device counter, so long cells start first and short ones fill
 * the tail; no CTA waits on another.  Each large bucket runs its own persistent
 * launch, in decreasing order of cost (a queue holding large cells ran them 11-28 %
 * slower: the specialized kernel keeps its plan in parameter space and a register
 * allocation of its own).  Pointers per bucket as in dpg_assemble (device memory);
 * flags as for dpg_assemble plus the claim size. */
typedef struct dpg_bucket_batch {
  dpg_plan* plan;
  int C;
  const double* nodes;
  const int8_t* parity;
  const double* coeff;
  double* K;
  double* l;
  double* S;
  double* s;
  int32_t* info;
} dpg_bucket_batch;

int dpg_assemble_multi(int n_buckets, const dpg_bucket_batch* buckets, void* stream, int flags);

/* Autotuner of the multi-bucket launch (no counterpart in the reference): times the
 * work queue of the given single-CTA buckets with claim sizes 1, 2, 4 and 8 cells
 * and returns the fastest in *chosen (pass it back as DPG_FLAG_CLAIM(*chosen); 1
 * when there are only large buckets).  The per-bucket shapes come from
 * dpg_plan_autotune on each plan beforehand. */
int dpg_multi_autotune(int n_buckets, const dpg_bucket_batch* buckets, void* stream, int flags, int* chosen);

/* The same multi-bucket launch recorded once in a CUDA graph and replayed:
 * for a fixed mesh re-assembled every step (new coefficients written into the
 * same buffers).  Capture uploads the bucket tables and allocates the
 * workspace (outside any stream capture of the caller); every launch then
 * reads the buffers named at capture time.  The graph holds the large buckets'
 * launches in decreasing order of cost, then the work queue of the single-CTA
 * buckets (whose counters reset themselves at the end of each launch).  Launches
 * of one graph must not overlap on the GPU (they share the workspace). */
typedef struct dpg_graph dpg_graph;
int dpg_graph_capture(int n_buckets, const dpg_bucket_batch* buckets, int flags, dpg_graph** out);
int dpg_graph_launch(dpg_graph* graph, void* stream);
int dpg_graph_destroy(dpg_graph* graph);

/* dpg_assemble without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory while
 * they assemble — an application whose GPU memory is already fully reserved by
 * its own pool (a framework's caching allocator, or a pre-sized arena shared by
 * several solver ranks), or a time-stepping loop that must not take allocation
 * latency or an out-of-memory failure in the middle of a step.
 * dpg_assemble takes its per-CTA scratch (the B tiles held between the B phase
 * and the triangular solve, and the Gram matrix's running sums) from a
 * stream-ordered allocation; this variant uses a fixed 32 MiB array that the
 * library reserves on every GPU that loads it, until the process exits.  Same
 * arguments, outputs and errors as dpg_assemble, plus:
 *   - the first call on a device looks the array up (cudaGetSymbolAddress) with
 *     that device current, and so does the first call after that device's
 *     context was destroyed and recreated (cudaDeviceReset); make those calls
 *     outside any stream capture;
 *   - large-bucket plans (more than 192 test rows or 120 trial columns after
 *     padding) are rejected with DPG_ERR_UNSUPPORTED, and so are buckets whose
 *     per-CTA scratch exceeds 32 MiB; otherwise the launch uses as many CTAs as
 *     fit (floor(32 MiB / per-CTA scratch), at most one per SM): the 3D hex k=2
 *     bucket (298 KiB per CTA) runs on 110 CTAs;
 *   - every call shares the one array: calls that overlap on the GPU (other
 *     streams, other threads, other plans) race and must be serialised by the
 *     caller.  The array keeps the last call's contents; every call writes the
 *     scratch it reads, so nothing needs clearing. */
int dpg_assemble_noalloc(dpg_plan* plan, int C, const double* nodes, const int8_t* parity,
                         const double* coeff, double* K, double* l, double* S, double* s,
                         int32_t* info, void* stream, int flags);

/* The reference bases and cubature rules the plans are built from, for checking
 * their conventions (host only; no GPU needed).  No counterpart in the reference as
 * a C call: they tabulate what Camellia gets from Intrepid through BasisFactory
 * (src/Basis/BasisFactory.cpp:122-420) and CubatureFactory
 * (src/Basis/CubatureFactory.cpp:25-53).
 * dpg_basis_tabulate: space DPG_SPACE_HGRAD (order n >= 0: Cn, nodal at the
 * Gauss-Lobatto points of [-1,1]^d, x fastest; triangles: the warp & blend lattice
 * on (0,0),(1,0),(0,1)) or DPG_SPACE_HDIV (order n >= 1: In, component-major; on
 * triangles RT_n).  out holds, per point and dof, d + 1 doubles: HGRAD value and
 * the d reference derivatives, HDIV the d value components and the divergence.
 * Returns the cardinality, or -(DPG_ERR_*) on an invalid argument.
 * dpg_cubature: the rule exact to `degree` (tensor Gauss on [-1,1]^d, collapsed
 * Gauss on the triangle); pts (npts, d) and wts (npts) may be NULL; returns npts,
 * or -(DPG_ERR_*) on an invalid argument. */
int dpg_basis_tabulate(int topology, int space, int n, int npts, const double* pts, double* out);
int dpg_cubature(int topology, int degree, double* pts, double* wts);

/* Thread-local description of the last error. */
const char* dpg_last_error_string(void);

/* Library version string and the compiled architecture. */
const char* dpg_version(void);

#ifdef __cplusplus
}
#endif

#endif /* DPG_B200_H */
