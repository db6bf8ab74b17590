// dpg_plan.h — per-bucket plan shared by the host builder and the sm_100a kernels.
//
// Layout conventions used by the kernels (all FP64):
//  * Test dofs are stored var by var, each var padded to a multiple of 8
//    ("test tiles"); trial dofs as [fields | traces | F column], each group padded
//    to a multiple of 8 ("trial tiles").  The F column (the load vector) rides
//    along as one extra trial column so y = L^-1 F and l = W^T y fall out of the
//    same triangular solve and Gram product as W and K.
//  * Reference features: every test var has four "slots" per dof and point,
//    HGRAD: (phi, dphi/dxi_0, dphi/dxi_1, dphi/dxi_2), HDIV: (v_0, .., v_{d-1}, div v)
//    (unused slots zero).  Physical operators are linear in the slots with
//    per-point coefficients from the Jacobian (the Piola maps), so every
//    geometric factor is folded into small per-point coupling matrices and the
//    slot tables themselves are per-bucket constants, copied to shared memory
//    by bulk (TMA) copies.  Staged layout per point: [var][slot][ldA].
//  * 8x8 tiles in shared memory use the "AK" layout: element (r, c) of a tile is at
//    ((c >> 2) * 8 + r) * 4 + (c & 3).  A-fragments of mma.m8n8k4 (thread (g,t)
//    holds A[g][4h+t]) and B-fragments of the transposed tile then read 32
//    consecutive doubles per k-step h: bank-conflict free.
#pragma once
#include <stdint.h>

#define DPG_MAXV 16       // max test vars / trial vars per bucket
#define DPG_MAX_BF 96     // max scalar bilinear products (after side expansion)
#define DPG_MAX_IP 64     // max inner-product entries
#define DPG_MAX_RHS 8
#define DPG_MAX_IPROWS 24
#define DPG_MAX_SEG 7     // volume + up to 6 sides
#define DPG_MAX_BLK 24    // active (test var, trial column tile) blocks per segment
#define DPG_MAX_PAIRS 36  // test var pairs a >= b
#define DPG_NWARPS 16
#define DPG_NTHREADS (DPG_NWARPS * 32)
#define DPG_CHG 8         // Gram quadrature points per staged chunk (4 when shared memory is short)
#define DPG_MAX_CHB 16    // max B quadrature points per staged chunk
#define DPG_MAX_BT 12     // max terms feeding one B block
#define DPG_MAX_BTW 12    // max active B tiles per warp per segment
#define DPG_MAX_QG 512    // max Gram-rule points
#define DPG_MAX_NBT 24    // max test tiles (N <= 192)
#define DPG_MAX_MBT 16    // max trial tiles incl. the F tile (one column tile per warp)
#define DPG_MAX_GT 12     // max 16x8 G blocks per warp
#define DPG_MAX_KT 9      // max lower K_ext tiles per warp: ceil(16*17/2 / 16)
#define DPG_ULD 12        // leading dim of a staged 8-column U block (conflict-free B-fragments)

struct DpgIPEnt {
  int row;      // (term, comp) row
  int gslot;    // global physical slot: var * 4 + slot
  double coef;
  int slot;     // coefficient slot, or -1
};

struct DpgBTerm {
  int trial_var, test_var, test_op;
  int kind;       // trial var kind; -1 = RHS (the F column)
  double coef;
  int slot, normal_comp;
  int col0, ncol; // device trial columns touched (contiguous)
};

// A boundary term whose test operator has a cell-independent side transform
// (HGRAD value; HDIV normal trace through the Piola identity
// (J v / det J) . n |J_s| = v . (t_0 x t_1) on the reference side), on one side.
// Per point it contributes factor(q) * W[q][c] to each of its entries c, with the
// cell-independent weights W = reference test value x trial value.
struct DpgSideTerm {
  int side;
  int pbase;        // first coefficient point of the side
  int slot;         // coefficient slot or -1
  int normal_comp;  // multiply by n_c, or -1
  int flux;         // multiply by the side parity
  int use_meas;     // 1: factor w |J_s| from the geometry; 0: the side weight is inside W
  double coef;
};

struct DpgBBlock {
  int var;        // test var
  int J;          // trial column tile
  int off;        // offset of the block inside a point's U region (doubles)
  int nt;         // terms feeding the block (segment-local indices)
  int terms[DPG_MAX_BT];
};

struct DpgSeg {
  int npts;                 // quadrature points
  int chunk, nchunk;        // points per staged chunk, number of chunks (chunk * nchunk >= npts)
  int side;                 // -1 volume, else side index
  const double* rec;        // [nchunk * chunk][rec_len] per-point records: reference slots, then trial values
  int rec_len;              // doubles per record (even)
  int geo0;                 // first point of the segment in the all-B-points geometry list
  int pbase;                // first coefficient point index of the segment
  int nblk;
  DpgBBlock blk[DPG_MAX_BLK];
  int ustride;              // doubles per point of staged U blocks
  int term0, nterm;         // range in the segment-sorted term list
  int tvoff[DPG_MAX_BF / 4];// offset of each (segment-local) term's trial values inside a record
  int tile0, ntile;         // active (I, J) tiles of the segment: btiles[tile0 .. tile0 + ntile)
};

struct DpgTrialVar {
  int kind, space, ncomp;
  int card_comp;  // dofs per component (fields) or per side (traces)
  int dev_off;    // first device trial column
  int user_off;   // first user trial index
  int per_side;   // traces: dofs per side
  const double* tabB;  // fields: ref values at B points [QBpad][card_comp]
  const double* tabS;  // fields: [ns][QSpad][card_comp]; traces: [QSpad][per_side]
};

struct DpgTestVar {
  int space;      // DPG_SPACE_HGRAD / HDIV
  int card;       // user dofs
  int dev_off;    // first device row
  int user_off;
  int ntile0, ntiles;  // tile range
  int ldA;        // padded leading dimension of staged slot rows (== 4 mod 16)
  int foff;       // offset of the var inside a point's staged slot block
};

// One 16x8 block of G for mma.m16n8k16: rows of test tiles (I, I+1) of one
// var, columns of test tile J.  The upper tile (I, I+1) of a diagonal block is
// computed and dropped.
struct DpgGTile {
  int16_t I, J;
  int16_t lda, ldb;
  int aoff, boff;  // A operand / B operand offsets inside a point's feature / h block
};

struct DpgPlanDev {
  int d, nv, ns;
  int N, M, nf, nt;
  int Np, NBT;              // padded test rows, test tiles
  int nfp, ntp, Mp, MBT;    // padded fields/traces, device trial columns incl F tile, trial tiles
  int nfb;                  // field tiles
  int fcol;                 // device column of F
  int QG, QB, QS, Ptot, nslots;
  int QGpad, QBpad, QSpad;
  int ntest, ntrial;
  DpgTestVar test[DPG_MAXV];
  DpgTrialVar trial[DPG_MAXV];
  // Gram
  int niprows, nipent;
  DpgIPEnt ipent[DPG_MAX_IP];
  int npairs;
  int pair_a[DPG_MAX_PAIRS], pair_b[DPG_MAX_PAIRS];
  int hoff[DPG_MAX_PAIRS];  // offset of h_{b->a} inside a point's h block
  int rowstart[DPG_MAX_IPROWS + 1];  // IP entries of row r: [rowstart[r], rowstart[r+1])
  int ngt;                  // lower 8x8 tiles of G: NBT (NBT + 1) / 2
  int ngb;                  // 16x8 G blocks
  const DpgGTile* gtiles;   // [ngb]
  int ngz;                  // lower tiles of G that no block writes (uncoupled test var pairs)
  const int* gzero;         // [ngz] their indices I (I + 1) / 2 + J
  int chg;                  // Gram points per staged chunk (DPG_CHG or DPG_CHG / 2)
  int featstride;           // doubles per point of staged slots (sum over vars of 4*ldA)
  int hstride;              // doubles per point of staged h blocks (sum over pairs)
  const double* frefG;      // [QGpad][featstride]
  const double* wG;         // [QGpad]
  const double* dNG;        // [QGpad][nv][d]
  // B and F
  int nseg;
  DpgSeg seg[DPG_MAX_SEG];
  int nbterm;
  DpgBTerm bterm[DPG_MAX_BF];  // sorted by segment
  int nbpts;                // all B points: volume then sides
  const double* dNB;        // [nbpts][nv][d]
  const double* wB;         // [nbpts]
  const double* tangB;      // [nbpts][6] reference side tangents (zero for volume points)
  int max_rec, max_chunk, max_ustride, max_nterm;
  const int4* btiles;       // active B tiles of all segments: (I, J, block, 0)
  // separable side terms: B[row][col] += sum_c sum_q W[q][c] factor_se(c)(q) over the
  // contributions c of each entry (row, col)
  int nse, nsent, ncon;
  const DpgSideTerm* se;    // [nse]
  const int4* sent;         // [nsent] (scratch element, first contribution, count, side term of the
                            //  first | 1 << 16 when the element has no other writer)
  const int* scon_se;       // [ncon] side term of each contribution
  const double* scon_w;     // [QS][ncon]
  // reverse mode (dpg_assemble_adjoint)
  int adj_ok;               // the adjoint's workspaces fit and every coefficient use is supported
  int ip_slots, b_slots, se_slots;  // coefficient slots occur in the IP / volume B and load / side terms
  const int* sadj_start;    // [nse + 1] contributions of each side term
  const int* sadj_con;      // contribution indices grouped by side term
  const int2* scon_rc;      // [ncon] (device row, device column) of each contribution
  // index maps
  const int* dev2user_trial;  // [Mp] -> user trial index, or -1
  const int* dev2user_test;   // [Np] -> user test index, or -1
  // shared memory layout (doubles)
  int sm_total;
  int sm_tiles;   // persistent: tile table copy
  int sm_nodes;   // persistent: cell vertices, flags, mbarriers, triangular index table (192 doubles)
  int sm_coef;    // per cell: coefficients [nslots][Ptot]
  int g_fref0, g_fref1, g_h, g_geo, g_D, g_beta;   // Gram phase (g_beta overlaps g_h)
  int sm_gt, sm_linv, sm_scale, sm_invd;           // factor
  int b_rec0, b_rec1, b_u, b_geo, b_fac;      // B phase
  int sm_w, sm_k;                                  // solve / Gram of W
  int a_sa, a_ldS;                                 // adjoint: S_A [MBT*8][a_ldS]
  int a_fs, a_xpf, a_ldx, a_geo, a_beta, a_cbar;   // adjoint pull-back
  size_t scratch_per_cta;                          // doubles of scratch per CTA: B tiles, then
                                                   // the Gram running sums at gsum_off
  size_t gsum_off;                                 // [ngb][32 lanes][4] Gram partial sums
  int gflush;                                      // staged Gram chunks between two flushes of the
                                                   // accumulators into the running sums (0: none)
  uint32_t gflushbits[DPG_NWARPS];                 // per warp: its blocks (bit u = its u-th) that
                                                   // take part in the flushes (var pairs that two
                                                   // or more graph-norm terms couple)
  // Large buckets (N > 192 or M > 120 after padding) run on dpg_big_kernel: per cell the
  // lower triangle of Z = [[G, E], [E^T, 0]] (E = [B^T | F]; rows/columns: device test rows,
  // then device trial columns) in a per-CTA global workspace.
  int big;
  int Zn, ldz;              // Z order (Np + Mp) and row stride (doubles)
  int nbe;                  // E-formation entries, one per (segment, term)
  int4 be[DPG_MAX_BF];      // (segment, segment-local term, first vt row, points)
  int ipmask[DPG_MAX_IPROWS];  // test vars each IP row touches (bit a)
  const int* u2d_trial;     // [M] user trial index -> device column
  const int* u2d_test;      // [N] user test index -> device row
  int bz_wq, bz_bh, bz_vt;  // per-CTA workspace after Z: w|J| at Gram points, per-point IP row
                            // factors [QG][rows][ntest][4], per-point term factors [vt rows][4]
  size_t bz_per_cta;        // doubles of per-CTA workspace
  int big_zk;               // formation k-chunk (16 or 32 points; dpg_plan_autotune picks it)
  int bs_sc, bs_col, bs_int, bs_nodes, bs_total;  // shared memory (doubles): scales, column
                                                  // records, ints, vertices; total
};
