// dpg_plan.h — per-bucket plan shared by the host builder and the sm_100a kernels.
//
// Layout conventions used by the kernels (all FP64):
//  * Test dofs are stored var by var, each var padded to a multiple of 8
//    ("test tiles"); trial dofs as [fields | traces | F column], each group padded
//    to a multiple of 8 ("trial tiles").  The F column (the load vector) rides
//    along as one extra trial column so y = L^-1 F and l = W^T y fall out of the
//    same triangular solve and Gram product as W and K.
//  * 8x8 tiles in shared memory use the "AK" layout: element (r, c) of a tile is at
//    ((c >> 2) * 8 + r) * 4 + (c & 3).  A-fragments of mma.m8n8k4 (thread (g,t)
//    holds A[g][4h+t]) and B-fragments of the transposed tile then read 32
//    consecutive doubles per k-step h: bank-conflict free.
#pragma once

#define DPG_MAXV 8        // max test vars / trial vars per bucket
#define DPG_MAX_BF 96     // max scalar bilinear products
#define DPG_MAX_IP 64     // max inner-product entries
#define DPG_MAX_RHS 8
#define DPG_MAX_FEAT 32   // 4 features per test var (padded) * DPG_MAXV
#define DPG_MAX_IPROWS 24
#define DPG_MAX_BOPS 24   // distinct (test var, op) pairs used by B terms in a segment
#define DPG_MAX_SEG 7     // volume + up to 6 sides
#define DPG_NWARPS 16
#define DPG_NTHREADS (DPG_NWARPS * 32)
#define DPG_CHUNK 4       // quadrature points per staged chunk (one mma k-step per point)
#define DPG_MAX_NBT 24    // max test tiles (N <= 192)
#define DPG_MAX_MBT 16    // max trial tiles incl. the F tile (one column tile per warp)
#define DPG_MAX_GT 19     // max lower G tiles per warp: ceil(24*25/2 / 16)
#define DPG_MAX_KT 9      // max lower K_ext tiles per warp: ceil(16*17/2 / 16)

struct DpgIPEnt {
  int row;      // (term, comp) row
  int gfeat;    // global feature index: var * 4 + local feature
  double coef;
  int slot;
};

struct DpgBTerm {
  int trial_var, trial_op, test_var, test_op;
  double coef;
  int slot, normal_comp;
  int seg;        // 0 = volume, 1 + s = side s
  int bop;        // index of (test var, test op) in the segment's op table
  int col0, ncol; // device trial columns touched (contiguous)
  int kind;       // trial var kind
  int tvar_comp;  // component (vector fields), 0 otherwise
};

struct DpgTrialVar {
  int kind, space, ncomp;
  int card_comp;  // dofs per component (fields) or per side (traces)
  int dev_off;    // first device trial column
  int user_off;   // first user trial index
  int per_side;   // traces: dofs per side
  const double* tabB;  // fields: ref values at B points [QB][card_comp]
  const double* tabS;  // fields: [ns][QS][card_comp]; traces: [QS][per_side]
};

struct DpgTestVar {
  int space;      // DPG_SPACE_HGRAD / HDIV
  int card;       // user dofs
  int dev_off;    // first device row
  int user_off;
  int ntile0, ntiles;  // tile range
  int nref;       // reference comps per dof: HGRAD 1 + d (value, grad), HDIV d + 1 (value, div)
  int nfeat;      // G features (<= 4)
  int feat_op[4];
  int ldA;        // padded leading dimension of staged operands (== 4 mod 16)
  const double* tabG;  // [QG][card][nref]
  const double* tabB;  // [QB][card][nref]
  const double* tabS;  // [ns][QS][card][nref]
};

struct DpgGTile {
  int I, J;       // tile coordinates (I >= J)
  int aoff, lda;  // A operand: offset inside a point's feature block, leading dim
  int boff, ldb;  // B operand: offset inside a point's h block
};

struct DpgBOp {
  int var, op;
  int off;        // offset inside a point's staged B-op block
};

struct DpgSeg {
  int npts;       // quadrature points (volume: QB; side: QS)
  int nops;
  DpgBOp ops[DPG_MAX_BOPS];
  int opstride;   // doubles per point of staged test ops
  int term0, nterm;  // range in the (segment-sorted) term list
  int rhs;        // 1: volume segment also carries the RHS (F column)
};

struct DpgPlanDev {
  int d, nv, ns;
  int N, M, nf, nt;
  int Np, NBT;              // padded test rows, test tiles
  int nfp, ntp, Mp, MBT;    // padded fields/traces, device trial columns incl F tile, trial tiles
  int nfb;                  // field tiles
  int fcol;                 // device column of F
  int QG, QB, QS, Ptot, nslots;
  int ntest, ntrial;
  DpgTestVar test[DPG_MAXV];
  DpgTrialVar trial[DPG_MAXV];
  // Gram
  int Ftot;                 // 4 * ntest
  int niprows, nipent;
  DpgIPEnt ipent[DPG_MAX_IP];
  int ngt;                  // lower G tiles
  const DpgGTile* gtiles;   // [ngt]
  int featstride;           // doubles per point of staged features (sum over vars of 4*ldA)
  int hstride;              // doubles per point of staged h blocks (sum over pairs)
  int hoff[DPG_MAXV][DPG_MAXV];  // offset of h_{b->a} block inside a point's h block (a >= b)
  // B and F
  int nseg;
  DpgSeg seg[DPG_MAX_SEG];
  int nbterm;
  DpgBTerm bterm[DPG_MAX_BF];  // sorted by segment
  int nrhs;
  DpgIPEnt rhs[DPG_MAX_RHS];   // (unused row), gfeat = test var * 16 + op, coef, slot
  int ldT;                     // leading dim of staged trial values (== 4 mod 16, >= Mp)
  // geometry tables
  const double* dNG;  // [QG][nv][d]
  const double* dNB;  // [QB][nv][d]
  const double* dNS;  // [ns][QS][nv][d]
  const double* wG;   // [QG]
  const double* wB;   // [QB]
  const double* wS;   // [QS]
  const double* sideT;  // [ns][QS][2][3] reference tangents (2D: one)
  // index maps
  const int* dev2user_trial;  // [Mp] -> user trial index, or -1
  const int* dev2user_test;   // [Np] -> user test index, or -1
  // shared memory layout (doubles)
  int sm_total;
  int sm_geo, sm_cmat, sm_feat, sm_h, sm_gt, sm_linv, sm_scale, sm_bops, sm_bval, sm_w, sm_k, sm_misc;
};
