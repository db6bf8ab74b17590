"""CPU emulation of reduced-precision tensor-core contractions for the Gram matrix G and
the stiffness B, applied term by term in the reference's order (each graph-norm term's
Gram block integrated on its own, IP.cpp:238-244 -> LinearTerm.cpp:470-606, then summed
in FP64), followed by the FP64 factored Cholesky solve and condensation of the oracle.

Recipes (A^T B over the contraction index k = (point, component)):
  * "bf16x3": A = A1 + A2, B = B1 + B2 with A1 = bf16(A), A2 = bf16(A - A1); products
    A1 B1 + A1 B2 + A2 B1 (exact in FP32), summed per MMA k-block of 16 (exactly here,
    which flatters the hardware), rounded to FP32 and accumulated in FP32 over the
    points of a chunk; chunks summed in FP64;
  * "bf16x6": three-way bf16 split, the six products A_i B_j with i + j <= 4;
  * "tf32x3": as bf16x3 with TF32 (10 stored mantissa bits) parts and k-blocks of 8;
  * "int8xK": Ozaki-style slicing.  Each column j of A = sqrt(w) L is scaled by a power
    of two so that |A_j| < 1 and cut into K slices of 7 bits (int8 in [-127, 127]);
    every slice product S_a^T S_b is exact (int32 accumulation on the tensor cores; an
    exact float64 product here, since every partial sum is an integer below 2^53) and
    the slice products are combined in FP64.  "int8xK" keeps all K^2 slice pairs, which
    makes the result the exact Gram matrix of the sliced operator; "int8xKt" keeps the
    pairs a + b <= K + 1 (the usual truncated Ozaki scheme).

TEST INFRASTRUCTURE ONLY (uses the oracle)."""
from __future__ import annotations

import numpy as np


def round_bf16(x):
    """Round float64 values to bfloat16 (8 significant bits), nearest-even."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = ((u + 0x7FFF + lsb) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def round_tf32(x):
    """Round float64 values to TF32 (11 significant bits), nearest-even."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 13) & 1
    u = ((u + 0xFFF + lsb) >> 13) << 13
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def split(x, rnd, n):
    parts, r = [], np.asarray(x, dtype=np.float64)
    for _ in range(n):
        p = rnd(r)
        parts.append(p)
        r = r - p
    return parts


def _fp32_mma(A, B, kblock, chunk_rows):
    """sum_k A[k,i] B[k,j]: exact k-block sums rounded to FP32, FP32 accumulation over a
    chunk of rows, FP64 sum of the chunks.  A (K, m), B (K, n), float64 inputs whose
    pairwise products are exact."""
    K = A.shape[0]
    out = np.zeros((A.shape[1], B.shape[1]))
    for c0 in range(0, K, chunk_rows):
        acc = np.zeros((A.shape[1], B.shape[1]), dtype=np.float32)
        for k0 in range(c0, min(K, c0 + chunk_rows), kblock):
            k1 = min(K, k0 + kblock, c0 + chunk_rows)
            blk = (A[k0:k1].T @ B[k0:k1]).astype(np.float32)
            acc = (acc + blk).astype(np.float32)
        out += acc.astype(np.float64)
    return out


def split_product(A, B, recipe, chunk_rows):
    if recipe == "bf16x3":
        (a1, a2), (b1, b2) = split(A, round_bf16, 2), split(B, round_bf16, 2)
        pairs, kb = [(a1, b1), (a1, b2), (a2, b1)], 16
    elif recipe == "bf16x6":
        a, b = split(A, round_bf16, 3), split(B, round_bf16, 3)
        pairs, kb = [(a[i], b[j]) for i in range(3) for j in range(3) if i + j <= 2], 16
    elif recipe == "tf32x3":
        (a1, a2), (b1, b2) = split(A, round_tf32, 2), split(B, round_tf32, 2)
        pairs, kb = [(a1, b1), (a1, b2), (a2, b1)], 8
    else:
        raise ValueError(recipe)
    # each product accumulates in FP32 on its own (one MMA chain per split pair); the
    # pair results are summed in FP64, smallest first
    out = np.zeros((A.shape[1], B.shape[1]))
    for pa, pb in reversed(pairs):
        out += _fp32_mma(pa, pb, kb, chunk_rows)
    return out


def int8_slices(A, nslices):
    """Per-column power-of-two scale and int8 slices: A[:, j] ~ 2^e[j] sum_a S_a[:, j] 128^-a."""
    amax = np.abs(A).max(axis=0)
    e = np.where(amax > 0, np.frexp(np.where(amax > 0, amax, 1.0))[1], 0).astype(np.int64)
    # |A / 2^e| < 1 (frexp gives amax = m 2^e with 0.5 <= m < 1)
    r = A / np.ldexp(1.0, e)[None, :]
    S = []
    for a in range(1, nslices + 1):
        s = np.trunc(np.ldexp(r, 7 * a))
        S.append(s)
        r = r - np.ldexp(s, -7 * a)
    return S, e


def ozaki_product(A, B, nslices, full):
    """A^T B with int8 slices of A and B (per-column scales), exact slice products."""
    Sa, ea = int8_slices(A, nslices)
    Sb, eb = int8_slices(B, nslices)
    pairs = [(a, b) for a in range(nslices) for b in range(nslices) if full or a + b <= nslices - 1]
    pairs.sort(key=lambda ab: -(ab[0] + ab[1]))  # smallest contributions first
    out = np.zeros((A.shape[1], B.shape[1]))
    for a, b in pairs:
        P = Sa[a].T @ Sb[b]  # integers below 2^53: exact in float64
        out += np.ldexp(P, -7 * (a + b + 2))
    return out * np.ldexp(1.0, ea)[:, None] * np.ldexp(1.0, eb)[None, :]


def contract(A, B, recipe, chunk_rows):
    """A^T B under a recipe ("fp64", "bf16x3", "bf16x6", "tf32x3", "int8xK", "int8xKt")."""
    if recipe == "fp64":
        return A.T @ B
    if recipe.startswith("int8x"):
        spec = recipe[5:]
        full = not spec.endswith("t")
        return ozaki_product(A, B, int(spec.rstrip("t")), full)
    return split_product(A, B, recipe, chunk_rows)


def gram(op, recipe, points_per_chunk=8):
    """G term by term: G = sum_t (sqrt(w) L_t)^T (sqrt(w) L_t) over (point, component)."""
    L, wm, rterm = op["L"], op["wm"], op["rterm"]
    QG, nT, N = L.shape
    G = np.zeros((N, N))
    for t in np.unique(rterm):
        rows = np.nonzero(rterm == t)[0]
        cols = np.nonzero(np.abs(L[:, rows, :]).sum(axis=(0, 1)) > 0)[0]
        A = (np.sqrt(wm)[:, None, None] * L[:, rows][:, :, cols]).reshape(QG * len(rows), len(cols))
        G[np.ix_(cols, cols)] += contract(A, A, recipe, points_per_chunk * len(rows))
    return G


def stiffness(op, recipe, rows_per_chunk=64):
    U, V = op["U"], op["V"]
    return contract(U, V, recipe, rows_per_chunk)


def assemble(oracle_mod, is_field, op, F, g_recipe, b_recipe, refine=False):
    """K, l, S, s of one cell with G and B from the recipes, F in FP64, the FP64 factored
    Cholesky solve (BF.cpp:924-1018) and condensation of the oracle.  refine=True adds
    one FP64 iterative-refinement step on X = G^-1 [B F] against the same G."""
    G = gram(op, g_recipe)
    B = stiffness(op, b_recipe)
    if not refine:
        K, l, info = oracle_mod.factored_cholesky_solve(G, B, F)
    else:
        import scipy.linalg as sl
        E = np.concatenate([B.T, F[:, None]], axis=1)
        c = sl.cho_factor(G, lower=True)
        X = sl.cho_solve(c, E)
        X = X + sl.cho_solve(c, E - G @ X)
        K = B @ X[:, :-1]
        K = 0.5 * (K + K.T)
        l = B @ X[:, -1]
        info = 0
    S, s, _ = oracle_mod.condense(is_field, K, l)
    return dict(G=G, B=B, K=K, l=l, S=S, s=s, info=info)
