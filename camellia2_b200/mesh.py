"""Synthetic meshes, side parities and per-point coefficients for the DPG
assembly workloads (seeded numpy PCG64 streams).

Vertex order per cell follows the shards topologies the reference uses
(quad: counter-clockwise from (-1,-1); hex: bottom face counter-clockwise,
then top face).  Side parities follow GlobalDofAssignment.cpp:158-258: a side
shared by two cells is +1 on the cell with the lower cell ID and -1 on the
other; boundary sides are +1.  Cell IDs are lexicographic, x fastest.
"""
from __future__ import annotations

import numpy as np


def quad_grid(nx, ny, jitter=0.0, seed=1, extent=(1.0, 1.0)):
    """nx*ny quads on [0,Lx]x[0,Ly]; interior nodes jittered by U[-jitter*h, jitter*h]
    per coordinate. Returns nodes (C,4,2) float64 and parity (C,4) int8."""
    rng = np.random.default_rng(seed)
    hx, hy = extent[0] / nx, extent[1] / ny
    X, Y = np.meshgrid(np.arange(nx + 1) * hx, np.arange(ny + 1) * hy, indexing="ij")
    if jitter:
        jx = rng.uniform(-jitter * hx, jitter * hx, size=X.shape)
        jy = rng.uniform(-jitter * hy, jitter * hy, size=Y.shape)
        interior = np.zeros_like(X, dtype=bool)
        interior[1:-1, 1:-1] = True
        X = X + np.where(interior, jx, 0.0)
        Y = Y + np.where(interior, jy, 0.0)
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")  # cell id = i + nx*j
    i = i.reshape(-1)
    j = j.reshape(-1)
    corners = [(i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1)]
    nodes = np.stack([np.stack([X[a, b], Y[a, b]], axis=-1) for a, b in corners], axis=1)
    par = np.ones((nx * ny, 4), dtype=np.int8)
    par[:, 0] = np.where(j > 0, -1, 1)       # bottom neighbour has the lower id
    par[:, 3] = np.where(i > 0, -1, 1)       # left neighbour has the lower id
    return np.ascontiguousarray(nodes), par


def tri_grid(nx, ny, jitter=0.0, seed=1, extent=(1.0, 1.0)):
    """nx*ny quads on [0,Lx]x[0,Ly], each cut along its diagonal into two
    counter-clockwise triangles (v00, v10, v11) and (v00, v11, v01); interior nodes
    jittered by U[-jitter*h, jitter*h].  Side s of a triangle joins its vertices s
    and s+1 (shards Triangle<3>).  Side parity: +1 on the boundary and for the
    lower cell id of a neighbour pair, -1 for the higher.  Returns nodes (C,3,2),
    parity (C,3)."""
    rng = np.random.default_rng(seed)
    hx, hy = extent[0] / nx, extent[1] / ny
    X, Y = np.meshgrid(np.arange(nx + 1) * hx, np.arange(ny + 1) * hy, indexing="ij")
    if jitter:
        jx = rng.uniform(-jitter * hx, jitter * hx, size=X.shape)
        jy = rng.uniform(-jitter * hy, jitter * hy, size=Y.shape)
        interior = np.zeros_like(X, dtype=bool)
        interior[1:-1, 1:-1] = True
        X = X + np.where(interior, jx, 0.0)
        Y = Y + np.where(interior, jy, 0.0)
    vid = lambda i, j: i * (ny + 1) + j  # noqa: E731
    cells = []
    for j in range(ny):
        for i in range(nx):
            v00, v10, v11, v01 = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
            cells.append((v00, v10, v11))
            cells.append((v00, v11, v01))
    cells = np.array(cells)
    P = np.stack([X.reshape(-1), Y.reshape(-1)], axis=-1)
    nodes = P[cells]
    owner = {}
    par = np.ones((len(cells), 3), dtype=np.int8)
    for c, tri in enumerate(cells):
        for s in range(3):
            key = tuple(sorted((tri[s], tri[(s + 1) % 3])))
            if key in owner:
                par[c, s] = -1  # the other cell has the lower id
            else:
                owner[key] = c
    return np.ascontiguousarray(nodes), par


def hex_grid(nx, ny, nz, jitter=0.0, seed=1, extent=(1.0, 1.0, 1.0)):
    """nx*ny*nz hexes; interior nodes jittered by U[-jitter*h, jitter*h].
    Returns nodes (C,8,3) float64 and parity (C,6) int8."""
    rng = np.random.default_rng(seed)
    h = [extent[0] / nx, extent[1] / ny, extent[2] / nz]
    G = np.stack(np.meshgrid(np.arange(nx + 1) * h[0], np.arange(ny + 1) * h[1], np.arange(nz + 1) * h[2],
                             indexing="ij"), axis=-1)
    if jitter:
        jit = np.stack([rng.uniform(-jitter * h[k], jitter * h[k], size=G.shape[:3]) for k in range(3)], axis=-1)
        interior = np.zeros(G.shape[:3], dtype=bool)
        interior[1:-1, 1:-1, 1:-1] = True
        G = G + np.where(interior[..., None], jit, 0.0)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.reshape(-1), j.reshape(-1), k.reshape(-1)  # cell id = i + nx*(j + ny*k)
    off = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    nodes = np.stack([G[i + a, j + b, k + c] for a, b, c in off], axis=1)
    par = np.ones((nx * ny * nz, 6), dtype=np.int8)
    par[:, 0] = np.where(j > 0, -1, 1)  # face y-
    par[:, 3] = np.where(i > 0, -1, 1)  # face x-
    par[:, 4] = np.where(k > 0, -1, 1)  # face z-
    return np.ascontiguousarray(nodes), par


def hex_trace_map(nx, ny, nz, k=2):
    """Conforming-shaped local-to-global map of the hex Poisson UW traces on hex_grid's
    cells: the H1 trace (k+1)^2 points per face and the L2 flux trace k^2 dofs per face,
    numbered face by face (faces x-, x+, y-, y+, z-, z+; points i + (k+1) j on the face's two
    tangent axes in increasing order).  Points are identified by their lattice position, so
    a trace point on a shared vertex, edge or face gets one global id for all the cells
    and faces touching it, as the GDA map of a conforming mesh does.  Returns gid (C, t)
    int64 with dense ids and the number of global dofs."""
    P = k * max(nx, ny, nz) + 1
    dims = (nx, ny, nz)
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    idx = np.stack([ii.reshape(-1), jj.reshape(-1), kk.reshape(-1)], axis=1)  # (C, 3), cell id = i + nx (j + ny k)
    C = idx.shape[0]
    nh, nq = (k + 1) ** 2, k * k
    h1 = np.empty((C, 6, nh), np.int64)
    fl = np.empty((C, 6, nq), np.int64)
    a_i, b_i = np.meshgrid(np.arange(k + 1), np.arange(k + 1), indexing="xy")  # point i + (k+1) j
    a_i, b_i = a_i.reshape(-1), b_i.reshape(-1)
    nfaces = [(dims[a] + 1) * dims[(a + 1) % 3] * dims[(a + 2) % 3] for a in range(3)]
    face_base = np.cumsum([0] + nfaces)
    for f in range(6):
        a, side = f // 2, f % 2
        b, c = [x for x in range(3) if x != a]
        pos = np.empty((C, nh, 3), np.int64)
        pos[:, :, a] = (k * (idx[:, a] + side))[:, None]
        pos[:, :, b] = k * idx[:, b][:, None] + a_i[None, :]
        pos[:, :, c] = k * idx[:, c][:, None] + b_i[None, :]
        h1[:, f] = pos[:, :, 0] + P * (pos[:, :, 1] + P * pos[:, :, 2])
        fid = face_base[a] + ((idx[:, a] + side) * dims[b] + idx[:, b]) * dims[c] + idx[:, c]
        fl[:, f] = P ** 3 + fid[:, None] * nq + np.arange(nq)[None, :]
    raw = np.concatenate([h1.reshape(C, -1), fl.reshape(C, -1)], axis=1)
    uniq, inv = np.unique(raw, return_inverse=True)
    return inv.reshape(C, -1).astype(np.int64), int(uniq.shape[0])


def uniform_coeff(C, n_slots, n_points, low=-1.0, high=1.0, seed=1):
    rng = np.random.default_rng(seed)
    return rng.uniform(low, high, size=(C, n_slots, n_points))


def cdr_coeff(C, info, seed=1):
    """Coefficients of the CDR workload: eps = exp(N(-4,1)) per point (slot 0 holds
    sqrt(eps)), beta = (cos t, sin t) with t ~ U[0,2pi) per cell, alpha = c ~ U[0,1],
    f ~ U[-1,1] per point."""
    rng = np.random.default_rng(seed)
    P = info["n_points_total"]
    co = np.empty((C, 5, P))
    eps = np.exp(rng.normal(-4.0, 1.0, size=(C, P)))
    theta = rng.uniform(0.0, 2 * np.pi, size=(C, 1))
    co[:, 0] = np.sqrt(eps)
    co[:, 1] = np.cos(theta)
    co[:, 2] = np.sin(theta)
    co[:, 3] = rng.uniform(0.0, 1.0, size=(C, P))
    co[:, 4] = rng.uniform(-1.0, 1.0, size=(C, P))
    return co


def forest_buckets(total=100_000, quad_frac=0.7, p_max=6, max_level=4, base_n=16, jitter=0.1, seed=1):
    """Cells of the uneven-cell Stokes workload as a synthetic refined forest.

    Each cell is a quad with probability quad_frac, else a triangle; its degree p is uniform
    on 1..p_max and its refinement level L is drawn from a geometric law (P(L) ~ 2^-L)
    truncated to 0..max_level.  A level-L cell of a base_n x base_n coarse grid of the unit
    square has size h = 1 / (base_n 2^L); it sits at a random position of the grid of its level
    and its vertices are jittered by U[-jitter h, jitter h].  The per-cell outputs depend on a
    neighbour only through the side parity, so cells are generated independently with random
    parities +-1 on their sides (hanging nodes change the global map, not the local matrices).

    Returns {(topology, p): (nodes (C, nv, 2), parity (C, nv) int8)} with topology 1 = quad,
    3 = triangle, and the cell counts in a deterministic order."""
    rng = np.random.default_rng(seed)
    is_quad = rng.uniform(size=total) < quad_frac
    p = rng.integers(1, p_max + 1, size=total)
    w = 0.5 ** np.arange(max_level + 1)
    level = rng.choice(max_level + 1, size=total, p=w / w.sum())
    out = {}
    for topo, nv, ref in ((1, 4, np.array([[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0]])),
                          (3, 3, np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]))):
        for pp in range(1, p_max + 1):
            sel = np.nonzero((is_quad == (topo == 1)) & (p == pp))[0]
            C = len(sel)
            if C == 0:
                continue
            n = base_n * 2 ** level[sel]
            h = 1.0 / n
            i = rng.integers(0, n)
            j = rng.integers(0, n)
            origin = np.stack([i * h, j * h], axis=-1)
            nodes = origin[:, None, :] + h[:, None, None] * ref[None, :, :]
            nodes = nodes + rng.uniform(-jitter, jitter, size=nodes.shape) * h[:, None, None]
            par = np.where(rng.uniform(size=(C, nv)) < 0.5, -1, 1).astype(np.int8)
            out[(topo, pp)] = (np.ascontiguousarray(nodes), par)
    return out
