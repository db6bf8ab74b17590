"""Workload builders shared by the tests (small versions of the bench configs)."""
import numpy as np

from camellia2_b200 import abi, formulation as fm, mesh


def poisson2d(k, dk, nx=3, ny=3, jitter=0.2, seed=1, load="random"):
    form = fm.PoissonFormulation(2)
    bucket = form.bucket(abi.TOPO_QUAD, k, dk)
    nodes, par = mesh.quad_grid(nx, ny, jitter, seed=seed)
    return form, bucket, nodes, par


def poisson3d(k, dk, n=2, jitter=0.1, seed=1):
    form = fm.PoissonFormulation(3)
    bucket = form.bucket(abi.TOPO_HEX, k, dk)
    nodes, par = mesh.hex_grid(n, n, n, jitter, seed=seed)
    return form, bucket, nodes, par


def cdr2d(k, dk, nx=3, ny=3, jitter=0.0, seed=1):
    form = fm.ConvectionDiffusionReactionFormulation(2)
    bucket = form.bucket(abi.TOPO_QUAD, k, dk)
    nodes, par = mesh.quad_grid(nx, ny, jitter, seed=seed)
    return form, bucket, nodes, par


def stokes2d(k, dk, nx=2, ny=2, jitter=0.1, seed=1):
    form = fm.StokesVGPFormulation(2)
    bucket = form.bucket(abi.TOPO_QUAD, k, dk)
    nodes, par = mesh.quad_grid(nx, ny, jitter, seed=seed)
    return form, bucket, nodes, par


def poisson_tri(k, dk, nx=2, ny=2, jitter=0.15, seed=1):
    form = fm.PoissonFormulation(2)
    bucket = form.bucket(abi.TOPO_TRI, k, dk)
    nodes, par = mesh.tri_grid(nx, ny, jitter, seed=seed)
    return form, bucket, nodes, par


def stokes_tri(k, dk, nx=2, ny=1, jitter=0.1, seed=1):
    form = fm.StokesVGPFormulation(2)
    bucket = form.bucket(abi.TOPO_TRI, k, dk)
    nodes, par = mesh.tri_grid(nx, ny, jitter, seed=seed)
    return form, bucket, nodes, par


def coeffs_for(bucket, info, C, seed=2):
    if bucket.n_slots == 0:
        return None
    if bucket.slot_names and bucket.slot_names[0] == "sqrt_eps":
        return mesh.cdr_coeff(C, info, seed=seed)
    return mesh.uniform_coeff(C, bucket.n_slots, info["n_points_total"], seed=seed)


def fp64_floor(oracle_mod, G, B, F, K, trials=4, seed=0):
    """Relative change of K when G is perturbed by random ~1-ulp relative noise."""
    from tests.conftest import rel_fro
    rng = np.random.default_rng(seed)
    worst = 0.0
    for _ in range(trials):
        E = rng.normal(size=G.shape)
        E = (E + E.T) / 2
        Kp, _, _ = oracle_mod.factored_cholesky_solve(G * (1 + 2e-16 * E), B, F)
        worst = max(worst, rel_fro(Kp, K))
    return worst


def check_against_truth(oracle_mod, bucket, nodes, par, co, got, ref, keys=("K", "l", "S", "s"), tol=1e-12,
                        factor=3.0):
    """Per cell, the GPU outputs `got` must match the FP64 oracle's `ref` to `tol`; on the
    cells where they do not (ill-conditioned Gram matrices: there two FP64 codes differ by
    their own rounding), both are compared with the extended-precision truth and the GPU's
    worst error over those cells must be at most `factor` times the oracle's worst.
    Returns the cells that needed the truth."""
    from tests.conftest import rel_fro
    import os
    C = nodes.shape[0]
    miss = [c for c in range(C) if max(rel_fro(got[k][c], ref[k][c]) for k in keys) >= tol]
    if not miss:
        return miss
    m = np.array(miss)
    truth = oracle_mod.OraclePlan(bucket, xp=True).assemble(nodes[m], par[m], None if co is None else co[m],
                                                           nthreads=os.cpu_count() or 1)
    for k in keys:
        e_gpu = max(rel_fro(got[k][c], truth[k][j]) for j, c in enumerate(miss))
        e_orc = max(rel_fro(ref[k][c], truth[k][j]) for j, c in enumerate(miss))
        assert e_gpu <= factor * e_orc + 1e-13, (k, e_gpu, e_orc)
    return miss
