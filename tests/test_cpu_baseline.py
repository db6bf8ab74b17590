"""The CPU baseline (oracle fast mode: a DGEMM per quadrature block as Intrepid's
integrate(COMP_BLAS), the factored Cholesky solve in LAPACK/BLAS) computes what the
checker computes: on cells of the configurations' meshes K, l, S, s agree with the
oracle within the FP64 floor of those meshes, and the one-process-per-core pool that
bench.py times runs and returns its sample."""
import numpy as np
import pytest

from camellia2_b200 import abi, formulation as fm, mesh
from tests.conftest import rel_fro
from tests.helpers import coeffs_for


@pytest.mark.parametrize("make,tol", [
    (lambda: (fm.PoissonFormulation(3).bucket(abi.TOPO_HEX, 2, 1), mesh.hex_grid(12, 12, 12, 0.1, seed=1)), 1e-10),
    (lambda: (fm.PoissonFormulation(2).bucket(abi.TOPO_QUAD, 2, 2), mesh.quad_grid(16, 16, 0.0, seed=1)), 1e-10),
    (lambda: (fm.ConvectionDiffusionReactionFormulation(2).bucket(abi.TOPO_QUAD, 3, 2),
              mesh.quad_grid(8, 8, 0.1, seed=1)), 1e-9),
    (lambda: (fm.StokesVGPFormulation(2).bucket(abi.TOPO_TRI, 3, 2), mesh.tri_grid(2, 2, 0.1, seed=1)), 1e-10),
], ids=["hex_k2", "quad_k2", "cdr_k3", "stokes_tri_p3"])
def test_fast_mode_matches_the_checker(oracle_mod, make, tol):
    bucket, (nodes, par) = make()
    P = oracle_mod.OraclePlan(bucket)
    idx = np.arange(min(24, nodes.shape[0]))
    co = coeffs_for(bucket, P.info, nodes.shape[0])
    co = None if co is None else co[idx]
    ref = P.assemble(nodes[idx], par[idx], co)
    got = P.assemble_blas(nodes[idx], par[idx], co, nthreads=2)
    assert (got["info"] == 0).all()
    for c in range(len(idx)):
        for k in ("K", "l", "S", "s"):
            assert rel_fro(got[k][c], ref[k][c]) < tol, (c, k)


def test_process_pool_runs_its_sample():
    from oracle.cpu_baseline import ProcessBaseline
    nodes, par = mesh.hex_grid(4, 4, 2, 0.1, seed=1)
    b = fm.PoissonFormulation(3).bucket(abi.TOPO_HEX, 2, 1)
    from oracle import oracle
    P = oracle.OraclePlan(b)
    co = mesh.uniform_coeff(nodes.shape[0], 1, P.info["n_points_total"], seed=1)
    with ProcessBaseline(("PoissonFormulation", (3, abi.TOPO_HEX, 2, 1)), nodes, par, co, cores=2) as pool:
        cells, dt = pool.run(3)
    assert cells == 6 and dt > 0
