"""DLS local matrices (dpg_assemble_dls; TBF::localStiffnessMatrixAndRHS_DLS,
BF.cpp:1169-1306): W = L^-1 B and y = L^-1 F with G = L L^T, against the oracle's
G, B, F and a dense Cholesky; and W^T W, W^T y reproduce dpg_assemble's K, l."""
import numpy as np
import pytest
import scipy.linalg as sla

torch = pytest.importorskip("torch")

from camellia2_b200 import lib as dlib  # noqa: E402
from tests.conftest import rel_fro  # noqa: E402
from tests.helpers import cdr2d, coeffs_for, poisson2d, poisson3d, stokes2d, stokes_tri  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [lambda: poisson3d(2, 1, 2, 0.1), lambda: poisson2d(2, 2, 2, 2, 0.2),
                                  lambda: cdr2d(3, 2, 2, 2, 0.1)])
def test_dls_matches_dense_factorisation(make, oracle_mod):
    form, bucket, nodes, par = make()
    plan = dlib.Plan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, plan.info, C)
    dev = [None if x is None else torch.as_tensor(x).cuda() for x in (nodes, par, co)]
    W, y, info = plan.dls(*dev)
    out = plan.assemble(*dev)
    torch.cuda.synchronize()
    assert int(info.abs().max()) == 0
    W, y = W.cpu().numpy(), y.cpu().numpy()
    K, l = out["K"].cpu().numpy(), out["l"].cpu().numpy()
    G, B, F = oracle_mod.OraclePlan(bucket).parts(nodes, par, co)
    for c in range(C):
        Lc = np.linalg.cholesky(G[c])
        assert rel_fro(W[c].T, sla.solve_triangular(Lc, B[c].T, lower=True)) < 1e-10
        assert rel_fro(y[c], sla.solve_triangular(Lc, F[c], lower=True)) < 1e-10
        assert rel_fro(W[c] @ W[c].T, K[c]) < 1e-12
        assert rel_fro(W[c] @ y[c], l[c]) < 1e-12


@pytest.mark.parametrize("make", [lambda: stokes2d(3, 2, 2, 2, 0.1), lambda: stokes_tri(4, 2, 1, 1, 0.1),
                                  lambda: stokes2d(6, 2, 1, 1, 0.1)],
                         ids=["stokes_quad_k3", "stokes_tri_k4", "stokes_quad_k6"])
def test_dls_large_buckets(make, oracle_mod):
    """Large-bucket plans (N > 192 or M > 120 after padding): the rows below the factored test
    block of Z are W^T = (L^-1 E)^T, read out as W and y.  Against the oracle's G, B, F and a dense
    Cholesky, and W W^T, W y against dpg_assemble's K, l.  These Gram matrices are much worse
    conditioned than the single-CTA buckets' (their FP64 K differ from the truth by up to 3e-9),
    so W is compared to 1e-8 and the products to 1e-10."""
    form, bucket, nodes, par = make()
    plan = dlib.Plan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, plan.info, C)
    dev = [None if x is None else torch.as_tensor(x).cuda() for x in (nodes, par, co)]
    W, y, info = plan.dls(*dev)
    out = plan.assemble(*dev)
    torch.cuda.synchronize()
    assert int(info.abs().max()) == 0
    W, y = W.cpu().numpy(), y.cpu().numpy()
    K, l = out["K"].cpu().numpy(), out["l"].cpu().numpy()
    G, B, F = oracle_mod.OraclePlan(bucket).parts(nodes, par, co)
    for c in range(C):
        Lc = np.linalg.cholesky(G[c])
        assert rel_fro(W[c].T, sla.solve_triangular(Lc, B[c].T, lower=True)) < 1e-8
        assert rel_fro(y[c], sla.solve_triangular(Lc, F[c], lower=True)) < 1e-8
        assert rel_fro(W[c] @ W[c].T, K[c]) < 1e-10
        assert rel_fro(W[c] @ y[c], l[c]) < 1e-10
