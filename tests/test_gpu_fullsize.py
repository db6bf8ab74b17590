"""The configurations at their full sizes (48^3 hexes, 256^2 and 128^2 quads), checked
through properties that do not depend on the mesh size, plus the oracle on a seeded
sample of cells spread over the whole mesh:

  - every cell's Gram matrix factors (info == 0);
  - K and S are symmetric to roundoff, per cell, over all cells;
  - cells are independent: a sub-range assembled on its own equals, bit for bit, the
    same cells of the full launch (no cross-cell state in the persistent kernel);
  - on the sampled cells the quadrature products G, B, F match the oracle to 1e-13
    (their accuracy does not depend on h), and K, l, S, s to 1e-12 or, where the
    cell's Gram conditioning puts two FP64 codes further apart (h = 1/48: cond(G) ~ 1e14),
    the GPU's error against the extended-precision truth is at most three times the FP64
    oracle's own.

The symmetry reductions run on the device in slices of cells, so no output leaves the
GPU except the sampled cells."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import abi, formulation as fm, lib as dlib, mesh  # noqa: E402
from tests.conftest import rel_fro  # noqa: E402
from tests.helpers import check_against_truth  # noqa: E402

pytestmark = pytest.mark.gpu


def _c5():
    bucket = fm.PoissonFormulation(3).bucket(abi.TOPO_HEX, 2, 1)
    nodes, par = mesh.hex_grid(48, 48, 48, 0.1, seed=1)
    return bucket, nodes, par, lambda P, C: mesh.uniform_coeff(C, 1, P, seed=1)


def _c2():
    bucket = fm.PoissonFormulation(2).bucket(abi.TOPO_QUAD, 4, 2)
    nodes, par = mesh.quad_grid(256, 256, 0.2, seed=1)
    return bucket, nodes, par, lambda P, C: mesh.uniform_coeff(C, 1, P, seed=1)


def _c4():
    bucket = fm.ConvectionDiffusionReactionFormulation(2).bucket(abi.TOPO_QUAD, 3, 2)
    nodes, par = mesh.quad_grid(128, 128, 0.1, seed=1)
    return bucket, nodes, par, None


def _max_asym(X, step=8192):
    worst = 0.0
    for c0 in range(0, X.shape[0], step):
        x = X[c0:c0 + step]
        d = (x - x.transpose(1, 2)).abs().amax(dim=(1, 2)) / x.abs().amax(dim=(1, 2)).clamp_min(1e-300)
        worst = max(worst, float(d.max()))
    return worst


@pytest.mark.parametrize("make", [_c5, _c2, _c4], ids=["c5_hex48", "c2_quad256", "c4_cdr128"])
def test_full_size_properties(make, oracle_mod):
    bucket, nodes, par, mkco = make()
    plan = dlib.Plan(bucket)
    C = nodes.shape[0]
    P = plan.info["n_points_total"]
    if mkco is not None:
        co = mkco(P, C)
    else:
        co = mesh.cdr_coeff(C, plan.info, seed=1)
    dn, dp, dc = (torch.as_tensor(np.ascontiguousarray(x)).cuda() for x in (nodes, par, co))
    out = plan.assemble(dn, dp, dc)
    torch.cuda.synchronize()
    assert int((out["info"] != 0).sum()) == 0
    assert _max_asym(out["K"]) < 1e-12
    assert _max_asym(out["S"]) < 1e-12
    # cells are independent: a sub-range on its own gives the same bits
    a, b = C // 3, C // 3 + 1000
    sub = plan.assemble(dn[a:b], dp[a:b], dc[a:b])
    torch.cuda.synchronize()
    for k in ("K", "l", "S", "s", "info"):
        assert torch.equal(sub[k], out[k][a:b]), k
    # oracle on a seeded sample: first and last cells plus 30 spread over the mesh
    rng = np.random.default_rng(11)
    pick = np.unique(np.concatenate([[0, C - 1], rng.choice(C, size=30, replace=False)]))
    O = oracle_mod.OraclePlan(bucket)
    ref = O.assemble(nodes[pick], par[pick], co[pick], parts=True)
    ip = torch.as_tensor(pick).cuda()
    got = {k: out[k][ip].cpu().numpy() for k in ("K", "l", "S", "s")}
    G, B, F = (x.cpu().numpy() for x in plan.parts(dn[ip], dp[ip], dc[ip]))
    for j in range(len(pick)):
        assert rel_fro(G[j], ref["G"][j]) < 1e-13
        assert rel_fro(B[j], ref["B"][j]) < 1e-13
        assert rel_fro(F[j], ref["F"][j]) < 1e-13
    check_against_truth(oracle_mod, bucket, nodes[pick], par[pick], None if co is None else co[pick], got, ref)
