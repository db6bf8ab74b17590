"""dpg_plan_autotune: the per-bucket choice of the Gram staging chunk (8 or 4 quadrature points,
which sets the shared-memory layout and the kernel instance) or, for large buckets, of the
formation k-chunk (32 or 16 points), timed on the caller's cells.  After
tuning, the plan's results still match the oracle at the parity bar (relative Frobenius error
<= 1e-12 per cell, or, where the Gram conditioning puts two FP64 codes further apart, an error
against the extended-precision truth at most three times the FP64 oracle's own)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import lib as dlib  # noqa: E402
from tests.conftest import rel_fro  # noqa: E402
from tests.helpers import check_against_truth, coeffs_for, poisson2d, poisson3d, stokes2d, stokes_tri  # noqa: E402

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("make", [lambda: poisson3d(2, 1, 3, 0.1), lambda: poisson2d(2, 2, 4, 4, 0.2),
                                  lambda: stokes_tri(3, 2, 3, 2, 0.1)])
def test_autotuned_plan_matches_oracle(make, oracle_mod):
    form, bucket, nodes, par = make()
    P = oracle_mod.OraclePlan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, P.info, C)
    ref = P.assemble(nodes, par, co, parts=True)
    plan = dlib.Plan(bucket)
    dn, dp, dc = _dev(nodes), _dev(par), None if co is None else _dev(co)
    chosen = plan.autotune(dn, dp, dc)
    assert chosen in (4, 8)
    out = plan.assemble(dn, dp, dc)
    torch.cuda.synchronize()
    o = {k: v.cpu().numpy() for k, v in out.items()}
    assert (o["info"] == 0).all()
    check_against_truth(oracle_mod, bucket, nodes, par, co, o, ref)


def test_autotune_large_bucket_picks_a_formation_chunk(oracle_mod):
    """Large-bucket plans tune the formation k-chunk (32 or 16 points); afterwards the results
    still match the oracle at the parity bar."""
    form, bucket, nodes, par = stokes2d(3, 2, 2, 1, 0.1)
    plan = dlib.Plan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, plan.info, C)
    dn, dp, dc = _dev(nodes), _dev(par), _dev(co)
    assert plan.autotune(dn, dp, dc) in (16, 32)
    out = plan.assemble(dn, dp, dc)
    torch.cuda.synchronize()
    o = {k: v.cpu().numpy() for k, v in out.items()}
    assert (o["info"] == 0).all()
    ref = oracle_mod.OraclePlan(bucket).assemble(nodes, par, co)
    check_against_truth(oracle_mod, bucket, nodes, par, co, o, ref)
