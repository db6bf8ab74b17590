"""dpg_plan_autotune: the per-bucket choice of the Gram staging chunk (8 or 4 quadrature points,
which sets the shared-memory layout and the kernel instance) timed on the caller's cells.  After
tuning, the plan's results still match the oracle at the parity bar (relative Frobenius error
<= 1e-12 per cell, or 5x the cell's FP64 floor where that floor exceeds 2e-13); large-bucket plans
have a single configuration and report 0."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import lib as dlib  # noqa: E402
from tests.conftest import rel_fro  # noqa: E402
from tests.helpers import coeffs_for, poisson2d, poisson3d, stokes2d, stokes_tri  # noqa: E402
from tests.test_gpu_parity import fp64_floor  # noqa: E402

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
    for c in range(C):
        tol = 1e-12
        errs = {k: rel_fro(o[k][c], ref[k][c]) for k in ("K", "l", "S", "s")}
        if max(errs.values()) >= tol:
            floor = fp64_floor(oracle_mod, ref["G"][c], ref["B"][c], ref["F"][c], ref["K"][c])
            if floor > 2e-13:
                tol = 5 * floor
        for k, e in errs.items():
            assert e < tol, (c, k, e, tol)


def test_autotune_large_bucket_has_one_configuration():
    form, bucket, nodes, par = stokes2d(3, 2, 1, 1, 0.1)
    plan = dlib.Plan(bucket)
    co = coeffs_for(bucket, plan.info, nodes.shape[0])
    assert plan.autotune(_dev(nodes), _dev(par), _dev(co)) == 0
