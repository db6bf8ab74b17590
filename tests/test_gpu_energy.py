"""Per-cell energy error (dpg_energy_error; TSolution::rankLocalEnergyError with
computeErrorRepresentation, Solution.cpp:2653-2722): sqrt(r^T G^-1 r), r = F - B x.

Checked against the oracle's G, B, F with a dense solve on random trial coefficients,
and on the consistency case: the interpolant of an exact linear solution (f = 0) has
zero residual, so its energy error vanishes to roundoff."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import lib as dlib  # noqa: E402
from tests.helpers import cdr2d, coeffs_for, poisson2d, poisson3d, stokes2d  # noqa: E402

pytestmark = pytest.mark.gpu


def _dev(x):
    return torch.as_tensor(np.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("make", [lambda: poisson3d(2, 1, 2, 0.1), lambda: poisson2d(4, 2, 2, 2, 0.2),
                                  lambda: cdr2d(3, 2, 2, 2, 0.1)])
def test_energy_error_matches_oracle(make, oracle_mod):
    form, bucket, nodes, par = make()
    plan = dlib.Plan(bucket)
    C, M = nodes.shape[0], plan.info["M"]
    co = coeffs_for(bucket, plan.info, C)
    x = np.random.default_rng(4).normal(size=(C, M))
    e, info = plan.energy_error(_dev(nodes), _dev(par), None if co is None else _dev(co), _dev(x))
    torch.cuda.synchronize()
    assert int(info.abs().max()) == 0
    e = e.cpu().numpy()
    G, B, F = oracle_mod.OraclePlan(bucket).parts(nodes, par, co)
    for c in range(C):
        r = F[c] - B[c].T @ x[c]
        ref = np.sqrt(r @ np.linalg.solve(G[c], r))
        assert abs(e[c] - ref) <= 1e-10 * ref, (c, e[c], ref)


def test_energy_error_of_exact_solution_vanishes(oracle_mod):
    from tests.test_formulation import _poisson_trial_interpolant
    form, bucket, nodes, par = poisson2d(2, 2, 3, 3, 0.2)
    plan = dlib.Plan(bucket)
    C = nodes.shape[0]
    co = np.zeros((C, 1, plan.info["n_points_total"]))
    a = np.array([0.7, 1.4])
    P = oracle_mod.OraclePlan(bucket)
    x = np.stack([_poisson_trial_interpolant(P, nodes[c], par[c], lambda X: X @ a + 0.3,
                                             lambda X: np.tile(a, (X.shape[0], 1)), 2, 2) for c in range(C)])
    e, info = plan.energy_error(_dev(nodes), _dev(par), _dev(co), _dev(x))
    torch.cuda.synchronize()
    xr = np.random.default_rng(1).normal(size=x.shape)
    e_rand, _ = plan.energy_error(_dev(nodes), _dev(par), _dev(co), _dev(xr))
    torch.cuda.synchronize()
    assert float(e.max()) < 1e-10 * float(e_rand.min())


@pytest.mark.parametrize("make", [lambda: poisson2d(2, 2, 2, 2, 0.1), lambda: stokes2d(3, 2, 2, 1, 0.1)],
                         ids=["single_cta", "large_bucket"])
def test_energy_error_is_nan_where_the_factorisation_fails(make):
    """Cells mirrored in x have det J < 0, so their Gram matrix is negative definite and its
    factorisation fails (info != 0): the energy error there is NaN, the other cells' are
    unchanged."""
    form, bucket, nodes, par = make()
    plan = dlib.Plan(bucket)
    C, M = nodes.shape[0], plan.info["M"]
    co = coeffs_for(bucket, plan.info, C)
    x = np.random.default_rng(4).normal(size=(C, M))
    bad = nodes.copy()
    bad[1, :, 0] = -bad[1, :, 0]  # cell 1 mirrored: negative Jacobian determinant
    dco = None if co is None else _dev(co)
    e0, info0 = plan.energy_error(_dev(nodes), _dev(par), dco, _dev(x))
    e1, info1 = plan.energy_error(_dev(bad), _dev(par), dco, _dev(x))
    torch.cuda.synchronize()
    e0, e1, info0, info1 = (t.cpu().numpy() for t in (e0, e1, info0, info1))
    assert (info0 == 0).all() and np.isfinite(e0).all()
    assert info1[1] != 0 and np.isnan(e1[1])
    keep = np.arange(C) != 1
    assert (info1[keep] == 0).all() and np.array_equal(e1[keep], e0[keep])
