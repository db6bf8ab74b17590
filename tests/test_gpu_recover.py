"""Field back-substitution after the global trace solve (dpg_recover_fields;
CondensedDofInterpreter::interpretGlobalCoefficients, CondensedDofInterpreter.cpp:
1229-1346): u_f = K_ff^-1 (l_f - K_ft t) per cell, with K, l from the GPU assembly.

Checked (1) against a dense solve of the same K, l on random trace values, and
(2) end to end on the consistency case: with the traces of an exact linear
solution (f = 0), the recovered fields are that solution's field interpolant."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import lib as dlib  # noqa: E402
from tests.conftest import rel_fro  # noqa: E402
from tests.helpers import coeffs_for, poisson2d, poisson3d  # noqa: E402

pytestmark = pytest.mark.gpu


def _dev(x):
    return torch.as_tensor(np.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("make", [lambda: poisson3d(2, 1, 2, 0.1), lambda: poisson2d(4, 2, 2, 2, 0.2),
                                  lambda: poisson2d(2, 2, 80, 80, 0.2)])
def test_recovered_fields_match_dense_solve(make):
    form, bucket, nodes, par = make()
    plan = dlib.Plan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, plan.info, C)
    out = plan.assemble(_dev(nodes), _dev(par), _dev(co))
    nf, nt = plan.info["n_field"], plan.info["n_trace"]
    t = np.random.default_rng(3).normal(size=(C, nt))
    u, info = plan.recover_fields(out["K"], out["l"], _dev(t))
    torch.cuda.synchronize()
    assert int(info.abs().max()) == 0
    K, l, u = out["K"].cpu().numpy(), out["l"].cpu().numpy(), u.cpu().numpy()
    for c in range(C):
        ref = np.linalg.solve(K[c][:nf, :nf], l[c][:nf] - K[c][:nf, nf:] @ t[c])
        assert rel_fro(u[c][:nf], ref) < 1e-10
        assert np.array_equal(u[c][nf:], t[c])


def test_recovered_fields_reproduce_exact_linear_solution(oracle_mod):
    from tests.test_formulation import _poisson_trial_interpolant
    form, bucket, nodes, par = poisson2d(2, 2, 3, 3, 0.2)
    plan = dlib.Plan(bucket)
    C = nodes.shape[0]
    co = np.zeros((C, 1, plan.info["n_points_total"]))  # f = 0 = -Laplace(u)
    out = plan.assemble(_dev(nodes), _dev(par), _dev(co))
    a = np.array([0.7, 1.4])
    u_ex = lambda X: X @ a + 0.3  # noqa: E731
    gu = lambda X: np.tile(a, (X.shape[0], 1))  # noqa: E731
    P = oracle_mod.OraclePlan(bucket)
    x = np.stack([_poisson_trial_interpolant(P, nodes[c], par[c], u_ex, gu, 2, 2) for c in range(C)])
    nf = plan.info["n_field"]
    u, info = plan.recover_fields(out["K"], out["l"], _dev(x[:, nf:]))
    torch.cuda.synchronize()
    assert int(info.abs().max()) == 0
    u = u.cpu().numpy()
    for c in range(C):
        assert rel_fro(u[c][:nf], x[c][:nf]) < 1e-10, c
