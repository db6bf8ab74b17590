"""Reverse mode (dpg_assemble_adjoint, no counterpart in the reference).

For J = sum_c (r_c^T K_c r_c + g_c^T l_c) with r, g ~ N(0, 1), Kbar = r r^T and
lbar = g; the coefficient gradient dJ/dcoeff (C, n_slots, n_points_total) is checked
against central finite differences of J, computed
  * with the oracle's FP64 forward (CPU restatement of BF.cpp:1385-1449) on a small
    mesh, along random unit directions in the full coefficient space and along
    single coordinates;
  * with this library's own forward on the CDR workload's shapes (128 x 128 quads
    in the bench; 16 x 16 here) along random directions.
The FD step h balances truncation (h^2) against the forward's roundoff (eps_J / h);
the test bound is 1e-6 relative plus that roundoff term.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import abi, formulation as fm, lib as dlib, mesh  # noqa: E402
from tests.helpers import coeffs_for  # noqa: E402

pytestmark = pytest.mark.gpu


def _loss(K, l, r, g):
    return float(np.einsum("ci,cij,cj->", r, K, r) + np.einsum("ci,ci->", g, l))


def _setup(which, nx, ny, seed=3):
    if which == "cdr":
        form = fm.ConvectionDiffusionReactionFormulation(2)
        bucket = form.bucket(abi.TOPO_QUAD, 3, 2)
    elif which == "poisson3d":  # the hex bucket of the bench (load f per point)
        form = fm.PoissonFormulation(3)
        bucket = form.bucket(abi.TOPO_HEX, 2, 1)
    else:
        form = fm.PoissonFormulation(2)
        bucket = form.bucket(abi.TOPO_QUAD, 2, 2)
    if which == "poisson3d":
        nodes, par = mesh.hex_grid(nx, ny, 1, 0.1, seed=seed)
    else:
        nodes, par = mesh.quad_grid(nx, ny, 0.15, seed=seed)
    plan = dlib.Plan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, plan.info, C, seed=seed)
    M = plan.info["M"]
    rng = np.random.default_rng(seed + 10)
    r = rng.normal(size=(C, M))
    g = rng.normal(size=(C, M))
    return bucket, plan, nodes, par, co, r, g


def _gpu_grad(plan, nodes, par, co, r, g):
    dev = lambda x: torch.as_tensor(x).cuda()  # noqa: E731
    Kbar = r[:, :, None] * r[:, None, :]
    cbar, info = plan.adjoint(dev(nodes), dev(par), dev(co), dev(Kbar), dev(g))
    torch.cuda.synchronize()
    assert int(info.abs().max()) == 0
    return cbar.cpu().numpy()


@pytest.mark.parametrize("which", ["cdr", "poisson", "poisson3d"])
def test_adjoint_matches_oracle_central_differences(which, oracle_mod):
    bucket, plan, nodes, par, co, r, g = _setup(which, 2, 1)
    orc = oracle_mod.OraclePlan(bucket)
    grad = _gpu_grad(plan, nodes, par, co, r, g)

    def J(c):
        o = orc.assemble(nodes, par, c)
        return _loss(o["K"], o["l"], r, g)

    J0 = J(co)
    h = 1e-5
    noise = 1e-12 * abs(J0) / h  # roundoff of J over the step
    rng = np.random.default_rng(7)
    worst = 0.0
    for _ in range(16):
        d = rng.normal(size=co.shape)
        d /= np.linalg.norm(d)
        fd = (J(co + h * d) - J(co - h * d)) / (2 * h)
        ad = float((grad * d).sum())
        worst = max(worst, abs(ad - fd) / (1e-6 * abs(fd) + noise))
        assert abs(ad - fd) <= 1e-6 * abs(fd) + noise, (ad, fd)
    flat = np.flatnonzero(np.abs(grad).reshape(-1) > 0)
    picks = rng.choice(flat, size=min(64, flat.size), replace=False)
    for idx in picks:
        d = np.zeros(co.size)
        d[idx] = 1.0
        d = d.reshape(co.shape)
        fd = (J(co + h * d) - J(co - h * d)) / (2 * h)
        ad = float(grad.reshape(-1)[idx])
        assert abs(ad - fd) <= 1e-6 * abs(fd) + noise, (idx, ad, fd)


def test_adjoint_matches_own_forward_directional():
    bucket, plan, nodes, par, co, r, g = _setup("cdr", 16, 16, seed=5)
    grad = _gpu_grad(plan, nodes, par, co, r, g)
    dn, dp = torch.as_tensor(nodes).cuda(), torch.as_tensor(par).cuda()

    def J(c):
        o = plan.assemble(dn, dp, torch.as_tensor(c).cuda())
        return _loss(o["K"].cpu().numpy(), o["l"].cpu().numpy(), r, g)

    J0 = J(co)
    h = 1e-5
    noise = 1e-12 * abs(J0) / h
    rng = np.random.default_rng(11)
    for _ in range(16):
        d = rng.normal(size=co.shape)
        d /= np.linalg.norm(d)
        fd = (J(co + h * d) - J(co - h * d)) / (2 * h)
        ad = float((grad * d).sum())
        assert abs(ad - fd) <= 1e-6 * abs(fd) + noise, (ad, fd)


def test_adjoint_zero_cells_and_unsupported_inputs():
    bucket, plan, nodes, par, co, r, g = _setup("cdr", 1, 1)
    e = torch.empty((0,), dtype=torch.float64, device="cuda")
    cbar, info = plan.adjoint(torch.empty((0, 4, 2), dtype=torch.float64, device="cuda"),
                              torch.empty((0, 4), dtype=torch.int8, device="cuda"), e, e, e)
    assert cbar.shape[0] == 0
