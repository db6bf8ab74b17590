"""The CPU oracle against the reference's own golden vectors and known answers.

unit_tests/BFTests.cpp and drivers/DPGTests/DPGTests.cpp of the reference hold
the only hand-computed values at this boundary; these tests restate them."""
import numpy as np
import pytest

from camellia2_b200 import abi
from tests.conftest import rel_fro


def test_factored_cholesky_identities(oracle_mod):
    # BFTests.cpp:28-72: identity G (5x5), rectangular identity B (4x5), F = 1
    G = np.eye(5)
    B = np.zeros((4, 5))
    B[np.arange(4), np.arange(4)] = 1.0
    F = np.ones(5)
    K, l, info = oracle_mod.factored_cholesky_solve(G, B, F)
    assert info == 0
    assert np.allclose(K, np.eye(4), atol=1e-14)
    assert np.allclose(l, 1.0, atol=1e-14)


@pytest.mark.parametrize("G,Bt,F,Kx,lx", [
    # BFTests.cpp:136-219 (column-major inputs transcribed to (trial, test) rows)
    ([[1, .5, 0], [.5, 1, 2], [0, 2, 8]], [[3, 1, 2], [2, 0, 2]], [1, 2, 3],
     [[13.5, 12.5], [12.5, 13.5]], [0.75, -1.75]),
    # BFTests.cpp:221-300
    ([[1, .5], [.5, 1]], [[3, 1], [2, 0]], [1, 2], [[28 / 3, 20 / 3], [20 / 3, 16 / 3]], [2, 0]),
    # BFTests.cpp:302-381
    ([[2, 0], [0, 4]], [[3, 1], [2, 0]], [1, 2], [[4.75, 3], [3, 2]], [2, 1]),
])
def test_factored_cholesky_golden(oracle_mod, G, Bt, F, Kx, lx):
    K, l, info = oracle_mod.factored_cholesky_solve(np.array(G, float), np.array(Bt, float), np.array(F, float))
    assert info == 0
    assert np.allclose(K, Kx, rtol=1e-14, atol=1e-14)
    assert np.allclose(l, lx, rtol=1e-14, atol=1e-14)


def test_factored_cholesky_reports_info(oracle_mod):
    G = np.diag([1.0, -1.0, 2.0])
    K, l, info = oracle_mod.factored_cholesky_solve(G, np.eye(3), np.ones(3))
    assert info == 2  # DPOTRF INFO: leading minor of order 2 not positive


def test_flux_stiffness_reference_quad(oracle_mod):
    """DPGTests.cpp:557-655: C1 trace on each side of the reference quad against the
    vertex-ordered C1 test basis has entries 2/3 and 1/3."""
    trial = [(abi.VAR_TRACE, abi.SPACE_HGRAD, 1)]
    test = [(abi.VAR_TEST, abi.SPACE_HGRAD, 1)]
    bf = [(0, abi.OP_VALUE, 0, abi.OP_VALUE, 1.0, -1, -1, 1)]
    h = abi.DescHolder(abi.TOPO_QUAD, trial, test, bf, [(0, 0, 0, abi.OP_VALUE, 1.0, -1)], [], 2, 2, 2, 0)
    P = oracle_mod.OraclePlan(h)
    nodes = np.array([[[-1, -1], [1, -1], [1, 1], [-1, 1]]], float)
    par = np.ones((1, 4), np.int8)
    G, B, F = P.parts(nodes, par)
    stiff = B[0].T  # (test, trial)
    # lexicographic C1 (ours) -> vertex-ordered C1 of the reference test: rows [0,1,3,2]
    stiff = stiff[[0, 1, 3, 2]]
    E = np.zeros((4, 8))
    E[0, [0, 1, 6, 7]] = [2 / 3, 1 / 3, 1 / 3, 2 / 3]
    E[1, [0, 1, 2, 3]] = [1 / 3, 2 / 3, 2 / 3, 1 / 3]
    E[2, [2, 3, 4, 5]] = [1 / 3, 2 / 3, 2 / 3, 1 / 3]
    E[3, [4, 5, 6, 7]] = [1 / 3, 2 / 3, 2 / 3, 1 / 3]
    assert np.abs(stiff - E).max() < 1e-14


@pytest.mark.parametrize("degree", range(0, 16))
def test_line_cubature_exact(oracle_mod, degree):
    # BasisCacheTests.cpp:60-82: a degree-d rule integrates x^d exactly on [-1,1]
    x, w = oracle_mod.cubature(1, degree)
    exact = 0.0 if degree % 2 else 2.0 / (degree + 1)
    assert abs((w * x[:, 0] ** degree).sum() - exact) < 1e-14


@pytest.mark.parametrize("topo,dim", [(abi.TOPO_QUAD, 2), (abi.TOPO_HEX, 3)])
@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_hgrad_nodal(oracle_mod, topo, dim, n):
    """HGRAD Cn is nodal at the tensor Gauss-Lobatto points, x fastest."""
    from numpy.polynomial.legendre import Legendre
    if n == 1:
        gll = np.array([-1.0, 1.0])
    else:
        gll = np.concatenate([[-1.0], np.sort(Legendre.basis(n).deriv().roots().real), [1.0]])
    grids = np.meshgrid(*([gll] * dim), indexing="ij")
    pts = np.stack([g.reshape(-1) for g in grids[::-1]], axis=1)[:, ::-1]
    # order points x fastest
    idx = np.arange(len(gll) ** dim)
    pts = np.stack([gll[(idx // (len(gll) ** k)) % len(gll)] for k in range(dim)], axis=1)
    val, grad, _ = oracle_mod.basis_tabulate(topo, abi.SPACE_HGRAD, n, pts)
    assert np.abs(val[:, :, 0] - np.eye(len(idx))).max() < 1e-12


@pytest.mark.parametrize("dim,topo", [(2, abi.TOPO_QUAD), (3, abi.TOPO_HEX)])
@pytest.mark.parametrize("n", [1, 2, 3])
def test_hdiv_span_and_divergence(oracle_mod, dim, topo, n):
    """HDIV In spans the tensor Raviart-Thomas space (dimension, unisolvence on
    random points) and div is the derivative of the normal-direction factor."""
    rng = np.random.default_rng(0)
    pts = rng.uniform(-1, 1, size=(200, dim))
    val, _, div = oracle_mod.basis_tabulate(topo, abi.SPACE_HDIV, n, pts)
    card = val.shape[1]
    assert card == (2 * n * (n + 1) if dim == 2 else 3 * n * n * (n + 1))
    A = val.transpose(0, 2, 1).reshape(-1, card)
    assert np.linalg.matrix_rank(A) == card
    # finite-difference divergence
    h = 1e-6
    fd = np.zeros_like(div)
    for k in range(dim):
        e = np.zeros(dim)
        e[k] = h
        vp, _, _ = oracle_mod.basis_tabulate(topo, abi.SPACE_HDIV, n, pts + e)
        vm, _, _ = oracle_mod.basis_tabulate(topo, abi.SPACE_HDIV, n, pts - e)
        fd += (vp[:, :, k] - vm[:, :, k]) / (2 * h)
    assert np.abs(fd - div).max() < 1e-6
