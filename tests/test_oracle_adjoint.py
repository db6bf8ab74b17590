"""The oracle's hand gradient (reverse mode; no counterpart in the reference) pinned by
central finite differences computed entirely in __float128.

For J = sum_c (r_c^T K_c r_c + g_c^T l_c) on cells of the 128^2 CDR workload (c4: field
degree 2, dk = 2; eps = exp(N(-4, 1)), beta = (cos t, sin t), c ~ U[0,1], f ~ U[-1,1]),
the gradient with respect to the per-point coefficient slots (sqrt(eps), beta_x, beta_y,
c, f) from Bbar = (Kbar + Kbar^T) X^T + lbar y^T, Gbar = -X Kbar_s X^T - ..., Fbar = X lbar
pulled back through the quadrature (oracle/dpg_oracle.cpp: adjoint_cell) matches
(J(c + h d) - J(c - h d)) / 2h at h = 1e-6 along 16 random directions and 64 single
coordinates.  In __float128 the difference carries only its truncation error (~1e-12
here), so the bound can be tight: 1e-9 relative."""
import numpy as np
import pytest

from camellia2_b200 import abi, formulation as fm, mesh

STEP = 1e-6


@pytest.fixture(scope="module")
def cdr_sample(oracle_mod):
    b = fm.ConvectionDiffusionReactionFormulation(2).bucket(abi.TOPO_QUAD, 3, 2)
    P = oracle_mod.OraclePlan(b)
    X = oracle_mod.OraclePlan(b, xp=True)
    nodes, par = mesh.quad_grid(128, 128, 0.1, seed=1)
    co = mesh.cdr_coeff(len(nodes), P.info, seed=1)
    idx = [0, 777, 9000, 16383]
    n, p, c = nodes[idx], par[idx], co[idx]
    rng = np.random.default_rng(5)
    M = P.info["M"]
    r = rng.normal(size=(len(idx), M))
    g = rng.normal(size=(len(idx), M))
    Kb = r[:, :, None] * r[:, None, :]
    return P, X, n, p, c, Kb, g


def test_hand_gradient_matches_extended_precision_differences(cdr_sample):
    P, X, n, p, c, Kb, g = cdr_sample
    grad = X.adjoint(n, p, c, Kb, g, nthreads=4)
    rng = np.random.default_rng(9)
    for _ in range(16):
        d = rng.normal(size=c.shape)
        d /= np.linalg.norm(d)
        fd = X.fd_directional(n, p, c, d, STEP, Kb, g, nthreads=4)
        assert abs(float((grad * d).sum()) - fd) <= 1e-9 * abs(fd), fd
    flat = np.flatnonzero(np.abs(grad).reshape(-1) > 0)
    for k in rng.choice(flat, size=64, replace=False):
        d = np.zeros(c.size)
        d[k] = 1.0
        d = d.reshape(c.shape)
        cell = int(np.unravel_index(k, c.shape)[0])
        s = slice(cell, cell + 1)
        fd = X.fd_directional(n[s], p[s], c[s], d[s], STEP, Kb[s], g[s])
        assert abs(float(grad.reshape(-1)[k]) - fd) <= 1e-9 * abs(fd) + 1e-15, (k, fd)


def test_fp64_hand_gradient_is_within_the_fp64_floor(cdr_sample):
    P, X, n, p, c, Kb, g = cdr_sample
    gx = X.adjoint(n, p, c, Kb, g, nthreads=4)
    g64 = P.adjoint(n, p, c, Kb, g)
    assert np.linalg.norm(g64 - gx) <= 1e-8 * np.linalg.norm(gx)


def test_loss_pair_keeps_extended_precision(cdr_sample):
    """J returned as (hi, lo): the difference of two nearby losses equals the oracle's own
    central difference."""
    P, X, n, p, c, Kb, g = cdr_sample
    d = np.random.default_rng(3).normal(size=c.shape)
    d /= np.linalg.norm(d)
    hi_p, lo_p = X.loss(n, p, c + STEP * d, Kb, g)
    hi_m, lo_m = X.loss(n, p, c - STEP * d, Kb, g)
    fd_pair = ((hi_p - hi_m) + (lo_p - lo_m)) / (2 * STEP)
    # the perturbed coefficients were rounded to double here, which moves J by ~1e-16 |c| / h
    fd = X.fd_directional(n, p, c, d, STEP, Kb, g)
    assert abs(fd_pair - fd) <= 1e-8 * abs(fd)
