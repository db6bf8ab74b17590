"""The product's reference bases and cubature rules (dpg_basis_tabulate, dpg_cubature:
the host tables every plan is built from) against constructions written here from the
definitions, independently of both the library and the oracle:

  * Gauss-Lobatto nodes as the roots of P_n' (numpy's Legendre class) plus the end points,
    Gauss nodes from numpy's leggauss; 1D Lagrange polynomials by Vandermonde solves;
  * HGRAD Cn on quads and hexes: tensor Lagrange at the Gauss-Lobatto nodes, x fastest
    (BasisFactory.cpp:122-420 with POINTTYPE_SPECTRAL);
  * HDIV In on quads and hexes: component c is a degree-n Lagrange polynomial at the
    Gauss-Lobatto nodes in direction c and degree n-1 at the Gauss nodes in the others,
    components one after the other, x fastest;
  * HGRAD Cn on the triangle: a warp & blend lattice computed here (Warburton's published
    construction, with Hesthaven & Warburton's alpha table) must be the nodal set of the
    product's functions (phi_k(x_j) = delta_kj), and its edge nodes the Gauss-Lobatto nodes;
  * RT_n on the triangle: the product's functions span (P_{n-1})^2 + x P~_{n-1} (a
    least-squares fit with monomials leaves no residual), are independent, and their
    divergence is the divergence of the fitted field;
  * cubature: tensor rules equal numpy's Gauss points and weights; the triangle rule
    integrates every monomial of degree <= its degree exactly (int x^a y^b = a! b! /
    (a + b + 2)!).
No GPU is needed: the tabulation is host code of libdpg_b200.so."""
import ctypes as ct
from math import factorial

import numpy as np
import pytest
from numpy.polynomial import legendre as npleg

from camellia2_b200 import abi, lib as dlib

TOL = 1e-12


def _tab(topo, space, n, pts):
    L = dlib.load()
    L.dpg_basis_tabulate.argtypes = [ct.c_int] * 4 + [ct.c_void_p] * 2
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    d = pts.shape[1]
    card = L.dpg_basis_tabulate(topo, space, n, 0, None, None)
    assert card > 0
    out = np.zeros((pts.shape[0], card, d + 1))
    assert L.dpg_basis_tabulate(topo, space, n, pts.shape[0], pts.ctypes.data_as(ct.c_void_p),
                                out.ctypes.data_as(ct.c_void_p)) == card
    return out


def _cub(topo, degree):
    L = dlib.load()
    L.dpg_cubature.argtypes = [ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p]
    n = L.dpg_cubature(topo, degree, None, None)
    d = abi.TOPO_INFO[topo][0]
    x, w = np.zeros((n, d)), np.zeros(n)
    L.dpg_cubature(topo, degree, x.ctypes.data_as(ct.c_void_p), w.ctypes.data_as(ct.c_void_p))
    return x, w


def gll(n):
    if n == 0:
        return np.zeros(1)
    inner = npleg.Legendre.basis(n).deriv().roots() if n > 1 else np.zeros(0)
    return np.concatenate([[-1.0], np.sort(inner.real), [1.0]])


def lagrange_1d(nodes, t):
    """Values and derivatives (len(t), len(nodes)) of the Lagrange polynomials on nodes."""
    m = len(nodes)
    V = np.vander(nodes, m, increasing=True)
    Cf = np.linalg.inv(V)  # column k: monomial coefficients of phi_k
    T = np.vander(t, m, increasing=True)
    dT = np.zeros_like(T)
    dT[:, 1:] = T[:, :-1] * np.arange(1, m)
    return T @ Cf, dT @ Cf


def _rand_pts(d, n=7, seed=3):
    return np.random.default_rng(seed).uniform(-1, 1, size=(n, d))


@pytest.mark.parametrize("topo,d", [(abi.TOPO_QUAD, 2), (abi.TOPO_HEX, 3)])
@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_hgrad_tensor_lagrange_at_gauss_lobatto(topo, d, n):
    pts = _rand_pts(d)
    got = _tab(topo, abi.SPACE_HGRAD, n, pts)
    x = gll(n)
    m = n + 1
    for q, p in enumerate(pts):
        vals = [lagrange_1d(x, np.array([p[k]])) for k in range(d)]
        for dof in range(m ** d):
            ii = [(dof // m ** k) % m for k in range(d)]
            v = np.prod([vals[k][0][0, ii[k]] for k in range(d)])
            assert abs(got[q, dof, 0] - v) < TOL
            for k in range(d):
                g = np.prod([vals[j][1][0, ii[j]] if j == k else vals[j][0][0, ii[j]] for j in range(d)])
                assert abs(got[q, dof, 1 + k] - g) < 10 * TOL


@pytest.mark.parametrize("topo,d", [(abi.TOPO_QUAD, 2), (abi.TOPO_HEX, 3)])
@pytest.mark.parametrize("n", [1, 2, 4])
def test_hdiv_tensor_raviart_thomas(topo, d, n):
    pts = _rand_pts(d, seed=5)
    got = _tab(topo, abi.SPACE_HDIV, n, pts)
    closed, opn = gll(n), npleg.leggauss(n)[0]
    for q, p in enumerate(pts):
        cl = [lagrange_1d(closed, np.array([p[k]])) for k in range(d)]
        op = [lagrange_1d(opn, np.array([p[k]])) for k in range(d)]
        dof = 0
        for comp in range(d):
            ext = [n + 1 if k == comp else n for k in range(d)]
            for idx in range(int(np.prod(ext))):
                ii, r = [], idx
                for k in range(d):
                    ii.append(r % ext[k])
                    r //= ext[k]
                f = np.prod([(cl if k == comp else op)[k][0][0, ii[k]] for k in range(d)])
                dv = np.prod([cl[k][1][0, ii[k]] if k == comp else op[k][0][0, ii[k]] for k in range(d)])
                want = np.zeros(d)
                want[comp] = f
                assert np.abs(got[q, dof, :d] - want).max() < TOL
                assert abs(got[q, dof, d] - dv) < 10 * TOL
                dof += 1
        assert dof == got.shape[1]


def warp_blend_lattice(N):
    """Warburton's warp & blend nodes on the triangle (0,0),(1,0),(0,1), written from the
    published construction: equidistant barycentric lattice, edge warp = interpolated
    displacement of the Gauss-Lobatto nodes, blended by 4 L_i L_j (1 + (alpha L_k)^2)."""
    alpopt = [0.0000, 0.0000, 1.4152, 0.1001, 0.2751, 0.9800, 1.0999, 1.2832, 1.3648, 1.4773, 1.4959,
              1.5743, 1.5770, 1.6223, 1.6258]
    alpha = alpopt[N - 1] if N < 16 else 5.0 / 3.0
    eq = np.linspace(-1, 1, N + 1)
    g = gll(N)

    def warp(r):
        # interpolant through (eq_i, g_i - eq_i), divided by 1 - r^2 (zero at the ends)
        Lr, _ = lagrange_1d(eq, np.atleast_1d(r))
        w = Lr @ (g - eq)
        zf = np.abs(r) < 1 - 1e-10
        return np.where(zf, w / np.where(zf, 1 - r * r, 1.0), 0.0)

    pts = []
    for i in range(N + 1):
        for j in range(N + 1 - i):
            L1, L3 = i / N, j / N
            L2 = 1 - L1 - L3
            x, y = -L2 + L3, (-L2 - L3 + 2 * L1) / np.sqrt(3)
            b1 = 4 * L2 * L3 * warp(L3 - L2)[0] * (1 + (alpha * L1) ** 2)
            b2 = 4 * L1 * L3 * warp(L1 - L3)[0] * (1 + (alpha * L2) ** 2)
            b3 = 4 * L1 * L2 * warp(L2 - L1)[0] * (1 + (alpha * L3) ** 2)
            x += b1 + np.cos(2 * np.pi / 3) * b2 + np.cos(4 * np.pi / 3) * b3
            y += np.sin(2 * np.pi / 3) * b2 + np.sin(4 * np.pi / 3) * b3
            # equilateral (vertices (-1,-1/sqrt3), (1,-1/sqrt3), (0,2/sqrt3)) -> reference triangle
            l1 = (np.sqrt(3) * y + 1) / 3
            l2 = (-3 * x - np.sqrt(3) * y + 2) / 6
            l3 = (3 * x - np.sqrt(3) * y + 2) / 6
            pts.append((l3, l1))  # xi = weight of vertex (1,0), eta = weight of vertex (0,1)
    return np.array(pts)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 6])
def test_triangle_hgrad_is_nodal_on_the_warp_blend_lattice(n):
    X = warp_blend_lattice(n)
    # edge eta = 0 carries the Gauss-Lobatto nodes mapped to [0, 1]
    edge = np.sort(X[np.abs(X[:, 1]) < 1e-14][:, 0])
    assert np.abs(edge - 0.5 * (1 + gll(n))).max() < TOL
    got = _tab(abi.TOPO_TRI, abi.SPACE_HGRAD, n, X)
    assert np.abs(got[:, :, 0] - np.eye(X.shape[0])).max() < 1e-11
    # gradients: differences of the product's own values along x and y
    pts = np.random.default_rng(2).uniform(0.05, 0.45, size=(5, 2))
    h = 1e-6
    for k in range(2):
        e = np.zeros(2)
        e[k] = h
        fd = (_tab(abi.TOPO_TRI, abi.SPACE_HGRAD, n, pts + e)[:, :, 0] -
              _tab(abi.TOPO_TRI, abi.SPACE_HGRAD, n, pts - e)[:, :, 0]) / (2 * h)
        assert np.abs(_tab(abi.TOPO_TRI, abi.SPACE_HGRAD, n, pts)[:, :, 1 + k] - fd).max() < 1e-7


@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_triangle_hdiv_spans_raviart_thomas(n):
    rng = np.random.default_rng(8)
    u = rng.uniform(size=(60, 2))
    pts = np.stack([u[:, 0] * (1 - u[:, 1]), u[:, 1]], axis=1)
    got = _tab(abi.TOPO_TRI, abi.SPACE_HDIV, n, pts)
    card = n * (n + 2)
    assert got.shape[1] == card
    # monomial basis of RT_n: (m, 0), (0, m) for monomials m of degree <= n-1, x m~ for degree n-1
    mono = [(a, b) for s in range(n) for a in range(s + 1) for b in [s - a]]
    hom = [(a, n - 1 - a) for a in range(n)]
    x, y = pts[:, 0], pts[:, 1]
    cols, divs = [], []
    for a, b in mono:
        m = x ** a * y ** b
        cols.append(np.concatenate([m, 0 * m]))
        divs.append(a * x ** max(a - 1, 0) * y ** b if a > 0 else 0 * m)
    for a, b in mono:
        m = x ** a * y ** b
        cols.append(np.concatenate([0 * m, m]))
        divs.append(b * x ** a * y ** max(b - 1, 0) if b > 0 else 0 * m)
    for a, b in hom:
        m = x ** a * y ** b
        cols.append(np.concatenate([x * m, y * m]))
        divs.append((n + 1) * m)  # div(x m) = 2 m + x . grad m = (2 + deg m) m
    A = np.stack(cols, axis=1)
    Dv = np.stack(divs, axis=1)
    assert A.shape[1] == card
    for dof in range(card):
        rhs = np.concatenate([got[:, dof, 0], got[:, dof, 1]])
        coef, *_ = np.linalg.lstsq(A, rhs, rcond=None)
        assert np.abs(A @ coef - rhs).max() < 1e-11
        assert np.abs(Dv @ coef - got[:, dof, 2]).max() < 1e-9
    V = np.concatenate([got[:, :, 0], got[:, :, 1]], axis=0)
    assert np.linalg.matrix_rank(V, tol=1e-10) == card


@pytest.mark.parametrize("topo,d", [(abi.TOPO_QUAD, 2), (abi.TOPO_HEX, 3)])
@pytest.mark.parametrize("degree", [0, 3, 8, 12])
def test_tensor_cubature_is_gauss(topo, d, degree):
    x, w = _cub(topo, degree)
    g, gw = npleg.leggauss(degree // 2 + 1)
    m = len(g)
    assert x.shape[0] == m ** d
    for q in range(m ** d):
        ii = [(q // m ** k) % m for k in range(d)]
        assert np.abs(x[q] - g[ii]).max() < TOL
        assert abs(w[q] - np.prod(gw[ii])) < TOL


@pytest.mark.parametrize("degree", [1, 4, 8, 12, 16])
def test_triangle_cubature_is_exact(degree):
    x, w = _cub(abi.TOPO_TRI, degree)
    for a in range(degree + 1):
        for b in range(degree + 1 - a):
            exact = factorial(a) * factorial(b) / factorial(a + b + 2)
            assert abs((w * x[:, 0] ** a * x[:, 1] ** b).sum() - exact) < 1e-14, (a, b)


def test_invalid_arguments_are_refused():
    L = dlib.load()
    L.dpg_basis_tabulate.argtypes = [ct.c_int] * 4 + [ct.c_void_p] * 2
    assert L.dpg_basis_tabulate(99, abi.SPACE_HGRAD, 2, 0, None, None) == -abi.DPG_ERR_INVALID_ARGUMENT
    assert L.dpg_basis_tabulate(abi.TOPO_QUAD, abi.SPACE_HDIV, 0, 0, None, None) == -abi.DPG_ERR_INVALID_ARGUMENT
