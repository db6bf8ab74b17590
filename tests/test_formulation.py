"""Formulation-level checks of the oracle (CPU): the compiled term tables follow
the reference formulations, and the assembled matrices satisfy basis-invariant
identities (consistency, optimal-test algebra, condensation)."""
import numpy as np
import pytest

from camellia2_b200 import abi, formulation as fm, mesh
from tests.conftest import rel_fro
from tests.helpers import poisson_tri, stokes_tri, cdr2d, coeffs_for, poisson2d, poisson3d


def test_poisson_graph_norm_terms():
    """BF.cpp:1040-1141 on PoissonFormulation: [div tau], [tau - grad v], [v], [tau]."""
    form = fm.PoissonFormulation(2)
    ip = form.bf().graphNorm()
    assert len(ip.terms) == 4
    ranks = [t.rank for t in ip.terms]
    assert ranks == [0, 1, 0, 1]
    ops = [[(a.var.name, a.op, a.coef.const) for a in c] for c in ip.terms[1].comps]
    assert ops[0] == [("tau", abi.OP_X, 1.0), ("v", abi.OP_DX, -1.0)]


def test_cdr_graph_norm_terms():
    """u -> sqrt_eps div tau - beta . grad v + alpha v ; sigma -> tau + sqrt_eps grad v."""
    form = fm.ConvectionDiffusionReactionFormulation(2)
    ip = form.bf().graphNorm()
    u_term = ip.terms[0].comps[0]
    got = sorted((a.var.name, a.op, a.coef.const, a.coef.slot) for a in u_term)
    want = sorted([("tau", abi.OP_DIV, 1.0, 0), ("v", abi.OP_DX, -1.0, 1), ("v", abi.OP_DY, -1.0, 2),
                   ("v", abi.OP_VALUE, 1.0, 3)])
    assert got == want


@pytest.mark.parametrize("k,dk,N,M,nf", [(2, 2, 65, 32, 12), (4, 2, 133, 84, 48), (3, 2, 96, 55, 27)])
def test_poisson2d_sizes(oracle_mod, k, dk, N, M, nf):
    form, bucket, nodes, par = poisson2d(k, dk, 2, 2)
    P = oracle_mod.OraclePlan(bucket)
    assert (P.info["N"], P.info["M"], P.info["n_field"]) == (N, M, nf)


def test_poisson3d_sizes(oracle_mod):
    form, bucket, nodes, par = poisson3d(2, 1, 1)
    P = oracle_mod.OraclePlan(bucket)
    i = P.info
    assert (i["N"], i["M"], i["n_field"], i["n_trace"]) == (172, 110, 32, 78)
    assert (i["Q_G"], i["Q_B"], i["Q_side"]) == (64, 27, 9)


def test_mesh_parities():
    nodes, par = mesh.quad_grid(3, 2)
    # cell 4 = (1,1): bottom neighbour 1 (lower id) -> -1; left neighbour 3 -> -1; right/top +1
    assert list(par[4]) == [-1, 1, 1, -1]
    assert list(par[0]) == [1, 1, 1, 1]
    nodes, par = mesh.hex_grid(2, 2, 2)
    assert list(par[7]) == [-1, 1, 1, -1, -1, 1]


def _poisson_trial_interpolant(P, nodes_c, par_c, u, grad_u, k, d):
    """Trial coefficients of the exact solution (u, sigma = grad u, u_hat = u, sigma_n_hat = parity * sigma.n)
    for Poisson UW on one cell, by nodal interpolation in reference coordinates."""
    from numpy.polynomial.legendre import Legendre

    def gll(p):
        if p == 0:
            return np.array([0.0])
        if p == 1:
            return np.array([-1.0, 1.0])
        return np.concatenate([[-1.0], np.sort(Legendre.basis(p).deriv().roots().real), [1.0]])

    def xmap(xi):
        if d == 2:
            ref = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], float)
        else:
            ref = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                            [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)
        N = np.prod(0.5 * (1 + xi[None, :] * ref), axis=1)
        return N @ nodes_c

    def tensor_pts(p, dim):
        g = gll(p)
        m = len(g)
        idx = np.arange(m ** dim)
        return np.stack([g[(idx // (m ** j)) % m] for j in range(dim)], axis=1)

    coeffs = []
    fp = tensor_pts(k - 1, d)
    X = np.array([xmap(x) for x in fp])
    coeffs += list(u(X))
    G = grad_u(X)
    for c in range(d):
        coeffs += list(G[:, c])
    # sides
    if d == 2:
        sv = [(0, 1), (1, 2), (2, 3), (3, 0)]
        ref = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], float)
    else:
        sv = [(0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (0, 4, 7, 3), (0, 3, 2, 1), (4, 5, 6, 7)]
        ref = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                        [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)

    def side_xi(s, tpt):
        if d == 2:
            a, b = ref[sv[s][0]], ref[sv[s][1]]
            return 0.5 * (1 - tpt[0]) * a + 0.5 * (1 + tpt[0]) * b
        u_, w_ = tpt
        Nq = [0.25 * (1 - u_) * (1 - w_), 0.25 * (1 + u_) * (1 - w_), 0.25 * (1 + u_) * (1 + w_),
              0.25 * (1 - u_) * (1 + w_)]
        return sum(Nq[a] * ref[sv[s][a]] for a in range(4))

    def side_normal(s):
        V = nodes_c[list(sv[s])]
        if d == 2:
            T = V[1] - V[0]
            n = np.array([T[1], -T[0]])
            return n / np.linalg.norm(n)
        n = np.cross(V[1] - V[0], V[3] - V[0])
        return n / np.linalg.norm(n)

    for s in range(len(sv)):  # u_hat: HGRAD C(k) on each side
        for tpt in tensor_pts(k, d - 1):
            coeffs.append(u(xmap(side_xi(s, tpt))[None, :])[0])
    for s in range(len(sv)):  # sigma_n_hat: C(k-1), times parity
        n = side_normal(s)
        for tpt in tensor_pts(k - 1, d - 1):
            x = xmap(side_xi(s, tpt))[None, :]
            coeffs.append(par_c[s] * float(grad_u(x)[0] @ n))
    return np.array(coeffs)


@pytest.mark.parametrize("dim,k,dk,jitter", [(2, 2, 2, 0.2), (2, 3, 1, 0.15), (3, 2, 1, 0.0)])
def test_poisson_consistency_linear(oracle_mod, dim, k, dk, jitter):
    """The interpolant of an exact linear solution satisfies B x = F (Delta u = 0 = f):
    pins Piola maps, normals, parities, side parametrisations and trace bases
    (idea of the formulation Consistency tests, StokesVGPFormulationTests.cpp:141-153).
    3D uses an affinely sheared mesh: a jittered hex has non-planar faces, on which
    sigma.n is not in the trace space."""
    if dim == 2:
        form, bucket, nodes, par = poisson2d(k, dk, 3, 3, jitter)
    else:
        form, bucket, nodes, par = poisson3d(k, dk, 2, jitter)
        nodes = nodes @ np.array([[1.0, 0.1, 0.05], [0.2, 0.9, 0.0], [0.0, 0.15, 1.1]])
    P = oracle_mod.OraclePlan(bucket)
    C = nodes.shape[0]
    coeff = np.zeros((C, 1, P.info["n_points_total"]))
    G, B, F = P.parts(nodes, par, coeff)
    a = np.arange(1, dim + 1) * 0.7
    u = lambda X: X @ a + 0.3  # noqa: E731
    gu = lambda X: np.tile(a, (X.shape[0], 1))  # noqa: E731
    for c in range(C):
        x = _poisson_trial_interpolant(P, nodes[c], par[c], u, gu, k, dim)
        r = B[c].T @ x
        assert np.abs(r).max() < 1e-12 * max(1.0, np.abs(B[c]).max())


def test_poisson_consistency_quadratic_affine(oracle_mod):
    """Quadratic exact solution on an affine (parallelogram) mesh with k = 3:
    B x = F with f = Laplacian(u) = const."""
    form, bucket, nodes, par = poisson2d(3, 2, 2, 2, 0.0)
    nodes = nodes @ np.array([[1.0, 0.2], [0.1, 0.9]])  # affine shear
    P = oracle_mod.OraclePlan(bucket)
    C = nodes.shape[0]
    lap = 2 * 0.5 + 2 * 0.25
    coeff = np.full((C, 1, P.info["n_points_total"]), lap)
    G, B, F = P.parts(nodes, par, coeff)
    u = lambda X: 0.5 * X[:, 0] ** 2 + 0.25 * X[:, 1] ** 2 + 0.1 * X[:, 0] * X[:, 1]  # noqa: E731
    gu = lambda X: np.stack([X[:, 0] + 0.1 * X[:, 1], 0.5 * X[:, 1] + 0.1 * X[:, 0]], axis=1)  # noqa: E731
    lap = 1.0 + 0.5
    coeff = np.full((C, 1, P.info["n_points_total"]), lap)
    G, B, F = P.parts(nodes, par, coeff)
    for c in range(C):
        x = _poisson_trial_interpolant(P, nodes[c], par[c], u, gu, 3, 2)
        r = B[c].T @ x - F[c]
        assert np.abs(r).max() < 1e-11 * max(1.0, np.abs(F[c]).max())


def test_gram_norm_of_constants(oracle_mod):
    """v = 1, tau = 0 has graph norm^2 = |K|; v = 0, tau = e1 has 2|K| (affine cell)."""
    form, bucket, nodes, par = poisson2d(2, 2, 1, 1, 0.0)
    nodes = nodes @ np.array([[1.0, 0.3], [0.0, 1.2]])
    P = oracle_mod.OraclePlan(bucket)
    G, B, F = P.parts(nodes, par, np.zeros((1, 1, P.info["n_points_total"])))
    area = abs(np.linalg.det(np.array([[1.0, 0.3], [0.0, 1.2]])))
    nv = 25
    c = np.zeros(65)
    c[:nv] = 1.0
    assert abs(c @ G[0] @ c - area) < 1e-12
    # tau = J^-1-consistent reference field for physical e1 on an affine map: tau_hat = det J J^-1 e1
    Jm = 0.5 * np.array([[1.0, 0.3], [0.0, 1.2]]).T  # x = A^T xi scaled by 1/2 for the unit cell
    th = np.linalg.det(Jm) * np.linalg.solve(Jm, np.array([1.0, 0.0]))
    c = np.zeros(65)
    nx_ = 4 * 5  # x-component dofs of HDIV I4
    c[nv:nv + nx_] = th[0]
    c[nv + nx_:] = th[1]
    assert abs(c @ G[0] @ c - 2 * area) < 1e-11


@pytest.mark.parametrize("builder,args", [(poisson2d, (2, 2)), (poisson3d, (2, 1)), (cdr2d, (3, 2))])
def test_optimal_test_algebra(oracle_mod, builder, args):
    """K = B^T G^-1 B, l = B^T G^-1 F, and CHOLESKY vs FACTORED_CHOLESKY agreement
    (BFTests.cpp:74-134), plus the Schur complement against a dense solve."""
    form, bucket, nodes, par = builder(*args, 2, 2) if builder is not poisson3d else builder(*args, 1)
    P = oracle_mod.OraclePlan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, P.info, C)
    out = P.assemble(nodes, par, co, parts=True)
    assert (out["info"] == 0).all()
    f = P.is_field.astype(bool)
    for c in range(C):
        G, B, F = out["G"][c], out["B"][c], out["F"][c]
        Ld = np.linalg.cholesky(G)
        W = np.linalg.solve(Ld, B.T)
        y = np.linalg.solve(Ld, F)
        assert rel_fro(out["K"][c], W.T @ W) < 1e-10
        assert rel_fro(out["l"][c], W.T @ y) < 1e-10
        K, l = out["K"][c], out["l"][c]
        D = K[np.ix_(f, f)]
        Bc = K[np.ix_(f, ~f)]
        S = K[np.ix_(~f, ~f)] - Bc.T @ np.linalg.solve(D, Bc)
        s = l[~f] - Bc.T @ np.linalg.solve(D, l[f])
        assert rel_fro(out["S"][c], S) < 1e-10
        assert rel_fro(out["s"][c], s) < 1e-10


def _tri_trial_interpolant(oracle_mod, nodes_c, par_c, u, grad_u, k):
    """Trial coefficients of an exact solution on one triangle (Poisson UW): fields at
    the warp & blend lattice of degree k-1, traces at Gauss-Lobatto points of each edge
    (edge s runs from vertex s to vertex s+1), sigma_n_hat = parity * sigma.n."""
    from numpy.polynomial.legendre import Legendre

    def gll(p):
        if p == 0:
            return np.array([0.0])
        if p == 1:
            return np.array([-1.0, 1.0])
        return np.concatenate([[-1.0], np.sort(Legendre.basis(p).deriv().roots().real), [1.0]])

    V = nodes_c
    xmap = lambda xi: V[0] + xi[..., :1] * (V[1] - V[0]) + xi[..., 1:2] * (V[2] - V[0])  # noqa: E731
    X = xmap(oracle_mod.tri_nodes(k - 1))
    coeffs = list(u(X))
    G = grad_u(X)
    coeffs += list(G[:, 0]) + list(G[:, 1])
    for s in range(3):
        a, b = V[s], V[(s + 1) % 3]
        for t in gll(k):
            coeffs.append(u((0.5 * (1 - t) * a + 0.5 * (1 + t) * b)[None, :])[0])
    for s in range(3):
        a, b = V[s], V[(s + 1) % 3]
        T = b - a
        n = np.array([T[1], -T[0]]) / np.linalg.norm(T)
        for t in gll(k - 1):
            x = (0.5 * (1 - t) * a + 0.5 * (1 + t) * b)[None, :]
            coeffs.append(par_c[s] * float(grad_u(x)[0] @ n))
    return np.array(coeffs)


def test_poisson_tri_sizes(oracle_mod):
    form, bucket, nodes, par = poisson_tri(2, 2)
    i = oracle_mod.OraclePlan(bucket).info
    assert (i["N"], i["M"], i["n_field"], i["n_trace"], i["n_sides"]) == (39, 24, 9, 15, 3)
    form, bucket, nodes, par = stokes_tri(1, 2)
    assert oracle_mod.OraclePlan(bucket).info["N"] == 60  # Stokes VGP tri p=1 (60 ... 295)


@pytest.mark.parametrize("k,dk,jitter", [(2, 2, 0.2), (3, 1, 0.15), (4, 2, 0.1)])
def test_poisson_tri_consistency_linear(oracle_mod, k, dk, jitter):
    """Triangles: the interpolant of an exact linear solution satisfies B x = F = 0;
    pins the triangle rule, the lattice basis of the fields, edge parametrisation,
    normals and parities."""
    form, bucket, nodes, par = poisson_tri(k, dk, 3, 2, jitter)
    P = oracle_mod.OraclePlan(bucket)
    C = nodes.shape[0]
    G, B, F = P.parts(nodes, par, np.zeros((C, 1, P.info["n_points_total"])))
    a = np.array([0.7, -1.3])
    u = lambda X: X @ a + 0.3  # noqa: E731
    gu = lambda X: np.tile(a, (X.shape[0], 1))  # noqa: E731
    for c in range(C):
        x = _tri_trial_interpolant(oracle_mod, nodes[c], par[c], u, gu, k)
        r = B[c].T @ x
        assert np.abs(r).max() < 1e-12 * max(1.0, np.abs(B[c]).max()), (c, np.abs(r).max())


def test_tri_mesh_parities():
    nodes, par = mesh.tri_grid(2, 1)
    # quad 0 holds cells 0 = (v00, v10, v11) and 1 = (v00, v11, v01); they share the
    # diagonal: side 2 of cell 0 and side 0 of cell 1
    assert par[0, 2] == 1 and par[1, 0] == -1
    # side 1 of cell 1 (v11 -> v01) lies on the top boundary
    assert par[1, 1] == 1
    # the edge x = h joins cell 0 (side 1, v10 -> v11) and cell 3 (side 2, v01 -> v00 of quad 1)
    assert par[0, 1] == 1 and par[3, 2] == -1
    # counter-clockwise vertices: positive signed areas
    e1, e2 = nodes[:, 1] - nodes[:, 0], nodes[:, 2] - nodes[:, 0]
    assert (e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0] > 0).all()
