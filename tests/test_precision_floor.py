"""The FP64 floor of the configurations, measured against the extended-precision truth
(the oracle built with __float128 arithmetic, oracle/liboracle_xp.so) on the same double
inputs.

At h = 1/48 (3D hex Poisson UW, k=2 dk=1) the graph-norm Gram matrix has cond(G) ~ 1e14:
its L2 terms scale with h^3 next to divergence terms scaling with 1/h^3.  Two facts follow
and are pinned here on cells of the 48^3 jittered mesh:

  * even with G, B and F computed exactly and rounded to double, the reference's FP64
    factored Cholesky solve (BF.cpp:924-1018) leaves K and S about 3e-11 from the truth,
    so no FP64 code -- Camellia's included -- can be within 1e-12 of the truth, or of
    another FP64 code, on this mesh;
  * summation order of the Gram quadrature matters at this conditioning: the oracle
    integrates each graph-norm term on its own (the reference's order, IP.cpp:238-244)
    and lands within ~5e-11 of the truth; rounding only the operator values (each
    G = L~^T W L~ then stays an exact Gram matrix) costs ~5e-12.

The c2 mesh (2D Poisson k=4 dk=2 on 256^2 quads, test degree 6) has a far higher floor
(~1e-8), c4 (CDR k=3 dk=2, 128^2) ~1e-10, c1 (16^2, unjittered) ~1e-11."""
import numpy as np
import pytest

from camellia2_b200 import abi, formulation as fm, mesh
from tests.conftest import rel_fro


def hex48_cells(oracle_mod, idx=(0, 1234, 55555, 110591)):
    b = fm.PoissonFormulation(3).bucket(abi.TOPO_HEX, 2, 1)
    P = oracle_mod.OraclePlan(b)
    nodes, par = mesh.hex_grid(48, 48, 48, 0.1, seed=1)
    co = mesh.uniform_coeff(len(nodes), 1, P.info["n_points_total"], seed=1)
    idx = list(idx)
    return b, P, nodes[idx], par[idx], co[idx]


@pytest.fixture(scope="module")
def cells48(oracle_mod):
    b, P, nodes, par, co = hex48_cells(oracle_mod)
    X = oracle_mod.OraclePlan(b, xp=True)
    return P, P.assemble(nodes, par, co, parts=True), X.assemble(nodes, par, co, parts=True, nthreads=4)


def test_gram_conditioning_at_48_cubed(cells48):
    P, o, x = cells48
    assert min(np.linalg.cond(G) for G in x["G"]) > 1e13


def test_extended_precision_oracle_agrees_on_the_quadrature(cells48):
    """The __float128 build computes the same quadrature: G, B, F agree to FP64 rounding."""
    P, o, x = cells48
    for c in range(o["G"].shape[0]):
        assert rel_fro(o["G"][c], x["G"][c]) < 1e-14
        assert rel_fro(o["B"][c], x["B"][c]) < 1e-14
        assert rel_fro(o["F"][c], x["F"][c]) < 1e-14
        assert x["info"][c] == 0


def test_fp64_floor_at_48_cubed(cells48, oracle_mod):
    """Correctly rounded G, B, F plus the FP64 solve: K is 1e-11..1e-10 from the truth."""
    P, o, x = cells48
    for c in range(o["G"].shape[0]):
        K, l, info = oracle_mod.factored_cholesky_solve(x["G"][c], x["B"][c], x["F"][c])
        assert info == 0
        e = rel_fro(K, x["K"][c])
        assert 1e-11 < e < 1e-10, e


def test_fp64_oracle_error_against_the_truth(cells48):
    """The FP64 oracle (the reference's per-term order) is within 1e-10 of the truth on
    K, l, S, s, and no closer than 1e-12 on K and S."""
    P, o, x = cells48
    for c in range(o["G"].shape[0]):
        for k in ("K", "l", "S", "s"):
            assert rel_fro(o[k][c], x[k][c]) < 1e-10, (c, k)
        assert rel_fro(o["K"][c], x["K"][c]) > 1e-12
        assert rel_fro(o["S"][c], x["S"][c]) > 1e-12


def test_structured_gram_errors_are_benign(cells48, oracle_mod):
    """Operator values rounded to about 2^-42 relative (per column), then summed exactly:
    G = L~^T W L~ is still a Gram matrix and S stays within the FP64 floor, while random
    relative errors of 2^-48 on G's entries already move S by more than 1e-10."""
    from tests import mixed_emulation as me
    b, P, nodes, par, co = hex48_cells(oracle_mod, idx=(0,))
    x = cells48[2]
    op = P.operators(nodes[0], par[0], co[0])
    G = me.gram(op, "int8x6")
    K, l, _ = oracle_mod.factored_cholesky_solve(G, x["B"][0], x["F"][0], xp=True)
    S, _, _ = oracle_mod.condense(P.is_field, K, l, xp=True)
    assert rel_fro(S, x["S"][0]) < 1e-10
    rng = np.random.default_rng(0)
    E = rng.normal(size=G.shape)
    Gp = x["G"][0] * (1 + 2.0 ** -48 * (E + E.T) / 2)
    K, l, _ = oracle_mod.factored_cholesky_solve(Gp, x["B"][0], x["F"][0], xp=True)
    S, _, _ = oracle_mod.condense(P.is_field, K, l, xp=True)
    assert rel_fro(S, x["S"][0]) > 1e-10


@pytest.mark.parametrize("p", [4, 6])
def test_triangle_rt_basis_is_well_conditioned(oracle_mod, p):
    """The triangle RT_n test basis (x psi with the PKD polynomials psi of exact degree n-1)
    keeps the Stokes VGP triangle buckets' FP64 floor (relative change of K under 1-ulp noise
    on G) at the level of the quad buckets: below 1e-11 on unit-size cells and below 1e-6 on
    the finest cells of the uneven-cell workload (h = 1/256), where every factorisation
    succeeds.  With x times monomials the floor was 1.4e-8 at h = 1 and the Gram matrix lost
    positive definiteness at h = 1/256 for p = 6."""
    from tests.helpers import fp64_floor
    b = fm.StokesVGPFormulation(2).bucket(abi.TOPO_TRI, p, 2)
    P = oracle_mod.OraclePlan(b)
    for base_n, bound in ((1, 1e-11), (256, 1e-6)):
        nodes, par = mesh.forest_buckets(2000, seed=3, base_n=base_n, max_level=0)[(abi.TOPO_TRI, p)]
        nodes, par = nodes[:2], par[:2]
        co = mesh.uniform_coeff(2, P.info["n_slots"], P.info["n_points_total"], seed=1)
        o = P.assemble(nodes, par, co, parts=True)
        assert (o["info"] == 0).all()
        floor = max(fp64_floor(oracle_mod, o["G"][c], o["B"][c], o["F"][c], o["K"][c], trials=2) for c in range(2))
        assert floor < bound, (base_n, floor)
