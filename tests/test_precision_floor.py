"""Why the bench runs the FP64 form: the accuracy the north star asks of a mixed
form (<= 1e-10 relative Frobenius on the condensed matrix S at the 48^3 bench
mesh) is below what any reduced-precision Gram matrix can give there.

On cells of the 48^3 jittered hex mesh (h = 1/48, 3D Poisson UW, k=2 dk=1) the
graph-norm Gram matrix has cond(G) ~ 1e14 (its L2 terms scale with h^3 next to
gradient terms scaling with h).  Random relative perturbations of G's entries of
size eps move S by roughly 1e5 * eps (oracle, FP64 otherwise):
    eps = 2^-53 -> 1.6e-11,  2^-48 -> 3.7e-10,  2^-24 (FP32) -> 6e-3,
while B tolerates 2^-40 (3.6e-12).  So G must be formed to nearly full FP64
accuracy; only B could drop precision, and B is a small share of the kernel.
This test pins those facts on four cells with the oracle (CPU)."""
import numpy as np
import pytest

from camellia2_b200 import abi, formulation as fm, mesh
from tests.conftest import rel_fro


@pytest.fixture(scope="module")
def cells48(oracle_mod):
    b = fm.PoissonFormulation(3).bucket(abi.TOPO_HEX, 2, 1)
    P = oracle_mod.OraclePlan(b)
    nodes, par = mesh.hex_grid(48, 48, 48, 0.1, seed=1)
    idx = [0, 1234, 55555, 110591]
    nodes, par = nodes[idx], par[idx]
    co = mesh.uniform_coeff(len(idx), 1, P.info["n_points_total"], seed=1)
    return P, P.assemble(nodes, par, co, parts=True)


def _worst_s_change(oracle_mod, P, o, eps, which, seed=0):
    rng = np.random.default_rng(seed)
    worst = 0.0
    for c in range(o["G"].shape[0]):
        G, B, F = o["G"][c], o["B"][c], o["F"][c]
        if which == "G":
            E = rng.normal(size=G.shape)
            G = G * (1 + eps * (E + E.T) / 2)
        else:
            B = B * (1 + eps * rng.normal(size=B.shape))
        K, l, _ = oracle_mod.factored_cholesky_solve(G, B, F)
        S, _, _ = oracle_mod.condense(P.is_field, K, l)
        S0, _, _ = oracle_mod.condense(P.is_field, o["K"][c], o["l"][c])
        worst = max(worst, rel_fro(S, S0))
    return worst


def test_gram_conditioning_at_48_cubed(cells48):
    P, o = cells48
    assert min(np.linalg.cond(G) for G in o["G"]) > 1e13


def test_reduced_precision_gram_misses_the_bar(cells48, oracle_mod):
    P, o = cells48
    assert _worst_s_change(oracle_mod, P, o, 2.0 ** -48, "G") > 1e-10  # 5 bits short of FP64 already fails
    assert _worst_s_change(oracle_mod, P, o, 2.0 ** -24, "G") > 1e-4   # an FP32-accurate G is far off


def test_fp64_gram_and_reduced_b_meet_the_bar(cells48, oracle_mod):
    P, o = cells48
    assert _worst_s_change(oracle_mod, P, o, 2.0 ** -53, "G") < 1e-10
    assert _worst_s_change(oracle_mod, P, o, 2.0 ** -40, "B") < 1e-10


@pytest.mark.parametrize("p", [4, 6])
def test_triangle_rt_basis_is_well_conditioned(oracle_mod, p):
    """The triangle RT_n test basis (x psi with the PKD polynomials psi of exact degree n-1)
    keeps the Stokes VGP triangle buckets' FP64 floor (relative change of K under 1-ulp noise
    on G) at the level of the quad buckets: below 1e-11 on unit-size cells and below 1e-6 on
    the finest cells of the uneven-cell workload (h = 1/256), where every factorisation
    succeeds.  With x times monomials the floor was 1.4e-8 at h = 1 and the Gram matrix lost
    positive definiteness at h = 1/256 for p = 6."""
    from tests.test_gpu_parity import fp64_floor
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
