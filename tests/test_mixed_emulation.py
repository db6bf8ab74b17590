"""Which reduced-precision contraction recipes can reach the mixed form's accuracy bar
(relative Frobenius error <= 1e-10 on the condensed matrix S) on the 48^3 hex mesh, each
applied term by term as the reference integrates the graph norm (IP.cpp:238-244), with
the FP64 factored Cholesky solve and condensation kept (BF.cpp:924-1018,
CondensedDofInterpreter.cpp:1138-1192).  Errors are measured against the
extended-precision truth and against the FP64 oracle (tests/mixed_emulation.py).

Measured on two cells (S error against the truth; the FP64 oracle's own is ~4e-11):
  G by bf16x3 (FP32 accumulation)    ~1               G by int8x5 (25 slice pairs)  ~1.5e-9
  G by tf32x3                        ~3e-3            G by int8x6 (36 pairs)        ~3e-11
  G by bf16x6                        ~2e-3            G by int8x7 truncated (28)    ~1.4e-9
  B by bf16x3                        ~1e-5            G by int8x8 truncated (36)    ~4e-11
                                                      B by int8x6                   ~5e-11
The split-precision recipes with FP32 accumulation miss the bar by 7 to 10 orders of
magnitude: their accumulation errors are relative to each term's largest products, and
at cond(G) ~ 1e14 the h^3-scaled terms underneath are lost.  Integer slicing with exact
accumulation (Ozaki) keeps G the exact Gram matrix of a sliced operator and meets the bar
from six slices on."""
import numpy as np
import pytest

from tests import mixed_emulation as me
from tests.conftest import rel_fro
from tests.test_precision_floor import hex48_cells


@pytest.fixture(scope="module")
def setup(oracle_mod):
    b, P, nodes, par, co = hex48_cells(oracle_mod, idx=(0, 55555))
    X = oracle_mod.OraclePlan(b, xp=True)
    x = X.assemble(nodes, par, co, parts=True, nthreads=2)
    o = P.assemble(nodes, par, co, parts=True)
    ops = [P.operators(nodes[c], par[c], co[c]) for c in range(2)]
    return P, o, x, ops


def _s_errors(oracle_mod, setup, g_recipe, b_recipe):
    P, o, x, ops = setup
    out = []
    for c in range(2):
        r = me.assemble(oracle_mod, P.is_field, ops[c], o["F"][c], g_recipe, b_recipe)
        out.append((rel_fro(r["S"], x["S"][c]), rel_fro(r["S"], o["S"][c]), rel_fro(r["K"], x["K"][c])))
    return np.array(out)


def test_operator_rows_reproduce_the_quadrature(setup):
    P, o, x, ops = setup
    for c in range(2):
        op = ops[c]
        G = np.einsum("q,qri,qrj->ij", op["wm"], op["L"], op["L"])
        assert rel_fro(G, o["G"][c]) < 1e-14
        assert rel_fro(op["U"].T @ op["V"], o["B"][c]) < 1e-14
        assert rel_fro(op["FV"].T @ op["fw"], o["F"][c]) < 1e-14


@pytest.mark.parametrize("recipe", ["bf16x3", "tf32x3", "bf16x6"])
def test_split_precision_gram_misses_the_bar(oracle_mod, setup, recipe):
    e = _s_errors(oracle_mod, setup, recipe, "fp64")
    assert e[:, 0].min() > 1e-4, e


def test_split_precision_stiffness_misses_the_bar(oracle_mod, setup):
    e = _s_errors(oracle_mod, setup, "fp64", "bf16x3")
    assert e[:, 0].min() > 1e-7, e


@pytest.mark.parametrize("recipe", ["int8x5", "int8x7t"])
def test_too_few_int8_slices_miss_the_bar(oracle_mod, setup, recipe):
    e = _s_errors(oracle_mod, setup, recipe, "fp64")
    assert e[:, 0].min() > 1e-10, e


@pytest.mark.parametrize("g_recipe,b_recipe", [("int8x6", "fp64"), ("int8x8t", "fp64"), ("int8x6", "int8x6")])
def test_int8_slicing_meets_the_bar(oracle_mod, setup, g_recipe, b_recipe):
    e = _s_errors(oracle_mod, setup, g_recipe, b_recipe)
    assert e[:, 0].max() < 1e-10, e  # against the truth
    assert e[:, 1].max() < 1e-10, e  # against the FP64 oracle
