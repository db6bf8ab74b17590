"""GPU parity against the extended-precision truth (the oracle built with __float128
arithmetic) on seeded samples of the configurations' full-size meshes, through the C ABI.

At these mesh sizes the graph-norm Gram matrices are so ill-conditioned that no FP64
code lands within 1e-12 of the exact result: with G, B, F computed exactly and rounded to
double, the reference's FP64 factored Cholesky solve alone leaves K about 3e-11 (48^3
hexes), 1e-8 (256^2 quads, test degree 6) or 1e-10 (128^2 CDR) from it.  Two FP64 codes
therefore differ at that level too.  The bar here is the one that means something: over
the sampled cells, the GPU's worst error against the truth (K, l, S, s; relative
Frobenius) is at most FACTOR times the FP64 oracle's worst.  The 48^3 hex workload must
in addition be within 1e-10 of the truth (the mixed form's bar)."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import abi, formulation as fm, lib as dlib, mesh  # noqa: E402
from tests.conftest import rel_fro  # noqa: E402

pytestmark = pytest.mark.gpu

FACTOR = 3.0
KEYS = ("K", "l", "S", "s")


def _sample(C, n, seed=11):
    rng = np.random.default_rng(seed)
    return np.unique(np.concatenate([[0, C - 1], rng.choice(C, size=n - 2, replace=False)]))


def _configs():
    uc = lambda info, C: mesh.uniform_coeff(C, 1, info["n_points_total"], seed=1)  # noqa: E731
    yield "c5_hex48", fm.PoissonFormulation(3).bucket(abi.TOPO_HEX, 2, 1), mesh.hex_grid(48, 48, 48, 0.1, seed=1), uc, 12
    yield "c2_quad256", fm.PoissonFormulation(2).bucket(abi.TOPO_QUAD, 4, 2), mesh.quad_grid(256, 256, 0.2, seed=1), uc, 8
    yield ("c4_cdr128", fm.ConvectionDiffusionReactionFormulation(2).bucket(abi.TOPO_QUAD, 3, 2),
           mesh.quad_grid(128, 128, 0.1, seed=1), lambda info, C: mesh.cdr_coeff(C, info, seed=1), 8)
    yield ("c1_quad16", fm.PoissonFormulation(2).bucket(abi.TOPO_QUAD, 2, 2), mesh.quad_grid(16, 16, 0.0, seed=1),
           lambda info, C: np.ones((C, 1, info["n_points_total"])), 8)
    yield ("stokes_quad_p6", fm.StokesVGPFormulation(2).bucket(abi.TOPO_QUAD, 6, 2), mesh.quad_grid(64, 64, 0.1, seed=2),
           lambda info, C: mesh.uniform_coeff(C, info["n_slots"], info["n_points_total"], seed=1), 3)


CONFIGS = {c[0]: c for c in _configs()}


def errors_against_truth(oracle_mod, name):
    """Per sampled cell: GPU and FP64-oracle relative errors against the truth."""
    _, bucket, (nodes, par), mkco, n = CONFIGS[name]
    plan = dlib.Plan(bucket)
    pick = _sample(nodes.shape[0], n)
    co = mkco(plan.info, nodes.shape[0])
    co = None if co is None else co[pick]
    nodes, par = nodes[pick], par[pick]
    dev = lambda x: None if x is None else torch.as_tensor(np.ascontiguousarray(x)).cuda()  # noqa: E731
    out = plan.assemble(dev(nodes), dev(par), dev(co))
    torch.cuda.synchronize()
    got = {k: out[k].cpu().numpy() for k in KEYS}
    assert int((out["info"] != 0).sum()) == 0
    ref = oracle_mod.OraclePlan(bucket).assemble(nodes, par, co)
    truth = oracle_mod.OraclePlan(bucket, xp=True).assemble(nodes, par, co, nthreads=os.cpu_count() or 1)
    e_gpu = {k: np.array([rel_fro(got[k][c], truth[k][c]) for c in range(len(pick))]) for k in KEYS}
    e_orc = {k: np.array([rel_fro(ref[k][c], truth[k][c]) for c in range(len(pick))]) for k in KEYS}
    return e_gpu, e_orc


@pytest.mark.parametrize("name", list(CONFIGS))
def test_gpu_error_bounded_by_the_oracles_own(oracle_mod, name):
    e_gpu, e_orc = errors_against_truth(oracle_mod, name)
    for k in KEYS:
        assert e_gpu[k].max() <= FACTOR * e_orc[k].max() + 1e-13, (k, e_gpu[k].max(), e_orc[k].max())
    if name == "c5_hex48":
        for k in KEYS:
            assert e_gpu[k].max() < 1e-10, (k, e_gpu[k].max())
