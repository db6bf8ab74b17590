"""CUDA path (through the C-ABI) against the CPU oracle on the same seeded inputs.

Tolerance: relative Frobenius error <= 1e-12 per cell for K, l, S, s (the FP64
bar of the north star), <= 1e-13 for the quadrature products G, B, F.  Where a
cell's Gram matrix is so ill-conditioned that two FP64 codes cannot agree to 1e-12
(test degree 6), both are compared with the extended-precision truth (the oracle
in __float128): the GPU's error there is at most three times the FP64 oracle's own."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import abi, lib as dlib, mesh  # noqa: E402
from tests.conftest import rel_fro  # noqa: E402
from tests.helpers import (cdr2d, check_against_truth, coeffs_for, fp64_floor, poisson2d, poisson3d,  # noqa: E402,F401
                           poisson_tri, stokes2d, stokes_tri)

pytestmark = pytest.mark.gpu

CASES = {
    "poisson2d_k2_dk2": lambda: poisson2d(2, 2, 3, 3, 0.2),       # c1 shapes (N=65, M=32)
    "poisson2d_k4_dk2": lambda: poisson2d(4, 2, 2, 3, 0.2),       # c2 shapes (N=133, M=84)
    "cdr2d_k3_dk2": lambda: cdr2d(3, 2, 3, 2, 0.1),               # c4 shapes (N=96, M=55)
    "poisson3d_k2_dk1": lambda: poisson3d(2, 1, 2, 0.1),          # c5 shapes (N=172, M=110)
    "poisson2d_k1_dk1": lambda: poisson2d(1, 1, 2, 2, 0.1),       # smallest bucket
    "poisson3d_k1_dk2": lambda: poisson3d(1, 2, 2, 0.1),
    "stokes2d_k1_dk2": lambda: stokes2d(1, 2, 2, 2, 0.1),         # c3 quad p=1 (N=96, M=31)
    "stokes2d_k2_dk2": lambda: stokes2d(2, 2, 2, 1, 0.1),         # c3 quad p=2 (N=155, M=68)
    "poisson_tri_k2_dk2": lambda: poisson_tri(2, 2, 2, 2, 0.15),  # triangles (N=39, M=24)
    "poisson_tri_k4_dk2": lambda: poisson_tri(4, 2, 2, 1, 0.15),
    "stokes_tri_k1_dk2": lambda: stokes_tri(1, 2, 2, 1, 0.1),     # c3 tri p=1 (N=60)
    "stokes_tri_k3_dk2": lambda: stokes_tri(3, 2, 1, 1, 0.1),     # c3 tri p=3 (N=133)
}


def _dev(a, dtype=None):
    t = torch.as_tensor(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


@pytest.fixture(scope="module")
def cases(oracle_mod):
    out = {}
    for name, make in CASES.items():
        form, bucket, nodes, par = make()
        P = oracle_mod.OraclePlan(bucket)
        C = nodes.shape[0]
        co = coeffs_for(bucket, P.info, C)
        ref = P.assemble(nodes, par, co, parts=True)
        out[name] = (bucket, nodes, par, co, ref, P.info)
    return out


@pytest.mark.parametrize("name", list(CASES))
def test_parts_match_oracle(cases, name):
    bucket, nodes, par, co, ref, info = cases[name]
    plan = dlib.Plan(bucket)
    assert plan.info == {**info, "precision": plan.info["precision"]}
    G, B, F = plan.parts(_dev(nodes), _dev(par), None if co is None else _dev(co))
    torch.cuda.synchronize()
    G, B, F = G.cpu().numpy(), B.cpu().numpy(), F.cpu().numpy()
    for c in range(nodes.shape[0]):
        assert rel_fro(G[c], ref["G"][c]) < 1e-13
        assert rel_fro(B[c], ref["B"][c]) < 1e-13
        assert rel_fro(F[c], ref["F"][c]) < 1e-13


@pytest.mark.parametrize("name", list(CASES))
def test_assemble_matches_oracle(cases, name, oracle_mod):
    bucket, nodes, par, co, ref, info = cases[name]
    plan = dlib.Plan(bucket)
    out = plan.assemble(_dev(nodes), _dev(par), None if co is None else _dev(co))
    torch.cuda.synchronize()
    o = {k: v.cpu().numpy() for k, v in out.items()}
    assert (o["info"] == 0).all()
    check_against_truth(oracle_mod, bucket, nodes, par, co, o, ref)


def test_host_api_matches_device_api(cases):
    bucket, nodes, par, co, ref, info = cases["poisson3d_k2_dk1"]
    plan = dlib.Plan(bucket)
    h = plan.assemble_host(nodes, par, co)
    d = plan.assemble(_dev(nodes), _dev(par), _dev(co))
    torch.cuda.synchronize()
    for k in ("K", "l", "S", "s", "info"):
        assert np.array_equal(h[k], d[k].cpu().numpy()), k


@pytest.mark.parametrize("flags,kept", [(1, ("S", "s", "info")), (2, ("K", "l", "info"))])
def test_host_api_output_flags(cases, flags, kept):
    """DPG_FLAG_NO_K (1) returns S, s alone, DPG_FLAG_NO_CONDENSE (2) K, l alone; what is
    returned equals the full call bit for bit."""
    bucket, nodes, par, co, ref, info = cases["poisson3d_k2_dk1"]
    plan = dlib.Plan(bucket)
    full = plan.assemble_host(nodes, par, co)
    part = {k: (np.empty_like(full[k]) if k in kept else None) for k in ("K", "l", "S", "s", "info")}
    plan.assemble_host(nodes, par, co, out=part, flags=flags)
    for k in kept:
        assert np.array_equal(part[k], full[k]), k


def test_empty_batch_is_ok(cases):
    bucket, nodes, par, co, ref, info = cases["poisson2d_k2_dk2"]
    plan = dlib.Plan(bucket)
    out = plan.assemble(_dev(nodes[:0]), _dev(par[:0]), _dev(co[:0]))
    torch.cuda.synchronize()
    assert out["K"].shape[0] == 0


@pytest.mark.parametrize("G,Bt,F,Kx,lx", [
    ([[1, .5, 0], [.5, 1, 2], [0, 2, 8]], [[3, 1, 2], [2, 0, 2]], [1, 2, 3], [[13.5, 12.5], [12.5, 13.5]],
     [0.75, -1.75]),
    ([[1, .5], [.5, 1]], [[3, 1], [2, 0]], [1, 2], [[28 / 3, 20 / 3], [20 / 3, 16 / 3]], [2, 0]),
    ([[2, 0], [0, 4]], [[3, 1], [2, 0]], [1, 2], [[4.75, 3], [3, 2]], [2, 1]),
])
def test_factored_cholesky_golden_gpu(G, Bt, F, Kx, lx):
    """BFTests.cpp:136-381 golden matrices through dpg_factored_cholesky_solve."""
    Gt = _dev(np.array([G], float))
    Bt_ = _dev(np.array([Bt], float))
    Ft = _dev(np.array([F], float))
    K, l, info = dlib.factoredCholeskySolve(Gt, Bt_, Ft)
    torch.cuda.synchronize()
    assert int(info[0]) == 0
    assert np.allclose(K[0].cpu().numpy(), Kx, rtol=1e-14, atol=1e-14)
    assert np.allclose(l[0].cpu().numpy(), lx, rtol=1e-14, atol=1e-14)


def test_factored_cholesky_random_batch(oracle_mod):
    rng = np.random.default_rng(5)
    C, N, M = 7, 45, 21
    A = rng.normal(size=(C, N, N))
    G = A @ A.transpose(0, 2, 1) + N * np.eye(N)
    B = rng.normal(size=(C, M, N))
    F = rng.normal(size=(C, N))
    K, l, info = dlib.factoredCholeskySolve(_dev(G), _dev(B), _dev(F))
    torch.cuda.synchronize()
    for c in range(C):
        Kr, lr, ir = oracle_mod.factored_cholesky_solve(G[c], B[c], F[c])
        assert rel_fro(K[c].cpu().numpy(), Kr) < 1e-13
        assert rel_fro(l[c].cpu().numpy(), lr) < 1e-13


def test_non_spd_gram_reports_info():
    """A Gram matrix with a non-positive leading minor: info = DPOTRF's INFO, no error."""
    G = np.array([np.diag([1.0, -1.0, 2.0]), np.eye(3)])
    B = np.array([np.eye(3), np.eye(3)])
    F = np.ones((2, 3))
    K, l, info = dlib.factoredCholeskySolve(_dev(G), _dev(B), _dev(F))
    torch.cuda.synchronize()
    assert info.cpu().tolist() == [2, 0]


def test_invalid_descriptor_is_rejected():
    h = abi.DescHolder(abi.TOPO_QUAD, [(abi.VAR_FIELD, abi.SPACE_HGRAD, 2)], [(abi.VAR_TEST, abi.SPACE_HGRAD, 2)],
                       [], [], [], 4, 4, 4, 0)
    with pytest.raises(dlib.DpgError) as e:
        dlib.Plan(h)
    assert e.value.code == abi.DPG_ERR_INVALID_ARGUMENT


def test_mixed_precision_is_refused():
    """No mixed-precision form is built: a plan asking for one is refused with
    DPG_ERR_UNSUPPORTED instead of silently running the FP64 form."""
    from camellia2_b200 import formulation as fm
    bucket = fm.PoissonFormulation(3).bucket(abi.TOPO_HEX, 2, 1, precision=abi.PREC_MIXED)
    with pytest.raises(dlib.DpgError) as e:
        dlib.Plan(bucket)
    assert e.value.code == abi.DPG_ERR_UNSUPPORTED
    assert "DPG_PREC_MIXED" in str(e.value)
