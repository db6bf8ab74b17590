"""Large buckets (N > 192 or M > 120 after padding: the Stokes VGP quads p >= 3 and
triangles p >= 4 of the uneven-cell workload, 2D Poisson k = 6, 3D Poisson k = 3) through
the C-ABI against the CPU oracle on the same seeded inputs.

Tolerance as in test_gpu_parity: relative Frobenius error <= 1e-12 per cell for K, l, S, s;
where a cell's Gram matrix puts two FP64 codes further apart, the GPU's error against the
extended-precision truth is at most three times the FP64 oracle's own."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import lib as dlib  # noqa: E402
from tests.conftest import rel_fro  # noqa: E402
from tests.helpers import check_against_truth, coeffs_for, poisson2d, poisson3d, stokes2d, stokes_tri  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = {
    "stokes2d_k3_dk2": lambda: stokes2d(3, 2, 2, 1, 0.1),       # N=228, M=119
    "stokes2d_k4_dk2": lambda: stokes2d(4, 2, 2, 1, 0.1),       # N=315, M=184
    "stokes2d_k5_dk2": lambda: stokes2d(5, 2, 1, 1, 0.1),       # N=416, M=263
    "stokes2d_k6_dk2": lambda: stokes2d(6, 2, 1, 1, 0.1),       # N=531, M=356
    "stokes_tri_k4_dk2": lambda: stokes_tri(4, 2, 1, 1, 0.1),   # N=180 (triangles)
    "stokes_tri_k6_dk2": lambda: stokes_tri(6, 2, 1, 1, 0.1),   # N=295, M=225
    "poisson2d_k6_dk1": lambda: poisson2d(6, 1, 2, 1, 0.2),     # N=176 but M=160: large by M
    "poisson3d_k3_dk1": lambda: poisson3d(3, 1, 1, 0.1),        # N=365, M=258 (3D alternative)
}


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def _check(oracle_mod, o, ref, bucket, nodes, par, co):
    assert (o["info"] == 0).all()
    check_against_truth(oracle_mod, bucket, nodes, par, co, o, ref)


@pytest.mark.parametrize("name", list(CASES))
def test_big_bucket_matches_oracle(name, oracle_mod):
    form, bucket, nodes, par = CASES[name]()
    P = oracle_mod.OraclePlan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, P.info, C)
    ref = P.assemble(nodes, par, co, parts=True)
    plan = dlib.Plan(bucket)
    assert plan.info == {**P.info, "precision": plan.info["precision"]}
    out = plan.assemble(_dev(nodes), _dev(par), None if co is None else _dev(co))
    torch.cuda.synchronize()
    _check(oracle_mod, {k: v.cpu().numpy() for k, v in out.items()}, ref, bucket, nodes, par, co)


def test_big_bucket_many_cells(oracle_mod):
    """More cells than CTAs: every CTA reuses its workspace for several cells."""
    form, bucket, nodes, par = stokes2d(3, 2, 20, 16, 0.15, seed=3)
    P = oracle_mod.OraclePlan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, P.info, C)
    ref = P.assemble(nodes, par, co, parts=True)
    plan = dlib.Plan(bucket)
    out = plan.assemble(_dev(nodes), _dev(par), _dev(co))
    torch.cuda.synchronize()
    _check(oracle_mod, {k: v.cpu().numpy() for k, v in out.items()}, ref, bucket, nodes, par, co)


def test_big_bucket_host_api_and_flags(oracle_mod):
    """Host buffers give the device call's results bit for bit; DPG_FLAG_NO_K returns S, s
    alone and DPG_FLAG_NO_CONDENSE K, l alone, equal to the full call."""
    form, bucket, nodes, par = stokes2d(4, 2, 2, 2, 0.1)
    C = nodes.shape[0]
    plan = dlib.Plan(bucket)
    co = coeffs_for(bucket, plan.info, C)
    d = plan.assemble(_dev(nodes), _dev(par), _dev(co))
    torch.cuda.synchronize()
    h = plan.assemble_host(nodes, par, co)
    for k in ("K", "l", "S", "s", "info"):
        assert np.array_equal(h[k], d[k].cpu().numpy()), k
    for flags, kept in ((1, ("S", "s", "info")), (2, ("K", "l", "info"))):
        part = {k: (np.empty_like(h[k]) if k in kept else None) for k in ("K", "l", "S", "s", "info")}
        plan.assemble_host(nodes, par, co, out=part, flags=flags)
        for k in kept:
            assert np.array_equal(part[k], h[k]), (flags, k)


def test_big_bucket_rejects_unsupported_entry_points():
    """Entry points the large-bucket kernel does not provide fail with DPG_ERR_UNSUPPORTED."""
    form, bucket, nodes, par = stokes2d(3, 2, 1, 1, 0.1)
    plan = dlib.Plan(bucket)
    co = coeffs_for(bucket, plan.info, 1)
    M = plan.info["M"]
    with pytest.raises(dlib.DpgError) as ei:
        plan.adjoint(_dev(nodes), _dev(par), _dev(co), _dev(np.eye(M)[None]), _dev(np.ones((1, M))))
    assert ei.value.code == 2


@pytest.mark.parametrize("name", ["stokes2d_k6_dk2", "stokes_tri_k4_dk2", "poisson3d_k3_dk1"])
def test_big_bucket_parts_match_oracle(name, oracle_mod):
    """dpg_assemble_parts on large buckets: G, B, F to 1e-13 relative Frobenius per cell."""
    form, bucket, nodes, par = CASES[name]()
    P = oracle_mod.OraclePlan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, P.info, C)
    ref = P.assemble(nodes, par, co, parts=True)
    plan = dlib.Plan(bucket)
    G, B, F = plan.parts(_dev(nodes), _dev(par), None if co is None else _dev(co))
    torch.cuda.synchronize()
    G, B, F = G.cpu().numpy(), B.cpu().numpy(), F.cpu().numpy()
    for c in range(C):
        assert rel_fro(G[c], ref["G"][c]) < 1e-13
        assert rel_fro(B[c], ref["B"][c]) < 1e-13
        assert rel_fro(F[c], ref["F"][c]) < 1e-13


def _mixed_buckets():
    """Single-CTA and large Stokes VGP buckets together (quads p = 2, 3, 5; triangles p = 3, 6)."""
    out = []
    for make, seed in ((lambda: stokes2d(2, 2, 2, 2, 0.1), 1), (lambda: stokes2d(3, 2, 3, 2, 0.1), 2),
                       (lambda: stokes_tri(3, 2, 2, 1, 0.1), 3), (lambda: stokes2d(5, 2, 2, 1, 0.1), 4),
                       (lambda: stokes_tri(6, 2, 1, 1, 0.1), 5)):
        form, bucket, nodes, par = make()
        plan = dlib.Plan(bucket)
        co = coeffs_for(bucket, plan.info, nodes.shape[0], seed=seed)
        out.append((plan, _dev(nodes), _dev(par), _dev(co)))
    return out


def test_multi_and_graph_with_large_buckets():
    """dpg_assemble_multi and a captured graph over single-CTA and large buckets reproduce
    dpg_assemble bucket by bucket, bit for bit, also after new coefficients are written into
    the captured buffers."""
    bs = _mixed_buckets()
    refs = [p.assemble(n, q, c) for p, n, q, c in bs]
    items = [(p, n, q, c, {k: v.fill_(7) for k, v in p.alloc_outputs(n.shape[0]).items()}) for p, n, q, c in bs]
    dlib.assemble_multi(items)
    torch.cuda.synchronize()
    for (p, n, q, c, out), ref in zip(items, refs):
        for k in ("K", "l", "S", "s", "info"):
            assert torch.equal(out[k], ref[k]), k
    g = dlib.Graph(items)
    for p, n, q, c, out in items:
        c.mul_(1.5).add_(0.1)
    g.launch()
    torch.cuda.synchronize()
    for p, n, q, c, out in items:
        ref = p.assemble(n, q, c)
        for k in ("K", "l", "S", "s", "info"):
            assert torch.equal(out[k], ref[k]), k
    g.close()


@pytest.mark.parametrize("name", ["stokes2d_k3_dk2", "stokes2d_k6_dk2", "stokes_tri_k4_dk2"])
def test_big_bucket_energy_error_matches_oracle(name, oracle_mod):
    """dpg_energy_error on large buckets: sqrt(r^T G^-1 r), r = F - B x, for random local trial
    coefficients x, against a dense solve with the oracle's G, B, F (1e-10 relative)."""
    form, bucket, nodes, par = CASES[name]()
    plan = dlib.Plan(bucket)
    C, M = nodes.shape[0], plan.info["M"]
    co = coeffs_for(bucket, plan.info, C)
    x = np.random.default_rng(4).normal(size=(C, M))
    e, info = plan.energy_error(_dev(nodes), _dev(par), _dev(co), _dev(x))
    torch.cuda.synchronize()
    assert int(info.abs().max()) == 0
    e = e.cpu().numpy()
    G, B, F = oracle_mod.OraclePlan(bucket).parts(nodes, par, co)
    for c in range(C):
        r = F[c] - B[c].T @ x[c]
        ref = np.sqrt(r @ np.linalg.solve(G[c], r))
        assert abs(e[c] - ref) <= 1e-10 * ref, (c, e[c], ref)


@pytest.mark.parametrize("make", [lambda: stokes2d(3, 2, 2, 2, 0.1), lambda: stokes2d(6, 2, 2, 1, 0.1),
                                  lambda: poisson2d(2, 2, 2, 2, 0.1)],
                         ids=["large_k3", "large_k6", "single_cta"])
def test_failed_factorisation_reports_the_oracle_info(make, oracle_mod):
    """A cell mirrored in x has det J < 0: its Gram matrix is negative definite, the factored
    Cholesky fails at the first pivot, and info holds the same 1-based column as the oracle's
    (DPOTRF INFO).  The other cells' outputs are bitwise those of a run without the bad cell."""
    form, bucket, nodes, par = make()
    P = oracle_mod.OraclePlan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, P.info, C)
    bad = nodes.copy()
    bad[1, :, 0] = -bad[1, :, 0]
    ref = P.assemble(bad, par, co)
    plan = dlib.Plan(bucket)
    dco = None if co is None else _dev(co)
    good = {k: v.cpu().numpy() for k, v in plan.assemble(_dev(nodes), _dev(par), dco).items()}
    out = {k: v.cpu().numpy() for k, v in plan.assemble(_dev(bad), _dev(par), dco).items()}
    torch.cuda.synchronize()
    assert ref["info"][1] != 0
    assert out["info"][1] == ref["info"][1]
    keep = np.arange(C) != 1
    assert (out["info"][keep] == 0).all() and (ref["info"][keep] == 0).all()
    for k in ("K", "l", "S", "s"):
        assert np.array_equal(out[k][keep], good[k][keep]), k
