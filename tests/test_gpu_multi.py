"""Multi-bucket assembly in one persistent launch (dpg_assemble_multi: the loop over
ElementType buckets of TSolution::populateStiffnessAndLoad, Solution.cpp:1131-1297)
and its CUDA-graph replay (dpg_graph_capture / dpg_graph_launch).  Both must
reproduce dpg_assemble bucket by bucket: the same phases run in the same order,
so the results are bitwise equal."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import lib as dlib  # noqa: E402
from tests.helpers import cdr2d, coeffs_for, poisson2d, poisson_tri, stokes_tri  # noqa: E402

pytestmark = pytest.mark.gpu


def _buckets():
    out = []
    for make, seed in ((lambda: poisson2d(2, 2, 3, 2, 0.2), 1), (lambda: cdr2d(3, 2, 2, 2, 0.1), 2),
                       (lambda: poisson_tri(2, 2, 2, 2, 0.1), 3), (lambda: stokes_tri(1, 2, 2, 1, 0.1), 4)):
        form, bucket, nodes, par = make()
        plan = dlib.Plan(bucket)
        C = nodes.shape[0]
        co = coeffs_for(bucket, plan.info, C, seed=seed)
        dev = lambda x: None if x is None else torch.as_tensor(x).cuda()  # noqa: E731
        out.append((plan, dev(nodes), dev(par), dev(co)))
    return out


def _fill(out):
    for v in out.values():
        v.fill_(7)
    return out


def test_multi_matches_per_bucket():
    bs = _buckets()
    refs = [p.assemble(n, q, c) for p, n, q, c in bs]
    items = [(p, n, q, c, _fill(p.alloc_outputs(n.shape[0]))) for p, n, q, c in bs]
    dlib.assemble_multi(items)
    torch.cuda.synchronize()
    for (p, n, q, c, out), ref in zip(items, refs):
        for k in ("K", "l", "S", "s", "info"):
            assert torch.equal(out[k], ref[k]), k


def test_graph_replays_with_new_coefficients():
    bs = _buckets()
    items = [(p, n, q, c, _fill(p.alloc_outputs(n.shape[0]))) for p, n, q, c in bs]
    g = dlib.Graph(items)
    g.launch()
    torch.cuda.synchronize()
    for p, n, q, c, out in items:
        ref = p.assemble(n, q, c)
        assert torch.equal(out["K"], ref["K"]) and torch.equal(out["S"], ref["S"])
    # new coefficients in the same buffers, replay
    for p, n, q, c, out in items:
        if c is not None:
            c.mul_(1.5).add_(0.1)
    g.launch()
    torch.cuda.synchronize()
    for p, n, q, c, out in items:
        ref = p.assemble(n, q, c)
        assert torch.equal(out["K"], ref["K"]) and torch.equal(out["l"], ref["l"])
    g.close()


def test_multi_rejects_missing_coefficients():
    p, n, q, c = _buckets()[1]  # CDR: five coefficient slots
    with pytest.raises(dlib.DpgError):
        dlib.assemble_multi([(p, n, q, None, p.alloc_outputs(n.shape[0]))])
