"""The multi-bucket launch (dpg_assemble_multi, dpg_graph_*, dpg_multi_autotune; the loop over
ElementType buckets of TSolution::populateStiffnessAndLoad, Solution.cpp:1131-1297): the
single-CTA buckets share one persistent launch whose CTAs claim cells from a device counter;
each large bucket runs its own persistent launch before the queue.

  * More cells than CTAs, buckets of both kinds, claim sizes 1, 3 and 8: each bucket's
    results equal dpg_assemble on that bucket bit for bit (the same phases in the same order).
  * A captured graph replayed three times, the outputs overwritten before each replay: every
    replay recomputes everything, so the queue's counters were reset at the end of the
    previous launch.
  * dpg_multi_autotune picks a claim size of 1, 2, 4 or 8, and a launch with it is bitwise
    equal to the default."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import lib as dlib  # noqa: E402
from tests.helpers import coeffs_for, poisson2d, poisson3d, stokes2d, stokes_tri  # noqa: E402

pytestmark = pytest.mark.gpu

KEYS = ("K", "l", "S", "s", "info")


def _dev(x):
    return None if x is None else torch.as_tensor(np.ascontiguousarray(x)).cuda()


@pytest.fixture(scope="module")
def buckets():
    """~420 cells in six buckets: Stokes quads p = 2 (single-CTA), 3, 4 (large), triangles
    p = 3 (single-CTA), 5 (large), and 3D Poisson hexes k = 2 (single-CTA)."""
    out = []
    for make, seed in ((lambda: stokes2d(2, 2, 10, 10, 0.1), 1), (lambda: stokes2d(3, 2, 8, 8, 0.1), 2),
                       (lambda: stokes2d(4, 2, 5, 4, 0.1), 3), (lambda: stokes_tri(3, 2, 6, 5, 0.1), 4),
                       (lambda: stokes_tri(5, 2, 3, 3, 0.1), 5), (lambda: poisson3d(2, 1, 4, 0.1), 6)):
        form, bucket, nodes, par = make()
        plan = dlib.Plan(bucket)
        co = coeffs_for(bucket, plan.info, nodes.shape[0], seed=seed)
        out.append((plan, _dev(nodes), _dev(par), _dev(co)))
    refs = [p.assemble(n, q, c) for p, n, q, c in out]
    torch.cuda.synchronize()
    assert sum(n.shape[0] for _, n, _, _ in out) > 2 * 148
    return out, refs


def _items(bs):
    return [(p, n, q, c, {k: v.fill_(7) for k, v in p.alloc_outputs(n.shape[0]).items()}) for p, n, q, c in bs]


def _same(items, refs):
    for (p, n, q, c, out), ref in zip(items, refs):
        for k in KEYS:
            assert torch.equal(out[k], ref[k]), k


@pytest.mark.parametrize("claim", [1, 3, 8])
def test_queue_matches_single_bucket_calls(buckets, claim):
    bs, refs = buckets
    items = _items(bs)
    dlib.assemble_multi(items, claim=claim)
    torch.cuda.synchronize()
    _same(items, refs)


def test_graph_replays_reset_the_queue(buckets):
    bs, refs = buckets
    items = _items(bs)
    g = dlib.Graph(items, claim=2)
    for _ in range(3):
        for *_, out in items:
            for v in out.values():
                v.fill_(7)
        g.launch()
        torch.cuda.synchronize()
        _same(items, refs)
    g.close()


def test_multi_autotune_picks_a_claim(buckets):
    bs, refs = buckets
    items = _items(bs)
    claim = dlib.multi_autotune(items)
    assert claim in (1, 2, 4, 8)
    items = _items(bs)
    dlib.assemble_multi(items, claim=claim)
    torch.cuda.synchronize()
    _same(items, refs)


def test_queue_with_only_large_buckets():
    form, bucket, nodes, par = stokes2d(3, 2, 13, 13, 0.1)
    plan = dlib.Plan(bucket)
    co = coeffs_for(bucket, plan.info, nodes.shape[0], seed=7)
    dn, dp, dc = _dev(nodes), _dev(par), _dev(co)
    ref = plan.assemble(dn, dp, dc)
    items = _items([(plan, dn, dp, dc)])
    dlib.assemble_multi(items, claim=4)
    torch.cuda.synchronize()
    _same(items, [ref])


def test_queue_after_autotuned_plans(buckets):
    """Plans tuned by dpg_plan_autotune (Gram chunk or formation chunk) keep their shapes in
    the queue launch: the queue equals their own dpg_assemble bit for bit."""
    bs, _ = buckets
    tuned = []
    for p, n, q, c in bs[:3]:
        p2 = dlib.Plan(p.holder)
        p2.autotune(n, q, c)
        tuned.append((p2, n, q, c))
    refs = [p.assemble(n, q, c) for p, n, q, c in tuned]
    items = _items(tuned)
    dlib.assemble_multi(items)
    torch.cuda.synchronize()
    _same(items, refs)
