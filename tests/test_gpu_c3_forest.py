"""The uneven-cell Stokes VGP workload at its full size (mesh.forest_buckets: 100,000 cells,
70 % quads and 30 % triangles, p uniform on 1..6, Delta p = 2, refinement levels 0..4; the
bench's seed), all twelve (topology, p) buckets in ONE dpg_assemble_multi call: the single-CTA
buckets through the work queue, the large buckets on the large-bucket kernel.

  - every cell's Gram matrix factors (info == 0);
  - K and S are symmetric to roundoff in every bucket;
  - one seeded cell per bucket matches the FP64 oracle to 1e-12 or, where the cell's Gram
    conditioning puts two FP64 codes further apart, the GPU's error against the
    extended-precision truth is at most three times the FP64 oracle's own.

Only the sampled cells leave the GPU."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import formulation as fm, lib as dlib, mesh  # noqa: E402
from tests.helpers import check_against_truth  # noqa: E402

pytestmark = pytest.mark.gpu


def _max_asym(X, step=4096):
    worst = 0.0
    for c0 in range(0, X.shape[0], step):
        x = X[c0:c0 + step]
        d = (x - x.transpose(1, 2)).abs().amax(dim=(1, 2)) / x.abs().amax(dim=(1, 2)).clamp_min(1e-300)
        worst = max(worst, float(d.max()))
    return worst


def test_c3_forest_full_size(oracle_mod):
    form = fm.StokesVGPFormulation(2)
    rng = np.random.default_rng(11)
    items, host = [], []
    for (topo, p), (nodes, par) in mesh.forest_buckets(100_000, seed=7).items():
        bucket = form.bucket(topo, p, 2)
        plan = dlib.Plan(bucket)
        C = nodes.shape[0]
        co = mesh.uniform_coeff(C, plan.info["n_slots"], plan.info["n_points_total"], seed=p)
        dev = [torch.as_tensor(np.ascontiguousarray(x)).cuda() for x in (nodes, par, co)]
        items.append((plan, *dev, plan.alloc_outputs(C)))
        host.append((bucket, nodes, par, co, int(rng.integers(0, C))))
    assert sum(it[1].shape[0] for it in items) == 100_000
    assert any(it[0].info["N"] > 192 for it in items) and any(it[0].info["N"] <= 192 for it in items)
    dlib.assemble_multi(items)
    torch.cuda.synchronize()
    for (plan, dn, dp, dc, out), (bucket, nodes, par, co, c) in zip(items, host):
        assert int((out["info"] != 0).sum()) == 0
        assert _max_asym(out["K"]) < 1e-12
        assert _max_asym(out["S"]) < 1e-12
        got = {k: out[k][c:c + 1].cpu().numpy() for k in ("K", "l", "S", "s")}
        sl = slice(c, c + 1)
        ref = oracle_mod.OraclePlan(bucket).assemble(nodes[sl], par[sl], co[sl])
        check_against_truth(oracle_mod, bucket, nodes[sl], par[sl], co[sl], got, ref)
