"""The uneven-cell Stokes workload generator (mesh.forest_buckets): cell counts per (topology, p)
bucket, counter-clockwise cells, sizes between the finest and the coarsest refinement level,
parities +-1, and a deterministic stream per seed."""
import numpy as np

from camellia2_b200 import mesh


def test_forest_buckets_shapes_and_mix():
    b = mesh.forest_buckets(20_000, seed=5)
    assert sum(n.shape[0] for n, _ in b.values()) == 20_000
    quads = sum(n.shape[0] for (t, _), (n, _) in b.items() if t == 1)
    assert abs(quads / 20_000 - 0.7) < 0.02
    assert sorted(p for (t, p) in b if t == 1) == [1, 2, 3, 4, 5, 6]
    for (topo, p), (nodes, par) in b.items():
        nv = 4 if topo == 1 else 3
        assert nodes.shape[1:] == (nv, 2) and par.shape == (nodes.shape[0], nv)
        assert set(np.unique(par)) <= {-1, 1}
        # counter-clockwise: positive signed area of the first three vertices
        a = nodes[:, 1] - nodes[:, 0]
        c = nodes[:, 2] - nodes[:, 0]
        assert (a[:, 0] * c[:, 1] - a[:, 1] * c[:, 0] > 0).all()
        # edge lengths between the level-4 and level-0 sizes of the 16 x 16 coarse grid (+-10 % jitter)
        h = np.linalg.norm(a, axis=1)
        assert h.min() > 0.7 / (16 * 16) and h.max() < 1.3 / 16


def test_forest_buckets_deterministic():
    a = mesh.forest_buckets(3000, seed=9)
    b = mesh.forest_buckets(3000, seed=9)
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(a[k][0], b[k][0]) and np.array_equal(a[k][1], b[k][1])
