"""The conforming-shaped trace map of the hex grid (mesh.hex_trace_map): the counts a
conforming GDA numbering of the k=2 hex Poisson UW traces has."""
import numpy as np

from camellia2_b200 import mesh


def test_hex_trace_map_counts():
    nx, ny, nz, k = 3, 2, 4, 2
    gid, n = mesh.hex_trace_map(nx, ny, nz, k)
    C = nx * ny * nz
    assert gid.shape == (C, 6 * (k + 1) ** 2 + 6 * k * k)
    # each cell: the (k+1)^3 - (k-1)^3 lattice points of its boundary plus 6 k^2 flux dofs
    assert all(len(np.unique(g)) == (k + 1) ** 3 - (k - 1) ** 3 + 6 * k * k for g in gid)
    lattice = (k * nx + 1) * (k * ny + 1) * (k * nz + 1) - C * (k - 1) ** 3
    faces = (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1)
    assert n == lattice + faces * k * k
    assert gid.min() == 0 and gid.max() == n - 1


def test_hex_trace_map_shares_faces_between_neighbours():
    gid, _ = mesh.hex_trace_map(2, 1, 1, 2)
    # cell 0's face x+ (face 1) is cell 1's face x- (face 0): same H1 points, same flux dofs
    h1 = lambda c, f: gid[c, 9 * f:9 * f + 9]  # noqa: E731
    fl = lambda c, f: gid[c, 54 + 4 * f:54 + 4 * f + 4]  # noqa: E731
    assert np.array_equal(h1(0, 1), h1(1, 0))
    assert np.array_equal(fl(0, 1), fl(1, 0))
    assert not set(fl(0, 0)) & set(fl(1, 1))
