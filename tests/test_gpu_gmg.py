"""Galerkin coarse operators for geometric multigrid (dpg_compose_map).

GMGOperator::computeCoarseStiffnessMatrix (GMGOperator.cpp:173-366) forms P^T A P from
the assembled fine matrix A = sum_c C_c^T S_c C_c.  Here the per-cell maps C_c P are
composed on the device and scattered with the cells' S, s; the result must equal the
dense P^T A P and P^T b built on the host.  The composed map itself is compared entry
by entry (bit for bit: one product per entry) with a host composition."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import lib as dlib  # noqa: E402
from tests.helpers import coeffs_for, poisson2d  # noqa: E402

pytestmark = pytest.mark.gpu


def _dev(x):
    return torch.as_tensor(x).cuda()


def _cells(seed=0):
    form, bucket, nodes, par = poisson2d(2, 2, 3, 3, 0.2)
    plan = dlib.Plan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, plan.info, C)
    out = plan.assemble(*(_dev(x) for x in (nodes, par, co)))
    torch.cuda.synchronize()
    return out["S"].cpu().numpy(), out["s"].cpu().numpy()


def _local_map(C, t, n_fine, rng):
    ptr, gid, w = [0], [], []
    for _ in range(C * t):
        for _ in range(rng.integers(1, 3)):
            gid.append(int(rng.integers(0, n_fine)))
            w.append(float(rng.uniform(0.25, 1.0)))
        ptr.append(len(gid))
    return np.array(ptr, np.int64), np.array(gid, np.int64), np.array(w)


def _prolongation(n_fine, n_coarse, rng, empty_rows=()):
    row_ptr, col, val = [0], [], []
    for r in range(n_fine):
        if r not in empty_rows:
            for c in sorted(rng.choice(n_coarse, size=int(rng.integers(1, 4)), replace=False)):
                col.append(int(c))
                val.append(float(rng.uniform(-1.0, 1.0)))
        row_ptr.append(len(col))
    return np.array(row_ptr, np.int64), np.array(col, np.int64), np.array(val)


def _compose_host(ptr, gid, w, prow, pcol, pval, n_fine):
    optr, ogid, ow = [0], [], []
    for r in range(len(ptr) - 1):
        for k in range(ptr[r], ptr[r + 1]):
            g = gid[k]
            if g < 0 or g >= n_fine:
                continue
            for j in range(prow[g], prow[g + 1]):
                ogid.append(pcol[j])
                ow.append(w[k] * pval[j])
        optr.append(len(ogid))
    return np.array(optr, np.int64), np.array(ogid, np.int64), np.array(ow)


def _dense_fine(S, s, ptr, gid, w, n):
    C, t = S.shape[0], S.shape[1]
    A, b = np.zeros((n, n)), np.zeros(n)
    for c in range(C):
        Cm = np.zeros((t, n))
        for a in range(t):
            for k in range(ptr[c * t + a], ptr[c * t + a + 1]):
                Cm[a, gid[k]] += w[k]
        A += Cm.T @ S[c] @ Cm
        b += Cm.T @ s[c]
    return A, b


def test_composed_map_matches_host_composition():
    rng = np.random.default_rng(3)
    C, t, n_fine, n_coarse = 7, 11, 30, 9
    ptr, gid, w = _local_map(C, t, n_fine, rng)
    prow, pcol, pval = _prolongation(n_fine, n_coarse, rng, empty_rows={4, 17})
    optr, ogid, ow, missing = dlib.compose_map(C, t, _dev(ptr), _dev(gid), _dev(w), n_fine, _dev(prow), _dev(pcol),
                                               _dev(pval))
    torch.cuda.synchronize()
    hptr, hgid, hw = _compose_host(ptr, gid, w, prow, pcol, pval, n_fine)
    assert int(missing.item()) == 0
    assert np.array_equal(optr.cpu().numpy(), hptr)
    assert np.array_equal(ogid.cpu().numpy(), hgid)
    assert np.array_equal(ow.cpu().numpy(), hw)


def test_coarse_operator_equals_pt_a_p():
    S, s = _cells()
    C, t = S.shape[0], S.shape[1]
    rng = np.random.default_rng(5)
    n_fine, n_coarse = 40, 14
    ptr, gid, w = _local_map(C, t, n_fine, rng)
    prow, pcol, pval = _prolongation(n_fine, n_coarse, rng)
    A, b = _dense_fine(S, s, ptr, gid, w, n_fine)
    P = np.zeros((n_fine, n_coarse))
    for r in range(n_fine):
        P[r, pcol[prow[r]:prow[r + 1]]] = pval[prow[r]:prow[r + 1]]
    Ac, bc = P.T @ A @ P, P.T @ b
    optr, ogid, ow, missing = dlib.compose_map(C, t, _dev(ptr), _dev(gid), _dev(w), n_fine, _dev(prow), _dev(pcol),
                                               _dev(pval))
    # full coarse graph
    row_ptr = np.arange(0, n_coarse * n_coarse + 1, n_coarse, dtype=np.int64)
    col = np.tile(np.arange(n_coarse, dtype=np.int64), n_coarse)
    vals = torch.zeros(col.shape[0], dtype=torch.float64, device="cuda")
    rhs = torch.zeros(n_coarse, dtype=torch.float64, device="cuda")
    miss2 = dlib.scatter_global(_dev(S), _dev(s), optr, ogid, ow, n_coarse, _dev(row_ptr), _dev(col), vals, rhs)
    torch.cuda.synchronize()
    assert int(missing.item()) == 0 and int(miss2.item()) == 0
    Ag = vals.cpu().numpy().reshape(n_coarse, n_coarse)
    assert np.linalg.norm(Ag - Ac) <= 1e-12 * np.linalg.norm(Ac)
    assert np.linalg.norm(rhs.cpu().numpy() - bc) <= 1e-12 * np.linalg.norm(bc)


def test_out_of_range_fine_ids_are_counted_and_skipped():
    rng = np.random.default_rng(9)
    C, t, n_fine, n_coarse = 3, 5, 12, 4
    ptr, gid, w = _local_map(C, t, n_fine, rng)
    gid = gid.copy()
    gid[0], gid[3] = -1, n_fine + 2
    prow, pcol, pval = _prolongation(n_fine, n_coarse, rng)
    optr, ogid, ow, missing = dlib.compose_map(C, t, _dev(ptr), _dev(gid), _dev(w), n_fine, _dev(prow), _dev(pcol),
                                               _dev(pval))
    torch.cuda.synchronize()
    hptr, hgid, hw = _compose_host(ptr, gid, w, prow, pcol, pval, n_fine)
    assert int(missing.item()) == 2
    assert np.array_equal(optr.cpu().numpy(), hptr)
    assert np.array_equal(ogid.cpu().numpy(), hgid)


def test_row_offsets_past_two_scan_levels():
    """More than 4096^2 local rows: the offsets take two levels of block scans."""
    rows = 4096 * 4096 + 12345
    t = 5
    C = rows // t
    rows = C * t
    g = torch.Generator(device="cuda").manual_seed(0)
    n_fine = 1000
    lens = torch.randint(0, 3, (rows,), device="cuda", generator=g, dtype=torch.int64)
    ptr = torch.zeros(rows + 1, dtype=torch.int64, device="cuda")
    ptr[1:] = torch.cumsum(lens, 0)
    nnz = int(ptr[-1].item())
    gid = torch.randint(0, n_fine, (nnz,), device="cuda", generator=g, dtype=torch.int64)
    plen = torch.randint(0, 4, (n_fine,), device="cuda", generator=g, dtype=torch.int64)
    prow = torch.zeros(n_fine + 1, dtype=torch.int64, device="cuda")
    prow[1:] = torch.cumsum(plen, 0)
    L = dlib.load()
    import ctypes as ct
    out_ptr = torch.empty(rows + 1, dtype=torch.int64, device="cuda")
    n = ct.c_int64(0)
    dlib._check(L.dpg_compose_map(C, t, dlib._ptr(ptr), dlib._ptr(gid), None, n_fine, dlib._ptr(prow), None, None,
                                  dlib._ptr(out_ptr), None, None, 0, ct.byref(n), None,
                                  dlib._stream_ptr(None)))
    per_entry = plen[gid]
    row_of_entry = torch.repeat_interleave(torch.arange(rows, device="cuda"), lens)
    cnt = torch.zeros(rows, dtype=torch.int64, device="cuda").index_add_(0, row_of_entry, per_entry)
    want = torch.zeros(rows + 1, dtype=torch.int64, device="cuda")
    want[1:] = torch.cumsum(cnt, 0)
    assert torch.equal(out_ptr, want)
    assert n.value == int(want[-1].item())
