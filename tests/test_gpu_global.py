"""Global assembly of the condensed cell systems (dpg_scatter_global; the GDA
interpretation C^T S C of GDAMinimumRule::interpretLocalData, GDAMinimumRule.cpp:
714-800, and the insertion of Solution.cpp:1263-1293) on a caller-owned CSR graph.

The cells' S, s come from the GPU assembly of a 2D Poisson mesh; each local trace dof
maps to one or two global dofs with weights (as hanging-node constraints do).  The
CSR values and the right-hand side must equal a dense accumulation of C^T S C and
C^T s on the host; entries outside the graph are counted, not written."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import lib as dlib  # noqa: E402
from tests.helpers import coeffs_for, poisson2d  # noqa: E402

pytestmark = pytest.mark.gpu


def _setup(seed=0):
    form, bucket, nodes, par = poisson2d(2, 2, 3, 3, 0.2)
    plan = dlib.Plan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, plan.info, C)
    out = plan.assemble(*(torch.as_tensor(x).cuda() for x in (nodes, par, co)))
    torch.cuda.synchronize()
    S, s = out["S"].cpu().numpy(), out["s"].cpu().numpy()
    t = S.shape[1]
    rng = np.random.default_rng(seed)
    n = 40
    ptr, gid, w = [0], [], []
    for c in range(C):
        for a in range(t):
            for _ in range(rng.integers(1, 3)):
                gid.append(int(rng.integers(0, n)))
                w.append(float(rng.uniform(0.25, 1.0)))
            ptr.append(len(gid))
    return S, s, np.array(ptr), np.array(gid), np.array(w), n


def _dense(S, s, ptr, gid, w, n):
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


def _graph(A, drop=None):
    rows, cols = np.nonzero(np.ones_like(A, dtype=bool) if drop is None else ~drop)
    row_ptr = np.zeros(A.shape[0] + 1, dtype=np.int64)
    np.add.at(row_ptr, rows + 1, 1)
    return np.cumsum(row_ptr), cols.astype(np.int64)


def test_scatter_matches_dense_accumulation():
    S, s, ptr, gid, w, n = _setup()
    A, b = _dense(S, s, ptr, gid, w, n)
    row_ptr, col = _graph(A)
    dev = lambda x: torch.as_tensor(x).cuda()  # noqa: E731
    vals = torch.zeros(col.shape[0], dtype=torch.float64, device="cuda")
    rhs = torch.zeros(n, dtype=torch.float64, device="cuda")
    missing = dlib.scatter_global(dev(S), dev(s), dev(ptr), dev(gid), dev(w), n, dev(row_ptr), dev(col), vals, rhs)
    torch.cuda.synchronize()
    assert int(missing.item()) == 0
    Ag = np.zeros((n, n))
    v = vals.cpu().numpy()
    for r in range(n):
        Ag[r, col[row_ptr[r]:row_ptr[r + 1]]] = v[row_ptr[r]:row_ptr[r + 1]]
    assert np.linalg.norm(Ag - A) <= 1e-12 * np.linalg.norm(A)
    assert np.linalg.norm(rhs.cpu().numpy() - b) <= 1e-12 * np.linalg.norm(b)


def test_entries_outside_the_graph_are_counted():
    S, s, ptr, gid, w, n = _setup(1)
    A, b = _dense(S, s, ptr, gid, w, n)
    drop = np.zeros((n, n), dtype=bool)
    drop[0, :] = True  # row 0 absent from the graph
    row_ptr, col = _graph(A, drop)
    gid = gid.copy()
    gid[0] = n + 5  # an index outside the system
    dev = lambda x: torch.as_tensor(x).cuda()  # noqa: E731
    vals = torch.zeros(col.shape[0], dtype=torch.float64, device="cuda")
    missing = dlib.scatter_global(dev(S), dev(s), dev(ptr), dev(gid), dev(w), n, dev(row_ptr), dev(col), vals)
    torch.cuda.synchronize()
    assert int(missing.item()) > 0
    assert np.isfinite(vals.cpu().numpy()).all()


def test_scatter_hex_conforming_map_matches_dense():
    """The hex grid's conforming-shaped trace map (each trace point shared by the faces and
    cells that touch it): the per-cell condensation onto distinct global dofs must give the
    dense C^T S C accumulation."""
    from camellia2_b200 import mesh
    from tests.helpers import poisson3d
    n = 3
    form, bucket, nodes, par = poisson3d(2, 1, n, 0.1)
    plan = dlib.Plan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, plan.info, C)
    out = plan.assemble(*(torch.as_tensor(x).cuda() for x in (nodes, par, co)))
    torch.cuda.synchronize()
    S, s = out["S"].cpu().numpy(), out["s"].cpu().numpy()
    t = S.shape[1]
    g, ng = mesh.hex_trace_map(n, n, n, 2)
    ptr = np.arange(C * t + 1, dtype=np.int64)
    gid = g.reshape(-1)
    w = np.ones(C * t)
    A, b = _dense(S, s, ptr, gid, w, ng)
    pattern = np.zeros((ng, ng), dtype=bool)
    for c in range(C):
        pattern[np.ix_(g[c], g[c])] = True
    row_ptr, col = _graph(A, ~pattern)
    dev = lambda x: torch.as_tensor(x).cuda()  # noqa: E731
    vals = torch.zeros(col.shape[0], dtype=torch.float64, device="cuda")
    rhs = torch.zeros(ng, dtype=torch.float64, device="cuda")
    missing = dlib.scatter_global(dev(S), dev(s), dev(ptr), dev(gid), None, ng, dev(row_ptr), dev(col), vals, rhs)
    torch.cuda.synchronize()
    assert int(missing.item()) == 0
    Ag = np.zeros((ng, ng))
    v = vals.cpu().numpy()
    for r in range(ng):
        Ag[r, col[row_ptr[r]:row_ptr[r + 1]]] = v[row_ptr[r]:row_ptr[r + 1]]
    assert np.linalg.norm(Ag - A) <= 1e-12 * np.linalg.norm(A)
    assert np.linalg.norm(rhs.cpu().numpy() - b) <= 1e-12 * np.linalg.norm(b)


def _to_dense_csr(vals, row_ptr, col, n):
    Ag = np.zeros((n, n))
    v = vals.cpu().numpy()
    for r in range(n):
        Ag[r, col[row_ptr[r]:row_ptr[r + 1]]] = v[row_ptr[r]:row_ptr[r + 1]]
    return Ag


def test_scatter_plan_matches_dense_and_accumulates():
    """dpg_scatter_plan_*: symbolic part once, numeric part twice (the values double)."""
    S, s, ptr, gid, w, n = _setup(2)
    C, t = S.shape[0], S.shape[1]
    A, b = _dense(S, s, ptr, gid, w, n)
    row_ptr, col = _graph(A)
    dev = lambda x: torch.as_tensor(x).cuda()  # noqa: E731
    plan = dlib.ScatterPlan(C, t, dev(ptr), dev(gid), dev(w), n, dev(row_ptr), dev(col))
    vals = torch.zeros(col.shape[0], dtype=torch.float64, device="cuda")
    rhs = torch.zeros(n, dtype=torch.float64, device="cuda")
    plan.apply(dev(S), dev(s), vals, rhs)
    torch.cuda.synchronize()
    assert int(plan.missing.item()) == 0
    assert np.linalg.norm(_to_dense_csr(vals, row_ptr, col, n) - A) <= 1e-12 * np.linalg.norm(A)
    assert np.linalg.norm(rhs.cpu().numpy() - b) <= 1e-12 * np.linalg.norm(b)
    plan.apply(dev(S), dev(s), vals, rhs)
    torch.cuda.synchronize()
    assert np.linalg.norm(_to_dense_csr(vals, row_ptr, col, n) - 2 * A) <= 1e-12 * np.linalg.norm(A)


def test_scatter_plan_counts_missing_at_creation():
    S, s, ptr, gid, w, n = _setup(1)
    C, t = S.shape[0], S.shape[1]
    A, b = _dense(S, s, ptr, gid, w, n)
    drop = np.zeros((n, n), dtype=bool)
    drop[0, :] = True
    row_ptr, col = _graph(A, drop)
    gid = gid.copy()
    gid[0] = n + 5
    dev = lambda x: torch.as_tensor(x).cuda()  # noqa: E731
    plan = dlib.ScatterPlan(C, t, dev(ptr), dev(gid), dev(w), n, dev(row_ptr), dev(col))
    vals = torch.zeros(col.shape[0], dtype=torch.float64, device="cuda")
    plan.apply(dev(S), None, vals)
    torch.cuda.synchronize()
    assert int(plan.missing.item()) > 0
    assert np.isfinite(vals.cpu().numpy()).all()


def test_scatter_plan_hex_map_equals_one_shot():
    from camellia2_b200 import mesh
    from tests.helpers import poisson3d
    n = 3
    form, bucket, nodes, par = poisson3d(2, 1, n, 0.1)
    p = dlib.Plan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, p.info, C)
    out = p.assemble(*(torch.as_tensor(x).cuda() for x in (nodes, par, co)))
    t = out["S"].shape[1]
    g, ng = mesh.hex_trace_map(n, n, n, 2)
    keys = np.unique((g[:, :, None] * ng + g[:, None, :]).reshape(-1))
    row_ptr = np.zeros(ng + 1, dtype=np.int64)
    np.add.at(row_ptr, keys // ng + 1, 1)
    row_ptr, col = np.cumsum(row_ptr), (keys % ng).astype(np.int64)
    dev = lambda x: torch.as_tensor(x).cuda()  # noqa: E731
    ptr, gid = dev(np.arange(C * t + 1, dtype=np.int64)), dev(g.reshape(-1))
    v1 = torch.zeros(col.shape[0], dtype=torch.float64, device="cuda")
    r1 = torch.zeros(ng, dtype=torch.float64, device="cuda")
    dlib.scatter_global(out["S"], out["s"], ptr, gid, None, ng, dev(row_ptr), dev(col), v1, r1)
    plan = dlib.ScatterPlan(C, t, ptr, gid, None, ng, dev(row_ptr), dev(col))
    v2, r2 = torch.zeros_like(v1), torch.zeros_like(r1)
    plan.apply(out["S"], out["s"], v2, r2)
    torch.cuda.synchronize()
    assert int(plan.missing.item()) == 0
    assert float((v1 - v2).abs().max()) <= 1e-13 * float(v1.abs().max())
    assert float((r1 - r2).abs().max()) <= 1e-13 * float(r1.abs().max())
