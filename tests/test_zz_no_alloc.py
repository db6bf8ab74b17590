"""dpg_assemble_noalloc — assembly for callers that cannot allocate device memory.

Some callers cannot let the library allocate device memory while they assemble:
an application whose GPU memory is already reserved by its own pool, or a
time-stepping loop that must not take allocation latency or an out-of-memory
failure in the middle of a step.  dpg_assemble_noalloc runs the same kernel as
dpg_assemble with its scratch in a fixed device array instead of a stream-ordered
allocation.  These tests call it through the C ABI twice in a row, on two
different inputs, and check each result against dpg_assemble on the same
inputs with the tolerance of the other parity tests (relative Frobenius 1e-12):
once on a few cells, once on 1,000 cells of the 3D hex bucket, whose 298 KiB of
scratch per CTA lets only 110 CTAs fit in the 32 MiB array, so every CTA walks
several cells on that capped grid.  Large-bucket plans are refused.  The file is
named so that pytest collects it last.
"""
import ctypes as ct

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import abi, formulation as fm, lib as dlib, mesh  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _rel(a, b):
    den = np.linalg.norm(b.reshape(-1))
    return float(np.linalg.norm((a - b).reshape(-1)) / (den if den > 0 else 1.0))


def _call(plan, nodes, parity, coeff, out):
    L = dlib.load()
    fn = L.dpg_assemble_noalloc
    fn.argtypes = [ct.c_void_p, ct.c_int] + [ct.c_void_p] * 8 + [ct.c_void_p, ct.c_int]
    fn.restype = ct.c_int
    p = lambda x: ct.c_void_p(x.data_ptr())  # noqa: E731
    return fn(plan.h, nodes.shape[0], p(nodes), p(parity), p(coeff), p(out["K"]), p(out["l"]), p(out["S"]),
              p(out["s"]), p(out["info"]), ct.c_void_p(torch.cuda.current_stream().cuda_stream), 0)


def _noalloc(plan, nodes, parity, coeff, out):
    rc = _call(plan, nodes, parity, coeff, out)
    assert rc == 0, dlib.load().dpg_last_error_string()


@pytest.mark.parametrize("shape", [(3, 3, 2), (10, 10, 10)], ids=["18_cells", "1000_cells_capped_grid"])
def test_noalloc_matches_dpg_assemble_on_two_calls(shape):
    bucket = fm.PoissonFormulation(3).bucket(abi.TOPO_HEX, 2, 1)
    plan = dlib.Plan(bucket)
    P = plan.info["n_points_total"]
    for call, seed in enumerate((11, 12)):
        nodes, par = mesh.hex_grid(*shape, 0.1, seed=seed)
        C = nodes.shape[0]
        co = mesh.uniform_coeff(C, 1, P, seed=seed)
        dn, dp, dc = (torch.as_tensor(x).cuda() for x in (nodes, par, co))
        ref = plan.assemble(dn, dp, dc)
        out = plan.alloc_outputs(C)
        for v in out.values():
            v.fill_(7)  # stale values must be overwritten
        _noalloc(plan, dn, dp, dc, out)
        torch.cuda.synchronize()
        r = {k: v.cpu().numpy() for k, v in ref.items()}
        o = {k: v.cpu().numpy() for k, v in out.items()}
        assert np.array_equal(o["info"], r["info"]), call
        for c in range(C):
            for k in ("K", "l", "S", "s"):
                assert _rel(o[k][c], r[k][c]) < TOL, (call, c, k)


def test_noalloc_refuses_large_buckets():
    """A large-bucket plan (Stokes VGP quads p = 3: 228 test rows) needs dpg_assemble."""
    bucket = fm.StokesVGPFormulation(2).bucket(abi.TOPO_QUAD, 3, 2)
    plan = dlib.Plan(bucket)
    nodes, par = mesh.quad_grid(2, 1, 0.1, seed=1)
    C = nodes.shape[0]
    co = mesh.uniform_coeff(C, plan.info["n_slots"], plan.info["n_points_total"], seed=1)
    dn, dp, dc = (torch.as_tensor(x).cuda() for x in (nodes, par, co))
    out = plan.alloc_outputs(C)
    assert _call(plan, dn, dp, dc, out) == abi.DPG_ERR_UNSUPPORTED
    assert b"large-bucket" in dlib.load().dpg_last_error_string()
