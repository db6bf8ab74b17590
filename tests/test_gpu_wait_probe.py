"""Failure detection without a GPU fault: every wait of the assembly kernels on a
staging copy (mbarrier) has an iteration limit.  The probe waits, with the same
routine, on a transaction that never arrives; the wait must end with the timeout
status (the value the kernels report in info) and the context must stay usable."""
import ctypes as ct

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import lib as dlib  # noqa: E402
from tests.helpers import coeffs_for, poisson2d  # noqa: E402

pytestmark = pytest.mark.gpu

TIMEOUT_STATUS = 0x7FFF0000


def test_bounded_wait_reports_timeout_and_context_survives():
    L = dlib.load()
    fn = L.dpg_debug_wait_probe
    fn.argtypes = [ct.c_int, ct.c_void_p, ct.c_void_p]
    fn.restype = ct.c_int
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    rc = fn(2000, ct.c_void_p(status.data_ptr()), ct.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.dpg_last_error_string()
    torch.cuda.synchronize()
    assert int(status.item()) == TIMEOUT_STATUS
    # the context still assembles
    form, bucket, nodes, par = poisson2d(2, 2, 2, 2, 0.1)
    plan = dlib.Plan(bucket)
    co = coeffs_for(bucket, plan.info, nodes.shape[0])
    out = plan.assemble(*(torch.as_tensor(x).cuda() for x in (nodes, par, co)))
    torch.cuda.synchronize()
    assert int(out["info"].abs().max()) == 0 and np.isfinite(out["K"].cpu().numpy()).all()
