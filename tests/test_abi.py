"""The C-ABI library loads and exports every entry point include/dpg_b200.h declares
(no GPU needed: no compute call is made)."""
import ctypes as ct
import os
import re

from camellia2_b200 import lib as dlib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "dpg_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(dpg_\w+)\s*\(", src, re.M)))


def test_header_declares_expected_entry_points():
    syms = declared_symbols()
    assert "dpg_assemble" in syms and "dpg_factored_cholesky_solve" in syms
    assert set(dlib.EXPORTED) <= set(syms)


def test_library_exports_every_declared_symbol():
    L = dlib.load()
    for s in declared_symbols():
        assert hasattr(L, s), s
    L.dpg_version.restype = ct.c_char_p
    assert b"sm_100a" in L.dpg_version()


def test_plan_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    from camellia2_b200 import abi, formulation as fm
    b = fm.PoissonFormulation(2).bucket(abi.TOPO_QUAD, 2, 2)
    try:
        dlib.Plan(b)
    except dlib.DpgError as e:
        assert e.code == abi.DPG_ERR_CUDA
    else:
        raise AssertionError("expected DpgError without a GPU")
