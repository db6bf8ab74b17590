"""ctypes binding of libdpg_b200.so (the C ABI in include/dpg_b200.h).

This is the host-side mirror of the reference's local-stiffness interface:
``Plan.localStiffnessMatrixAndRHS`` returns what TBF::localStiffnessMatrixAndRHS
(BF.cpp:1309-1496) returns, ``Plan.interpretLocalData``-style condensed outputs
come from the same launch, ``factoredCholeskySolve`` mirrors
TBF::factoredCholeskySolve (BF.cpp:924-1018).  torch is used only to hold
device memory and streams.  There is no CPU fallback: if the library cannot be
loaded or no GPU is present, calls raise.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdpg_b200.so")
_LIB = None

EXPORTED = [
    "dpg_plan_create", "dpg_plan_destroy", "dpg_plan_query", "dpg_assemble", "dpg_assemble_host",
    "dpg_assemble_parts", "dpg_factored_cholesky_solve", "dpg_assemble_adjoint", "dpg_assemble_multi",
    "dpg_last_error_string", "dpg_version",
]


class DpgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dpg error {code}: {msg}")
        self.code = code


def load():
    """Load the CUDA library (raises if it is missing: there is no fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m camellia2_b200.build`")
    L = ct.CDLL(LIB_PATH)
    vp, i, d = ct.c_void_p, ct.c_int, ct.c_double
    L.dpg_plan_create.argtypes = [vp, ct.POINTER(vp)]
    L.dpg_plan_destroy.argtypes = [vp]
    L.dpg_plan_query.argtypes = [vp, vp]
    L.dpg_plan_autotune.argtypes = [vp, i, vp, vp, vp, vp, ct.POINTER(i)]
    L.dpg_assemble.argtypes = [vp, i] + [vp] * 8 + [vp, i]
    L.dpg_assemble_host.argtypes = [vp, i] + [vp] * 8 + [i]
    L.dpg_assemble_parts.argtypes = [vp, i] + [vp] * 6 + [vp]
    L.dpg_factored_cholesky_solve.argtypes = [i, i, i] + [vp] * 6 + [vp]
    L.dpg_assemble_adjoint.argtypes = [vp, i] + [vp] * 7 + [vp]
    L.dpg_assemble_multi.argtypes = [i, vp, vp, i]
    L.dpg_multi_autotune.argtypes = [i, vp, vp, i, ct.POINTER(i)]
    L.dpg_recover_fields.argtypes = [vp, i] + [vp] * 5 + [vp]
    L.dpg_energy_error.argtypes = [vp, i] + [vp] * 6 + [vp]
    L.dpg_assemble_dls.argtypes = [vp, i] + [vp] * 6 + [vp]
    L.dpg_scatter_global.argtypes = [i, i] + [vp] * 3 + [ct.c_int64] + [vp] * 8
    L.dpg_scatter_plan_create.argtypes = [i, i] + [vp] * 3 + [ct.c_int64] + [vp] * 4 + [ct.POINTER(vp)]
    L.dpg_scatter_plan_apply.argtypes = [vp] * 6
    L.dpg_scatter_plan_destroy.argtypes = [vp]
    L.dpg_compose_map.argtypes = [i, i] + [vp] * 3 + [ct.c_int64] + [vp] * 6 + [ct.c_int64, ct.POINTER(ct.c_int64),
                                                                               vp, vp]
    L.dpg_graph_capture.argtypes = [i, vp, i, ct.POINTER(vp)]
    L.dpg_graph_launch.argtypes = [vp, vp]
    L.dpg_graph_destroy.argtypes = [vp]
    L.dpg_last_error_string.restype = ct.c_char_p
    L.dpg_version.restype = ct.c_char_p
    _LIB = L
    return L


def _check(rc):
    if rc != 0:
        raise DpgError(rc, load().dpg_last_error_string().decode())


def _ptr(x):
    """Device or host address of a torch tensor / numpy array (None -> NULL)."""
    if x is None:
        return None
    if hasattr(x, "data_ptr"):
        return ct.c_void_p(x.data_ptr())
    return x.ctypes.data_as(ct.c_void_p)


def _stream_ptr(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return ct.c_void_p(stream.cuda_stream)


class Plan:
    """One bucket (Camellia ElementType) compiled for the GPU."""

    def __init__(self, bucket):
        self.holder = getattr(bucket, "holder", bucket)
        L = load()
        h = ct.c_void_p()
        _check(L.dpg_plan_create(self.holder.ptr(), ct.byref(h)))
        self.h = h
        info = abi.PlanInfo()
        _check(L.dpg_plan_query(self.h, ct.byref(info)))
        self.info = info.as_dict()

    def close(self):
        if getattr(self, "h", None):
            load().dpg_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ device
    def alloc_outputs(self, C, device="cuda"):
        import torch
        i = self.info
        M, t = i["M"], i["n_trace"]
        f64 = dict(dtype=torch.float64, device=device)
        return dict(K=torch.empty((C, M, M), **f64), l=torch.empty((C, M), **f64),
                    S=torch.empty((C, t, t), **f64), s=torch.empty((C, t), **f64),
                    info=torch.empty((C,), dtype=torch.int32, device=device))

    def assemble(self, nodes, parity, coeff=None, out=None, stream=None, flags=0):
        """Device tensors in, device tensors out (asynchronous on `stream`)."""
        C = nodes.shape[0]
        if out is None:
            out = self.alloc_outputs(C, nodes.device)
        _check(load().dpg_assemble(self.h, C, _ptr(nodes), _ptr(parity), _ptr(coeff), _ptr(out["K"]),
                                   _ptr(out["l"]), _ptr(out["S"]), _ptr(out["s"]), _ptr(out["info"]),
                                   _stream_ptr(stream), flags))
        return out

    def localStiffnessMatrixAndRHS(self, nodes, parity, coeff=None):
        o = self.assemble(nodes, parity, coeff)
        return o["K"], o["l"]

    def autotune(self, nodes, parity, coeff=None, stream=None):
        """dpg_plan_autotune: time the candidate shapes on these cells (device tensors) and keep
        the faster; returns the chosen Gram staging chunk (single-CTA plans: 8 or 4) or the
        formation k-chunk (large-bucket plans: 32 or 16)."""
        chosen = ct.c_int(0)
        _check(load().dpg_plan_autotune(self.h, nodes.shape[0], _ptr(nodes), _ptr(parity), _ptr(coeff),
                                        _stream_ptr(stream), ct.byref(chosen)))
        return chosen.value

    def parts(self, nodes, parity, coeff=None, stream=None):
        import torch
        C = nodes.shape[0]
        i = self.info
        N, M = i["N"], i["M"]
        f64 = dict(dtype=torch.float64, device=nodes.device)
        G = torch.zeros((C, N, N), **f64)
        B = torch.zeros((C, M, N), **f64)
        F = torch.zeros((C, N), **f64)
        _check(load().dpg_assemble_parts(self.h, C, _ptr(nodes), _ptr(parity), _ptr(coeff), _ptr(G), _ptr(B),
                                         _ptr(F), _stream_ptr(stream)))
        return G, B, F

    def adjoint(self, nodes, parity, coeff, Kbar, lbar=None, stream=None):
        """dJ/dcoeff (C, n_slots, n_points_total) for a loss J(K, l) with Kbar = dJ/dK (C,M,M)
        and lbar = dJ/dl (C,M); device tensors (dpg_assemble_adjoint)."""
        import torch
        C = nodes.shape[0]
        i = self.info
        cbar = torch.zeros((C, i["n_slots"], i["n_points_total"]), dtype=torch.float64, device=nodes.device)
        info = torch.empty((C,), dtype=torch.int32, device=nodes.device)
        _check(load().dpg_assemble_adjoint(self.h, C, _ptr(nodes), _ptr(parity), _ptr(coeff),
                                           _ptr(Kbar.contiguous()), _ptr(None if lbar is None else lbar.contiguous()),
                                           _ptr(cbar), _ptr(info), _stream_ptr(stream)))
        return cbar, info

    def dls(self, nodes, parity, coeff=None, stream=None):
        """dpg_assemble_dls: W = L^-1 B (C, M, N) and y = L^-1 F (C, N), G = L L^T."""
        import torch
        C = nodes.shape[0]
        i = self.info
        W = torch.empty((C, i["M"], i["N"]), dtype=torch.float64, device=nodes.device)
        y = torch.empty((C, i["N"]), dtype=torch.float64, device=nodes.device)
        info = torch.empty((C,), dtype=torch.int32, device=nodes.device)
        _check(load().dpg_assemble_dls(self.h, C, _ptr(nodes), _ptr(parity), _ptr(coeff), _ptr(W), _ptr(y), _ptr(info),
                                       _stream_ptr(stream)))
        return W, y, info

    def energy_error(self, nodes, parity, coeff, local_coeff, stream=None):
        """dpg_energy_error: per-cell energy error sqrt(r^T G^-1 r), r = F - B x, of the
        local trial coefficients x (C, M); device tensors."""
        import torch
        C = nodes.shape[0]
        e = torch.empty((C,), dtype=torch.float64, device=nodes.device)
        info = torch.empty((C,), dtype=torch.int32, device=nodes.device)
        _check(load().dpg_energy_error(self.h, C, _ptr(nodes), _ptr(parity), _ptr(coeff), _ptr(local_coeff.contiguous()),
                                       _ptr(e), _ptr(info), _stream_ptr(stream)))
        return e, info

    def recover_fields(self, K, l, trace_coeff, stream=None):
        """dpg_recover_fields: local coefficients [u_f | t] (C, M) from K, l and the cells'
        trace coefficients t (C, n_trace) after the global solve; device tensors."""
        import torch
        C = K.shape[0]
        u = torch.empty((C, self.info["M"]), dtype=torch.float64, device=K.device)
        info = torch.empty((C,), dtype=torch.int32, device=K.device)
        _check(load().dpg_recover_fields(self.h, C, _ptr(K.contiguous()), _ptr(l.contiguous()),
                                         _ptr(trace_coeff.contiguous()), _ptr(u), _ptr(info), _stream_ptr(stream)))
        return u, info

    # -------------------------------------------------------------------- host
    def assemble_host(self, nodes, parity, coeff=None, out=None, flags=0):
        """Host arrays (numpy or CPU torch, pinned is fastest) in and out."""
        C = nodes.shape[0]
        i = self.info
        M, t = i["M"], i["n_trace"]
        if out is None:
            out = dict(K=np.empty((C, M, M)), l=np.empty((C, M)), S=np.empty((C, t, t)), s=np.empty((C, t)),
                       info=np.empty((C,), dtype=np.int32))
        _check(load().dpg_assemble_host(self.h, C, _ptr(nodes), _ptr(parity), _ptr(coeff), _ptr(out["K"]),
                                        _ptr(out["l"]), _ptr(out["S"]), _ptr(out["s"]), _ptr(out["info"]), flags))
        return out


def factoredCholeskySolve(G, B, F, stream=None):
    """Batched TBF::factoredCholeskySolve on device tensors G (C,N,N), B (C,M,N), F (C,N).
    Returns K (C,M,M), l (C,M), info (C,)."""
    import torch
    C, N, _ = G.shape
    M = B.shape[1]
    K = torch.empty((C, M, M), dtype=torch.float64, device=G.device)
    l = torch.empty((C, M), dtype=torch.float64, device=G.device)
    info = torch.empty((C,), dtype=torch.int32, device=G.device)
    _check(load().dpg_factored_cholesky_solve(C, N, M, _ptr(G.contiguous()), _ptr(B.contiguous()),
                                              _ptr(F.contiguous()), _ptr(K), _ptr(l), _ptr(info),
                                              _stream_ptr(stream)))
    return K, l, info


class BucketBatch(ct.Structure):
    """dpg_bucket_batch: one bucket's cells and buffers in a multi-bucket call."""
    _fields_ = [("plan", ct.c_void_p), ("C", ct.c_int)] + [(n, ct.c_void_p) for n in
                                                           ("nodes", "parity", "coeff", "K", "l", "S", "s", "info")]


def _batches(items):
    """items: list of (Plan, nodes, parity, coeff, out) with device tensors."""
    arr = (BucketBatch * len(items))()
    for k, (plan, nodes, parity, coeff, out) in enumerate(items):
        b = arr[k]
        b.plan = plan.h.value if hasattr(plan.h, "value") else plan.h
        b.C = nodes.shape[0]
        for name, t in (("nodes", nodes), ("parity", parity), ("coeff", coeff), ("K", out["K"]), ("l", out["l"]),
                        ("S", out["S"]), ("s", out["s"]), ("info", out["info"])):
            setattr(b, name, None if t is None else t.data_ptr())
    return arr


def assemble_multi(items, stream=None, flags=0, claim=None):
    """dpg_assemble_multi: several buckets, single-CTA and large, in one persistent launch with a
    dynamic work queue; `claim` cells are taken from the queue at a time (flags bits 8-15)."""
    arr = _batches(items)
    if claim is not None:
        flags = (flags & 0xff) | ((int(claim) & 0xff) << 8)
    _check(load().dpg_assemble_multi(len(items), ct.cast(arr, ct.c_void_p), _stream_ptr(stream), flags))


def multi_autotune(items, stream=None, flags=0):
    """dpg_multi_autotune: the fastest claim size (cells per queue claim) for these buckets."""
    arr = _batches(items)
    chosen = ct.c_int(0)
    _check(load().dpg_multi_autotune(len(items), ct.cast(arr, ct.c_void_p), _stream_ptr(stream), flags,
                                     ct.byref(chosen)))
    return chosen.value


class Graph:
    """dpg_graph_capture / dpg_graph_launch: a captured multi-bucket launch replayed on
    the buffers named at capture time."""

    def __init__(self, items, flags=0, claim=None):
        self._keep = items  # the buffers must outlive the graph
        if claim is not None:
            flags = (flags & 0xff) | ((int(claim) & 0xff) << 8)
        arr = _batches(items)
        h = ct.c_void_p()
        _check(load().dpg_graph_capture(len(items), ct.cast(arr, ct.c_void_p), flags, ct.byref(h)))
        self.h = h

    def launch(self, stream=None):
        _check(load().dpg_graph_launch(self.h, _stream_ptr(stream)))

    def close(self):
        if getattr(self, "h", None):
            load().dpg_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scatter_global(S, s, map_ptr, map_gid, map_w, n_global, row_ptr, col_idx, values, rhs=None, stream=None):
    """dpg_scatter_global: values += sum_c C_c^T S_c C_c, rhs += sum_c C_c^T s_c on the
    CSR graph (row_ptr, col_idx); returns the number of skipped entries.  Device tensors
    (int64 maps and graph, float64 data)."""
    import torch
    C, t = S.shape[0], S.shape[1]
    missing = torch.zeros((1,), dtype=torch.int32, device=S.device)
    _check(load().dpg_scatter_global(C, t, _ptr(map_ptr), _ptr(map_gid), _ptr(map_w), int(n_global), _ptr(row_ptr),
                                     _ptr(col_idx), _ptr(S.contiguous()), _ptr(None if s is None else s.contiguous()),
                                     _ptr(values), _ptr(rhs), _ptr(missing), _stream_ptr(stream)))
    return missing


def compose_map(C, t, map_ptr, map_gid, map_w, n_fine, p_row_ptr, p_col, p_val, stream=None):
    """dpg_compose_map: the per-cell local-to-coarse maps C_c P (size query, then fill).
    Returns (ptr, gid, w, missing) as device tensors; scatter_global with them and the
    cells' S, s assembles the Galerkin coarse operator P^T A P and load P^T b."""
    import torch
    dev = map_ptr.device
    L, sp = load(), _stream_ptr(stream)
    out_ptr = torch.empty((C * t + 1,), dtype=torch.int64, device=dev)
    missing = torch.zeros((1,), dtype=torch.int32, device=dev)
    n = ct.c_int64(0)
    args = (_ptr(map_ptr), _ptr(map_gid), _ptr(map_w), int(n_fine), _ptr(p_row_ptr), _ptr(p_col), _ptr(p_val))
    _check(L.dpg_compose_map(C, t, *args, _ptr(out_ptr), None, None, 0, ct.byref(n), _ptr(missing), sp))
    gid = torch.empty((max(n.value, 1),), dtype=torch.int64, device=dev)
    w = torch.empty((max(n.value, 1),), dtype=torch.float64, device=dev)
    missing.zero_()
    _check(L.dpg_compose_map(C, t, *args, _ptr(out_ptr), _ptr(gid), _ptr(w), n.value, ct.byref(n), _ptr(missing), sp))
    return out_ptr, gid[:n.value], w[:n.value], missing


class ScatterPlan:
    """dpg_scatter_plan_*: the global scatter's symbolic part once (map and graph fixed),
    then apply(S, s, values, rhs) per assembly.  `missing` (device int32) holds the
    count of contributions the graph has no place for."""

    def __init__(self, C, t, map_ptr, map_gid, map_w, n_global, row_ptr, col_idx, stream=None):
        import torch
        self.missing = torch.zeros((1,), dtype=torch.int32, device=map_ptr.device)
        h = ct.c_void_p()
        self._keep = (map_ptr, map_gid, map_w, row_ptr, col_idx)
        _check(load().dpg_scatter_plan_create(C, t, _ptr(map_ptr), _ptr(map_gid), _ptr(map_w), int(n_global),
                                              _ptr(row_ptr), _ptr(col_idx), _ptr(self.missing), _stream_ptr(stream),
                                              ct.byref(h)))
        self.h = h

    def apply(self, S, s, values, rhs=None, stream=None):
        _check(load().dpg_scatter_plan_apply(self.h, _ptr(S.contiguous()), _ptr(None if s is None else s.contiguous()),
                                             _ptr(values), _ptr(rhs), _stream_ptr(stream)))

    def __del__(self):
        if getattr(self, "h", None) and _LIB is not None:
            _LIB.dpg_scatter_plan_destroy(self.h)
            self.h = None
