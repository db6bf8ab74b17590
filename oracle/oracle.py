"""ctypes binding of the CPU oracle (oracle/dpg_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the camellia2_b200 package.

Two builds of the same source: liboracle.so computes in FP64 (the oracle the GPU
path is compared with); liboracle_xp.so computes in __float128 (`xp=True` below),
the extended-precision truth for the same double inputs, used to measure how far
each FP64 code lies from the exact result.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

from camellia2_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


def build():
    subprocess.check_call(["bash", os.path.join(_HERE, "build.sh")])


def lib(xp=False):
    if xp not in _LIBS:
        path = os.path.join(_HERE, "liboracle_xp.so" if xp else "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ct.CDLL(path)
        L.orc_plan_create.restype = ct.c_void_p
        L.orc_plan_create.argtypes = [ct.c_void_p]
        L.orc_plan_destroy.argtypes = [ct.c_void_p]
        L.orc_plan_query.argtypes = [ct.c_void_p, ct.c_void_p]
        L.orc_assemble.argtypes = [ct.c_void_p, ct.c_int] + [ct.c_void_p] * 11 + [ct.c_int]
        L.orc_factored_cholesky_solve.argtypes = [ct.c_int, ct.c_int] + [ct.c_void_p] * 5
        L.orc_condense.argtypes = [ct.c_int] + [ct.c_void_p] * 5
        L.orc_trial_is_field.argtypes = [ct.c_void_p, ct.c_void_p]
        L.orc_basis_tabulate.argtypes = [ct.c_int] * 4 + [ct.c_void_p] * 4
        L.orc_cubature.argtypes = [ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p]
        L.orc_tri_cubature.argtypes = [ct.c_int, ct.c_void_p, ct.c_void_p]
        L.orc_tri_nodes.argtypes = [ct.c_int, ct.c_void_p]
        L.orc_cell_operators.argtypes = [ct.c_void_p] * 12
        L.orc_adjoint.argtypes = [ct.c_void_p, ct.c_int] + [ct.c_void_p] * 6 + [ct.c_int]
        L.orc_fd_directional.argtypes = [ct.c_void_p, ct.c_int] + [ct.c_void_p] * 4 + [ct.c_double] + [ct.c_void_p] * 2 + [ct.c_int]
        L.orc_fd_directional.restype = ct.c_double
        L.orc_loss.argtypes = [ct.c_void_p, ct.c_int] + [ct.c_void_p] * 6 + [ct.c_int]
        if not xp:
            L.orc_set_blas.argtypes = [ct.c_void_p] * 5
            L.orc_assemble_blas.argtypes = [ct.c_void_p, ct.c_int] + [ct.c_void_p] * 8 + [ct.c_int]
        L.orc_last_error.restype = ct.c_char_p
        assert L.orc_precision() == (1 if xp else 0)
        _LIBS[xp] = L
    return _LIBS[xp]


def _p(a):
    return None if a is None else a.ctypes.data_as(ct.c_void_p)


_BLAS_READY = False


def enable_blas():
    """Hand scipy's BLAS/LAPACK (scipy.linalg.cython_blas / cython_lapack: the OpenBLAS
    scipy bundles, Fortran LP64 interface) to the FP64 oracle's fast mode."""
    global _BLAS_READY
    if _BLAS_READY:
        return
    import scipy.linalg.cython_blas as cb
    import scipy.linalg.cython_lapack as cl
    get_name = ct.pythonapi.PyCapsule_GetName
    get_name.restype, get_name.argtypes = ct.c_char_p, [ct.py_object]
    get_ptr = ct.pythonapi.PyCapsule_GetPointer
    get_ptr.restype, get_ptr.argtypes = ct.c_void_p, [ct.py_object, ct.c_char_p]

    def fn(mod, name):
        cap = mod.__pyx_capi__[name]
        return get_ptr(cap, get_name(cap))

    ptrs = [fn(cb, "dgemm"), fn(cb, "dgemv"), fn(cb, "dsyrk"), fn(cb, "dtrsm"), fn(cl, "dpotrf")]
    if lib().orc_set_blas(*[ct.c_void_p(x) for x in ptrs]) != 0:
        raise RuntimeError("oracle fast mode: BLAS entry points missing")
    _BLAS_READY = True


class OraclePlan:
    """One bucket on the CPU.  xp=True computes in __float128 (the truth)."""

    def __init__(self, bucket_or_holder, xp=False):
        holder = getattr(bucket_or_holder, "holder", bucket_or_holder)
        self.holder = holder
        self.L = lib(xp)
        self.xp = xp
        self.h = self.L.orc_plan_create(holder.ptr())
        if not self.h:
            raise RuntimeError("oracle plan: " + self.L.orc_last_error().decode())
        info = abi.PlanInfo()
        self.L.orc_plan_query(self.h, ct.byref(info))
        self.info = info.as_dict()
        self.is_field = np.zeros(self.info["M"], dtype=np.int32)
        self.L.orc_trial_is_field(self.h, _p(self.is_field))

    def __del__(self):
        try:
            self.L.orc_plan_destroy(self.h)
        except Exception:
            pass

    def assemble(self, nodes, parity, coeff=None, parts=False, nthreads=1):
        i = self.info
        C = nodes.shape[0]
        N, M, t = i["N"], i["M"], i["n_trace"]
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        parity = np.ascontiguousarray(parity, dtype=np.int8)
        if coeff is not None:
            coeff = np.ascontiguousarray(coeff, dtype=np.float64)
        out = {}
        if parts:
            out["G"] = np.zeros((C, N, N))
            out["B"] = np.zeros((C, M, N))
            out["F"] = np.zeros((C, N))
        out["K"] = np.zeros((C, M, M))
        out["l"] = np.zeros((C, M))
        out["S"] = np.zeros((C, t, t))
        out["s"] = np.zeros((C, t))
        out["info"] = np.zeros(C, dtype=np.int32)
        self.L.orc_assemble(self.h, C, _p(nodes), _p(parity), _p(coeff), _p(out.get("G")), _p(out.get("B")),
                           _p(out.get("F")), _p(out["K"]), _p(out["l"]), _p(out["S"]), _p(out["s"]),
                           _p(out["info"]), nthreads)
        return out

    def adjoint(self, nodes, parity, coeff, Kbar, lbar, nthreads=1):
        """Hand gradient of J = sum_c <Kbar_c, K_c> + <lbar_c, l_c> with respect to the
        coefficient slots, (C, n_slots, n_points_total)."""
        C = nodes.shape[0]
        cbar = np.zeros((C, self.info["n_slots"], self.info["n_points_total"]))
        arr = lambda a, t=np.float64: np.ascontiguousarray(a, dtype=t)  # noqa: E731
        self.L.orc_adjoint(self.h, C, _p(arr(nodes)), _p(arr(parity, np.int8)), _p(arr(coeff)), _p(arr(Kbar)),
                           _p(arr(lbar)), _p(cbar), nthreads)
        return cbar

    def loss(self, nodes, parity, coeff, Kbar, lbar, nthreads=1):
        """J = sum_c <Kbar_c, K_c> + <lbar_c, l_c> as an unevaluated pair of doubles (hi, lo)."""
        arr = lambda a, t=np.float64: np.ascontiguousarray(a, dtype=t)  # noqa: E731
        out = np.zeros(2)
        self.L.orc_loss(self.h, nodes.shape[0], _p(arr(nodes)), _p(arr(parity, np.int8)), _p(arr(coeff)),
                        _p(arr(Kbar)), _p(arr(lbar)), _p(out), nthreads)
        return float(out[0]), float(out[1])

    def fd_directional(self, nodes, parity, coeff, direction, h, Kbar, lbar, nthreads=1):
        """Central difference of J = sum_c <Kbar_c, K_c> + <lbar_c, l_c> along `direction`
        (same shape as coeff) with step h, all in the build's arithmetic (xp=True: the
        perturbed coefficients and the difference in __float128)."""
        arr = lambda a, t=np.float64: np.ascontiguousarray(a, dtype=t)  # noqa: E731
        return float(self.L.orc_fd_directional(self.h, nodes.shape[0], _p(arr(nodes)), _p(arr(parity, np.int8)),
                                               _p(arr(coeff)), _p(arr(direction)), float(h), _p(arr(Kbar)),
                                               _p(arr(lbar)), nthreads))

    def operators(self, nodes, parity, coeff=None):
        """Quadrature operator rows of ONE cell (nodes (nv, d), parity (ns,), coeff
        (n_slots, P) or None): G = sum_q wm[q] L[q]^T L[q] (rows = graph-norm term
        components, rterm their terms), B = U^T V, F = FV^T fw."""
        i = self.info
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        parity = np.ascontiguousarray(parity, dtype=np.int8)
        cf = None if coeff is None else np.ascontiguousarray(coeff, dtype=np.float64)
        dims = np.zeros(3, dtype=np.int32)
        self.L.orc_cell_operators(self.h, _p(nodes), _p(parity), _p(cf), _p(dims), *([None] * 7))
        nT, nB, nF = (int(x) for x in dims)
        N, M, QG = i["N"], i["M"], i["Q_G"]
        out = dict(L=np.zeros((QG, nT, N)), wm=np.zeros(QG), rterm=np.zeros(nT, dtype=np.int32),
                   U=np.zeros((nB, M)), V=np.zeros((nB, N)), fw=np.zeros(nF), FV=np.zeros((nF, N)))
        self.L.orc_cell_operators(self.h, _p(nodes), _p(parity), _p(cf), _p(dims),
                                  *(_p(out[k]) for k in ("L", "wm", "rterm", "U", "V", "fw", "FV")))
        return out

    def assemble_blas(self, nodes, parity, coeff=None, nthreads=1):
        """Fast mode (the CPU baseline): the same outputs with every quadrature contraction a
        DGEMM per block and the dense solve in LAPACK/BLAS, each call on one BLAS thread
        (threads = cells in parallel)."""
        from threadpoolctl import threadpool_limits
        assert not self.xp
        enable_blas()
        i = self.info
        C = nodes.shape[0]
        M, t = i["M"], i["n_trace"]
        arr = lambda a, ty=np.float64: np.ascontiguousarray(a, dtype=ty)  # noqa: E731
        out = dict(K=np.zeros((C, M, M)), l=np.zeros((C, M)), S=np.zeros((C, t, t)), s=np.zeros((C, t)),
                   info=np.zeros(C, dtype=np.int32))
        with threadpool_limits(limits=1, user_api="blas"):
            rc = self.L.orc_assemble_blas(self.h, C, _p(arr(nodes)), _p(arr(parity, np.int8)),
                                          _p(None if coeff is None else arr(coeff)), _p(out["K"]), _p(out["l"]),
                                          _p(out["S"]), _p(out["s"]), _p(out["info"]), nthreads)
        if rc != 0:
            raise RuntimeError(self.L.orc_last_error().decode())
        return out

    def parts(self, nodes, parity, coeff=None):
        i = self.info
        C = nodes.shape[0]
        N, M = i["N"], i["M"]
        G, B, F = np.zeros((C, N, N)), np.zeros((C, M, N)), np.zeros((C, N))
        self.L.orc_assemble(self.h, C, _p(np.ascontiguousarray(nodes, dtype=np.float64)),
                           _p(np.ascontiguousarray(parity, dtype=np.int8)),
                           _p(None if coeff is None else np.ascontiguousarray(coeff, dtype=np.float64)),
                           _p(G), _p(B), _p(F), None, None, None, None, None, 1)
        return G, B, F


def factored_cholesky_solve(G, B, F, xp=False):
    """Single cell: G (N,N), B (M,N) [stiffnessEnriched layout], F (N)."""
    G = np.ascontiguousarray(G, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    F = np.ascontiguousarray(F, dtype=np.float64)
    N, M = G.shape[0], B.shape[0]
    K, l = np.zeros((M, M)), np.zeros(M)
    info = lib(xp).orc_factored_cholesky_solve(N, M, _p(G), _p(B), _p(F), _p(K), _p(l))
    return K, l, info


def condense(is_field, K, l, xp=False):
    is_field = np.ascontiguousarray(is_field, dtype=np.int32)
    K = np.ascontiguousarray(K, dtype=np.float64)
    l = np.ascontiguousarray(l, dtype=np.float64)
    t = int((is_field == 0).sum())
    S, s = np.zeros((t, t)), np.zeros(t)
    err = lib(xp).orc_condense(K.shape[0], _p(is_field), _p(K), _p(l), _p(S), _p(s))
    return S, s, err


def basis_tabulate(topo, space, n, pts):
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    npts = pts.shape[0]
    # size generously, then trim
    big = 4096
    d = pts.shape[1]
    val = np.zeros((npts, big * d))
    grad = np.zeros((npts, big * d))
    div = np.zeros((npts, big))
    card = lib().orc_basis_tabulate(topo, space, n, npts, _p(pts), _p(val), _p(grad), _p(div))
    vdim = d if space == abi.SPACE_HDIV else 1
    flat_v = val.reshape(-1)[: npts * card * vdim].reshape(npts, card, vdim)
    flat_g = grad.reshape(-1)[: npts * card * d].reshape(npts, card, d)
    flat_d = div.reshape(-1)[: npts * card].reshape(npts, card)
    return flat_v, flat_g, flat_d


def cubature(dim, degree):
    n = (degree // 2 + 1) ** dim
    pts, wts = np.zeros((n, dim)), np.zeros(n)
    lib().orc_cubature(dim, degree, _p(pts), _p(wts))
    return pts, wts


def tri_cubature(degree):
    n = lib().orc_tri_cubature(degree, None, None)
    pts, wts = np.zeros((n, 2)), np.zeros(n)
    lib().orc_tri_cubature(degree, _p(pts), _p(wts))
    return pts, wts


def tri_nodes(n):
    m = lib().orc_tri_nodes(n, None)
    pts = np.zeros((m, 2))
    lib().orc_tri_nodes(n, _p(pts))
    return pts
