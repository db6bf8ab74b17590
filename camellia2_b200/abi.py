"""ctypes mirror of include/dpg_b200.h (structs and constants).

The same flat descriptor feeds the CUDA library and, in the tests, the CPU
oracle; both read it with the layout declared in the C header.
"""
import ctypes as ct

DPG_ABI_VERSION = 1

DPG_OK = 0
DPG_ERR_INVALID_ARGUMENT = 1
DPG_ERR_UNSUPPORTED = 2
DPG_ERR_CUDA = 3
DPG_ERR_OUT_OF_MEMORY = 4
DPG_ERR_TIMEOUT = 5
DPG_ERR_BAD_PLAN = 6

TOPO_QUAD, TOPO_HEX, TOPO_TRI = 1, 2, 3
SPACE_HGRAD, SPACE_HDIV, SPACE_HVOL, SPACE_VECTOR_HVOL = 1, 2, 3, 4
VAR_FIELD, VAR_TRACE, VAR_FLUX, VAR_TEST = 1, 2, 3, 4
OP_VALUE, OP_X, OP_Y, OP_Z, OP_DX, OP_DY, OP_DZ, OP_DIV, OP_DOT_NORMAL = range(9)
PREC_FP64, PREC_MIXED = 0, 1
FLAG_NO_K, FLAG_NO_CONDENSE = 1, 2

TOPO_INFO = {
    # key: (space_dim, n_vertices, n_sides)
    TOPO_QUAD: (2, 4, 4),
    TOPO_HEX: (3, 8, 6),
    TOPO_TRI: (2, 3, 3),
}


class VarDesc(ct.Structure):
    _fields_ = [("kind", ct.c_int), ("space", ct.c_int), ("poly_order", ct.c_int)]


class BFTerm(ct.Structure):
    _fields_ = [
        ("trial_var", ct.c_int), ("trial_op", ct.c_int),
        ("test_var", ct.c_int), ("test_op", ct.c_int),
        ("coef", ct.c_double), ("slot", ct.c_int),
        ("normal_comp", ct.c_int), ("boundary", ct.c_int),
    ]


class IPEntry(ct.Structure):
    _fields_ = [
        ("term", ct.c_int), ("comp", ct.c_int), ("test_var", ct.c_int),
        ("test_op", ct.c_int), ("coef", ct.c_double), ("slot", ct.c_int),
    ]


class RHSTerm(ct.Structure):
    _fields_ = [("test_var", ct.c_int), ("test_op", ct.c_int), ("coef", ct.c_double), ("slot", ct.c_int)]


class BucketDesc(ct.Structure):
    _fields_ = [
        ("abi_version", ct.c_int), ("topology", ct.c_int),
        ("n_trial", ct.c_int), ("trial", ct.POINTER(VarDesc)),
        ("n_test", ct.c_int), ("test", ct.POINTER(VarDesc)),
        ("n_bf", ct.c_int), ("bf", ct.POINTER(BFTerm)),
        ("n_ip", ct.c_int), ("ip", ct.POINTER(IPEntry)),
        ("n_rhs", ct.c_int), ("rhs", ct.POINTER(RHSTerm)),
        ("cub_degree_G", ct.c_int), ("cub_degree_B", ct.c_int), ("cub_degree_side", ct.c_int),
        ("n_slots", ct.c_int), ("precision", ct.c_int),
    ]


class PlanInfo(ct.Structure):
    _fields_ = [
        ("N", ct.c_int), ("M", ct.c_int), ("n_field", ct.c_int), ("n_trace", ct.c_int),
        ("space_dim", ct.c_int), ("n_vertices", ct.c_int), ("n_sides", ct.c_int),
        ("Q_G", ct.c_int), ("Q_B", ct.c_int), ("Q_side", ct.c_int), ("n_points_total", ct.c_int),
        ("n_slots", ct.c_int), ("precision", ct.c_int),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class BucketBatch(ct.Structure):
    _fields_ = [
        ("plan", ct.c_void_p), ("C", ct.c_int),
        ("nodes", ct.c_void_p), ("parity", ct.c_void_p), ("coeff", ct.c_void_p),
        ("K", ct.c_void_p), ("l", ct.c_void_p), ("S", ct.c_void_p), ("s", ct.c_void_p),
        ("info", ct.c_void_p),
    ]


class DescHolder:
    """Owns the ctypes arrays a BucketDesc points into."""

    def __init__(self, topology, trial, test, bf, ip, rhs, degG, degB, degS, n_slots, precision=PREC_FP64):
        self.trial = (VarDesc * max(1, len(trial)))(*[VarDesc(*t) for t in trial])
        self.test = (VarDesc * max(1, len(test)))(*[VarDesc(*t) for t in test])
        self.bf = (BFTerm * max(1, len(bf)))(*[BFTerm(*t) for t in bf])
        self.ip = (IPEntry * max(1, len(ip)))(*[IPEntry(*t) for t in ip])
        self.rhs = (RHSTerm * max(1, len(rhs)))(*[RHSTerm(*t) for t in rhs])
        self.desc = BucketDesc(
            DPG_ABI_VERSION, topology,
            len(trial), self.trial, len(test), self.test,
            len(bf), self.bf, len(ip), self.ip, len(rhs), self.rhs,
            degG, degB, degS, n_slots, precision,
        )
        self.tuples = dict(topology=topology, trial=list(trial), test=list(test), bf=list(bf), ip=list(ip),
                           rhs=list(rhs), degG=degG, degB=degB, degS=degS, n_slots=n_slots, precision=precision)

    def with_precision(self, precision):
        t = dict(self.tuples)
        t["precision"] = precision
        return DescHolder(t["topology"], t["trial"], t["test"], t["bf"], t["ip"], t["rhs"], t["degG"],
                          t["degB"], t["degS"], t["n_slots"], precision)

    def ptr(self):
        return ct.byref(self.desc)
