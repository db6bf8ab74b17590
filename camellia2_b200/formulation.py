"""Host-side mirror of Camellia's problem-definition API for the DPG assembly path.

Names and meaning follow the reference:
  VarFactory.fieldVar/traceVar/fluxVar/testVar    src/include/VarFactory.h
  Var ops .div() .grad() .dot_normal() .dx() ...  src/include/Var.h
  LinearTerm algebra (function * var, +, -)       src/ScratchPad/LinearTerm.cpp
  BF.addTerm / BF.graphNorm                       src/ScratchPad/BF.cpp:1040-1141
  RHS.addTerm                                     src/Problem/RHS.cpp
  PoissonFormulation (ULTRAWEAK)                  src/Formulations/PoissonFormulation.cpp:26-80
  ConvectionDiffusionReactionFormulation (UW)     src/Formulations/ConvectionDiffusionReactionFormulation.cpp:38-111
  StokesVGPFormulation (steady)                   src/Formulations/StokesVGPFormulation.cpp:224-407

A BF is compiled (``compile_bucket``) into the flat term tables of
include/dpg_b200.h: every vector dot product expanded into scalar products,
every coefficient reduced to ``constant * slot`` where a slot is a
per-quadrature-point coefficient array supplied at assembly time.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

from . import abi

# ----------------------------------------------------------------------------
# Coefficient functions
# ----------------------------------------------------------------------------


@dataclass(frozen=True)
class Fn:
    """Scalar coefficient: const * slot(x) * n_comp(x) (slot/normal optional)."""
    const: float = 1.0
    slot: Optional[int] = None
    normal: Optional[int] = None

    def __mul__(self, other):
        if isinstance(other, (int, float)):
            return Fn(self.const * other, self.slot, self.normal)
        if isinstance(other, Fn):
            if self.slot is not None and other.slot is not None:
                raise NotImplementedError("products of two per-point coefficients are not supported")
            if self.normal is not None and other.normal is not None:
                raise NotImplementedError("products of two normal components are not supported")
            return Fn(self.const * other.const,
                      self.slot if self.slot is not None else other.slot,
                      self.normal if self.normal is not None else other.normal)
        if isinstance(other, VecFn):
            return VecFn([self * c for c in other.comps])
        if isinstance(other, (Var, LinearTerm)):
            return _as_lt(other).scaled(self)
        return NotImplemented

    __rmul__ = __mul__

    def __neg__(self):
        return Fn(-self.const, self.slot, self.normal)


@dataclass(frozen=True)
class VecFn:
    comps: List[Fn]

    def __mul__(self, other):
        if isinstance(other, (int, float)):
            return VecFn([c * other for c in self.comps])
        if isinstance(other, Fn):
            return VecFn([c * other for c in self.comps])
        if isinstance(other, (Var, LinearTerm)):
            lt = _as_lt(other)
            if lt.rank == 0:  # vector function times scalar term -> vector term
                return LinearTerm(1, [[a.scaled(c) for a in lt.comps[0]] for c in self.comps])
            # vector . vector -> scalar term
            atoms = []
            for c, comp in zip(self.comps, lt.comps):
                atoms += [a.scaled(c) for a in comp]
            return LinearTerm(0, [atoms])
        return NotImplemented

    __rmul__ = __mul__

    def __neg__(self):
        return VecFn([-c for c in self.comps])

    def spatialComponent(self, i):  # 1-based, as in Camellia
        return self.comps[i - 1]


def constant(c):
    return Fn(float(c))


def slot(i):
    return Fn(1.0, int(i))


def normal(space_dim):
    return VecFn([Fn(1.0, None, k) for k in range(space_dim)])


# ----------------------------------------------------------------------------
# Variables and linear terms
# ----------------------------------------------------------------------------


@dataclass(frozen=True)
class Atom:
    coef: Fn
    var: "Var"
    op: int

    def scaled(self, f):
        return Atom(self.coef * f, self.var, self.op)

    @property
    def boundary_only(self):
        return (self.op == abi.OP_DOT_NORMAL or self.coef.normal is not None
                or self.var.kind in (abi.VAR_TRACE, abi.VAR_FLUX))


class LinearTerm:
    """A (scalar, rank 0) or vector (rank 1, one entry per component) sum of atoms."""

    def __init__(self, rank, comps):
        self.rank = rank
        self.comps = comps

    def scaled(self, f):
        if isinstance(f, (int, float)):
            f = Fn(float(f))
        return LinearTerm(self.rank, [[a.scaled(f) for a in comp] for comp in self.comps])

    def __add__(self, other):
        other = _as_lt(other)
        if self.rank != other.rank or len(self.comps) != len(other.comps):
            raise ValueError("rank mismatch in LinearTerm sum")
        return LinearTerm(self.rank, [a + b for a, b in zip(self.comps, other.comps)])

    def __sub__(self, other):
        return self + (-_as_lt(other))

    def __neg__(self):
        return self.scaled(-1.0)

    def __mul__(self, f):
        if isinstance(f, (int, float, Fn, VecFn)):
            return f * self
        return NotImplemented

    def __rmul__(self, f):
        if isinstance(f, (int, float)):
            return self.scaled(float(f))
        return f.__mul__(self)

    def non_boundary_part(self):
        return LinearTerm(self.rank, [[a for a in comp if not a.boundary_only] for comp in self.comps])

    def is_empty(self):
        return all(len(c) == 0 for c in self.comps)


def _as_lt(x):
    if isinstance(x, LinearTerm):
        return x
    if isinstance(x, Var):
        return x.value()
    raise TypeError(f"cannot use {type(x)} as a LinearTerm")


class Var:
    def __init__(self, vf, vid, name, kind, space):
        self.vf, self.id, self.name, self.kind, self.space = vf, vid, name, kind, space

    def __repr__(self):
        return f"Var({self.name})"

    def __hash__(self):
        return hash((id(self.vf), self.id))

    def __eq__(self, other):
        return isinstance(other, Var) and other.vf is self.vf and other.id == self.id

    @property
    def vector_valued(self):
        return self.space in (abi.SPACE_HDIV, abi.SPACE_VECTOR_HVOL)

    def _lt(self, rank, ops):
        return LinearTerm(rank, [[Atom(Fn(), self, op)] for op in ops])

    def value(self):
        d = self.vf.space_dim
        if self.vector_valued:
            return self._lt(1, [abi.OP_X + k for k in range(d)])
        return self._lt(0, [abi.OP_VALUE])

    def grad(self):
        return self._lt(1, [abi.OP_DX + k for k in range(self.vf.space_dim)])

    def div(self):
        return self._lt(0, [abi.OP_DIV])

    def dot_normal(self):
        return self._lt(0, [abi.OP_DOT_NORMAL])

    def di(self, i):  # 1-based
        return self._lt(0, [abi.OP_DX + i - 1])

    def dx(self):
        return self.di(1)

    def dy(self):
        return self.di(2)

    def dz(self):
        return self.di(3)

    def spatialComponent(self, i):  # 1-based
        return self._lt(0, [abi.OP_X + i - 1])

    x = lambda self: self.spatialComponent(1)  # noqa: E731
    y = lambda self: self.spatialComponent(2)  # noqa: E731
    z = lambda self: self.spatialComponent(3)  # noqa: E731

    def __neg__(self):
        return -self.value()

    def __add__(self, o):
        return self.value() + o

    def __sub__(self, o):
        return self.value() - o

    def __mul__(self, f):
        return f * self.value()

    __rmul__ = __mul__


class VarFactory:
    """IDs are assigned in creation order, as Camellia's VarFactory does."""

    def __init__(self, space_dim):
        self.space_dim = space_dim
        self.vars: List[Var] = []

    def _new(self, name, kind, space):
        v = Var(self, len(self.vars), name, kind, space)
        self.vars.append(v)
        return v

    def fieldVar(self, name, space=abi.SPACE_HVOL):
        return self._new(name, abi.VAR_FIELD, space)

    def traceVar(self, name, space=abi.SPACE_HGRAD):
        return self._new(name, abi.VAR_TRACE, space)

    def fluxVar(self, name, space=abi.SPACE_HVOL):
        return self._new(name, abi.VAR_FLUX, space)

    def testVar(self, name, space):
        return self._new(name, abi.VAR_TEST, space)

    def trialVars(self):
        return [v for v in self.vars if v.kind != abi.VAR_TEST]

    def testVars(self):
        return [v for v in self.vars if v.kind == abi.VAR_TEST]


class IP:
    def __init__(self):
        self.terms: List[LinearTerm] = []

    def addTerm(self, lt):
        self.terms.append(_as_lt(lt))


class RHS:
    def __init__(self):
        self.terms: List[LinearTerm] = []

    def addTerm(self, lt):
        lt = _as_lt(lt)
        if lt.rank != 0:
            raise ValueError("RHS terms must be scalar")
        self.terms.append(lt)


class BF:
    def __init__(self, vf: VarFactory):
        self.vf = vf
        self.terms: List[Tuple[LinearTerm, LinearTerm]] = []

    def addTerm(self, trial, test):
        trial, test = _as_lt(trial), _as_lt(test)
        if trial.rank != test.rank:
            raise ValueError("trial and test terms must have the same rank")
        self.terms.append((trial, test))

    def graphNorm(self, trial_weights: Optional[Dict[int, float]] = None, weight_l2_test=1.0) -> IP:
        """TBF::graphNorm (BF.cpp:1040-1141): one term per field var collecting the
        (non-boundary) test terms it multiplies, then an L2 term per test var."""
        trial_weights = trial_weights or {}
        d = self.vf.space_dim
        per_var: Dict[int, LinearTerm] = {}
        for trial, test in self.terms:
            test_nb = test.non_boundary_part()
            if test_nb.is_empty():
                continue
            for ci, comp in enumerate(trial.comps):
                for a in comp:
                    if a.var.kind != abi.VAR_FIELD or a.boundary_only:
                        continue
                    if a.var.vector_valued:
                        target_rank, target_comp = 1, a.op - abi.OP_X
                    else:
                        target_rank, target_comp = 0, 0
                    src = test_nb.comps[ci]
                    contrib = [x.scaled(a.coef) for x in src]
                    if a.var.id not in per_var:
                        per_var[a.var.id] = LinearTerm(target_rank, [[] for _ in range(d if target_rank else 1)])
                    per_var[a.var.id].comps[target_comp] += contrib
        ip = IP()
        for vid in sorted(per_var):
            w = 1.0
            if vid in trial_weights:
                if trial_weights[vid] <= 0:
                    raise ValueError("variable weights must be positive.")
                w = 1.0 / trial_weights[vid] ** 0.5
            ip.addTerm(per_var[vid].scaled(w))
        for v in self.vf.testVars():
            ip.addTerm(v.value().scaled(weight_l2_test ** 0.5))
        return ip


# ----------------------------------------------------------------------------
# Compilation into the flat bucket descriptor
# ----------------------------------------------------------------------------


def _basis_degree(var, k):
    """Intrepid basis degree of a var of H1Order k (BasisFactory.cpp:122-420)."""
    if var.kind == abi.VAR_TEST:
        return k
    if var.kind == abi.VAR_FIELD:
        return k - 1
    return k if var.space == abi.SPACE_HGRAD else k - 1


@dataclass
class Bucket:
    """One ElementType: topology + polynomial orders + the compiled tables."""
    holder: abi.DescHolder
    topology: int
    k: int
    dk: int
    n_slots: int
    slot_names: List[str] = field(default_factory=list)

    def desc(self):
        return self.holder.desc


def compile_bucket(bf: BF, ip: IP, rhs: Optional[RHS], topology: int, k: int, dk: int,
                   slot_names=(), precision=abi.PREC_FP64, cubature_enrichment=0) -> Bucket:
    vf = bf.vf
    trial_vars = vf.trialVars()
    test_vars = vf.testVars()
    tr_index = {v.id: i for i, v in enumerate(trial_vars)}
    te_index = {v.id: i for i, v in enumerate(test_vars)}
    trial = [(v.kind, v.space, k) for v in trial_vars]
    test = [(v.kind, v.space, k + dk) for v in test_vars]

    bf_terms = []
    for trial_lt, test_lt in bf.terms:
        for ci in range(len(trial_lt.comps)):
            for a in trial_lt.comps[ci]:
                for b in test_lt.comps[ci]:
                    f = a.coef * b.coef
                    boundary = int(a.boundary_only or b.boundary_only)
                    bf_terms.append((tr_index[a.var.id], a.op, te_index[b.var.id], b.op, f.const,
                                     -1 if f.slot is None else f.slot,
                                     -1 if f.normal is None else f.normal, boundary))
    ip_entries = []
    for t, lt in enumerate(ip.terms):
        for ci, comp in enumerate(lt.comps):
            for a in comp:
                if a.boundary_only:
                    raise NotImplementedError("boundary IP terms are not supported")
                ip_entries.append((t, ci, te_index[a.var.id], a.op, a.coef.const,
                                   -1 if a.coef.slot is None else a.coef.slot))
    rhs_terms = []
    if rhs is not None:
        for lt in rhs.terms:
            for a in lt.comps[0]:
                rhs_terms.append((te_index[a.var.id], a.op, a.coef.const, -1 if a.coef.slot is None else a.coef.slot))

    max_test = max(_basis_degree(v, k + dk) for v in test_vars)
    max_trial = max(_basis_degree(v, k) for v in trial_vars)
    traces = [v for v in trial_vars if v.kind != abi.VAR_FIELD]
    max_trace = max((_basis_degree(v, k) for v in traces), default=max_trial)
    degG = 2 * max_test + cubature_enrichment
    degB = max_trial + max_test + cubature_enrichment
    degS = max_trace + max_test + cubature_enrichment
    n_slots = 0
    for t in bf_terms:
        n_slots = max(n_slots, t[5] + 1)
    for t in ip_entries:
        n_slots = max(n_slots, t[5] + 1)
    for t in rhs_terms:
        n_slots = max(n_slots, t[3] + 1)
    n_slots = max(n_slots, len(slot_names))
    holder = abi.DescHolder(topology, trial, test, bf_terms, ip_entries, rhs_terms, degG, degB, degS, n_slots,
                            precision)
    return Bucket(holder, topology, k, dk, n_slots, list(slot_names))


# ----------------------------------------------------------------------------
# Formulations
# ----------------------------------------------------------------------------


class PoissonFormulation:
    """Ultraweak Poisson, conforming traces (PoissonFormulation.cpp:26-80):
       b = (u, div tau) + (sigma, tau) - <u_hat, tau.n> - (sigma, grad v) + <sigma_n_hat, v>.
    Load slot 0 = f at the quadrature points."""

    def __init__(self, space_dim, use_conforming_traces=True):
        vf = VarFactory(space_dim)
        self.vf = vf
        self.u = vf.fieldVar("u")
        self.sigma = vf.fieldVar("sigma", abi.SPACE_VECTOR_HVOL)
        self.u_hat = vf.traceVar("u_hat", abi.SPACE_HGRAD if use_conforming_traces else abi.SPACE_HVOL)
        self.sigma_n_hat = vf.fluxVar("sigma_n_hat")
        self.v = vf.testVar("v", abi.SPACE_HGRAD)
        self.tau = vf.testVar("tau", abi.SPACE_HDIV)
        bf = BF(vf)
        bf.addTerm(self.u, self.tau.div())
        bf.addTerm(self.sigma, self.tau)
        bf.addTerm(-self.u_hat, self.tau.dot_normal())
        bf.addTerm(-self.sigma, self.v.grad())
        bf.addTerm(self.sigma_n_hat, self.v)
        self._bf = bf

    def bf(self):
        return self._bf

    def rhs(self, f=None):
        r = RHS()
        r.addTerm((slot(0) if f is None else f) * self.v)
        return r

    def bucket(self, topology, k, dk, precision=abi.PREC_FP64, constant_load=None):
        f = constant(constant_load) if constant_load is not None else None
        return compile_bucket(self._bf, self._bf.graphNorm(), self.rhs(f), topology, k, dk,
                              slot_names=[] if f is not None else ["f"], precision=precision)


class ConvectionDiffusionReactionFormulation:
    """Ultraweak CDR (ConvectionDiffusionReactionFormulation.cpp:95-103), 2D:
       b = (sigma, tau) + (sqrt_eps u, div tau) - <sqrt_eps u_hat, tau.n>
           + (sqrt_eps sigma - beta u, grad v) - <sigma_n, v> + (alpha u, v).
    Per-point slots: 0 = sqrt(eps), 1 = beta_x, 2 = beta_y, 3 = alpha (c), 4 = f."""
    SLOTS = ["sqrt_eps", "beta_x", "beta_y", "alpha", "f"]

    def __init__(self, space_dim=2):
        if space_dim != 2:
            raise NotImplementedError("CDR mirror is 2D")
        vf = VarFactory(space_dim)
        self.vf = vf
        sq = slot(0)
        beta = VecFn([slot(1), slot(2)])
        alpha = slot(3)
        self.u = vf.fieldVar("u")
        self.sigma = vf.fieldVar("sigma", abi.SPACE_VECTOR_HVOL)
        self.uhat = vf.traceVar("uhat", abi.SPACE_HGRAD)
        self.sigma_n = vf.fluxVar("sigma_n")
        self.v = vf.testVar("v", abi.SPACE_HGRAD)
        self.tau = vf.testVar("tau", abi.SPACE_HDIV)
        bf = BF(vf)
        bf.addTerm(self.sigma, self.tau)
        bf.addTerm(sq * self.u, self.tau.div())
        bf.addTerm(-(sq * self.uhat), self.tau.dot_normal())
        bf.addTerm(sq * self.sigma - beta * self.u, self.v.grad())
        bf.addTerm(-self.sigma_n, self.v)
        bf.addTerm(alpha * self.u, self.v)
        self._bf = bf

    def bf(self):
        return self._bf

    def rhs(self):
        r = RHS()
        r.addTerm(slot(4) * self.v)
        return r

    def bucket(self, topology, k, dk, precision=abi.PREC_FP64):
        return compile_bucket(self._bf, self._bf.graphNorm(), self.rhs(), topology, k, dk,
                              slot_names=self.SLOTS, precision=precision)


class StokesVGPFormulation:
    """Steady velocity-gradient-pressure Stokes (StokesVGPFormulation.cpp:224-407), 2D,
    conforming velocity traces, mu constant."""

    def __init__(self, space_dim=2, mu=1.0):
        if space_dim != 2:
            raise NotImplementedError("Stokes VGP mirror is 2D")
        vf = VarFactory(space_dim)
        self.vf = vf
        d = space_dim
        u = [vf.fieldVar("u1"), vf.fieldVar("u2")]
        p = vf.fieldVar("p")
        s11, s12, s21, s22 = (vf.fieldVar(n) for n in ("sigma11", "sigma12", "sigma21", "sigma22"))
        sigma = [[s11, s12], [s21, s22]]
        u_hat = [vf.traceVar("u1_hat", abi.SPACE_HGRAD), vf.traceVar("u2_hat", abi.SPACE_HGRAD)]
        tn = [vf.fluxVar("t1n"), vf.fluxVar("t2n")]
        v = [vf.testVar("v1", abi.SPACE_HGRAD), vf.testVar("v2", abi.SPACE_HGRAD)]
        tau = [vf.testVar("tau1", abi.SPACE_HDIV), vf.testVar("tau2", abi.SPACE_HDIV)]
        q = vf.testVar("q", abi.SPACE_HGRAD)
        n = normal(d)
        bf = BF(vf)
        for d1 in range(d):
            bf.addTerm(u[d1], tau[d1].div())
            for d2 in range(d):
                bf.addTerm(constant(1.0 / mu) * sigma[d1][d2], tau[d1].spatialComponent(d2 + 1))
            bf.addTerm(-u_hat[d1], tau[d1].dot_normal())
        for d1 in range(d):
            for d2 in range(d):
                bf.addTerm(sigma[d1][d2], v[d1].di(d2 + 1))
            bf.addTerm(-p, v[d1].di(d1 + 1))
            bf.addTerm(tn[d1], v[d1])
        for d1 in range(d):
            bf.addTerm(-u[d1], q.di(d1 + 1))
            bf.addTerm(n.spatialComponent(d1 + 1) * u_hat[d1], q)
        self._bf = bf
        self.u, self.p, self.sigma, self.u_hat, self.tn, self.v, self.tau, self.q = u, p, sigma, u_hat, tn, v, tau, q

    def bf(self):
        return self._bf

    def rhs(self):
        r = RHS()
        r.addTerm(slot(0) * self.v[0])
        r.addTerm(slot(1) * self.v[1])
        return r

    def bucket(self, topology, k, dk, precision=abi.PREC_FP64):
        return compile_bucket(self._bf, self._bf.graphNorm(), self.rhs(), topology, k, dk,
                              slot_names=["f1", "f2"], precision=precision)
