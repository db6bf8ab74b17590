"""Reverse mode through torch.autograd on the CDR workload (c4: 128 x 128 quads, field
degree 2, dk = 2), the wrapper living in the test harness only.

AssembleKL is a torch.autograd.Function whose forward is dpg_assemble (K, l from the
per-point coefficient slots) and whose backward is dpg_assemble_adjoint (C ABI).  The
leaves are the workload's physical coefficients -- eps per point, the convection angle
theta per cell (beta = (cos theta, sin theta)), the reaction c per point and the load f per
point -- and torch's own chain rule maps them onto the slots (sqrt(eps), beta_x, beta_y,
c, f).  For J = sum_e (r_e^T K_e r_e + g_e^T l_e), r, g ~ N(0, 1), the gradient of every
leaf is checked on sampled cells of the full mesh:
  * against the oracle's hand gradient computed in __float128 (the same chain rule applied
    in numpy), relative error <= 1e-8 per leaf;
  * against central finite differences with step 1e-6 of the extended-precision forward
    (J returned as a pair of doubles), along 16 random unit directions in the sample's
    (eps, theta, c, f) space and 64 single coordinates: within 1e-6 relative;
  * in slot space, the raw adjoint against the oracle's __float128 central difference
    (truncation-limited), within 1e-8 relative.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from camellia2_b200 import abi, formulation as fm, lib as dlib, mesh  # noqa: E402

pytestmark = pytest.mark.gpu

STEP = 1e-6
NTH = os.cpu_count() or 1


class AssembleKL(torch.autograd.Function):
    """(K, l) of a bucket as a function of its coefficient slots (C, n_slots, points)."""

    @staticmethod
    def forward(ctx, coeff, plan, nodes, parity):
        out = plan.assemble(nodes, parity, coeff.contiguous())
        assert int(out["info"].abs().max()) == 0
        ctx.save_for_backward(coeff)
        ctx.plan, ctx.nodes, ctx.parity = plan, nodes, parity
        return out["K"], out["l"]

    @staticmethod
    def backward(ctx, Kbar, lbar):
        (coeff,) = ctx.saved_tensors
        C, M = coeff.shape[0], ctx.plan.info["M"]
        if Kbar is None:
            Kbar = torch.zeros((C, M, M), dtype=torch.float64, device=coeff.device)
        if lbar is None:
            lbar = torch.zeros((C, M), dtype=torch.float64, device=coeff.device)
        cbar, info = ctx.plan.adjoint(ctx.nodes, ctx.parity, coeff.contiguous(), Kbar.contiguous(),
                                      lbar.contiguous())
        assert int(info.abs().max()) == 0
        return cbar, None, None, None


def slots_of(eps, theta, c, f):
    """Coefficient slots (sqrt(eps), beta_x, beta_y, c, f) from the physical leaves."""
    P = eps.shape[1]
    bx = torch.cos(theta)[:, None].expand(-1, P)
    by = torch.sin(theta)[:, None].expand(-1, P)
    return torch.stack([torch.sqrt(eps), bx, by, c, f], dim=1)


def slots_np(eps, theta, c, f):
    P = eps.shape[1]
    return np.stack([np.sqrt(eps), np.repeat(np.cos(theta)[:, None], P, 1), np.repeat(np.sin(theta)[:, None], P, 1),
                     c, f], axis=1)


@pytest.fixture(scope="module")
def c4():
    bucket = fm.ConvectionDiffusionReactionFormulation(2).bucket(abi.TOPO_QUAD, 3, 2)
    plan = dlib.Plan(bucket)
    nodes, par = mesh.quad_grid(128, 128, 0.1, seed=1)
    C, P, M = nodes.shape[0], plan.info["n_points_total"], plan.info["M"]
    rng = np.random.default_rng(1)
    eps = np.exp(rng.normal(-4.0, 1.0, size=(C, P)))
    theta = rng.uniform(0.0, 2 * np.pi, size=C)
    c = rng.uniform(0.0, 1.0, size=(C, P))
    f = rng.uniform(-1.0, 1.0, size=(C, P))
    r = rng.normal(size=(C, M))
    g = rng.normal(size=(C, M))
    dev = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()  # noqa: E731
    leaves = [dev(x).requires_grad_() for x in (eps, theta, c, f)]
    K, l = AssembleKL.apply(slots_of(*leaves), plan, dev(nodes), dev(par))
    dr, dg = dev(r), dev(g)
    J = torch.einsum("ci,cij,cj->", dr, K, dr) + torch.einsum("ci,ci->", dg, l)
    J.backward()
    torch.cuda.synchronize()
    grads = [x.grad.cpu().numpy() for x in leaves]
    pick = np.unique(np.concatenate([[0, C - 1], rng.choice(C, size=6, replace=False)]))
    return dict(bucket=bucket, plan=plan, nodes=nodes, par=par, params=(eps, theta, c, f), r=r, g=g, grads=grads,
                pick=pick, J=float(J.detach()))


def _sample(c4, cells):
    eps, theta, c, f = c4["params"]
    r, g = c4["r"][cells], c4["g"][cells]
    return (c4["nodes"][cells], c4["par"][cells], (eps[cells], theta[cells], c[cells], f[cells]),
            r[:, :, None] * r[:, None, :], g)


def test_leaf_gradients_match_the_extended_precision_hand_gradient(c4, oracle_mod):
    X = oracle_mod.OraclePlan(c4["bucket"], xp=True)
    nodes, par, (eps, theta, c, f), Kb, lb = _sample(c4, c4["pick"])
    cbar = X.adjoint(nodes, par, slots_np(eps, theta, c, f), Kb, lb, nthreads=NTH)
    ref = [cbar[:, 0] / (2 * np.sqrt(eps)),
           (-np.sin(theta)[:, None] * cbar[:, 1] + np.cos(theta)[:, None] * cbar[:, 2]).sum(axis=1),
           cbar[:, 3], cbar[:, 4]]
    for name, got, want in zip(("eps", "theta", "c", "f"), c4["grads"], ref):
        got = got[c4["pick"]]
        assert np.linalg.norm(got - want) <= 1e-8 * np.linalg.norm(want), name


def test_leaf_gradients_match_central_differences(c4, oracle_mod):
    X = oracle_mod.OraclePlan(c4["bucket"], xp=True)
    pick = c4["pick"]
    nodes, par, params, Kb, lb = _sample(c4, pick)
    grads = [gr[pick] for gr in c4["grads"]]

    def J(ps, cells=slice(None)):
        hi, lo = X.loss(nodes[cells], par[cells], slots_np(*[p[cells] for p in ps]), Kb[cells], lb[cells],
                        nthreads=NTH)
        return hi, lo

    def fd(dirs, cells=slice(None)):
        hp, lp = J([p + STEP * d for p, d in zip(params, dirs)], cells)
        hm, lm = J([p - STEP * d for p, d in zip(params, dirs)], cells)
        return ((hp - hm) + (lp - lm)) / (2 * STEP)

    rng = np.random.default_rng(17)
    for _ in range(16):
        dirs = [rng.normal(size=p.shape) for p in params]
        nrm = np.sqrt(sum(float((d * d).sum()) for d in dirs))
        dirs = [d / nrm for d in dirs]
        ad = sum(float((gr * d).sum()) for gr, d in zip(grads, dirs))
        ref = fd(dirs)
        assert abs(ad - ref) <= 1e-6 * abs(ref), (ad, ref)
    sizes = [p.size for p in params]
    for k in rng.choice(sum(sizes), size=64, replace=False):
        which = int(np.searchsorted(np.cumsum(sizes), k, side="right"))
        local = int(k - sum(sizes[:which]))
        idx = np.unravel_index(local, params[which].shape)
        cell = int(idx[0])
        dirs = [np.zeros_like(p) for p in params]
        dirs[which][idx] = 1.0
        ad = float(grads[which][idx])
        ref = fd(dirs, slice(cell, cell + 1))
        assert abs(ad - ref) <= 1e-6 * abs(ref) + 1e-14, (which, idx, ad, ref)


def test_slot_gradient_matches_extended_precision_differences(c4, oracle_mod):
    """The raw adjoint (slot space) along random directions, against the oracle's difference
    taken entirely in __float128 (truncation-limited at step 1e-6)."""
    X = oracle_mod.OraclePlan(c4["bucket"], xp=True)
    pick = c4["pick"]
    nodes, par, params, Kb, lb = _sample(c4, pick)
    co = slots_np(*params)
    dev = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()  # noqa: E731
    cbar, info = c4["plan"].adjoint(dev(nodes), dev(par), dev(co), dev(Kb), dev(lb))
    torch.cuda.synchronize()
    assert int(info.abs().max()) == 0
    cbar = cbar.cpu().numpy()
    rng = np.random.default_rng(23)
    for _ in range(16):
        d = rng.normal(size=co.shape)
        d /= np.linalg.norm(d)
        ref = X.fd_directional(nodes, par, co, d, STEP, Kb, lb, nthreads=NTH)
        assert abs(float((cbar * d).sum()) - ref) <= 1e-8 * abs(ref), ref
