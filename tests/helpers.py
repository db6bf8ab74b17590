"""Workload builders shared by the tests (small versions of the bench configs)."""
import numpy as np

from camellia2_b200 import abi, formulation as fm, mesh


def poisson2d(k, dk, nx=3, ny=3, jitter=0.2, seed=1, load="random"):
    form = fm.PoissonFormulation(2)
    bucket = form.bucket(abi.TOPO_QUAD, k, dk)
    nodes, par = mesh.quad_grid(nx, ny, jitter, seed=seed)
    return form, bucket, nodes, par


def poisson3d(k, dk, n=2, jitter=0.1, seed=1):
    form = fm.PoissonFormulation(3)
    bucket = form.bucket(abi.TOPO_HEX, k, dk)
    nodes, par = mesh.hex_grid(n, n, n, jitter, seed=seed)
    return form, bucket, nodes, par


def cdr2d(k, dk, nx=3, ny=3, jitter=0.0, seed=1):
    form = fm.ConvectionDiffusionReactionFormulation(2)
    bucket = form.bucket(abi.TOPO_QUAD, k, dk)
    nodes, par = mesh.quad_grid(nx, ny, jitter, seed=seed)
    return form, bucket, nodes, par


def stokes2d(k, dk, nx=2, ny=2, jitter=0.1, seed=1):
    form = fm.StokesVGPFormulation(2)
    bucket = form.bucket(abi.TOPO_QUAD, k, dk)
    nodes, par = mesh.quad_grid(nx, ny, jitter, seed=seed)
    return form, bucket, nodes, par


def poisson_tri(k, dk, nx=2, ny=2, jitter=0.15, seed=1):
    form = fm.PoissonFormulation(2)
    bucket = form.bucket(abi.TOPO_TRI, k, dk)
    nodes, par = mesh.tri_grid(nx, ny, jitter, seed=seed)
    return form, bucket, nodes, par


def stokes_tri(k, dk, nx=2, ny=1, jitter=0.1, seed=1):
    form = fm.StokesVGPFormulation(2)
    bucket = form.bucket(abi.TOPO_TRI, k, dk)
    nodes, par = mesh.tri_grid(nx, ny, jitter, seed=seed)
    return form, bucket, nodes, par


def coeffs_for(bucket, info, C, seed=2):
    if bucket.n_slots == 0:
        return None
    if bucket.slot_names and bucket.slot_names[0] == "sqrt_eps":
        return mesh.cdr_coeff(C, info, seed=seed)
    return mesh.uniform_coeff(C, bucket.n_slots, info["n_points_total"], seed=seed)
