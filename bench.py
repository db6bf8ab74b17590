#!/usr/bin/env python
"""Benchmark: condensed DPG cells/s on one B200 (3D hex Poisson ultraweak, 48^3 cells).

Workload (the north-star configuration): 48x48x48 hexes on the unit cube,
interior nodes jittered by U[-0.1h, 0.1h] (seeded), Poisson ultraweak DPG with
H1Order k = 2 (L2 fields of degree 1), test enrichment 1 (v in H1 and tau in
H(div) of degree 3: N = 172, M = 110), f ~ U[-1,1] per quadrature point.
One step = full local assembly + field condensation of all 110,592 cells
(K, l, S, s and info written for every cell).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank assembles its own 48^3 mesh (weak scaling, no
collective on the data path); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "condensed DPG cells/s on 1 B200: mixed vs FP64 form at ≤1e-10 rel err"
# Algorithmic work per c5 cell (reference's operation count: full contractions,
# N^3/3 Cholesky, full TRSM, lower SYRK, condensation): 26.40 MFLOP.
def flops_parts(N, M, nf, nt, QG, QB, QS, nsides, d):
    nv, ntau = 64, 108  # c5 test var sizes (v: HGRAD C3 hex, tau: HDIV I3 hex)
    FG = 2 * ntau * ntau * QG * 1 + 2 * N * N * QG * d + 2 * nv * nv * QG + 2 * ntau * ntau * QG * d
    FB = 2 * (8 * ntau + 24 * ntau * d + 24 * nv * d) * QB + nsides * 2 * (9 * ntau + 4 * nv) * QS
    Fsolve = N ** 3 / 3 + N * N * M + N * M * (M + 1) + N * N + 2 * N * M
    Fcond = 2 * nf ** 3 / 3 + 2 * nf * nf * nt + 2 * nt * nt * nf + 2 * nf * nf + 2 * nt * nf
    return FG, FB, Fsolve, Fcond


def algorithmic_flops_per_cell(*a):
    return sum(flops_parts(*a))


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=48, help="cells per direction (48 -> 110,592 cells)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-extra", action="store_true", help="skip the other configurations' timings")
    p.add_argument("--no-next", action="store_true",
                   help="skip the timings of the kernels after the assembly (recovery, energy, DLS, scatter)")
    p.add_argument("--c3-bucket", default=None, metavar="quad_pK|tri_pK",
                   help="small case for profiler captures: one Stokes VGP bucket (Delta p = 2) of the "
                        "uneven-cell workload on --c3-cells jittered cells, one warm-up launch and one timed "
                        "launch; prints one JSON line")
    p.add_argument("--c3-cells", type=int, default=148)
    p.add_argument("--case", default=None, choices=["c2", "c4"],
                   help="small case for profiler captures: the 2D Poisson k=4 (c2) or CDR k=3 (c4) bucket on "
                        "--case-n x --case-n jittered quads, one warm-up launch and one timed launch; prints one "
                        "JSON line")
    p.add_argument("--case-n", type=int, default=64)
    return p.parse_args()


def run_case(args):
    """One launch of the c2 or c4 bucket on a small jittered quad mesh (small case for ncu)."""
    import torch
    from camellia2_b200 import abi, formulation as fm, lib, mesh
    n = args.case_n
    nodes, par = mesh.quad_grid(n, n, 0.2 if args.case == "c2" else 0.1, seed=1)
    if args.case == "c2":
        plan = lib.Plan(fm.PoissonFormulation(2).bucket(abi.TOPO_QUAD, 4, 2))
        co = mesh.uniform_coeff(nodes.shape[0], 1, plan.info["n_points_total"], seed=1)
    else:
        plan = lib.Plan(fm.ConvectionDiffusionReactionFormulation(2).bucket(abi.TOPO_QUAD, 3, 2))
        co = mesh.cdr_coeff(nodes.shape[0], plan.info, seed=1)
    C = nodes.shape[0]
    dev = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()  # noqa: E731
    dn, dp, dc = dev(nodes), dev(par), dev(co)
    out = plan.alloc_outputs(C)
    plan.assemble(dn, dp, dc, out=out)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    plan.assemble(dn, dp, dc, out=out)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    print(json.dumps({"case": args.case, "N": plan.info["N"], "M": plan.info["M"], "cells": C, "ms": ms,
                      "cells_per_s": C / ms * 1e3, "info_nonzero_cells": int((out["info"] != 0).sum().item())}))


def run_c3_bucket(args):
    """One bucket of the uneven-cell Stokes workload (small case for ncu captures)."""
    import torch
    from camellia2_b200 import abi, formulation as fm, lib, mesh
    kind, p = args.c3_bucket.split("_p")
    topo = abi.TOPO_QUAD if kind == "quad" else abi.TOPO_TRI
    plan = lib.Plan(fm.StokesVGPFormulation(2).bucket(topo, int(p), 2))
    n = int(np.ceil(np.sqrt(args.c3_cells)))
    nodes, par = (mesh.quad_grid(n, n, 0.1, seed=1) if topo == abi.TOPO_QUAD else mesh.tri_grid(n, n, 0.1, seed=1))
    nodes, par = nodes[:args.c3_cells], par[:args.c3_cells]
    C = nodes.shape[0]
    co = mesh.uniform_coeff(C, plan.info["n_slots"], plan.info["n_points_total"], seed=1)
    dev = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()  # noqa: E731
    dn, dp, dc = dev(nodes), dev(par), dev(co)
    out = plan.alloc_outputs(C)
    plan.assemble(dn, dp, dc, out=out)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    plan.assemble(dn, dp, dc, out=out)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    print(json.dumps({"c3_bucket": args.c3_bucket, "N": plan.info["N"], "M": plan.info["M"], "cells": C, "ms": ms,
                      "cells_per_s": C / ms * 1e3, "info_nonzero_cells": int((out["info"] != 0).sum().item())}))


def build_workload(n, seed):
    from camellia2_b200 import abi, formulation as fm, mesh
    bucket = fm.PoissonFormulation(3).bucket(abi.TOPO_HEX, 2, 1)
    nodes, par = mesh.hex_grid(n, n, n, 0.1, seed=seed)
    return bucket, nodes, par


def make_coeff(C, P, seed):
    rng = np.random.default_rng(seed + 1000)
    return rng.uniform(-1.0, 1.0, size=(C, 1, P))


def other_configs(torch):
    """Device throughput (CUDA events, inputs resident) of the other configurations the
    path covers, on seeded synthetic meshes of their sizes: c2 (2D Poisson UW k=4 dk=2,
    256^2 jittered quads), c4 (2D CDR UW k=3 dk=2, 128^2 quads, forward and reverse
    mode with J = sum r^T K r + g^T l), and the c3 buckets one CTA holds (Stokes VGP
    quads p=1,2 and triangles p=1..3, Delta p=2) in one multi-bucket launch.  Context
    for the headline, not bench lines."""
    from camellia2_b200 import abi, formulation as fm, lib, mesh

    def timeit(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    dev = lambda x: torch.as_tensor(np.ascontiguousarray(x)).cuda()  # noqa: E731
    res = {}
    # c2
    b = fm.PoissonFormulation(2).bucket(abi.TOPO_QUAD, 4, 2)
    plan = lib.Plan(b)
    nodes, par = mesh.quad_grid(256, 256, 0.2, seed=1)
    C = nodes.shape[0]
    co = mesh.uniform_coeff(C, 1, plan.info["n_points_total"], seed=1)
    dn, dp, dc = dev(nodes), dev(par), dev(co)
    out = plan.alloc_outputs(C)
    ms = timeit(lambda: plan.assemble(dn, dp, dc, out=out))
    res["c2_poisson2d_k4_256sq"] = {"cells": C, "ms": ms, "cells_per_s": C / ms * 1e3}
    del out
    # c4 forward and reverse
    b = fm.ConvectionDiffusionReactionFormulation(2).bucket(abi.TOPO_QUAD, 3, 2)
    plan = lib.Plan(b)
    nodes, par = mesh.quad_grid(128, 128, 0.1, seed=1)
    C = nodes.shape[0]
    co = mesh.cdr_coeff(C, plan.info, seed=1)
    dn, dp, dc = dev(nodes), dev(par), dev(co)
    out = plan.alloc_outputs(C)
    ms = timeit(lambda: plan.assemble(dn, dp, dc, out=out))
    res["c4_cdr2d_k3_128sq"] = {"cells": C, "ms": ms, "cells_per_s": C / ms * 1e3}
    M = plan.info["M"]
    rng = np.random.default_rng(5)
    r = rng.normal(size=(C, M))
    Kbar, lbar = dev(r[:, :, None] * r[:, None, :]), dev(rng.normal(size=(C, M)))
    ms = timeit(lambda: plan.adjoint(dn, dp, dc, Kbar, lbar))
    res["c4_cdr2d_k3_128sq_adjoint"] = {"cells": C, "ms": ms, "cells_per_s": C / ms * 1e3}
    del out, Kbar
    # c3 buckets that fit one CTA, one multi-bucket launch
    items, total = [], 0
    for topo, k, make in ((abi.TOPO_QUAD, 1, mesh.quad_grid), (abi.TOPO_QUAD, 2, mesh.quad_grid),
                          (abi.TOPO_TRI, 1, mesh.tri_grid), (abi.TOPO_TRI, 2, mesh.tri_grid),
                          (abi.TOPO_TRI, 3, mesh.tri_grid)):
        pl = lib.Plan(fm.StokesVGPFormulation(2).bucket(topo, k, 2))
        nodes, par = make(64, 64 if topo == abi.TOPO_QUAD else 32, 0.1, seed=k)
        C = nodes.shape[0]
        co = mesh.uniform_coeff(C, pl.info["n_slots"], pl.info["n_points_total"], seed=k)
        items.append((pl, dev(nodes), dev(par), dev(co), pl.alloc_outputs(C)))
        total += C
    ms = timeit(lambda: lib.assemble_multi(items))
    res["c3_stokes_quads_p1_2_tris_p1_3_multi"] = {"cells": total, "ms": ms, "cells_per_s": total / ms * 1e3}
    del items
    res["c3_stokes_forest_100k_graph"] = c3_forest(torch, timeit, dev)
    return res


def c3_forest(torch, timeit, dev, total=100_000):
    """The uneven-cell Stokes VGP workload: ~100k cells (70 % quads, 30 % triangles, p uniform
    on 1..6, Delta p = 2, refinement level geometric on 0..4, jittered), twelve (topology, p)
    buckets in ONE persistent launch with a dynamic work queue (single-CTA and large buckets
    alike, longest cells first), captured in a CUDA graph.  Tuned first: each bucket's shape by
    dpg_plan_autotune on its own cells (Gram staging chunk for single-CTA buckets, formation
    k-chunk for large ones), then the queue's claim size by dpg_multi_autotune.  Per-bucket
    device times come from single-bucket launches."""
    from camellia2_b200 import formulation as fm, lib, mesh
    form = fm.StokesVGPFormulation(2)
    items, keys, per = [], [], {}
    for (topo, p), (nodes, par) in mesh.forest_buckets(total, seed=7).items():
        pl = lib.Plan(form.bucket(topo, p, 2))
        C = nodes.shape[0]
        co = mesh.uniform_coeff(C, pl.info["n_slots"], pl.info["n_points_total"], seed=p)
        items.append((pl, dev(nodes), dev(par), dev(co), pl.alloc_outputs(C)))
        keys.append(("quad" if topo == 1 else "tri") + f"_p{p}")
    for key, (pl, dn, dp, dc, out) in zip(keys, items):
        C = dn.shape[0]
        N, M = pl.info["N"], pl.info["M"]
        shape = pl.autotune(dn, dp, dc)  # per-bucket shape, timed on these cells
        big = shape in (16, 32)  # formation k-chunk of a large-bucket plan (Gram chunks are 8 or 4)
        ms = timeit(lambda: pl.assemble(dn, dp, dc, out=out), reps=1)
        per[key] = {"cells": C, "N": N, "M": M, "ms": round(ms, 3), "cells_per_s": round(C / ms * 1e3),
                    "kernel": "large-bucket" if big else "single-CTA",
                    ("formation_chunk" if big else "gram_chunk"): shape}
    claim = lib.multi_autotune(items)
    g = lib.Graph(items, claim=claim)
    ms = timeit(g.launch, reps=2)
    bad = sum(int((it[4]["info"] != 0).sum().item()) for it in items)
    g.close()
    n = sum(it[1].shape[0] for it in items)
    return {"cells": n, "ms": ms, "cells_per_s": n / ms * 1e3, "info_nonzero_cells": bad, "queue_claim": claim,
            "launches_per_assembly": 1, "buckets": per}


def measured_hbm_gbs():
    """HBM copy bandwidth measured on this GPU model (MEASURED_PEAKS.json beside this file)."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        return 6650.0


def next_rows(torch, plan, info, n, d_nodes, d_par, d_co, out, peak_tflops, hbm_gbs):
    """The per-cell kernels that follow the assembly (field recovery, energy error, DLS
    local matrices, global scatter of S, s) timed on the same 48^3 workload, inputs
    resident (CUDA events, 3 launches after one warm-up), each with its roofline."""
    from camellia2_b200 import lib, mesh

    def timeit(fn, reps=5):
        # median of single launches, after one warm-up
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(statistics.median(ts))

    C, M, N, nf, nt = d_nodes.shape[0], info["M"], info["N"], info["n_field"], info["n_trace"]
    FG, FB, _, _ = flops_parts(N, M, nf, nt, info["Q_G"], info["Q_B"], info["Q_side"], info["n_sides"],
                               info["space_dim"])
    res = {}
    g = torch.Generator(device=d_nodes.device).manual_seed(7)
    tr = torch.rand((C, nt), dtype=torch.float64, device=d_nodes.device, generator=g) * 2 - 1
    u = [None]

    def rec():
        u[0], _ = plan.recover_fields(out["K"], out["l"], tr)
    ms = timeit(rec)
    by = 8 * (nf * M + nf + nt + M)  # K rows of the fields (K_ff | K_ft), l_f, t in; u out
    res["recover_fields"] = {"ms": ms, "cells_per_s": C / ms * 1e3, "bound": "hbm", "bytes_per_cell": by,
                             "achieved_gbs": by * C / ms * 1e-6, "frac_of_measured_hbm": by * C / ms * 1e-6 / hbm_gbs}
    fl = FG + FB + N ** 3 / 3 + N * N + 2 * N * M + 2 * N
    ms = timeit(lambda: plan.energy_error(d_nodes, d_par, d_co, u[0]))
    res["energy_error"] = {"ms": ms, "cells_per_s": C / ms * 1e3, "bound": "tensor", "flops_per_cell": fl,
                           "achieved_tflops": fl * C / ms * 1e-9, "frac_of_measured_fp64": fl * C / ms * 1e-9 / peak_tflops}
    del u[0]
    fl = FG + FB + N ** 3 / 3 + N * N * M + N * N
    ms = timeit(lambda: plan.dls(d_nodes, d_par, d_co))
    res["dls"] = {"ms": ms, "cells_per_s": C / ms * 1e3, "bound": "tensor", "flops_per_cell": fl,
                  "achieved_tflops": fl * C / ms * 1e-9, "frac_of_measured_fp64": fl * C / ms * 1e-9 / peak_tflops,
                  "out_bytes_per_cell": 8 * (M * N + N)}
    # reverse mode: dJ/df per point for J = sum_c (r^T K r + g^T l)
    rr = torch.rand((C, M), dtype=torch.float64, device=d_nodes.device, generator=g) - 0.5
    Kbar = rr[:, :, None] * rr[:, None, :]
    lbar = torch.rand((C, M), dtype=torch.float64, device=d_nodes.device, generator=g) - 0.5
    ms = timeit(lambda: plan.adjoint(d_nodes, d_par, d_co, Kbar, lbar))
    res["adjoint"] = {"ms": ms, "cells_per_s": C / ms * 1e3,
                      "what": "dpg_assemble_adjoint: Gram, B, Cholesky, X = G^-1 [B | F] recomputed, pull-back to f"}
    del Kbar, lbar, rr
    torch.cuda.empty_cache()
    # global scatter with the conforming-shaped trace map of the hex grid
    gid_np, ng = mesh.hex_trace_map(n, n, n, 2)
    gid = torch.as_tensor(gid_np, device=d_nodes.device)
    keys = (gid[:, :, None] * ng + gid[:, None, :]).reshape(-1)
    keys = torch.unique(keys)
    rows, cols = keys // ng, keys % ng
    del keys
    row_ptr = torch.zeros(ng + 1, dtype=torch.int64, device=d_nodes.device)
    row_ptr[1:] = torch.cumsum(torch.bincount(rows, minlength=ng), 0)
    del rows
    nnz = cols.shape[0]
    ptr = torch.arange(C * nt + 1, dtype=torch.int64, device=d_nodes.device)
    gflat = gid.reshape(-1).contiguous()
    vals = torch.empty(nnz, dtype=torch.float64, device=d_nodes.device)
    rhs = torch.empty(ng, dtype=torch.float64, device=d_nodes.device)
    miss = [None]

    def scat():
        vals.zero_()
        rhs.zero_()
        miss[0] = lib.scatter_global(out["S"], out["s"], ptr, gflat, None, ng, row_ptr, cols, vals, rhs)
    ms = timeit(scat)
    by = 8 * C * (nt * nt + nt) + 16 * C * nt + 16 * nnz + 8 * (ng + 1) + 8 * ng
    res["scatter_global"] = {"ms": ms, "cells_per_s": C / ms * 1e3, "bound": "hbm", "n_global": ng, "nnz": nnz,
                             "bytes": by, "achieved_gbs": by / ms * 1e-6, "frac_of_measured_hbm": by / ms * 1e-6 / hbm_gbs,
                             "missing": int(miss[0].item()),
                             "map": "hex trace points identified by lattice position (50 global dofs per cell)"}
    # the same with the symbolic part done once (dpg_scatter_plan_*)
    t0 = time.perf_counter()
    splan = lib.ScatterPlan(C, nt, ptr, gflat, None, ng, row_ptr, cols)
    torch.cuda.synchronize()
    create_ms = (time.perf_counter() - t0) * 1e3

    def scat_plan():
        vals.zero_()
        rhs.zero_()
        splan.apply(out["S"], out["s"], vals, rhs)
    ms = timeit(scat_plan)
    gs = np.sort(gid_np, axis=1)
    pairs = int((((gs[:, 1:] != gs[:, :-1]).sum(axis=1) + 1) ** 2).sum())
    by = 8 * C * (nt * nt + nt) + 4 * pairs + 8 * nnz + 8 * ng
    res["scatter_global_plan_apply"] = {"ms": ms, "cells_per_s": C / ms * 1e3, "bound": "hbm", "bytes": by,
                                        "distinct_pairs": pairs, "achieved_gbs": by / ms * 1e-6,
                                        "frac_of_measured_hbm": by / ms * 1e-6 / hbm_gbs,
                                        "plan_create_ms_wall": create_ms, "missing": int(splan.missing.item())}
    del splan, vals, cols, row_ptr
    torch.cuda.empty_cache()
    return res


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sms.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sms)}


def fp64_peak_tflops(torch):
    """Live FP64 peak on this GPU: torch float64 GEMM 8192^3, best of 3."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


C5_BUCKET_ARGS = ("PoissonFormulation", (3, 2, 2, 1))  # 3D, TOPO_HEX, k = 2, dk = 1


def _baseline_pool(nodes, par, coeff, cores, max_per_worker=4096):
    """Oracle fast mode (BLAS/LAPACK per block, one BLAS thread) in one spawned process per
    host core, like Camellia's one MPI rank per core (oracle/cpu_baseline.py)."""
    from oracle.cpu_baseline import ProcessBaseline
    m = min(nodes.shape[0], max_per_worker * cores)
    return ProcessBaseline(C5_BUCKET_ARGS, nodes[:m], par[:m], coeff[:m], cores=cores)


def _sample_size(pool, budget_s):
    cells, dt = pool.run(4)  # warm-up and calibration
    cells, dt = pool.run(16)
    return max(4, min(pool.capacity, int(budget_s / max(dt / 16, 1e-6))))


def cpu_baseline(bucket, nodes, par, coeff, budget_s=10.0):
    """The oracle's fast mode on all host cores (one process per core), on a bounded
    sample of the same cells."""
    cores = os.cpu_count() or 1
    with _baseline_pool(nodes, par, coeff, cores) as pool:
        per = _sample_size(pool, budget_s)
        cells, dt = pool.run(per)
    return {"value": cells / dt, "unit": "cells/s", "cores": cores, "kind": "port",
            "sample": f"{cells} cells of the 48^3 jittered hex mesh ({per} per process), full K/l/S/s per cell; "
                      f"{cores} processes, one per host core, each on one BLAS thread (oracle fast mode: "
                      "DGEMM per quadrature block, LAPACK/BLAS solve)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = args.n
    bucket, nodes, par = build_workload(n, 1)
    from oracle import oracle
    P = oracle.OraclePlan(bucket)
    coeff = make_coeff(nodes.shape[0], P.info["n_points_total"], 1)
    cores = os.cpu_count() or 1
    with _baseline_pool(nodes, par, coeff, cores) as pool:
        per = _sample_size(pool, 3.0)  # each step a bounded sample of about 3 s
        for _ in range(args.warmup):
            pool.run(4)
        times, cells = [], 0
        for _ in range(args.steps):
            cells, dt = pool.run(per)
            times.append(dt)
    ms = 1e3 * statistics.mean(times)
    value = cells / (ms * 1e-3)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"3D hex Poisson ultraweak DPG, {n}^3 jittered hexes, k=2 dk=1 (N=172, M=110)",
                   "cells": int(nodes.shape[0]), "sample_cells_per_step": cells},
        "cpu_baseline": {"value": value, "unit": "cells/s", "cores": cores, "kind": "port",
                         "sample": f"{cells} cells per step ({per} per process), {cores} processes, one per host "
                                   "core, each on one BLAS thread: the oracle's fast mode (DGEMM per quadrature "
                                   "block, LAPACK/BLAS solve); the reference itself is not buildable here "
                                   "(Trilinos/MOAB absent)"},
        "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.c3_bucket:
        run_c3_bucket(args)
        return
    if args.case:
        run_case(args)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from camellia2_b200 import lib
    from camellia2_b200.shard import max_over_ranks

    n = args.n
    bucket, nodes, par = build_workload(n, 1 + rank)
    plan = lib.Plan(bucket)
    info = plan.info
    C = nodes.shape[0]
    coeff = make_coeff(C, info["n_points_total"], 1 + rank)
    dev = torch.device("cuda", local)
    d_nodes = torch.as_tensor(nodes, device=dev)
    d_par = torch.as_tensor(par, device=dev)
    d_co = torch.as_tensor(coeff, device=dev)
    out = plan.alloc_outputs(C, dev)
    stream = torch.cuda.current_stream()

    # parity spot check against the oracle on the first cells (rank 0)
    parity = None
    if rank == 0:
        from oracle import oracle
        m = 16
        ref = oracle.OraclePlan(bucket).assemble(nodes[:m], par[:m], coeff[:m], nthreads=os.cpu_count() or 1)
        plan.assemble(d_nodes[:m], d_par[:m], d_co[:m], out={k: v[:m] for k, v in out.items()})
        torch.cuda.synchronize()
        parity = {}
        for k in ("K", "l", "S", "s"):
            a = out[k][:m].cpu().numpy()
            parity[k] = float(max(np.linalg.norm(a[c] - ref[k][c]) / np.linalg.norm(ref[k][c]) for c in range(m)))

    for _ in range(args.warmup):
        plan.assemble(d_nodes, d_par, d_co, out=out)
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.assemble(d_nodes, d_par, d_co, out=out, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = clk.stop()
    ms_total = max_over_ranks(e0.elapsed_time(e1), dev)
    ms = ms_total / args.steps
    value = world * C / (ms * 1e-3)
    bad = int((out["info"] != 0).sum().item())

    # ---- end to end through the host C-ABI call (pinned host buffers) -----------
    e2e = e2e_cond = None
    if not args.no_e2e:
        h_nodes = torch.as_tensor(nodes).pin_memory()
        h_par = torch.as_tensor(par).pin_memory()
        h_co = torch.as_tensor(coeff).pin_memory()
        M, t = info["M"], info["n_trace"]
        hout = {"K": torch.empty((C, M, M), dtype=torch.float64).pin_memory(),
                "l": torch.empty((C, M), dtype=torch.float64).pin_memory(),
                "S": torch.empty((C, t, t), dtype=torch.float64).pin_memory(),
                "s": torch.empty((C, t), dtype=torch.float64).pin_memory(),
                "info": torch.empty((C,), dtype=torch.int32).pin_memory()}
        plan.assemble_host(h_nodes, h_par, h_co, out=hout)  # warm-up (workspace)
        e_steps = max(1, min(args.steps, 3))
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(e_steps):
            plan.assemble_host(h_nodes, h_par, h_co, out=hout)
        f1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(f0.elapsed_time(f1) / e_steps, dev)
        h2d = sum(x.numel() * x.element_size() for x in (h_nodes, h_par, h_co))
        d2h = sum(x.numel() * x.element_size() for x in hout.values())
        e2e = {"value": world * C / (ems * 1e-3), "unit": "cells/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": ems,
               "path": "dpg_assemble_host (C ABI), pinned host buffers, 2-stream chunked copies"}
        # The same call with DPG_FLAG_NO_K: only the condensed S, s come back (the reference's
        # CondensedDofInterpreter recomputes K per cell when it holds none, CondensedDofInterpreter.cpp:106).
        hc = {"S": hout["S"], "s": hout["s"], "info": hout["info"], "K": None, "l": None}
        plan.assemble_host(h_nodes, h_par, h_co, out=hc, flags=1)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        f0.record(stream)
        for _ in range(e_steps):
            plan.assemble_host(h_nodes, h_par, h_co, out=hc, flags=1)
        f1.record(stream)
        torch.cuda.synchronize()
        cms = max_over_ranks(f0.elapsed_time(f1) / e_steps, dev)
        e2e_cond = {"value": world * C / (cms * 1e-3), "unit": "cells/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": sum(x.numel() * x.element_size() for x in (hout["S"], hout["s"], hout["info"])),
                    "ms_per_step": cms, "path": "dpg_assemble_host with DPG_FLAG_NO_K (S, s and info only)"}

    if rank == 0:
        peak = fp64_peak_tflops(torch)
        fl = algorithmic_flops_per_cell(info["N"], info["M"], info["n_field"], info["n_trace"], info["Q_G"],
                                        info["Q_B"], info["Q_side"], info["n_sides"], info["space_dim"])
        achieved = fl * C / (ms * 1e-3) / 1e12
        traffic = None
        tp = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tp):
            try:
                traffic = json.load(open(tp)).get("dpg_cell_kernel_fp64_bytes_per_launch")
            except Exception:
                traffic = None
        cpu = None if args.no_cpu else cpu_baseline(bucket, nodes, par, coeff)
        M_, t_ = info["M"], info["n_trace"]
        out_bytes = 8 * C * (M_ * M_ + M_ + t_ * t_ + t_) + 4 * C
        in_bytes = C * (8 * info["n_vertices"] * info["space_dim"] + info["n_sides"] +
                        8 * info["n_slots"] * info["n_points_total"])
        line = {
            "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"3D hex Poisson ultraweak DPG, {n}^3 jittered hexes (0.1h), k=2 dk=1 "
                                   f"(N={info['N']}, M={info['M']}, f={info['n_field']}, t={info['n_trace']})",
                       "cells": C, "form": "fp64",
                       "l2": f"no flush: each step reads {in_bytes / 1e9:.2f} GB and writes {out_bytes / 1e9:.1f} GB "
                             f"({'>' if out_bytes > 126e6 else '<'} 126 MB L2)",
                       "parallelism": f"{world} GPU(s), cells sharded (weak), no data-path collective"},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "flops_per_cell": fl, "peak_source": "measured live: torch float64 GEMM 8192^3 (DMMA d884), FP64 tensor pipe"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "e2e_condensed": e2e_cond,
            "gpu_launches": args.steps,
            "clocks": clocks,
            "parity_vs_oracle_max_rel": parity,
            "info_nonzero_cells": bad,
            "other_configs": None if args.no_extra else other_configs(torch),
            "next_rows": None if args.no_next else next_rows(torch, plan, info, n, d_nodes, d_par, d_co, out, peak,
                                                             measured_hbm_gbs()),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
