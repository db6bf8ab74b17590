"""CPU baseline of the assembly: the oracle's fast mode (oracle/dpg_oracle.cpp:
assemble_cell_blas -- every quadrature contraction a DGEMM per block, the dense solve in
LAPACK/BLAS, as Camellia's BF::localStiffnessMatrixAndRHS does through Intrepid and
Teuchos) on all host cores, one process per core, each on one BLAS thread.  This mirrors
Camellia's execution model, one MPI rank per core with no threading inside a rank.

TEST INFRASTRUCTURE ONLY (bench.py's CPU-baseline and reference legs; tests/).  The
worker processes are started with the spawn method, so they never inherit a CUDA
context, and they import neither torch nor the CUDA library.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import time


def _worker(conn, bucket_args, nodes, par, coeff):
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    from camellia2_b200 import formulation as fm
    from oracle import oracle
    form, args = bucket_args
    bucket = getattr(fm, form)(args[0]).bucket(*args[1:])
    P = oracle.OraclePlan(bucket)
    n = nodes.shape[0]
    while True:
        cmd = conn.recv()
        if cmd is None:
            break
        m = min(n, int(cmd))
        t0 = time.perf_counter()
        out = P.assemble_blas(nodes[:m], par[:m], None if coeff is None else coeff[:m])
        dt = time.perf_counter() - t0
        conn.send((dt, int((out["info"] != 0).sum())))
    conn.close()


class ProcessBaseline:
    """`cores` worker processes, worker w holding cells w, w + cores, ... of the sample.

    bucket_args = (formulation class name, (space_dim, topology, k, dk)) so each worker
    builds the same bucket; run(per_worker) assembles that many cells in every worker and
    returns (cells, seconds of the slowest worker)."""

    def __init__(self, bucket_args, nodes, par, coeff, cores=None):
        self.cores = cores or os.cpu_count() or 1
        ctx = mp.get_context("spawn")
        self.conns, self.procs = [], []
        for w in range(self.cores):
            a, b = ctx.Pipe()
            sl = slice(w, None, self.cores)
            p = ctx.Process(target=_worker, args=(b, bucket_args, nodes[sl].copy(), par[sl].copy(),
                                                  None if coeff is None else coeff[sl].copy()), daemon=True)
            p.start()
            self.conns.append(a)
            self.procs.append(p)
        self.capacity = min(nodes[w::self.cores].shape[0] for w in range(self.cores))

    def run(self, per_worker):
        per_worker = min(per_worker, self.capacity)
        for c in self.conns:
            c.send(per_worker)
        res = [c.recv() for c in self.conns]
        failed = sum(r[1] for r in res)
        if failed:
            raise RuntimeError(f"CPU baseline: {failed} cells with a failed factorisation")
        return per_worker * self.cores, max(r[0] for r in res)

    def close(self):
        for c in self.conns:
            try:
                c.send(None)
            except (BrokenPipeError, OSError):
                pass
        for p in self.procs:
            p.join(timeout=10)
            if p.is_alive():
                p.kill()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
