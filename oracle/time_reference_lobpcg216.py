"""Times the reference's distributed real LOBPCG (LOBPCG::Eigen_d_multi_mpi,
lobpcg_d_multi_mpi.h:882-1572, through oracle/_ref) on the 216-atom 3x3x3 diamond cell
(120^3, atoms displaced by seeded Gaussian sigma 0.05 bohr, 528 states) for a few
iterations on one rank, DGEMMs on OpenBLAS threads, and prints one JSON line with the
seconds of every iteration and of the reference's own watch sections.

This is the CPU comparator of the GPU engine's 216-atom solve. It needs about 52 GB of
host memory (7 blocks of 528 states x 1.73 M points) and several minutes per iteration,
so it is run by hand, not by the test suite or the bench:

    python oracle/time_reference_lobpcg216.py --iters 3 --threads 8
"""
import argparse
import json
import os
import platform
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import oracle as O  # noqa: E402
from qumasun_b200.cell import build_cell  # noqa: E402


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--iters", type=int, default=3)
    p.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    p.add_argument("--states", type=int, default=528)
    a = p.parse_args()
    cell = build_cell(reps=(3, 3, 3), displacement=0.05, seed=2024)
    rng = np.random.default_rng(2024)
    X = rng.uniform(-0.5, 0.5, size=(a.states, cell.N))  # the solver works on this array in place
    t0 = time.perf_counter()
    r = O.ref_lobpcg_d_mpi(cell, X, a.iters, threads=a.threads, in_place=True)
    wall = time.perf_counter() - t0
    its = r["iteration_s"]
    out = {"workload": "diamond216_120cube_528states_fd8_reference_Eigen_d_multi_mpi_one_rank",
           "iterations": r["iters"], "iteration_s": [round(v, 2) for v in its],
           "steady_iteration_s": round(its[-1], 2) if len(its) > 1 else None,
           "phase_s": {k: round(v, 2) for k, v in r["phase_s"].items()},
           "wall_s": round(wall, 1), "openblas_threads": a.threads, "host_cpus": os.cpu_count(),
           "cpu": platform.processor() or platform.machine(),
           "note": "H applications single-threaded (the reference has no OpenMP); the first iteration "
                   "solves the 2n pencil (P starts from zero)"}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
