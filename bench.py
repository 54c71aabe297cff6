#!/usr/bin/env python3
"""Benchmark of the Kohn-Sham H|psi> path on the B200 (and the reference CPU arm).

Workload (one "step"): one application of H = V + V_NL - 1/2 Lap (8th-order FD)
to a batch of 256 states of the 64-atom diamond cell on an 80^3 grid, FP64,
states resident in HBM (1.05 GB of states in, 1.05 GB out: larger than L2, so
no flush is needed between steps). ``value`` is algorithmic HBM GB/s of the
whole apply:  bytes = N*ns*2*8 (read psi, write H psi) + N*8 (V)
                    + n_atoms*4*n_sphere*8 (projector tables).
``e2e`` is the same metric through the host-buffer C entry point
(qg_hamiltonian_apply_host_d) with pinned host states: H2D + apply + D2H.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun each rank applies H to its own 256 states on its own GPU
(weak scaling, no data-path collective); ``value`` is the total over ranks
divided by the max over ranks of the device time.
"""
from __future__ import annotations

import argparse
import math
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NS = 256
REPS = (2, 2, 2)
# The dominant kernel of the apply and its DRAM bytes (dram__bytes_read.sum +
# dram__bytes_write.sum) per state of this workload, from an ncu capture of the same bench
# at 32 states; traffic grows in proportion to the states, so a full launch is scaled.
STENCIL_KERNEL = "k_stencil_rows<double, 8, 80> (FD stencil + V, two rows per thread, V in the ring)"
STENCIL_DRAM_BYTES_PER_STATE = (138647296 + 92578048) / 32
FD_ORDER = 8
WORKLOAD = "diamond64_80cube_Hpsi"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-sweep", action="store_true", help="skip the FD order 2/4/6/8 x FP64/FP32 sweep")
    p.add_argument("--no-lobpcg", action="store_true", help="skip the LOBPCG time-to-solution legs")
    p.add_argument("--no-lobpcg216", action="store_true",
                   help="skip the 216-atom 120^3 LOBPCG leg (FP64 vs BF16x3 Gram, about a minute)")
    p.add_argument("--states", type=int, default=NS, help="states per apply (smaller for profiling captures)")
    p.add_argument("--no-e2e", action="store_true", help="skip the host-buffer (e2e) leg")
    p.add_argument("--no-kpoint", action="store_true", help="skip the k-point leg (64 Monkhorst-Pack points)")
    p.add_argument("--no-cells", action="store_true",
                   help="skip the 16-cell leg (8- to 64-atom cells solved one by one and together)")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the engine's default launch shapes (profiling captures)")
    p.add_argument("--no-scf", action="store_true",
                   help="skip the SCF-step leg (density, potential, Taylor-4 step, nonlocal forces)")
    p.add_argument("--no-learned", action="store_true",
                   help="skip the learned-preconditioner leg (GPU training and an unseen-cell comparison)")
    p.add_argument("--only", choices=["kpoint", "gram", "cells", "netapply"], default=None,
                   help="run one leg alone and print its JSON (profiling captures)")
    p.add_argument("--kpoints", type=int, default=64, help="k-points of the k-point leg (4x4x4 grid order)")
    p.add_argument("--gram-rows", type=int, default=1_728_000, help="rows N of the --only gram leg")
    p.add_argument("--gram-cols", type=int, default=1584, help="columns m of the --only gram leg")
    return p.parse_args()


def algorithmic_bytes(cell, ns, elem=8, n_sphere_pts=None):
    N = cell.N
    proj = (n_sphere_pts if n_sphere_pts is not None else 0) * 4 * elem
    return N * ns * 2 * elem + N * elem + proj


def chunk_states(N, elem):
    """States per L2-resident chunk, as the engine picks them (chunk_states, hamiltonian.cu)."""
    for c in (16, 8, 4, 2):
        if c * N * elem <= 20.0e6:
            return c
    return 1


def sphere_points(cell):
    """Projector points with a nonzero table value, summed over atoms."""
    import numpy as np
    tot = 0
    for per_k in cell.cubes:
        nz = None
        for (_, _, w) in per_k:
            m = w != 0.0
            nz = m if nz is None else (nz | m)
        tot += int(nz.sum()) if nz is not None else 0
    return tot


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# --------------------------------------------------------------- CPU arms
def _ref_worker(args):
    """One single-thread process applying the reference H to a slice of states."""
    reps, ns, seed, order = args
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    import numpy as np
    import oracle as O
    from qumasun_b200.cell import build_cell, initial_states
    cell = build_cell(reps=reps, fd_order=order)
    X = initial_states(ns, cell.N, seed=seed)
    t0 = time.perf_counter()
    O.hamiltonian_apply(cell, X, impl="ref" if O.ref_available() else "port")
    return time.perf_counter() - t0


def cpu_reference_rate(states_per_proc=2, procs=None, order=FD_ORDER):
    """States/s of the reference CPU H-apply on the host cores: `procs` concurrent
    single-thread processes on disjoint state slices (the reference runs one
    state per OpeA call, single-threaded per rank)."""
    import multiprocessing as mp
    import oracle as O
    procs = procs or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        times = pool.map(_ref_worker, [(REPS, states_per_proc, 100 + i, order) for i in range(procs)])
    wall = time.perf_counter() - t0
    per_state = max(times) / states_per_proc
    kind = "reference" if O.ref_available() else "port"
    return dict(states_per_s=procs / per_state, cores=procs, kind=kind,
                sample=f"{procs} processes x {states_per_proc} states of the 80^3 64-atom cell, "
                       f"FD order {order}, one thread each (max process time {max(times):.2f} s, wall {wall:.1f} s)")


_REF_W = {}


def _ref_arm_init(reps, ns, seed, order):
    """Pool initialiser of the reference arm: each single-thread process builds the
    cell and its own slice of seeded states once."""
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    from qumasun_b200.cell import build_cell, initial_states
    cell = build_cell(reps=reps, fd_order=order)
    _REF_W["cell"] = cell
    _REF_W["X"] = initial_states(ns, cell.N, seed=seed + os.getpid() % 1000)


def _ref_arm_apply(_):
    """Applies the reference H to this process's slice of states; returns seconds."""
    import oracle as O
    t0 = time.perf_counter()
    O.hamiltonian_apply(_REF_W["cell"], _REF_W["X"], impl="ref" if O.ref_available() else "port")
    return time.perf_counter() - t0


def bench_config(cell, ws):
    """The `config` both arms print (same keys and values, so the two lines compare)."""
    return {"workload": WORKLOAD, "n_states": NS, "grid": [cell.nx, cell.ny, cell.nz], "atoms": cell.n_atoms,
            "fd_order": FD_ORDER, "parallelism": f"states-replicated x{ws}",
            "l2": "inputs larger than L2 (1.05 GB states), no flush"}


def run_reference_arm(a):
    """The reference's own CPU H-apply (oracle/_ref, else the oracle port) on the host
    cores: every step applies H to all 256 states of the workload, split over one
    single-thread process per core (the reference applies H one state per OpeA call,
    single-threaded per rank). Warm-up steps run the same work untimed. Under torchrun
    only rank 0 runs."""
    import multiprocessing as mp
    import oracle as O
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from qumasun_b200.cell import build_cell
    cell = build_cell(reps=REPS)
    nsph = sphere_points(cell)
    per_state_bytes = algorithmic_bytes(cell, NS, n_sphere_pts=nsph) / NS
    procs = max(1, min(os.cpu_count() or 1, NS))
    while NS % procs:
        procs -= 1
    per_proc = NS // procs
    ctx = mp.get_context("spawn")
    step_s = []
    with ctx.Pool(procs, initializer=_ref_arm_init, initargs=(REPS, per_proc, 100, FD_ORDER)) as pool:
        for _ in range(a.warmup):
            pool.map(_ref_arm_apply, range(procs), chunksize=1)
        t_all = time.perf_counter()
        for _ in range(max(1, a.steps)):
            t0 = time.perf_counter()
            pool.map(_ref_arm_apply, range(procs), chunksize=1)
            step_s.append(time.perf_counter() - t0)
            if time.perf_counter() - t_all > 240:  # bound the arm's run time on slow hosts
                break
    sec = sum(step_s) / len(step_s)
    gbs = NS * per_state_bytes / sec / 1e9
    kind = "reference" if O.ref_available() else "port"
    sample = (f"{len(step_s)} timed steps, each all {NS} states of the 80^3 64-atom cell (FD order {FD_ORDER}) "
              f"over {procs} single-thread processes x {per_proc} states; {a.warmup} untimed warm-up steps")
    line = {
        "metric": "H|psi> GB/s (algorithmic)", "value": round(gbs, 3), "unit": "GB/s",
        "impl": "reference", "n_gpus": a.gpus, "steps": len(step_s), "warmup": a.warmup,
        "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(cell, ws),
        "state_applications_per_s": round(NS / sec, 3),
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": procs, "kind": kind, "sample": sample},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def lobpcg_diamond8(ctx, cpu=True):
    """Time to the 16 lowest eigenpairs of the 8-atom 40^3 cell (FD order 8) from
    seeded uniform(-0.5, 0.5) states, GPU FP64 LOBPCG, next to the reference's
    EigenLOBPCG_d_multi timed on a bounded sample of its iterations."""
    import numpy as np
    from qumasun_b200 import Hamiltonian
    from qumasun_b200.cell import build_cell, initial_states
    gold = np.load(os.path.join(ROOT, "tests", "golden", "lobpcg_diamond8.npz"))
    cell = build_cell()
    ns = int(gold["ns"])
    X0 = initial_states(ns, cell.N, seed=int(gold["seed"]))
    H = Hamiltonian(ctx, cell)
    H.lobpcg(X0, max_iter=5, precond=1)  # warm-up (library handles, workspace, FFT plans)

    def solve(precond):
        t0 = time.perf_counter()
        r = H.lobpcg(X0, max_iter=3000, precond=precond)
        wall = time.perf_counter() - t0
        rep = r["report"]
        return {"seconds": round(wall, 4), "device_ms": round(rep["ms_total"], 2), "iterations": rep["iterations"],
                "converged": bool(rep["converged"]), "restarts": rep["restarts"],
                "max_abs_ev_error_vs_reference_Ha": float(np.abs(r["ev"] - gold["ev"]).max()),
                "phase_ms": {k: round(rep[k], 2) for k in ("ms_hamiltonian", "ms_gram", "ms_eigensolve",
                                                           "ms_rotate", "ms_vector")}}

    faithful = solve(0)   # the reference's unpreconditioned iteration
    plain = solve(1)      # FP64 with the kinetic preconditioner
    H.close()
    wall = plain["seconds"]
    out = {"workload": "diamond8_40cube_16states_fd8", "fp64_kinetic_preconditioner": plain,
           "fp64_reference_iteration": faithful, "seconds": wall,
           "reference_iterations": int(gold["iters"])}
    if cpu:
        try:
            import oracle as O
            k = 25
            t1 = time.perf_counter()
            rr = O.ref_lobpcg_d_multi(cell, X0, k)
            per_it = (time.perf_counter() - t1) / max(1, rr["iters"])
            out["reference_cpu"] = {"seconds_extrapolated": round(per_it * int(gold["iters"]), 2),
                                    "seconds_per_iteration": round(per_it, 4), "cores": 1,
                                    "kind": "reference" if O.ref_available() else "port",
                                    "sample": f"{rr['iters']} iterations of EigenLOBPCG_d_multi, extrapolated to "
                                              f"the reference's {int(gold['iters'])}"}
            out["speedup_vs_reference_cpu"] = round(per_it * int(gold["iters"]) / wall, 1)
        except Exception as ex:
            out["reference_cpu"] = {"failed": str(ex)}
    return out


def monkhorst_pack(n, a0):
    """n x n x n Monkhorst-Pack Bloch vectors (bohr^-1) of a cubic cell with edge a0:
    k = (2r - n - 1) / (2n) * 2 pi / a0 per axis, r = 1..n."""
    f = [(2 * r - n - 1) / (2 * n) for r in range(1, n + 1)]
    b = 2 * math.pi / a0
    return [(b * fx, b * fy, b * fz) for fz in f for fy in f for fx in f]


def kpoint_leg(ctx, n_k=64, steps=10, rank=0, ws=1):
    """Complex k-point operator on the 8-atom 40^3 cell, 16 states per k-point, over a
    4x4x4 Monkhorst-Pack grid: (1) H_k|psi> throughput of the complex apply (rank 0),
    (2) time to the 16 lowest eigenpairs at every k-point (FP64 complex LOBPCG, kinetic
    preconditioner). With several ranks the k-points are sharded by longest-processing-
    time assignment (qumasun_b200.shard), one GPU per rank, no collective on the data
    path; the time is the max over ranks and rank 0 gathers the eigenvalues."""
    import numpy as np
    import torch
    from qumasun_b200 import Hamiltonian
    from qumasun_b200.cell import build_cell, initial_states
    from qumasun_b200.shard import run_sharded
    cell = build_cell()
    N, ns = cell.N, 16
    mp = monkhorst_pack(4, 6.74)
    ks = mp[:n_k]
    H = Hamiltonian(ctx, cell, kvec=mp[0])
    apply = None
    if rank == 0:
        gen = torch.Generator(device="cuda").manual_seed(77)
        X = torch.rand(ns, 2 * N, dtype=torch.float64, device="cuda", generator=gen) - 0.5
        HX = torch.empty_like(X)
        for _ in range(3):
            H.apply_z(X, HX)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            H.apply_z(X, HX)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        phases = sorted((H.apply_timed_z(ns, X.data_ptr(), HX.data_ptr()) for _ in range(5)), key=lambda p: p[1])[2]
        nbytes = N * ns * 32 + N * 8
        apply = {"ms": round(ms, 4), "GBs": round(nbytes / (ms * 1e-3) / 1e9, 1),
                 "state_apps_per_s": round(ns / (ms * 1e-3), 1),
                 "phase_ms": {"projection": round(phases[0], 4), "stencil_V": round(phases[1], 4),
                              "scatter": round(phases[2], 4)}}
        del X, HX
    solves = None
    if n_k > 0:
        X0 = initial_states(ns, 2 * N, seed=1234)

        def solve(i):
            H.set_kvector(ks[i])
            r = H.lobpcg_z(X0, max_iter=500, precond=1, tol=1e-10)
            return {"ev": r["ev"].tolist(), "iterations": r["report"]["iterations"],
                    "device_ms": r["report"]["ms_total"]}

        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = run_sharded([1.0] * n_k, solve)
        wall = time.perf_counter() - t0
        if ws > 1:
            import torch.distributed as dist
            t = torch.tensor([wall], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            wall = float(t.item())
        if rank == 0:
            evs = np.array([res[i]["ev"] for i in range(n_k)])
            its = [res[i]["iterations"] for i in range(n_k)]
            # time reversal: E(k) = E(-k); the Monkhorst-Pack grid holds both of each pair
            pair = float(max(np.abs(np.sort(evs[i]) - np.sort(evs[n_k - 1 - i])).max() for i in range(n_k)))
            solves = {"mode": "one solve per k-point (qg_lobpcg_z)", "k_points": n_k, "states_per_k": ns,
                      "ranks": ws, "seconds": round(wall, 3),
                      "device_ms": round(sum(res[i]["device_ms"] for i in range(n_k)), 1),
                      "iterations_max": int(max(its)), "iterations_mean": round(float(np.mean(its)), 1),
                      "band_min_Ha": float(evs.min()), "band_max_Ha": float(evs.max()),
                      "max_abs_ev_diff_k_vs_minus_k_Ha": pair}
    batched = None
    if rank == 0 and n_k > 0:
        # all k-points in one solve: one H launch per phase for every k-point's states
        Xb = torch.from_numpy(np.stack([initial_states(ns, 2 * N, seed=1234)] * n_k)).cuda().contiguous()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rb = H.lobpcg_zk(np.array(ks), Xb, max_iter=500, precond=1, tol=1e-10)
        torch.cuda.synchronize()
        wb = time.perf_counter() - t0
        evb = rb["ev"]
        diff = None
        if solves is not None:
            diff = float(max(np.abs(np.sort(evb[i]) - np.sort(np.array(res[i]["ev"]))).max() for i in range(n_k)))
        batched = {"mode": "all k-points in one solve (qg_lobpcg_zk_device)", "k_points": n_k, "seconds": round(wb, 3),
                   "device_ms": round(rb["report"]["ms_total"], 1), "iterations": rb["report"]["iterations"],
                   "phase_ms": {k_: round(rb["report"][k_], 1) for k_ in ("ms_hamiltonian", "ms_gram", "ms_eigensolve",
                                                                         "ms_rotate", "ms_vector")},
                   "converged": bool(rb["report"]["converged"]), "max_abs_ev_diff_vs_one_by_one_Ha": diff}
        del Xb
    H.close()
    if rank != 0:
        return None
    return {"workload": "diamond8_40cube_16states_mp4x4x4_fd8_complex", "apply": apply, "lobpcg": solves,
            "lobpcg_batched": batched}


def learned_leg(ctx, steps=1500):
    """Learned preconditioner: (residual, correction) pairs from LOBPCG iterates on four
    8-atom 40^3 cells, GPU training with the engine's own forward/backward kernels, then
    LOBPCG with the kinetic preconditioner against kinetic + learned correction on an
    unseen 8-atom cell (atoms displaced by sigma 0.1 bohr), 16 states, 14 converged."""
    from qumasun_b200 import learned as LP
    from qumasun_b200.cell import build_cell
    t0 = time.perf_counter()
    data = []
    for i, c in enumerate(LP.default_training_cells()):
        R, Cc, V = LP.residual_pairs(ctx, c, 16, (2, 4, 7, 11, 16), seed=100 + i)
        data.append(((c.nx, c.ny, c.nz), R, Cc, V))
    t1 = time.perf_counter()
    nn, hist = LP.train(ctx, data, steps=steps, log_every=max(1, steps // 5))
    t2 = time.perf_counter()
    hc = build_cell(displacement=0.1, seed=99)
    Rh, Ch, Vh = LP.residual_pairs(ctx, hc, 16, (3, 8), seed=77)
    held = LP.held_out_loss(nn, [((hc.nx, hc.ny, hc.nz), Rh, Ch, Vh)])
    cmp = LP.compare(ctx, nn, build_cell(displacement=0.1, seed=98), 16, n_converge=14)
    apply_ms = network_apply_times(nn)
    nn.close()
    return {"workload": "diamond8_40cube_train4cells_eval_unseen_sigma0.1", "pairs": sum(d[1].shape[0] for d in data),
            "pair_generation_s": round(t1 - t0, 2), "training_steps": steps, "training_s": round(t2 - t1, 2),
            "loss_history": [[s_, round(l_, 4)] for s_, l_ in hist], "held_out_loss": round(held, 4),
            "lobpcg_unseen_cell": cmp, "network_apply_80cube_64states": apply_ms}


def netapply_leg(ctx, steps=5):
    """The learned preconditioner's network alone (seeded random parameters, no
    training): 64 residuals at 80^3, tensor-core against CUDA-core layers."""
    import numpy as np
    from qumasun_b200 import LearnedPreconditioner
    nn = LearnedPreconditioner(ctx)
    nn.set_params(np.random.default_rng(4).normal(0, 0.1, nn.n_params).astype(np.float32))
    out = network_apply_times(nn, reps=max(1, steps))
    nn.close()
    return {"workload": "learned_network_80cube_64states", **out}


def network_apply_times(nn, grid=(80, 80, 80), ns=64, reps=5):
    """One application of the trained network to 64 residuals on the 80^3 grid (15.1k
    multiply-adds per voxel), CUDA events: the layers on the tensor cores against the
    CUDA-core kernels."""
    import torch
    N = grid[0] * grid[1] * grid[2]
    g = torch.Generator(device="cuda").manual_seed(3)
    R = torch.rand(ns, N, dtype=torch.float64, device="cuda", generator=g) - 0.5
    V = torch.rand(N, dtype=torch.float64, device="cuda", generator=g) - 4.0
    out = torch.zeros_like(R)
    res = {}
    for name, on in (("tensor_cores", True), ("cuda_cores", False)):
        nn.set_tensor_cores(on)
        for _ in range(2):
            nn.apply(grid, R, V, 4.0, out=out)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            nn.apply(grid, R, V, 4.0, out=out)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        res[name] = {"ms": round(ms, 3), "TMAC_per_s": round(15120.0 * N * ns / (ms * 1e-3) / 1e12, 2)}
    nn.set_tensor_cores(True)
    return res


def cells_leg():
    """16 cells of uneven size solved together: 4 each of the 8-atom (40^3), 16-atom
    (80x40x40), 32-atom (80x80x40) and 64-atom (80^3) diamond supercells, atoms displaced
    by seeded Gaussian sigma 0.05 bohr, 2 states per atom to 1e-10 (plus a 1/8 guard
    band), kinetic-preconditioned FP64 LOBPCG. Each cell has its own context and stream.
    Times the 16 solves one after another and all at once (qg_lobpcg_cells_device) and
    checks that both give the same eigenvalues."""
    import numpy as np
    import torch
    from qumasun_b200 import Context, Hamiltonian
    from qumasun_b200.cell import build_cell, initial_states
    from qumasun_b200.engine import lobpcg_cells
    shapes = [(1, 1, 1), (2, 1, 1), (2, 2, 1), (2, 2, 2)]
    cells, X0, nconv = [], [], []
    for i in range(16):
        reps = shapes[i // 4]
        cell = build_cell(reps=reps, displacement=0.05, seed=100 + i)
        nc = 2 * cell.n_atoms
        cells.append(cell)
        nconv.append(nc)
        X0.append(initial_states(nc + nc // 8, cell.N, seed=200 + i))
    ctxs = [Context(0) for _ in cells]
    hams = [Hamiltonian(c, cell) for c, cell in zip(ctxs, cells)]
    # one by one (each cell on its own context, the contexts used in turn)
    t0 = time.perf_counter()
    one = []
    for c in range(16):
        r = hams[c].lobpcg_device(torch.from_numpy(X0[c]).cuda(), None, max_iter=1000, precond=1,
                                  n_converge=nconv[c])
        one.append(r)
    torch.cuda.synchronize()
    t_one = time.perf_counter() - t0
    Xs = [torch.from_numpy(x).cuda() for x in X0]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out, rc = lobpcg_cells(hams, Xs, max_iter=1000, precond=1, n_converge=nconv)
    torch.cuda.synchronize()
    t_all = time.perf_counter() - t0
    diff = max(float(np.abs(out[c]["ev"][:nconv[c]] - one[c]["ev"][:nconv[c]]).max()) for c in range(16))
    res = {"workload": "16_cells_8to64_atoms_40to80_grids_sigma0.05_2states_per_atom_fd8",
           "cells": [{"atoms": cells[c].n_atoms, "grid": [cells[c].nx, cells[c].ny, cells[c].nz],
                      "states": int(X0[c].shape[0]), "converge": nconv[c],
                      "iterations": out[c]["report"]["iterations"], "converged": bool(out[c]["report"]["converged"])}
                     for c in range(16)],
           "seconds_one_by_one": round(t_one, 3), "seconds_together": round(t_all, 3),
           "speedup_together": round(t_one / t_all, 3), "status": rc,
           "max_abs_ev_diff_together_vs_one_by_one_Ha": diff}
    for h in hams:
        h.close()
    for c in ctxs:
        c.close()
    return res


def lobpcg_diamond216(ctx):
    """Time to the 480 lowest eigenpairs (528 solved, a 48-state guard band) of the
    216-atom 3x3x3 cell (120^3, atoms displaced by seeded Gaussian sigma 0.05 bohr),
    kinetic-preconditioned GPU LOBPCG from the same seeded uniform(-0.5, 0.5) states:
    FP64 Gram products against split-BF16x3 (QG_MIXED_BF16X3) and FP32 (QG_FP32) Gram
    products, which must agree on the 480 eigenvalues to 1e-8 Ha, and the FP64 solve once
    more with the projection sums split over 2-block clusters (iteration-count sensitivity)."""
    import numpy as np
    import torch
    from qumasun_b200 import Hamiltonian
    from qumasun_b200.cell import build_cell
    cell = build_cell(reps=(3, 3, 3), displacement=0.05, seed=2024)
    ns, nconv = 528, 480
    H = Hamiltonian(ctx, cell)
    gen = torch.Generator(device="cuda").manual_seed(2024)
    X0 = torch.rand(ns, cell.N, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    runs = {}
    evs = {}
    # fp64_proj2: the FP64 solve again with every atom's projection summed over a 2-block
    # cluster (a change in the last bits of H), the sensitivity check of the iteration
    for name, prec in (("fp64", 0), ("bf16x3_gram", 2), ("fp32_gram", 1), ("fp64_proj2", 0),
                       ("fp64_int8_gram", 3)):
        H.set_nonlocal_blocking(project_parts=2 if name == "fp64_proj2" else 0)
        X = X0.clone()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = H.lobpcg_device(X, None, max_iter=300, precond=1, shift=1.0, n_converge=nconv, precision=prec)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        rep = r["report"]
        evs[name] = r["ev"][:nconv]
        runs[name] = {"seconds": round(wall, 3), "device_ms": round(rep["ms_total"], 1),
                      "iterations": rep["iterations"], "converged": bool(rep["converged"]),
                      "mixed_iterations": rep["mixed_iterations"], "restarts": rep["restarts"],
                      "max_residual": rep["max_residual"],
                      "phase_ms": {k: round(rep[k], 1) for k in ("ms_hamiltonian", "ms_gram", "ms_eigensolve",
                                                                 "ms_rotate", "ms_vector")}}
        del X
    H.close()
    diff = float(np.abs(evs["fp64"] - evs["bf16x3_gram"]).max())
    diff32 = float(np.abs(evs["fp64"] - evs["fp32_gram"]).max())
    diffp2 = float(np.abs(evs["fp64"] - evs["fp64_proj2"]).max())
    diffi8 = float(np.abs(evs["fp64"] - evs["fp64_int8_gram"]).max())
    return {"workload": "diamond216_120cube_480of528states_fd8_kinetic_precond", **runs,
            "max_abs_ev_diff_mixed_vs_fp64_Ha": diff,
            "max_abs_ev_diff_fp32_gram_vs_fp64_Ha": diff32,
            "max_abs_ev_diff_proj2_vs_fp64_Ha": diffp2,
            "max_abs_ev_diff_int8_gram_vs_fp64_Ha": diffi8,
            "speedup_int8_gram_vs_fp64": round(runs["fp64"]["seconds"] / runs["fp64_int8_gram"]["seconds"], 3),
            "speedup_mixed_vs_fp64": round(runs["fp64"]["seconds"] / runs["bf16x3_gram"]["seconds"], 3),
            "speedup_fp32_gram_vs_fp64": round(runs["fp64"]["seconds"] / runs["fp32_gram"]["seconds"], 3)}


def scf_leg(ctx, X, cell, steps=10, cpu=True):
    """The SCF-step neighbours of the eigensolver on the 64-atom 80^3 cell: density of the
    256 states (qg_density_d), the Poisson + LDA potential (qg_potential_lda_d) at 80^3 and
    120^3, one Taylor-4 step of 64 complex states (qg_td_taylor4_z: four H applications
    and the updates) and the nonlocal energies and forces of the 256 states
    (qg_nonlocal_force_d); device times by CUDA events. With cpu=True the reference's
    TimeEvoH4 and ForceNonlocal (oracle/_ref) are timed on one state each, single-thread."""
    import numpy as np
    import torch
    from qumasun_b200 import Hamiltonian, Poisson, density
    from qumasun_b200.cell import build_cell, initial_states
    ns, N = X.shape
    occ = np.where(np.arange(ns) < 128, 2.0, 0.0)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {"workload": "diamond64_80cube_scf_step_neighbours"}
    rho = torch.zeros(N, dtype=torch.float64, device="cuda")
    ms = timed(lambda: density(ctx, X, occ, rho=rho), steps)
    nocc = int((occ > 0).sum())
    out["density"] = {"states": ns, "occupied": nocc, "ms": round(ms, 4),
                      "GBs": round((nocc * N * 8 + N * 8) / (ms * 1e-3) / 1e9, 1)}
    pot = {}
    for reps_ in ((2, 2, 2), (3, 3, 3)):
        c = build_cell(reps=reps_)
        P = Poisson(ctx, (c.nx, c.ny, c.nz), (c.hx, c.hy, c.hz))
        r = torch.from_numpy(0.02 + 0.3 * np.exp(c.V / 4.0)).cuda()
        v = torch.from_numpy(c.V).cuda()
        pot[f"{c.nx}cube"] = {"ms": round(timed(lambda: P.potential(r, v), steps), 4)}
        P.close()
    out["potential_lda"] = pot
    Hk = Hamiltonian(ctx, cell, kvec=(0.0582, 0.0582, 0.0582))
    Z = (torch.rand(64, 2 * N, dtype=torch.float64, device="cuda") - 0.5) * 1e-2
    ms = timed(lambda: Hk.td_taylor4(Z, 0.002), 3)
    out["taylor4"] = {"states": 64, "ms_per_step": round(ms, 3), "state_steps_per_s": round(64 / (ms * 1e-3), 1)}
    Hk.close()
    H = Hamiltonian(ctx, cell)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f, e, ev = H.nonlocal_force(X, occ)
    out["nonlocal_force"] = {"states": ns, "occupied": nocc, "seconds": round(time.perf_counter() - t0, 4),
                             "ev_sum_Ha": ev}
    H.close()
    if cpu:
        try:
            import oracle as O
            Z1 = initial_states(1, 2 * N, seed=5) * 1e-2
            t1 = time.perf_counter()
            O.td_taylor4(cell, (0.0582, 0.0582, 0.0582), 0.002, Z1, impl="ref")
            tt = time.perf_counter() - t1
            X1 = X[:1].cpu().numpy()
            t1 = time.perf_counter()
            O.nonlocal_force(cell, X1, np.array([2.0]), impl="ref")
            tf = time.perf_counter() - t1
            out["reference_cpu"] = {"taylor4_s_per_state": round(tt, 3), "force_s_per_state": round(tf, 3),
                                    "cores": 1, "kind": "reference",
                                    "sample": "QUMASUN::TimeEvoH4 and ForceNonlocal (with Gradient8th) on one "
                                              "state of the 80^3 64-atom cell, single thread"}
            out["speedup_taylor4_vs_reference_cpu_per_state"] = round(tt / (ms * 1e-3 / 64), 1)
        except Exception as ex:
            out["reference_cpu"] = {"failed": str(ex)}
    return out


# --------------------------------------------------------------- GPU arm
def run_gpu_arm(a):
    import numpy as np
    import torch
    import torch.distributed as dist

    global NS
    NS = a.states

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from qumasun_b200 import Context, Hamiltonian
    from qumasun_b200.cell import build_cell

    cell = build_cell(reps=REPS)
    nsph = sphere_points(cell)
    ctx = Context(local)
    stream = torch.cuda.Stream(device=local)
    ctx.set_stream(stream.cuda_stream)
    H = Hamiltonian(ctx, cell, fd_order=FD_ORDER)
    N = cell.N
    gen = torch.Generator(device="cuda").manual_seed(1000 + rank)
    with torch.cuda.stream(stream):
        X = torch.rand(NS, N, dtype=torch.float64, device="cuda", generator=gen) - 0.5
        HX = torch.empty_like(X)
    stream.synchronize()
    nbytes = algorithmic_bytes(cell, NS, n_sphere_pts=nsph)
    launches_per_step = H.launches_per_apply(NS)

    def barrier():
        if ws > 1:
            dist.barrier()

    def max_over_ranks(v):
        if ws == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # the engine's autotuner picks the bit-identical launch shapes on these states
    tuned = None
    if not a.no_autotune:
        with torch.cuda.stream(stream):
            tuned = H.autotune(X, HX)
    stream.synchronize()
    ctx.set_stream(stream.cuda_stream)
    # warm-up
    for _ in range(max(3, a.warmup)):
        H.apply_device(NS, X.data_ptr(), HX.data_ptr())
    stream.synchronize()

    # timed region: device events on the launching stream
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(a.steps):
            H.apply_device(NS, X.data_ptr(), HX.data_ptr())
        e1.record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1) / a.steps
    ms_max = max_over_ranks(ms)
    gbs = nbytes * ws / (ms_max * 1e-3) / 1e9

    # dominant-kernel roofline: per-phase device times of one apply
    phases = sorted((H.apply_timed(NS, X.data_ptr(), HX.data_ptr()) for _ in range(5)), key=lambda p: p[1])
    ms_proj, ms_sten, ms_scat = phases[2]
    # the stencil kernel: psi in, H psi out, V once
    sten_bytes = N * NS * 2 * 8 + N * 8
    peak, peak_kind = measured_peak_hbm()
    sten_gbs = sten_bytes / (ms_sten * 1e-3) / 1e9
    phase_ms = {"projection": round(ms_proj, 4), "stencil_V": round(ms_sten, 4), "scatter": round(ms_scat, 4)}

    # e2e through the host-buffer entry point with pinned host states
    e2e = None
    if not a.no_e2e:
        Xh = torch.empty(NS, N, dtype=torch.float64, pin_memory=True)
        Xh.copy_(X.cpu())
        HXh = torch.empty_like(Xh).pin_memory()
        e2e_steps = max(2, min(a.steps, 5))
        H.apply_host_ptr(NS, Xh.data_ptr(), HXh.data_ptr())  # warm the staging buffers
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            H.apply_host_ptr(NS, Xh.data_ptr(), HXh.data_ptr())
        e2e_s = (time.perf_counter() - t0) / e2e_steps
        e2e_s = max_over_ranks(e2e_s)
        e2e = {"value": round(nbytes * ws / e2e_s / 1e9, 2), "unit": "GB/s", "h2d_bytes_per_step": NS * N * 8,
               "d2h_bytes_per_step": NS * N * 8, "seconds_per_step": round(e2e_s, 5)}

    # the legs that only rank 0 runs (sweep, learned, LOBPCG, cells) run in single-GPU
    # runs only: with several ranks the others would wait at the final barrier for longer
    # than the process group's timeout; the multi-GPU line carries the headline metric and
    # the sharded k-point leg
    solo = ws == 1
    sweep = {}
    if not a.no_sweep and solo:
        for order in (2, 4, 6, 8):
            Ho = Hamiltonian(ctx, cell, fd_order=order)
            for dt in ("f64", "f32"):
                Xs = X if dt == "f64" else X.float()
                HXs = torch.empty_like(Xs)
                for _ in range(3):
                    Ho.apply_device(NS, Xs.data_ptr(), HXs.data_ptr(), dtype=dt)
                stream.synchronize()
                s0 = torch.cuda.Event(enable_timing=True)
                s1 = torch.cuda.Event(enable_timing=True)
                s0.record(stream)
                for _ in range(5):
                    Ho.apply_device(NS, Xs.data_ptr(), HXs.data_ptr(), dtype=dt)
                s1.record(stream)
                stream.synchronize()
                m = s0.elapsed_time(s1) / 5
                el = 8 if dt == "f64" else 4
                sweep[f"o{order}_{dt}"] = {"ms": round(m, 4),
                                           "GBs": round(algorithmic_bytes(cell, NS, el, nsph) / (m * 1e-3) / 1e9, 1),
                                           "state_apps_per_s": round(NS / (m * 1e-3), 1)}
                del Xs, HXs
            Ho.close()

    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        try:
            r = cpu_reference_rate(states_per_proc=1)
            per_state = nbytes / NS
            cpu = {"value": round(r["states_per_s"] * per_state / 1e9, 3), "unit": "GB/s", "cores": r["cores"],
                   "kind": r["kind"], "sample": r["sample"],
                   "state_applications_per_s": round(r["states_per_s"], 3)}
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "GB/s", "cores": 0, "kind": "port", "sample": f"failed: {ex}"}
        if sweep and cpu and cpu.get("value") is not None:
            # the reference CPU H-apply at every FD order of the sweep (FP64: the reference's
            # H path is double only), same processes and sample as the order-8 baseline
            for order in (2, 4, 6, 8):
                try:
                    r = (cpu_reference_rate(states_per_proc=1, order=order) if order != FD_ORDER
                         else {"states_per_s": cpu["state_applications_per_s"]})
                    sw = sweep[f"o{order}_f64"]
                    sw["reference_cpu_state_apps_per_s"] = round(r["states_per_s"], 2)
                    sw["reference_cpu_GBs"] = round(r["states_per_s"] * nbytes / NS / 1e9, 3)
                    sw["speedup_vs_reference_cpu"] = round(sw["state_apps_per_s"] / r["states_per_s"], 1)
                except Exception as ex:
                    sweep[f"o{order}_f64"]["reference_cpu_state_apps_per_s"] = f"failed: {ex}"

    scf = None
    if solo and not a.no_scf:
        scf = scf_leg(ctx, X, cell, cpu=not a.no_cpu_baseline)
    kp = None
    if not a.no_kpoint:
        kp = kpoint_leg(ctx, n_k=a.kpoints, rank=rank, ws=ws)
    lrn = None
    if solo and not a.no_learned:
        lrn = learned_leg(ctx)
    cells_res = None
    if solo and not a.no_cells:
        cells_res = cells_leg()
    lob = None
    lob216 = None
    if solo and not a.no_lobpcg:
        lob = lobpcg_diamond8(ctx, cpu=(ws == 1 and not a.no_cpu_baseline))
        if not a.no_lobpcg216:
            del X, HX
            torch.cuda.empty_cache()
            lob216 = lobpcg_diamond216(ctx)

    if rank == 0:
        line = {
            "metric": "H|psi> GB/s (algorithmic)", "value": round(gbs, 2), "unit": "GB/s",
            "n_gpus": ws, "steps": a.steps, "warmup": max(3, a.warmup), "ms_per_step": round(ms_max, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": bench_config(cell, ws),
            "state_applications_per_s": round(NS * ws / (ms_max * 1e-3), 1),
            "autotuned": tuned,
            "roofline": {"bound": "hbm", "kernel": STENCIL_KERNEL,
                         "achieved": round(sten_gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(sten_gbs / peak, 4), "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": sten_bytes, "launches": 1,
                         "ms_per_launch": round(ms_sten, 5),
                         "traffic": (int(STENCIL_DRAM_BYTES_PER_STATE * NS) if STENCIL_DRAM_BYTES_PER_STATE
                                     else None),
                         "traffic_note": "ncu capture at 32 states scaled by states",
                         "phase_ms_per_apply": phase_ms,
                         "whole_apply_frac": round(gbs / peak, 4)},
            "e2e": e2e,
            "gpu_launches": launches_per_step * a.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        if sweep:
            line["sweep"] = sweep
        if lob:
            line["lobpcg"] = lob
        if lob216:
            line["lobpcg_216"] = lob216
        if kp:
            line["kpoint"] = kp
        if scf:
            line["scf"] = scf
        if lrn:
            line["learned_preconditioner"] = lrn
        if cells_res:
            line["cells"] = cells_res
        print(json.dumps(line), flush=True)
    H.close()
    ctx.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def gram_leg(ctx, N=1_728_000, m=1584, steps=5):
    """Split-BF16 Gram products of the mixed-precision LOBPCG at the 216-atom cell's
    shape (N = 120^3 rows, m = 3 x 528 columns): the tcgen05 kernel with 3 and 2
    pieces, the cuBLAS BF16 path and the int8 7-slice (FP64-accurate) kernel against
    FP64 DGEMM, time and max error."""
    import ctypes as C
    import torch
    from qumasun_b200.engine import lib
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.rand(m, N, dtype=torch.float64, device="cuda", generator=g) - 0.5
    A /= A.norm(dim=1, keepdim=True)
    Cm = torch.zeros(m, m, dtype=torch.float64, device="cuda")
    ref = A @ A.T
    out = {"N": N, "m": m}
    for pieces in (3, 2, 0, 7):
        rc = lib().qg_gram_mixed_d(ctx.h, N, m, C.c_void_p(A.data_ptr()), None, 1.0, C.c_void_p(Cm.data_ptr()), pieces)
        if rc != 0:
            out[f"pieces{pieces}"] = {"status": rc}
            continue
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            lib().qg_gram_mixed_d(ctx.h, N, m, C.c_void_p(A.data_ptr()), None, 1.0, C.c_void_p(Cm.data_ptr()), pieces)
        torch.cuda.synchronize()
        sec = (time.perf_counter() - t0) / steps
        out[f"pieces{pieces}"] = {"ms": round(sec * 1e3, 2), "max_abs_err": float((Cm - ref).abs().max().item()),
                                  "effective_TFLOPs": round(2.0 * N * m * m / sec / 1e12, 1)}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        torch.mm(A, A.T)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    out["fp64_dgemm"] = {"ms": round(ms, 2), "TFLOPs": round(2.0 * N * m * m / (ms * 1e-3) / 1e12, 1)}
    return out


def run_only(a):
    import torch
    from qumasun_b200 import Context
    torch.cuda.set_device(0)
    ctx = Context(0)
    ctx.use_torch_stream()
    if a.only == "gram":
        out = gram_leg(ctx, N=a.gram_rows, m=a.gram_cols, steps=a.steps)
    elif a.only == "cells":
        out = cells_leg()
    elif a.only == "netapply":
        out = netapply_leg(ctx, steps=a.steps)
    else:
        out = kpoint_leg(ctx, n_k=a.kpoints, steps=a.steps)
    print(json.dumps(out), flush=True)
    ctx.close()
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference_arm(a)
    if a.only:
        return run_only(a)
    return run_gpu_arm(a)


if __name__ == "__main__":
    sys.exit(main())
