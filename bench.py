#!/usr/bin/env python
"""Benchmark: ms per pressure-Poisson solve to 1e-6 relative residual on one B200.

Workload (synthetic, seeded; the reference publishes no dataset or numbers):
the adaptive sphere octree on [0,1]^3 with h0 = 1/8 -- tiles within 0.05 of
the surface of a solid sphere (centre (0.5,0.5,0.5), radius 0.1) refined to
level 6 (512^3 effective), within 0.15 to level 5 (256^3), the rest level 4
(128^3), 2:1 graded; the sphere is a Neumann cut-cell boundary with face
fractions from its analytic SDF; Dirichlet outer walls; rhs = volume-weighted
divergence of a face velocity summing 16 random Fourier modes (wavenumbers
1..8, amplitudes N(0,1), seed 1).  Solver: FAS mu-cycle (mu = 2) preconditioned
CG, omega = 1.5, level_iters = 2, coarsest_iters = 10, R_matrix = 0.5, FP32
vectors with FP64 dot products, tolerance 1e-6 -- the reference simulator's
call (cirrus_cutcell/FluidEuler.cu:702-706).

A step is one full solve from x = 0.  `value` is device time per solve with
the inputs resident in HBM (a device-to-device restore of b, which the solve
overwrites, is inside the timed region); `e2e` is the same solve through the
C ABI with host buffers (b copied in from pinned memory, x copied out).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (the path does not shard).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "cirrus-amg_b200"))

import numpy as np  # noqa: E402

METRIC = "ms per Poisson solve to 1e-6 rel. residual: learned/mixed vs plain MG, 1×B200"
UNIT = "ms"
COEFF, U, BSAVE = 6, 10, 15
SHELL = [4, 6, 5, 0.5, 0.5, 0.5, 0.1, 0.05, 0.15]  # coarse, fine, mid level, centre, radius, fine band, mid band
SPHERES = [(0.5, 0.5, 0.5, 0.1)]
WORKLOAD = "adaptive sphere octree 128^3/256^3/512^3 (h0=1/8, levels 4/5/6), Neumann cut-cell sphere r=0.1, Fourier-divergence rhs seed 1"
SOLVE = dict(max_iters=100, tol=1e-6, level_iters=2, coarsest_iters=10, sync_stride=1, omega=1.5, mu=2)
BYTES_PER_CELL_GS = 27  # x 4 + rhs 4 + 4 coefficients 16 + type 1 + half of x written 2


def fourier_modes(seed=1, n=16):
    rng = np.random.default_rng(seed)
    k = rng.integers(1, 9, size=(n, 3)).astype(np.float64)
    amp = rng.standard_normal((n, 3))
    ph = rng.uniform(0.0, 2.0 * np.pi, n)
    return k, amp, ph


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic_per_cell():
    """DRAM bytes per cell of one GS launch from the committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", "k_gs_pipe_sphere.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.startswith("dram_bytes_per_cell:"):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    return None
    return None


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.lines = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
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
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def replica_time(total_ms, world, device=None):
    """Whole-job time of N independent replicas: the slowest rank's device time
    (all_reduce MAX over the default process group; identity for one rank)."""
    if world <= 1:
        return total_ms
    import torch
    import torch.distributed as dist

    t = torch.tensor([total_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def per_solve_ms(total_ms, steps, world):
    """ms per solve of the whole job: N replicas each ran `steps` solves in `total_ms`."""
    return total_ms / (steps * world)


def build_workload(cmg):
    G = cmg.HADeviceGrid(0.125, 10, 16)
    G.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    G.rebuild()
    G.refine_case(cmg.CASE_SHELL, SHELL)
    G.set_leaf_cell_types_case(cmg.CASE_UNIFORM)
    G.cutcell_sphere_coeffs(COEFF, SPHERES, 0.5)
    k, amp, ph = fourier_modes(1)
    G.face_velocity_fourier(U, k, amp, ph)
    G.divergence(U, COEFF, 1)
    G.copy(1, BSAVE)
    G.synchronize()
    return G


def make_solver(cmg):
    s = cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0)
    s.omega = SOLVE["omega"]
    s.mu_cycle_repeat_times = SOLVE["mu"]
    # CMG_SOLVE_MODE=stream launches kernel by kernel (for ncu launch lists)
    if os.environ.get("CMG_SOLVE_MODE", "graph") == "stream":
        s.set_launch_mode(use_graph=False)
    return s


def solve_args():
    return (False, SOLVE["max_iters"], SOLVE["tol"], SOLVE["level_iters"], SOLVE["coarsest_iters"], SOLVE["sync_stride"], False)


def cpu_baseline_fp64(G, cmg):
    """FP64 Jacobi-preconditioned CG (the algorithm of Eigen's default
    ConjugateGradient) on the same operator assembled into CSR, all host cores."""
    from oracle import oracle as O

    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(O.CASE_SHELL, SHELL)
    g.alloc(16)
    lv, ijk, ty = G.tiles()
    olv, oijk, oty = g.tiles()
    if not (np.array_equal(lv, olv) and np.array_equal(ijk, oijk) and np.array_equal(ty, oty)):
        return {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": "topology mismatch"}
    g.cell_types()[:] = G.download_cell_types()
    for a in range(4):
        g.channel(COEFF + a)[:] = G.download(COEFF + a)
    b = G.download(BSAVE)
    rp, ci, va, rt, rc = g.assemble(COEFF)
    bb = b[rt, rc].astype(np.float64)
    t0 = time.perf_counter()
    x, its, rel = O.csr_solve(rp, ci, va, bb, 1e-6, 4000, 0)
    dt = time.perf_counter() - t0
    return {"value": dt * 1e3, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"one full FP64 Jacobi-CG solve of the workload to 1e-6 ({len(bb)} unknowns, {its} iterations, "
                      f"rel {rel:.2e}); OpenMP over all host threads"}


def run_ours(args, rank, world, local_rank):
    import torch

    import cmg

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    G = build_workload(cmg)
    S = make_solver(cmg)
    ntiles, maxl, nleaf = G.info()
    lv, ijk, ty = G.tiles()
    ct = G.download_cell_types()
    leaf_cells = int(nleaf) * 512
    interior = int(((ct == cmg.INTERIOR) & (ty[:, None] == cmg.LEAF)).sum())

    def one_solve():
        G.copy(BSAVE, 1)
        return S.solve(G, *solve_args())

    for _ in range(max(args.warmup, 1)):
        it, rel = one_solve()
    torch.cuda.synchronize()

    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    iters, rels, per_ms, launches = [], [], [], 0
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        torch.cuda.nvtx.range_push("solve")
        it, rel = one_solve()
        torch.cuda.nvtx.range_pop()
        iters.append(it)
        rels.append(rel)
        per_ms.append(S.last_solve_ms())
        launches += S.last_solve_launches()
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = replica_time(e0.elapsed_time(e1), world, dev)
    if world > 1:
        dist.barrier()

    # true residual of the last solution, FP32 operator apply on the device
    x = G.download(0)
    G.full_neg_lap(0, COEFF, 3)
    ax = G.download(3)
    b = G.download(BSAVE)
    m = (ty[:, None] == cmg.LEAF) & (ct == cmg.INTERIOR)
    true_rel = float(np.linalg.norm((b - ax)[m].astype(np.float64)) / np.linalg.norm(b[m].astype(np.float64)))

    # e2e: the same solve through the C ABI with pinned host buffers
    count = ntiles * 512
    b_host = torch.from_numpy(G.download(BSAVE).reshape(-1)).pin_memory()
    x_host = torch.empty(count, dtype=torch.float32).pin_memory()
    S.solve_host(G, b_host.data_ptr(), x_host.data_ptr(), count, SOLVE["max_iters"], SOLVE["tol"], SOLVE["level_iters"],
                 SOLVE["coarsest_iters"], SOLVE["sync_stride"], False)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_wall = time.perf_counter()
    f0.record()
    for _ in range(args.steps):
        S.solve_host(G, b_host.data_ptr(), x_host.data_ptr(), count, SOLVE["max_iters"], SOLVE["tol"], SOLVE["level_iters"],
                     SOLVE["coarsest_iters"], SOLVE["sync_stride"], False)
    f1.record()
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1) / args.steps
    e2e_wall_ms = (time.perf_counter() - t_wall) * 1e3 / args.steps

    # roofline of the dominant kernel: the pipelined red-black GS launch (k_gs_pipe) on the
    # finest level, as the cycle runs it (x starts at 0, so it is 0 on cells that are not
    # INTERIOR); L2 flushed (a 256 MB write) before every measured pair of launches
    L = maxl
    active = int(((lv == L) & ((ty == cmg.LEAF) | (ty == cmg.NONLEAF))).sum())
    cells = active * 512
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    G.copy(BSAVE, 1)
    G.fill(4, 0.0)
    reps, gs_ms = 20, []
    torch.cuda.nvtx.range_push("roofline")
    for r in range(reps + 2):
        flush.fill_(float(r))
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        S.gauss_seidel_masked(G, 1, 0, L, 4, 1)
        a1.record()
        torch.cuda.synchronize()
        if r >= 2:
            gs_ms.append(a0.elapsed_time(a1) / 2.0)
    torch.cuda.nvtx.range_pop()
    gs_ms.sort()
    launch_ms = gs_ms[len(gs_ms) // 2]
    peak, peak_kind = measured_peaks()
    alg_bytes = BYTES_PER_CELL_GS * cells
    achieved = alg_bytes / (launch_ms * 1e-3) / 1e9
    tpc = profile_traffic_per_cell()

    result = None
    if rank == 0:
        per_solve = per_solve_ms(total_ms, args.steps, world)
        result = {
            "metric": METRIC,
            "value": round(per_solve, 4),
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(total_ms / args.steps, 4),
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": WORKLOAD,
                "method": "plain FP32 FAS mu-cycle (mu=2) MG-PCG, FP64 dots",
                "tiles": ntiles, "leaf_tiles": nleaf, "leaf_cells": leaf_cells, "interior_cells": interior, "max_level": maxl,
                "pcg_iters": iters[-1], "rel_residual_recurrence": rels[-1], "rel_residual_true_fp32_apply": true_rel,
                "solve_ms_p50": sorted(per_ms)[len(per_ms) // 2],
                "l2": f"inputs larger than L2: {16 * ntiles * 2048 / 1e6:.0f} MB of channel planes per grid",
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "e2e_wall_ms": round(e2e_wall_ms, 4),
            },
            "e2e": {"value": round(e2e_ms, 4), "unit": UNIT, "h2d_bytes_per_step": count * 4, "d2h_bytes_per_step": count * 4},
            "gpu_launches": int(launches),
            "roofline": {
                "kernel": f"k_gs_pipe (pipelined red-black Gauss-Seidel pass, level {L}, {active} tiles)",
                "bound": "hbm",
                "achieved": round(achieved, 1),
                "peak": peak,
                "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                "peak_kind": peak_kind,
                "algorithmic_bytes_per_launch": alg_bytes,
                "launch_ms": round(launch_ms, 5),
                "traffic": (round(tpc * cells) if tpc else None),
            },
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline_fp64(G, cmg)
    return result


def run_reference(args):
    """The reference's algorithm for this path on the host cores: the oracle's
    restatement of AMGSolver::solve (src/AMGSolver.cu:1399), OpenMP over all
    host threads, on the same workload."""
    from oracle import oracle as O

    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(O.CASE_SHELL, SHELL)
    g.alloc(16)
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    g.cutcell_sphere_coeffs(COEFF, SPHERES, 0.5)
    k, amp, ph = fourier_modes(1)
    g.face_velocity_fourier(U, k, amp, ph)
    g.divergence(U, COEFF, 1)
    b = g.channel(1).copy()
    steps = max(1, min(args.steps, 5))
    warm = min(args.warmup, 1)
    times, it, rel = [], 0, 0.0
    for s in range(warm + steps):
        g.channel(1)[:] = b
        t0 = time.perf_counter()
        it, rel = g.amg_solve(COEFF, omega=SOLVE["omega"], mu=SOLVE["mu"], max_iters=SOLVE["max_iters"], tol=SOLVE["tol"],
                              level_iters=SOLVE["level_iters"], coarsest_iters=SOLVE["coarsest_iters"], sync_stride=1)
        dt = (time.perf_counter() - t0) * 1e3
        if s >= warm:
            times.append(dt)
    v = sum(times) / len(times)
    sample = (f"{steps} full solves of the workload ({it} PCG iterations, rel {rel:.2e}) by the C restatement of "
              f"AMGSolver::solve, OpenMP; the reference's own solver is CUDA-only")
    return {
        "impl": "reference",
        "metric": METRIC, "value": round(v, 3), "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": warm,
        "ms_per_step": round(v, 3), "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": WORKLOAD, "method": "reference FAS mu-cycle MG-PCG on host cores"},
        "cpu_baseline": {"value": round(v, 3), "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": sample},
        "e2e": {"value": round(v, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return

    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    res = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
