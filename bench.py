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
                  [--workload sphere|uniform64|batched64]

--workload uniform64: the uniform 64^3 grid (level 3), all cells INTERIOR,
Dirichlet walls, rhs N(0,1) per cell (numpy default_rng(0)) minus its mean.
--workload batched64: 64 independent octrees (seed 2): finest level 4 or 5 within
0.05 of the surfaces of 1-3 solid spheres (radius U(0.05, 0.15), centres
U(0.2, 0.8)^3), level 3 elsewhere, 2:1 graded, each with its own Fourier-
divergence rhs; a step solves all 64 in one persistent kernel launch inside a CUDA
graph (cmg_batch_solve, schedule picked by its autotuner); the metric is solves per
second, with p50/p99 of each octree's solve time inside the launch.  The same batch
as 64 graph launches on 16 streams (cmg_amg_solve_batch) is reported beside it.

N > 1 runs N independent replicas: one solve works on one octree in one GPU's memory,
and the path has no partition that avoids an exchange per sweep.
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
# algorithmic bytes per cell of the other tile steps of a solve (float planes, 1-byte types)
BYTES_PER_CELL = dict(
    restrict=26,  # x 4 + rhs 4 + coefficients 16 + type 1 read, the parent's x and rhs (8 B per 8 cells) written
    fas=33,       # x 4 + rhs 4 + coefficients 16 + type 1 read, rhs 4 + saved x 4 written
    prolong=10,   # x 4 + type 1 read, the parent's x and saved x (8 B per 8 cells) read, x 4 written
    apply=25,     # p 4 + coefficients 16 + type 1 read, Ap 4 written
    xr=25,        # x, r, p, Ap 16 + type 1 read, x and r 8 written
    dot=8,        # two planes read
    pupdate=13,   # p, z 8 + type 1 read, p 4 written
    fill=4,       # z = 0 on every tile
    coarse=29,    # levels 0-1 (9 tiles): x, rhs, saved x, coefficients, type read, x written once per visit
)


def solve_algorithmic_bytes(G, mu, level_iters, iters, finest_iters=-1):
    """Algorithmic DRAM bytes of one plain solve of octree G that took `iters` PCG iterations:
    every tile step of the FAS mu-cycle (a level-l step runs mu^(top-l) times per cycle) and
    of the PCG vector updates, each plane read or written once per step.  finest_iters >= 0:
    the sweeps of the finest level (the autotuner's setting), else level_iters."""
    lv, _, ty = G.tiles()
    import cmg

    top = int(lv.max())
    act = [int(((lv == l) & (ty != cmg.GHOST)).sum()) for l in range(top + 1)]
    alll = [int((lv == l).sum()) for l in range(top + 1)]
    nonleaf = [int(((lv == l) & (ty == cmg.NONLEAF)).sum()) for l in range(top + 1)]
    nleaf = int((ty == cmg.LEAF).sum())
    B, c = BYTES_PER_CELL, 512
    cycle = 0.0
    for l in range(2, top + 1):
        v = mu ** (top - l)
        li = finest_iters if (l == top and finest_iters >= 0) else level_iters
        # li sweeps before and li after the coarse correction, two colour passes each
        step = 4 * li * act[l] * BYTES_PER_CELL_GS + act[l] * B["restrict"] + nonleaf[l - 1] * B["fas"] + alll[l] * B["prolong"]
        cycle += v * step * c
    cycle += (mu ** max(top - 1, 0)) * 9 * c * B["coarse"] + len(lv) * c * B["fill"]
    leaf_iter = nleaf * c * (B["apply"] + B["xr"] + B["dot"] + B["pupdate"])
    return iters * cycle + iters * leaf_iter + nleaf * c * (B["dot"] + B["fill"])


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


WORKLOADS = {
    "sphere": WORKLOAD,
    "uniform64": "uniform 64^3 grid (h0=1/8, level 3), all cells INTERIOR, Dirichlet walls, rhs N(0,1) seed 0 minus mean",
    "batched64": "64 adaptive octrees (seed 2): finest level 4 or 5 within 0.05 of 1-3 solid spheres r~U(0.05,0.15), "
                 "centres U(0.2,0.8)^3, level 3 elsewhere; Fourier-divergence rhs per octree",
    "moving_sphere": "sequence of adaptive sphere octrees (levels 4/5/6, r=0.1) with the sphere centre moving on a circle of "
                     "radius 0.25 around (0.5,0.5,0.5) in the z=0.5 plane at 1 revolution per 400 steps; octree, cut-cell "
                     "operator and Fourier-divergence rhs (seed 1) rebuilt per step",
}
BATCH_STREAMS = 16


def moving_sphere_spec(step):
    """Position `step` of the moving-sphere sequence: centre on a circle of radius 0.25, 400 steps per turn."""
    th = 2.0 * np.pi * step / 400.0
    c = (0.5 + 0.25 * np.cos(th), 0.5 + 0.25 * np.sin(th), 0.5)
    return dict(case="shell", params=[4, 6, 5, c[0], c[1], c[2], 0.1, 0.05, 0.15], spheres=[(c[0], c[1], c[2], 0.1)],
                rhs=("fourier", 1))


def instance_specs(name):
    """The octrees of a workload: refinement case and parameters, cut-cell spheres, rhs."""
    if name == "sphere":
        return [dict(case="shell", params=SHELL, spheres=SPHERES, rhs=("fourier", 1))]
    if name == "moving_sphere":
        return [moving_sphere_spec(0)]
    if name == "uniform64":
        return [dict(case="uniform", params=[3, 3], spheres=None, rhs=("normal", 0))]
    rng = np.random.default_rng(2)
    specs = []
    for i in range(64):
        finest = int(rng.integers(4, 6))
        ns = int(rng.integers(1, 4))
        sph = [tuple(float(v) for v in rng.uniform(0.2, 0.8, 3)) + (float(rng.uniform(0.05, 0.15)),) for _ in range(ns)]
        params = [3, finest, 0.05, ns] + [v for sp in sph for v in sp]
        specs.append(dict(case="multi", params=params, spheres=sph, rhs=("fourier", 100 + i)))
    return specs


def normal_rhs(ty, seed, leaf):
    """N(0,1) per LEAF cell in tile order, mean removed, 0 elsewhere."""
    rng = np.random.default_rng(seed)
    m = ty == leaf
    n = int(m.sum())
    v = rng.standard_normal(n * 512).astype(np.float32)
    v -= v.mean(dtype=np.float64).astype(np.float32)
    b = np.zeros((ty.size, 512), np.float32)
    b[m] = v.reshape(n, 512)
    return b


def build_grid(cmg, spec):
    """One octree on the device with its operator and rhs (b in channel 1 and BSAVE)."""
    case = {"shell": cmg.CASE_SHELL, "uniform": cmg.CASE_UNIFORM, "multi": cmg.CASE_MULTI_SPHERE}[spec["case"]]
    G = cmg.HADeviceGrid(0.125, 10, 16)
    G.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    G.rebuild()
    G.refine_case(case, spec["params"], on_device=True)  # the octree built in device memory
    G.set_leaf_cell_types_case(cmg.CASE_UNIFORM)
    if spec["spheres"]:
        G.cutcell_sphere_coeffs(COEFF, spec["spheres"], 0.5)
    else:
        cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0).prepareTypesAndCoeffs(G)
    kind, seed = spec["rhs"]
    if kind == "fourier":
        k, amp, ph = fourier_modes(seed)
        G.face_velocity_fourier(U, k, amp, ph)
        G.divergence(U, COEFF, 1)
    else:
        G.upload(1, normal_rhs(G.tiles()[2], seed, cmg.LEAF))
    G.copy(1, BSAVE)
    G.synchronize()
    return G


def build_oracle_grid(O, spec):
    """The same octree, operator and rhs (channel 1) in the oracle."""
    case = {"shell": O.CASE_SHELL, "uniform": O.CASE_UNIFORM, "multi": O.CASE_MULTI_SPHERE}[spec["case"]]
    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(case, spec["params"])
    g.alloc(16)
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    if spec["spheres"]:
        g.cutcell_sphere_coeffs(COEFF, spec["spheres"], 0.5)
    else:
        g.coarsen_types_and_coeffs(COEFF, 0.5)
    kind, seed = spec["rhs"]
    if kind == "fourier":
        k, amp, ph = fourier_modes(seed)
        g.face_velocity_fourier(U, k, amp, ph)
        g.divergence(U, COEFF, 1)
    else:
        g.channel(1)[:] = normal_rhs(g.tiles()[2], seed, O.LEAF)
    return g


def build_workload(cmg, name="sphere"):
    return build_grid(cmg, instance_specs(name)[0])


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


def cpu_baseline_fp64(G, cmg, spec, what="the workload", solutions=None):
    """FP64 Jacobi-preconditioned CG (the algorithm of Eigen's default
    ConjugateGradient) on the same operator assembled into CSR, all host cores.
    With `solutions` ({name: [tiles, 512] array}), the FP64 solution is refined after the
    timed solve (one residual-correction solve, to ~1e-10) and each solution's relative L2
    error against it over the unknowns is reported."""
    from oracle import oracle as O

    case = {"shell": O.CASE_SHELL, "uniform": O.CASE_UNIFORM, "multi": O.CASE_MULTI_SPHERE}[spec["case"]]
    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(case, spec["params"])
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
    out = {"value": dt * 1e3, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
           "sample": f"one full FP64 Jacobi-CG solve of {what} to 1e-6 ({len(bb)} unknowns, {its} iterations, "
                     f"rel {rel:.2e}); OpenMP over all host threads"}
    if solutions:
        r = bb - O.csr_matvec(rp, ci, va, x)
        dx, its2, rel2 = O.csr_solve(rp, ci, va, r, 1e-4, 4000, 0)
        xr = x + dx
        res = np.linalg.norm(bb - O.csr_matvec(rp, ci, va, xr)) / np.linalg.norm(bb)
        nx = np.linalg.norm(xr)
        out["error_vs_fp64"] = {name: float(np.linalg.norm(sol[rt, rc].astype(np.float64) - xr) / nx)
                                for name, sol in solutions.items()}
        out["error_vs_fp64"]["fp64_reference_rel_residual"] = float(res)
    return out


def roofline_gs(G, S, cmg, torch, dev):
    """Roofline of the dominant kernel: the pipelined red-black GS launch (k_gs_pipe) on the
    finest level, as the cycle runs it (x starts at 0, so it is 0 on cells that are not
    INTERIOR), CUDA events on the grid's stream (the default stream here); L2 flushed (a
    256 MB write) before every measured pair of launches."""
    ntiles, L, nleaf = G.info()
    lv, ijk, ty = G.tiles()
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
    return launch_ms, achieved, alg_bytes, L, active, cells, peak, peak_kind, profile_traffic_per_cell()


def roofline_entry(launch_ms, achieved, alg_bytes, L, active, cells, peak, peak_kind, tpc):
    return {
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
    }


def training_rhs(cmg, G, spec, n):
    """Right-hand sides of the learned smoother's training pairs: the workload's rhs kind with
    other seeds (normal: 100..; Fourier divergence: 200..); never the timed rhs."""
    kind, _ = spec["rhs"]
    out = []
    _, _, ty = G.tiles()
    for i in range(n):
        if kind == "fourier":
            k, amp, ph = fourier_modes(200 + i)
            G.face_velocity_fourier(U, k, amp, ph)
            G.divergence(U, COEFF, 1)
            out.append(G.download(1))
        else:
            out.append(normal_rhs(ty, 100 + i, cmg.LEAF))
    return out


LEARNED_INFERENCE = ["mma.sync"]  # set from --learned-inference
LEARNED = dict(hidden=8, epochs=30, batch=256, lr=2e-3, damping=0.5, loss="energy", iters=(1, 2, 3, 5), rhs=10, max_tiles=1250,
               octrees=3)
# the network as the learned-preconditioner spec states it: conv 8->32, four residual blocks of
# two 3x3x3 convs at 32 channels, conv 32->1, inference and training on tcgen05
LEARNED_DEEP = dict(LEARNED, hidden=32, epochs=20, lr=1e-3, damping=0.25)
NETWORKS = {8: "conv 8->8, conv 8->8, conv 8->1 (3x3x3, BF16 operands)",
            32: "conv 8->32, 4 residual blocks of two 3x3x3 convs at 32 channels, conv 32->1 (BF16 operands)"}


def random_octree_specs(spec, k, seed=300):
    """k octrees like `spec` with the sphere moved and resized at random (centre U(0.3, 0.7)^3,
    radius U(0.07, 0.13), seeded): the training octrees of the learned smoother.  A uniform
    workload has one octree, so it trains on its own (with other right-hand sides)."""
    if spec["case"] != "shell":
        return [spec]
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(k):
        c = tuple(float(v) for v in rng.uniform(0.3, 0.7, 3))
        r = float(rng.uniform(0.07, 0.13))
        p = list(spec["params"])
        p[3:7] = [c[0], c[1], c[2], r]
        out.append(dict(case="shell", params=p, spheres=[c + (r,)], rhs=spec["rhs"]))
    return out


def collect_training_pairs(cmg, spec, S):
    """Training pairs of the learned smoother: plain solves of right-hand sides of the
    workload's kind (training seeds, never the timed rhs) on random octrees like the
    workload's (random_octree_specs), LEARNED["rhs"] right-hand sides in all."""
    import learned

    specs = random_octree_specs(spec, LEARNED["octrees"])
    per = max(1, LEARNED["rhs"] // len(specs))
    parts = []
    for i, sp in enumerate(specs):
        G = build_grid(cmg, sp)
        rhs = training_rhs(cmg, G, sp, per)
        # channels 10-12 (the face velocity, spent once the rhs exist) hold z, the FAS x0 and A z
        parts.append(learned.collect_pairs(G, S, COEFF, rhs, iters=LEARNED["iters"], max_tiles=LEARNED["max_tiles"], z_ch=U, x0_ch=U + 1,
                                           az_ch=U + 2, seed=i))
        del G
    return {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}


def learned_block(cmg, torch, spec, steps, world, dev, cfg=LEARNED, pairs=None):
    """The learned finest-level smoother on one workload: pairs from plain solves on random
    octrees like the workload's (collect_training_pairs, or the given pairs), trained on the
    GPU with the settings cfg, then the timed rhs solved plain and learned, each timed over
    `steps` solves with CUDA events (the learned solve's true-residual judge included).
    Returns the result and the pairs."""
    import learned

    S = make_solver(cmg)
    t0 = time.perf_counter()
    if pairs is None:
        pairs = collect_training_pairs(cmg, spec, S)
    G = build_grid(cmg, spec)
    t1 = time.perf_counter()
    net, losses = learned.train(pairs, hidden=cfg["hidden"], epochs=cfg["epochs"], batch=cfg["batch"], lr=cfg["lr"], seed=0,
                                damping=cfg["damping"], loss=cfg["loss"])
    torch.cuda.synchronize()
    t2 = time.perf_counter()

    def timed(use_net):
        S.set_learned(net if use_net else None)
        for _ in range(3):
            G.copy(BSAVE, 1)
            S.solve(G, *solve_args())
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            G.copy(BSAVE, 1)
            it, rel = S.solve(G, *solve_args())
        b.record()
        torch.cuda.synchronize()
        return replica_time(a.elapsed_time(b), world, dev) / steps, it, G.download(0)

    plain_ms, plain_it, xp = timed(False)
    ms, it, xl = timed(True)
    true_rel, fell_back, learned_it = S.learned_status()
    S.set_learned(None)
    _, _, ty = G.tiles()
    lm = ty == cmg.LEAF
    return {"hidden": cfg["hidden"], "network": NETWORKS[cfg["hidden"]], "loss": cfg["loss"],
            "kernels": "tcgen05 inference and training" if cfg["hidden"] == 32 else LEARNED_INFERENCE[0] + " inference, mma.sync training",
            "damping": cfg["damping"], "train_pairs": int(pairs["rho"].shape[0]), "collect_s": round(t1 - t0, 3),
            "train_s": round(t2 - t1, 3), "epochs": cfg["epochs"], "loss_first_epoch": float(losses[0]),
            "loss_last_epoch": float(losses[-1]), "plain_ms": round(plain_ms, 4), "plain_pcg_iters": plain_it,
            "learned_ms": round(ms, 4), "pcg_iters": it, "learned_pcg_iters": learned_it, "fell_back": fell_back,
            "rel_residual_true": true_rel,
            "rel_l2_vs_plain_solution": float(np.linalg.norm((xl - xp)[lm].astype(np.float64)) /
                                              np.linalg.norm(xp[lm].astype(np.float64)))}, pairs


def learned_on_tuned(cmg, torch, G, S2, best, spec, steps, world, dev):
    """The learned finest-level smoother on top of the autotuned cycle: training pairs from the
    residual the tuned cycle leaves (other right-hand sides of the same octree), the net trained
    on the GPU, then the timed rhs solved by the tuned cycle without and with it."""
    import learned

    t0 = time.perf_counter()
    rhs = training_rhs(cmg, G, spec, LEARNED["rhs"])
    pairs = learned.collect_pairs(G, S2, COEFF, rhs, iters=LEARNED["iters"], max_tiles=LEARNED["max_tiles"], z_ch=U, x0_ch=U + 1,
                                  az_ch=U + 2, level_iters=best[2], coarsest_iters=best[3])
    net, losses = learned.train(pairs, hidden=LEARNED["hidden"], epochs=LEARNED["epochs"], batch=LEARNED["batch"],
                                lr=LEARNED["lr"], seed=0, damping=LEARNED["damping"], loss=LEARNED["loss"])
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    args_t = (False, SOLVE["max_iters"], SOLVE["tol"], best[2], best[3], SOLVE["sync_stride"], False)

    def timed(use_net):
        S2.set_learned(net if use_net else None)
        for _ in range(3):
            G.copy(BSAVE, 1)
            S2.solve(G, *args_t)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            G.copy(BSAVE, 1)
            it, _ = S2.solve(G, *args_t)
        b.record()
        torch.cuda.synchronize()
        return replica_time(a.elapsed_time(b), world, dev) / steps, it

    tuned_ms, tuned_it = timed(False)
    ms, it = timed(True)
    true_rel, fell_back, learned_it = S2.learned_status()
    S2.set_learned(None)
    return {"trained_on": "residuals the tuned cycle leaves on other right-hand sides of the same octree",
            "train_and_collect_s": round(train_s, 3), "loss_first_epoch": float(losses[0]), "loss_last_epoch": float(losses[-1]),
            "tuned_ms": round(tuned_ms, 4), "tuned_pcg_iters": tuned_it, "learned_on_tuned_ms": round(ms, 4),
            "learned_pcg_iters": learned_it, "fell_back": fell_back, "rel_residual_true": true_rel}


def run_sequence(args, rank, world, local_rank):
    """The moving-sphere sequence: --steps positions, each with its own octree, cut-cell
    operator and rhs; at each position the plain and the learned solve (trained once, on
    random sphere octrees) are timed on the device.  value = mean plain ms
    per solve; the learned figures sit in config."""
    import torch

    import cmg
    import learned

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    spec0 = moving_sphere_spec(0)
    S = make_solver(cmg)
    t0 = time.perf_counter()
    pairs = collect_training_pairs(cmg, spec0, S)  # random sphere octrees, not the sequence's
    cfg = LEARNED_DEEP if args.learned_net == "residual" else LEARNED
    net, losses = learned.train(pairs, hidden=cfg["hidden"], epochs=cfg["epochs"], batch=cfg["batch"], lr=cfg["lr"], seed=0,
                                damping=cfg["damping"], loss=cfg["loss"])
    train_s = time.perf_counter() - t0
    G = build_grid(cmg, spec0)
    rhs = training_rhs(cmg, G, spec0, 1)
    # the autotuned smoother, tuned once at position 0 on a training rhs
    St = make_solver(cmg)
    G.upload(1, rhs[0])
    best, _ = St.autotune(G, max_iters=SOLVE["max_iters"], relative_tolerance=SOLVE["tol"], repeats=2)
    targs = (False, SOLVE["max_iters"], SOLVE["tol"], best[2], best[3], SOLVE["sync_stride"], False) if best else None
    del G
    for _ in range(args.warmup):  # warm both graphs on the first position
        G = build_grid(cmg, spec0)
        for use in (None, net):
            S.set_learned(use)
            G.copy(BSAVE, 1)
            S.solve(G, *solve_args())
    sampler = ClockSampler(local_rank)
    sampler.start()
    plain_ms, learned_ms, plain_it, learned_it, fallbacks, true_rel, setup_s, launches = [], [], [], [], 0, [], 0.0, 0
    tuned_ms, tuned_it = [], []
    for k in range(args.steps):
        t1 = time.perf_counter()
        G = build_grid(cmg, moving_sphere_spec(k))
        setup_s += time.perf_counter() - t1
        S.set_learned(None)
        G.copy(BSAVE, 1)
        it, _ = S.solve(G, *solve_args())
        plain_ms.append(S.last_solve_ms())
        plain_it.append(it)
        launches += S.last_solve_launches()
        S.set_learned(net)
        G.copy(BSAVE, 1)
        it, _ = S.solve(G, *solve_args())
        learned_ms.append(S.last_solve_ms())
        launches += S.last_solve_launches()
        tr, fb, lit = S.learned_status()
        learned_it.append(lit)
        fallbacks += int(fb)
        true_rel.append(tr)
        S.set_learned(None)
        if targs:
            G.copy(BSAVE, 1)
            it, _ = St.solve(G, *targs)
            tuned_ms.append(St.last_solve_ms())
            tuned_it.append(it)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    mp, ml = float(np.mean(plain_ms)), float(np.mean(learned_ms))
    return {
        "metric": METRIC, "value": round(mp, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(mp, 4), "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": WORKLOADS["moving_sphere"], "method": "plain FP32 FAS mu-cycle (mu=2) MG-PCG, FP64 dots",
            "timing": "device time of each solve's graph (CUDA events inside the library); the octree, operator and rhs set-up of each position is outside it (its host wall time is octree_setup_ms_per_step)",
            "l2": "inputs larger than L2: ~550 MB of channel planes per octree",
            "plain_pcg_iters": [min(plain_it), max(plain_it)], "octree_setup_ms_per_step": round(setup_s * 1e3 / max(args.steps, 1), 2),
            "learned_preconditioner": {
                "hidden": cfg["hidden"], "network": NETWORKS[cfg["hidden"]], "loss": cfg["loss"], "damping": cfg["damping"],
                "inference_kernel": "tcgen05" if cfg["hidden"] == 32 else LEARNED_INFERENCE[0], "trained_on": "3 random sphere octrees, 10 right-hand sides (none of the sequence's)", "train_and_collect_s": round(train_s, 3),
                "loss_first_epoch": float(losses[0]), "loss_last_epoch": float(losses[-1]),
                "ms_mean": round(ml, 4), "learned_pcg_iters": [min(learned_it), max(learned_it)], "fell_back": fallbacks,
                "rel_residual_true_max": float(max(true_rel)), "plain_ms_mean": round(mp, 4)},
            "autotuned_smoother": None if not targs else {
                "tuned_on": "position 0, one training rhs", "omega": best[0], "mu": best[1], "level_iters": best[2],
                "coarsest_iters": best[3], "finest_iters": best[4], "ms_mean": round(float(np.mean(tuned_ms)), 4),
                "pcg_iters": [min(tuned_it), max(tuned_it)], "speedup_vs_plain": round(mp / float(np.mean(tuned_ms)), 3)},
        },
        "gpu_launches": int(launches),
        "clocks": clocks,
    }


def run_ours(args, rank, world, local_rank):
    import torch

    import cmg

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    spec = instance_specs(args.workload)[0]
    G = build_grid(cmg, spec)
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

    # the mixed-precision preconditioner, timed the same way on the same solve, against the
    # FP32 solution above: 16-bit operator storage in the smoothing sweeps; the FP64 direct
    # coarsest solve alone (timed against the reference's coarsest sweeps); and the whole
    # mixed mode (BF16 storage, FP64 true residual every 10 iterations, direct coarsest)
    x32 = G.download(0)
    mixed, mixed_x = {}, {"fp32": x32}
    # (operator storage, x/rhs of levels >= 3 in BF16, true residual every N, direct coarsest)
    mixed_modes = {"bf16": ("bf16", False, 0, False), "fp16": ("fp16", False, 0, False),
                   "bf16_operator_x_rhs": ("bf16", True, 0, False),
                   "bf16_operator_x_rhs_replace10": ("bf16", True, 10, False),
                   "fp32_direct_coarsest": ("fp32", False, 0, True),
                   "bf16_operator_x_rhs_replace10_direct_coarsest": ("bf16", True, 10, True)}
    for mode, (storage, cycle16, every, direct) in mixed_modes.items():
        S.set_storage(storage)
        S.set_cycle_bf16(cycle16)
        S.set_residual_replacement(every)
        S.set_coarsest_direct(direct)
        for _ in range(3):
            one_solve()
        torch.cuda.synchronize()
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record()
        for _ in range(args.steps):
            it_m, rel_m = one_solve()
        m1.record()
        torch.cuda.synchronize()
        xm = G.download(0)
        mixed_x[mode] = xm
        lm = ty == cmg.LEAF
        mixed[mode] = {"ms": round(replica_time(m0.elapsed_time(m1), world, dev) / args.steps, 4), "pcg_iters": it_m,
                       "rel_residual_recurrence": rel_m, "residual_replacements": S.last_replacements(),
                       "rel_l2_vs_fp32_solution": float(np.linalg.norm((xm - x32)[lm].astype(np.float64)) /
                                                        np.linalg.norm(x32[lm].astype(np.float64)))}
    S.set_storage("fp32")
    S.set_cycle_bf16(False)
    S.set_residual_replacement(0)
    S.set_coarsest_direct(False)
    one_solve()
    torch.cuda.synchronize()

    # the learned finest-level smoother on the uniform 64^3 grid and on this workload
    learned_res = []
    if not args.no_learned:
        for name in dict.fromkeys(["uniform64", args.workload]):
            spec_n = dict(instance_specs(name)[0], name=name)
            res, pairs = learned_block(cmg, torch, spec_n, args.steps, world, dev)
            learned_res.append(dict(res, workload=WORKLOADS[name]))
            res, _ = learned_block(cmg, torch, spec_n, args.steps, world, dev, cfg=LEARNED_DEEP, pairs=pairs)
            learned_res.append(dict(res, workload=WORKLOADS[name]))

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

    launch_ms, achieved, alg_bytes, L, active, cells, peak, peak_kind, tpc = roofline_gs(G, S, cmg, torch, dev)

    # the autotuned smoother: omega, mu and the sweep counts learned by timing solves of another
    # right-hand side (training seed), then the timed rhs solved with them (FP32, and with the
    # BF16 operator storage); a second solver object, so the plain solver above is untouched
    tuned = None
    if not args.no_learned:
        S2 = make_solver(cmg)
        G.upload(1, training_rhs(cmg, G, spec, 1)[0])
        t0 = time.perf_counter()
        best, table = S2.autotune(G, max_iters=SOLVE["max_iters"], relative_tolerance=SOLVE["tol"], repeats=2)
        tune_s = time.perf_counter() - t0
        if best is not None:
            def timed_tuned(storage, cycle16=False):
                S2.set_storage(storage)
                S2.set_cycle_bf16(cycle16)
                args_t = (False, SOLVE["max_iters"], SOLVE["tol"], best[2], best[3], SOLVE["sync_stride"], False)
                for _ in range(3):
                    G.copy(BSAVE, 1)
                    S2.solve(G, *args_t)
                torch.cuda.synchronize()
                a, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                for _ in range(args.steps):
                    G.copy(BSAVE, 1)
                    torch.cuda.nvtx.range_push("tuned_solve")
                    it_t, _ = S2.solve(G, *args_t)
                    torch.cuda.nvtx.range_pop()
                b_.record()
                torch.cuda.synchronize()
                return replica_time(a.elapsed_time(b_), world, dev) / args.steps, it_t, G.download(0)

            ms_t, it_t, mixed_x["tuned"] = timed_tuned("fp32")
            ms_tb, it_tb, mixed_x["tuned_bf16"] = timed_tuned("bf16")
            ms_tc, it_tc, mixed_x["tuned_bf16_operator_x_rhs"] = timed_tuned("bf16", True)
            S2.set_storage("fp32")
            S2.set_cycle_bf16(False)
            on_top = learned_on_tuned(cmg, torch, G, S2, best, spec, args.steps, world, dev)
            tuned = {"tuned_on": "one training rhs of the same octree (seed 100 / Fourier seed 200), never the timed one",
                     "tune_s": round(tune_s, 3), "candidates": len(table),
                     "omega": best[0], "mu": best[1], "level_iters": best[2], "coarsest_iters": best[3], "finest_iters": best[4],
                     "ms": round(ms_t, 4), "pcg_iters": it_t, "ms_bf16_storage": round(ms_tb, 4), "pcg_iters_bf16_storage": it_tb,
                     "ms_bf16_operator_x_rhs": round(ms_tc, 4), "pcg_iters_bf16_operator_x_rhs": it_tc,
                     "plain_setting": {"omega": SOLVE["omega"], "mu": SOLVE["mu"], "level_iters": SOLVE["level_iters"],
                                       "coarsest_iters": SOLVE["coarsest_iters"]},
                     "learned_smoother_on_top": on_top}

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
                "workload": WORKLOADS[args.workload],
                "method": "plain FP32 FAS mu-cycle (mu=2) MG-PCG, FP64 dots",
                "tiles": ntiles, "leaf_tiles": nleaf, "leaf_cells": leaf_cells, "interior_cells": interior, "max_level": maxl,
                "pcg_iters": iters[-1], "rel_residual_recurrence": rels[-1], "rel_residual_true_fp32_apply": true_rel,
                "solve_ms_p50": sorted(per_ms)[len(per_ms) // 2],
                "l2": f"inputs larger than L2: {16 * ntiles * 2048 / 1e6:.0f} MB of channel planes per grid",
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "e2e_wall_ms": round(e2e_wall_ms, 4),
                "mixed_precision_preconditioner": mixed,
                "learned_preconditioner": learned_res,
                "autotuned_smoother": tuned,
            },
            "e2e": {"value": round(e2e_ms, 4), "unit": UNIT, "h2d_bytes_per_step": count * 4, "d2h_bytes_per_step": count * 4},
            "gpu_launches": int(launches),
            "roofline": roofline_entry(launch_ms, achieved, alg_bytes, L, active, cells, peak, peak_kind, tpc),
            "clocks": clocks,
        }
        # the whole solve against the HBM roofline: algorithmic bytes of every cycle and PCG step
        # (solve_algorithmic_bytes) over the solve's time, of the measured copy bandwidth
        sb = solve_algorithmic_bytes(G, SOLVE["mu"], SOLVE["level_iters"], iters[-1])
        result["config"]["whole_solve_hbm"] = {
            "algorithmic_bytes": int(sb), "ms": round(per_solve, 4), "achieved_gbs": round(sb / per_solve / 1e6, 1),
            "per_vcycle_hbm_frac": round(sb / per_solve / 1e6 / peak, 4), "peak_gbs": peak, "peak_kind": peak_kind}
        if tuned is not None:
            tb = solve_algorithmic_bytes(G, tuned["mu"], tuned["level_iters"], tuned["pcg_iters"], tuned["finest_iters"])
            tuned["whole_solve_hbm"] = {"algorithmic_bytes": int(tb), "achieved_gbs": round(tb / tuned["ms"] / 1e6, 1),
                                        "per_vcycle_hbm_frac": round(tb / tuned["ms"] / 1e6 / peak, 4)}
            tuned["speedup_vs_plain"] = round(per_solve / tuned["ms"], 3)
            tuned["speedup_vs_plain_bf16_storage"] = round(per_solve / tuned["ms_bf16_storage"], 3)
            tuned["speedup_vs_plain_bf16_operator_x_rhs"] = round(per_solve / tuned["ms_bf16_operator_x_rhs"], 3)
        if world == 1 and not args.no_cpu_baseline:
            cb = cpu_baseline_fp64(G, cmg, spec, solutions=mixed_x)
            err = cb.pop("error_vs_fp64", None)
            result["cpu_baseline"] = cb
            if err:
                result["config"]["solution_error_vs_fp64"] = err
    return result


BATCH_METRIC = "Poisson solves per second to 1e-6 rel. residual, 64 batched adaptive octrees, 1×B200"
BATCH_UNIT = "solves/s"
# candidate schedules of the persistent batch: (blocks per small group, split, slots per block)
BATCH_SCHEDULES = [(g, sp, ns) for ns in (6, 8) for g, sp in ((4, 0.0), (6, 0.0), (8, 0.0), (2, 1.0), (4, 1.0), (4, 1.2))] + [(4, 1.0, 4)]


def run_batched(args, rank, world, local_rank):
    """64 independent octrees per step, all solved by ONE persistent cooperative kernel launch
    inside a CUDA graph (cmg_batch_solve): groups of blocks take the octrees from a device
    queue, largest first; the schedule (slots per block, group sizes, groups of their own for
    the largest octrees) is picked by the batch autotuner.  The same batch as 64 graph
    launches on BATCH_STREAMS streams (cmg_amg_solve_batch) is timed beside it."""
    import torch

    import cmg

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    specs = instance_specs("batched64")[:max(1, args.batch_instances)]
    grids = [build_grid(cmg, sp) for sp in specs]
    solvers = [make_solver(cmg) for _ in specs]
    n = len(grids)
    infos = [G.info() for G in grids]
    sargs = (SOLVE["max_iters"], SOLVE["tol"], SOLVE["level_iters"], SOLVE["coarsest_iters"], SOLVE["sync_stride"], False)
    batch = cmg.PersistentBatch(solvers, grids)
    fixed = None
    if args.batch_schedule:
        g_, sp_, ns_ = args.batch_schedule.split(",")
        fixed = (int(g_), float(sp_), int(ns_))

    def restore():
        for G in grids:
            G.copy(BSAVE, 1)

    def one_batch(b_host=None, x_host=None, solve_args=None):
        if b_host is None:
            restore()
        return batch.solve(*(solve_args or sargs), b_host=b_host, x_host=x_host)

    def timed(steps, fn, **kw):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = []
        for _ in range(steps):
            torch.cuda.nvtx.range_push("batch")
            out.append(fn(**kw))
            torch.cuda.nvtx.range_pop()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    # the schedule: the autotuner times the candidates (the schedule never changes a result)
    restore()
    t0 = time.perf_counter()
    if fixed is None:
        cands = BATCH_SCHEDULES
        sched, sched_table = batch.autotune(cands, *sargs[:4], repeats=2)
    else:
        cands, sched, sched_table = [], fixed, []
        batch.set_schedule(*fixed)
    sched_s = time.perf_counter() - t0
    slots, gblocks, ngroups, dedicated, resident = batch.schedule()

    for _ in range(max(args.warmup, 1)):
        one_batch()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    t_ms, out = timed(args.steps, one_batch)
    clocks = sampler.stop()
    total_ms = replica_time(t_ms, world, dev)
    per = sorted(m for _, _, ms, _ in out for m in ms)
    launch_ms = sorted(bms for _, _, _, bms in out)
    its = [i for it, _, _, _ in out for i in it]
    rels = [r for _, rel, _, _ in out for r in rel]

    # e2e: the same batch through the C ABI with pinned host buffers for b and x
    b_host = [torch.from_numpy(G.download(BSAVE).reshape(-1)).pin_memory() for G in grids]
    x_host = [torch.empty_like(b).pin_memory() for b in b_host]
    hb = dict(b_host=[b.data_ptr() for b in b_host], x_host=[x.data_ptr() for x in x_host])
    one_batch(**hb)
    e2e_ms, _ = timed(args.steps, one_batch, **hb)
    e2e_ms = replica_time(e2e_ms, world, dev)
    nbytes = sum(b.numel() * 4 for b in b_host)

    # roofline of the one kernel: algorithmic bytes of all 64 solves / its CUDA-event time
    alg = sum(solve_algorithmic_bytes(G, SOLVE["mu"], SOLVE["level_iters"], it) for G, it in zip(grids, out[0][0]))
    lms = launch_ms[len(launch_ms) // 2]
    peak, peak_kind = measured_peaks()
    achieved = alg / (lms * 1e-3) / 1e9
    roof = {"kernel": f"k_batch_solve (persistent batch: {slots} slots per block, {ngroups} groups, {dedicated} of them for one octree each)",
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "peak_kind": peak_kind, "algorithmic_bytes_per_launch": int(alg), "launch_ms": round(lms, 4), "traffic": None}

    # the same batch as separate graph launches on BATCH_STREAMS streams
    nstreams = max(1, args.streams)
    streams = [torch.cuda.Stream(device=dev) for _ in range(nstreams)]
    for i, G in enumerate(grids):
        G.set_stream(streams[i % nstreams].cuda_stream)

    def ms_batch(solve_args=None):
        restore()
        return cmg.solve_batch(solvers, grids, *(solve_args or sargs))

    def timed_streams(steps, solve_args=None):
        ms_batch(solve_args)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for st in streams:
            st.wait_event(e0)
        res = [ms_batch(solve_args) for _ in range(steps)]
        for st in streams:
            ev = torch.cuda.Event()
            ev.record(st)
            torch.cuda.current_stream().wait_event(ev)
        e1.record()
        torch.cuda.synchronize()
        return replica_time(e0.elapsed_time(e1), world, dev), res

    ms_t, ms_out = timed_streams(args.steps)
    ms_per = sorted(m for _, _, ms in ms_out for m in ms)
    multistream = {"streams": nstreams, "solves_per_s": round(n * args.steps * world / (ms_t / 1e3), 2),
                   "solve_ms_p50": ms_per[len(ms_per) // 2], "solve_ms_p99": ms_per[min(len(ms_per) - 1, int(0.99 * len(ms_per)))]}
    for G in grids:
        G.set_stream(0)

    # the autotuned smoother: tuned once on octree 0 with a training rhs, applied to all 64
    tuned = None
    if not args.no_learned:
        G0 = grids[0]
        G0.upload(1, training_rhs(cmg, G0, specs[0], 1)[0])
        t0 = time.perf_counter()
        best, table = solvers[0].autotune(G0, max_iters=SOLVE["max_iters"], relative_tolerance=SOLVE["tol"], repeats=2)
        tune_s = time.perf_counter() - t0
        if best is not None:
            for S in solvers:
                S.omega, S.mu_cycle_repeat_times, S.finest_iters = best[0], best[1], best[4]
            targs = (SOLVE["max_iters"], SOLVE["tol"], best[2], best[3], SOLVE["sync_stride"], False)
            restore()
            tsched = fixed
            if fixed is None:
                tsched, _ = batch.autotune(BATCH_SCHEDULES, *targs[:4], repeats=1)
            one_batch(solve_args=targs)
            t_t, out_t = timed(args.steps, one_batch, solve_args=targs)
            per_t = sorted(m for _, _, ms, _ in out_t for m in ms)
            its_t = [i for it, _, _, _ in out_t for i in it]
            for i, G in enumerate(grids):
                G.set_stream(streams[i % nstreams].cuda_stream)
            ms_tt, _ = timed_streams(args.steps, targs)
            for G in grids:
                G.set_stream(0)
            tuned = {"tuned_on": "octree 0, one training rhs (Fourier seed 200)", "tune_s": round(tune_s, 3),
                     "omega": best[0], "mu": best[1], "level_iters": best[2], "coarsest_iters": best[3], "finest_iters": best[4],
                     "schedule": list(tsched) if tsched is not None else None,
                     "solves_per_s": round(n * args.steps * world / (replica_time(t_t, world, dev) / 1e3), 2),
                     "multistream_solves_per_s": round(n * args.steps * world / (ms_tt / 1e3), 2),
                     "pcg_iters_mean": round(float(np.mean(its_t)), 2), "pcg_iters_max": int(max(its_t)),
                     "rel_residual_max": max(r for _, rel, _, _ in out_t for r in rel),
                     "solve_ms_p50": per_t[len(per_t) // 2], "solve_ms_p99": per_t[min(len(per_t) - 1, int(0.99 * len(per_t)))]}
            for S in solvers:
                S.omega, S.mu_cycle_repeat_times, S.finest_iters = SOLVE["omega"], SOLVE["mu"], -1

    result = None
    if rank == 0:
        value = n * args.steps * world / (total_ms / 1e3)
        result = {
            "metric": BATCH_METRIC, "value": round(value, 2), "unit": BATCH_UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {
                "workload": WORKLOADS["batched64"], "method": "plain FP32 FAS mu-cycle (mu=2) MG-PCG, FP64 dots, batched",
                "execution": "one persistent cooperative kernel launch per batch, inside a CUDA graph",
                "schedule": {"slots_per_block": slots, "small_group_blocks": gblocks, "groups": ngroups, "dedicated_groups": dedicated,
                             "resident_blocks": resident, "split": (sched[1] if sched is not None and not isinstance(sched, int) else 0.0),
                             "tune_s": round(sched_s, 3),
                             "candidates_ms": {str(tuple(c) if not isinstance(c, int) else c): round(m, 2) for c, m in zip(cands, sched_table)}},
                "instances": n, "tiles": int(sum(i[0] for i in infos)),
                "leaf_cells": int(sum(i[2] for i in infos)) * 512, "finest_levels": sorted({int(i[1]) for i in infos}),
                "pcg_iters_mean": round(float(np.mean(its)), 2), "pcg_iters_max": int(max(its)), "rel_residual_max": max(rels),
                "solve_ms_p50": per[len(per) // 2], "solve_ms_p99": per[min(len(per) - 1, int(0.99 * len(per)))],
                "per_solve_ms_is": "each octree's solve time inside the launch (device clock)",
                "launch_ms_median": round(lms, 4),
                "multistream": multistream,
                "l2": f"inputs larger than L2: {16 * sum(i[0] for i in infos) * 2048 / 1e9:.1f} GB of channel planes",
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "autotuned_smoother": tuned,
            },
            "e2e": {"value": round(n * args.steps * world / (e2e_ms / 1e3), 2), "unit": BATCH_UNIT, "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes},
            "gpu_launches": int(args.steps),
            "roofline": roof,
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            cb = cpu_baseline_fp64(grids[0], cmg, specs[0], "octree 0 of the batch")
            if cb["value"]:
                cb["sample"] += "; solves/s = 1000 / its ms"
                cb["value"] = 1000.0 / cb["value"]
            cb["unit"] = BATCH_UNIT
            result["cpu_baseline"] = cb
    return result


def run_reference(args):
    """The reference's algorithm for this path on the host cores: the oracle's
    restatement of AMGSolver::solve (src/AMGSolver.cu:1399), OpenMP over all
    host threads, on the same workload (for the batch: a sample of its octrees)."""
    from oracle import oracle as O

    specs = instance_specs(args.workload)
    batched = args.workload == "batched64"
    sample_specs = specs[:2] if batched else specs[:1]
    steps = max(1, min(args.steps, 2 if batched else 5))
    warm = min(args.warmup, 1)
    times, it, rel = [], 0, 0.0
    for sp in sample_specs:
        g = build_oracle_grid(O, sp)
        b = g.channel(1).copy()
        for st in range(warm + steps):
            g.channel(1)[:] = b
            t0 = time.perf_counter()
            it, rel = g.amg_solve(COEFF, omega=SOLVE["omega"], mu=SOLVE["mu"], max_iters=SOLVE["max_iters"], tol=SOLVE["tol"],
                                  level_iters=SOLVE["level_iters"], coarsest_iters=SOLVE["coarsest_iters"], sync_stride=1)
            dt = (time.perf_counter() - t0) * 1e3
            if st >= warm:
                times.append(dt)
    ms = sum(times) / len(times)
    if batched:
        v, unit, metric, hib = 1000.0 / ms, BATCH_UNIT, BATCH_METRIC, True
        sample = (f"{steps} solves each of octrees 0 and 1 of the batch by the C restatement of AMGSolver::solve, OpenMP; "
                  f"solves/s = 1000 / mean ms ({ms:.1f} ms); the reference's own solver is CUDA-only")
    else:
        v, unit, metric, hib = ms, UNIT, METRIC, False
        sample = (f"{steps} full solves of the workload ({it} PCG iterations, rel {rel:.2e}) by the C restatement of "
                  f"AMGSolver::solve, OpenMP; the reference's own solver is CUDA-only")
    return {
        "impl": "reference",
        "metric": metric, "value": round(v, 3), "unit": unit, "n_gpus": 1, "steps": steps, "warmup": warm,
        "ms_per_step": round(ms, 3), "higher_is_better": hib, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": WORKLOADS[args.workload], "method": "reference FAS mu-cycle MG-PCG on host cores"},
        "cpu_baseline": {"value": round(v, 3), "unit": unit, "cores": os.cpu_count(), "kind": "port", "sample": sample},
        "e2e": {"value": round(v, 3), "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-smoother comparison")
    ap.add_argument("--learned-inference", default="mma.sync", choices=["mma.sync", "tcgen05"],
                    help="inference kernel of the learned smoother")
    ap.add_argument("--workload", default="sphere", choices=sorted(WORKLOADS))
    ap.add_argument("--learned-net", default="small", choices=["small", "residual"],
                    help="moving_sphere: the learned smoother's net (small: 3 convs at 8 channels; residual: 4 residual blocks at 32)")
    ap.add_argument("--streams", type=int, default=BATCH_STREAMS, help="streams of the batched workload")
    ap.add_argument("--batch-instances", type=int, default=64, help="batched workload: solve only its first N octrees (profiling)")
    ap.add_argument("--batch-schedule", default=None,
                    help="batched workload: a fixed schedule 'group_blocks,split,slots' instead of the autotuned one (profiling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl != "reference":
        import cmg

        LEARNED_INFERENCE[0] = args.learned_inference
        cmg.set_learned_inference(args.learned_inference)

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
    runner = {"batched64": run_batched, "moving_sphere": run_sequence}.get(args.workload, run_ours)
    res = runner(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
