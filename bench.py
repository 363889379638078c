"""Benchmark of the IBPM time step on B200.

Workload: the 1024 x 1024, 5-level, 628-point cylinder at Re 100, dt 0.001
with seeded vorticity noise (amplitude 1e-3) -- the FP64 GPU configuration;
synthetic inputs.  One "step" is one advance! of the whole case.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank runs an independent replica of the case
(the single case does not shard); value = total steps/s over ranks.
`--impl reference` times the CPU restatement of the reference (the oracle, all
host threads) on the same workload; under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "immersedbodies.jl_b200")
METRIC = "IBPM steps/s on 1 B200, chosen form vs plain FP64 GPU at |ΔC_D,C_L|≤1e-4"
WORKLOAD = "cylinder_re100_1024: 1024x1024 cells x 5 levels, 628 body points, Re 100, dt 0.001, FP64 plain path"


def load_package():
    name = "immersedbodies_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def step_bytes_model(nx: int, ny: int, L: int, npanel: int, s: float = 1.0) -> float:
    """Algorithmic HBM bytes of one static-body step: one read and one write of every
    field each pass touches, with each 2D DST-diagonalised solve counted as three
    full passes.  G, Q are one level of circulation / flux in bytes.

    nonlinear + rhs L(Q+4G); A and Ainv solves 12GL; two vort2flux
    2(6GL + L(G+Q) + 1.25G(L-1)); projection 6G + 2GL; B^-1 matvec 8(2np)^2."""
    G = 8.0 * (nx - 1) * (ny - 1) * s
    Q = 8.0 * ((nx + 1) * ny + nx * (ny + 1)) * s
    return (L * (Q + 4 * G) + 12 * G * L + 2 * (6 * G * L + L * (G + Q) + 1.25 * G * (L - 1)) + 6 * G + 2 * G * L
            + 8.0 * (2 * npanel) ** 2)


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# dominant kernel classes, each from one ncu capture (constants, not measured by
# this run); the command of each capture is in NCU_TRAFFIC_RUN.
NCU_TRAFFIC = {"ypass": 8454912.0, "xpass": 8417792.0}
NCU_TRAFFIC_RUN = {"ypass": "ncu --set full --clock-control none -k regex:ypass_kernel -s 210 -c 1 python bench.py "
                            "--steps 1 --warmup 3 --no-cpu-baseline --no-chosen --no-learned --no-ensemble: one "
                            "single-level launch (1023^2 FP64), cold-cache replay",
                   "xpass": "ncu --set full --clock-control none --nvtx --nvtx-include timed/ -k regex:xpass_kernel "
                            "-s 1 -c 1 python bench.py --steps 2 --warmup 3 --no-cpu-baseline --no-chosen --no-learned "
                            "--no-ensemble: one single-level launch (1023^2 FP64, vort2flux level 5), cold-cache replay"}


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def read_tensor_peak():
    """Dense BF16 TFLOP/s of this pool's B200s for a kernel timed alone (burst)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def tensor_core_rebuild_report(ib, device: int, steps: int = 10, warmup: int = 3):
    """The preconditioner's B assembled on the tensor cores, rebuilt every step of
    the moving-body workload (512^2 x 4 levels, 101-point plate, k = 0.55; 202
    columns per batched solve): steps/s per product count against the FP64
    direct start (CUDA events on the solver's stream), and, from one profiled
    step (events around each launch group, eager launches), the tensor-core
    passes' algorithmic FLOP rate against the measured BF16 peak."""
    peak, src = read_tensor_peak()
    out = {"workload": "pitching_plate_512: preconditioned CG rebuilt every step, B assembled from 202 columns; "
                       "tensor-core passes: 4 nprod P^3 algorithmic flops per field and solve (P = 512)",
           "fp64_direct_start": direct_start_run(ib, device, steps, warmup, 101, 0)}
    for products in (3, 1):
        run = direct_start_run(ib, device, steps, warmup, 101, products)
        s = ib.GpuCnabSolver(ib.State(ib.configs.pitching_plate(0.55)),
                             cg=dict(reltol=0.0, abstol=1e-10, maxiter=5000), device=device)
        s.set_warm_start(None, mode="preconditioned", depth=1)
        s.set_rebuild_transform(products)
        for _ in range(2):
            s.advance_()
        s.profile(True)
        s.advance_()
        n, ms, flops = s.profile_read("tcdst")
        nl, msl, bytes_l = s.profile_read("tclines")
        s.profile(False)
        del s
        achieved = flops / (ms / 1000.0) / 1e12
        out[f"products_{products}"] = {
            "steps_per_s": run["value"], "ms_per_step": run["ms_per_step"],
            "cg_iterations_mean": run["cg_iterations_mean"],
            "passes": {"launch_groups": n, "ms": ms, "tflops": flops / 1e12,
                       "achieved_tflops_s": achieved, "peak_tflops_s": peak, "peak_source": src,
                       "frac": achieved / peak},
            "lines": {"launches": nl, "ms": msl, "achieved_gb_s": bytes_l / (msl / 1000.0) / 1e9}}
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(v: float, pg, device) -> float:
    """The largest v over all ranks; every rank calls it at the same point (pg is
    torch.distributed or None for one process; device holds the reduction buffer:
    "cuda" under NCCL, "cpu" under gloo)."""
    if pg is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, steps: int, max_ms: float) -> float:
    """Steps/s of the whole job: every rank ran `steps` steps of its own replica and
    the slowest rank took max_ms."""
    return world * steps / (max_ms / 1000.0)


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_time_oracle(ib, steps: int, warmup: int, threads: int):
    """Steps/s of the CPU oracle (FP64 restatement of the reference) on the same case."""
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle import oracle as orc

    used = orc.set_threads(threads)
    prob = ib.configs.cylinder_re100_1024()
    st = ib.configs.seed_vorticity(ib.State(prob))
    s = orc.OracleSolver(st, timing_only=True)
    for _ in range(warmup):
        s.advance_(pull=False)
    t = time.perf_counter()
    for _ in range(steps):
        s.advance_(pull=False)
    dt = time.perf_counter() - t
    return steps / dt, used


def warm_start_report(ib, device: int, train_steps: int = 100, eval_steps: int = 100):
    """CG iterations and steps/s of the moving-body case (the 512^2 x 4-level
    pitching and plunging plate, 101 points, Re 500, dt 0.002, CG to an absolute
    residual of 1e-10) at a held-out reduced frequency k = 0.55, with the
    reference's start (the previous solution), the extrapolated start, the
    learned start, the projection onto the last 16 solutions, the direct start
    (B assembled and inverted on the GPU every step, or every 8th) and CG
    preconditioned by that inverse rebuilt every 8th or 32nd step (B assembled
    with the FP64 transforms, or on the tensor cores with three or one BF16
    products: "tc3", "tc1"); the network is
    trained on samples of k = 0.25, 0.45, 0.65 and 0.85 generated by the solver
    (after a 60-step start-up).  Every run takes the same steps, so their final
    forces differ only by the CG tolerance."""
    import torch

    cg = dict(reltol=0.0, abstol=1e-10, maxiter=5000)

    def make(k):
        return ib.GpuCnabSolver(ib.State(ib.configs.pitching_plate(k)), cg=cg, device=device)

    t0 = time.perf_counter()
    X, T = ib.warmstart.make_training_set(make, (0.25, 0.45, 0.65, 0.85), train_steps, skip=60)
    t_collect = time.perf_counter() - t0
    net = ib.WarmStartNet(seed=2026, device=device)
    net.fit_normalisation(X, T)
    t0 = time.perf_counter()
    losses = np.concatenate([net.train(X, T, epochs=200, batch=64, lr=1e-3),
                             net.train(X, T, epochs=200, batch=64, lr=2e-4, seed=8)])
    t_train = time.perf_counter() - t0
    out, forces = {}, {}
    runs = (("previous", "previous", 16), ("extrapolated", "extrapolated", 16), ("learned", "learned", 16),
            ("projected", "projected", 16), ("direct", "direct", 1), ("direct_every_8", "direct", 8),
            ("preconditioned_every_8", "preconditioned", 8), ("preconditioned_every_32", "preconditioned", 32),
            ("preconditioned_extrapolated_every_8", "preconditioned_extrapolated", 8),
            ("preconditioned_extrapolated_every_32", "preconditioned_extrapolated", 32),
            ("preconditioned_extrapolated_tc3_every_8", "preconditioned_extrapolated", 8, 3),
            ("preconditioned_extrapolated_tc3_every_32", "preconditioned_extrapolated", 32, 3),
            ("preconditioned_extrapolated_tc1_every_8", "preconditioned_extrapolated", 8, 1),
            ("preconditioned_extrapolated_tc1_every_32", "preconditioned_extrapolated", 32, 1))
    for label, mode, depth, *tc in runs:
        s = make(0.55)
        if mode != "previous":
            s.set_warm_start(net if mode == "learned" else None, mode=mode, depth=depth)
        if tc:
            s.set_rebuild_transform(tc[0])
        for _ in range(60):  # start-up transient, excluded
            s.advance_()
        stream = torch.cuda.ExternalStream(s.stream_handle())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        it, r0, coef = [], [], []
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(eval_steps):
            s.advance_()
            inf = s.info()
            it.append(inf.last_cg_iters)
            r0.append(inf.first_cg_residual)
            coef.append(list(inf.warm_start_coef))
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        forces[label] = np.asarray(s.total_force(), dtype=np.float64).copy()
        out[label] = {"cg_iterations_mean": float(np.mean(it)), "first_residual_geomean": float(np.exp(np.mean(np.log(np.maximum(r0, 1e-300))))),
                      "steps_per_s": eval_steps / (ms / 1000.0),
                      "galerkin_coef_median": [float(v) for v in np.median(np.asarray(coef), axis=0)]}
        if mode == "learned":
            Xh, Th, _ = ib.warmstart.collect_samples(s, 30)
            ph = net.forward(Xh)
            out[label]["held_out_r2"] = float(1 - ((ph - Th) ** 2).sum() / ((Th - Th.mean(axis=(0, 2), keepdims=True)) ** 2).sum())
        del s
    for label in out:
        f0 = forces["previous"]
        out[label]["max_force_diff_vs_previous_rel"] = float(np.abs(forces[label] - f0).max() / np.abs(f0).max())
    base = out["previous"]
    return {"workload": "pitching_plate_512: 512x512 cells x 4 levels, 101-point plate pitching 30 deg and plunging "
                        "0.25 chord, Re 500, dt 0.002; CG to |r| <= 1e-10; held-out k = 0.55",
            "training": {"samples": int(X.shape[0]), "ks": [0.25, 0.45, 0.65, 0.85], "collect_s": t_collect,
                         "train_s": t_train, "epochs": int(losses.size), "loss_first": float(losses[0]),
                         "loss_last": float(losses[-1])},
            "modes": out,
            "iterations_vs_previous": {m: out[m]["cg_iterations_mean"] / base["cg_iterations_mean"] for m in out},
            "steps_per_s_vs_previous": {m: out[m]["steps_per_s"] / base["steps_per_s"] for m in out}}


def mixed_precision_plate_report(ib, device: int, steps: int = 200, timed: int = 50):
    """The mixed-precision workload as configured: flat plate of chord 1 at 30 deg,
    Re 200, 1024^2 cells x 5 levels, 201 points, dt 0.001, from rest.  The FP64
    engine and each reduced-precision form ("mixed": level 1 in FP64, levels 2..5
    in FP32 -- the chosen form; "fp32": every level in FP32) are stepped side by
    side for `steps` steps; the largest |dC_D|, |dC_L| over those steps and over
    their second half, past the impulsive start (C = 2F / (U^2 c), U = c = 1),
    and the vorticity relative L2 at the end are reported, then each engine's
    steps/s over `timed` further steps (CUDA events on its stream)."""
    import torch

    prob = ib.configs.plate_aoa30_1024()

    def rate(s):
        stream = torch.cuda.ExternalStream(s.stream_handle())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        s.advance_many(timed)
        e1.record(stream)
        torch.cuda.synchronize()
        return timed / (e0.elapsed_time(e1) / 1000.0)

    out = {"workload": "plate_aoa30_1024: flat plate chord 1 at 30 deg, Re 200, 1024x1024 cells x 5 levels, "
                       "201 points, dt 0.001, from rest",
           "steps_compared": steps,
           "bar": "|dC_D|,|dC_L| <= 1e-4 and vorticity rel-L2 <= 1e-5 vs FP64"}
    v64 = None
    for prec in ("mixed", "fp32"):
        s64 = ib.GpuCnabSolver(ib.State(prob), device=device)
        sx = ib.GpuCnabSolver(ib.State(prob), device=device, precision=prec)
        dmax, cmax, dlate = 0.0, 0.0, 0.0
        for k in range(steps):
            s64.advance_()
            sx.advance_()
            c64, cx = 2 * np.asarray(s64.total_force()), 2 * np.asarray(sx.total_force())
            d = float(np.abs(c64 - cx).max())
            dmax = max(dmax, d)
            cmax = max(cmax, float(np.abs(c64).max()))
            if 2 * k >= steps:
                dlate = max(dlate, d)
        g64, gx = s64.getstate().Gamma, sx.getstate().Gamma
        vort = float(np.linalg.norm(gx - g64) / np.linalg.norm(g64))
        if v64 is None:
            v64 = rate(s64)
        vx = rate(sx)
        out[prec] = {"steps_per_s": vx, "ratio_vs_fp64": vx / v64, "max_abs_dCD_dCL": dmax,
                     "max_abs_dCD_dCL_second_half": dlate, "max_abs_C": cmax, "vorticity_rel_l2": vort,
                     "meets_bar": bool(dmax <= 1e-4 and vort <= 1e-5)}
        del s64, sx
    out.update({"chosen_form": "mixed", "fp64_steps_per_s": v64, "ratio": out["mixed"]["ratio_vs_fp64"],
                "meets_bar": out["mixed"]["meets_bar"]})
    return out


def direct_start_run(ib, device: int, steps: int, warmup: int, npts: int = 101, products: int = 0):
    """The direct CG start alone (B assembled and inverted on the GPU every step)
    on the 512^2 x 4-level pitching plate at k = 0.55 with `npts` points (B has
    2 npts columns): `warmup` steps, then `steps` steps timed with CUDA events on
    the solver's stream, the last of them inside the NVTX range "direct_step"
    (the range a kernel-launch list or a profile selects).  With products 1 or 3
    the step is the preconditioned mode rebuilt every step, its B assembled on
    the tensor cores with that many BF16 products."""
    import torch

    s = ib.GpuCnabSolver(ib.State(ib.configs.pitching_plate(0.55, npts=npts)),
                         cg=dict(reltol=0.0, abstol=1e-10, maxiter=5000), device=device)
    if products:
        s.set_warm_start(None, mode="preconditioned", depth=1)
        s.set_rebuild_transform(products)
    else:
        s.set_warm_start(None, mode="direct", depth=1)
    for _ in range(warmup):
        s.advance_()
    stream = torch.cuda.ExternalStream(s.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    it = []
    torch.cuda.synchronize()
    l0 = s.kernel_launches()
    e0.record(stream)
    for k in range(steps):
        if k == steps - 1:
            torch.cuda.nvtx.range_push("direct_step")
        s.advance_()
        it.append(s.info().last_cg_iters)
        if k == steps - 1:
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    what = f"preconditioned CG rebuilt every step, B on the tensor cores ({products} BF16 products)" if products \
        else "direct CG start"
    return {"metric": f"moving-body steps/s, {what}", "value": 1000.0 / ms, "unit": "steps/s",
            "ms_per_step": ms, "steps": steps, "warmup": warmup, "cg_iterations_mean": float(np.mean(it)),
            "gpu_launches_per_step": (s.kernel_launches() - l0) / steps,
            "config": {"workload": f"pitching_plate_512: 512x512 cells x 4 levels, {npts}-point plate, Re 500, dt 0.002, "
                                   "k = 0.55; CG to |r| <= 1e-10", "precision": "fp64"}}


def ensemble_report(ib, device: int, pg=None, rank: int = 0, world: int = 1, seed: int = 2026, n: int = 128,
                    steps: int = 10):
    """Case-steps/s of one seeded ensemble of n independent FP32 cases (finest
    grids of {256, 384, 512} x 256 cells at h 0.01, 3 levels, seeded cylinders or
    plates, Re ~ U[50, 300], dt 0.002) stepped together (ibpm_ensemble_advance),
    against the same cases stepped one after another.  Under torchrun the cases
    are sharded over the ranks by cost (no collective on the data path); each
    rank times its shard with CUDA events on the current stream bracketing the
    call (which returns after every case's stream has finished), the slowest
    rank's time counts, and every case's C_D, C_L are gathered at the end."""
    import torch

    probs = ib.configs.ensemble_cases(n, seed=seed)
    costs = [ib.ensemble.case_cost(p) for p in probs]
    parts = ib.ensemble.shard_cases(costs, world)
    mine = parts[rank]
    red = "cuda" if pg else "cpu"
    t0 = time.perf_counter()
    solvers = [ib.GpuCnabSolver(ib.State(probs[k]), precision="fp32", device=device) for k in mine]
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0
    ens = ib.Ensemble(solvers)
    groups = ens.groups() if hasattr(ens, "groups") else None
    ens.advance_(3, fetch_forces=False)
    torch.cuda.synchronize()
    # one untimed step inside the NVTX range a kernel-launch list selects
    torch.cuda.nvtx.range_push("ensemble_step")
    ens.advance_(1, fetch_forces=False)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if pg:
        pg.barrier()
    e0.record()
    ens.advance_(steps, fetch_forces=False)
    e1.record()
    torch.cuda.synchronize()
    ms_conc = max_over_ranks(e0.elapsed_time(e1), pg, red)
    forces = ib.ensemble.gather_case_forces(n, mine, [2 * s.total_force() for s in solvers], pg, red)
    ens.close()
    # each case alone captures its own step graph on its first step: keep that out of the timed leg
    for s in solvers:
        s.advance_many(1)
    torch.cuda.synchronize()
    e0.record()
    for s in solvers:
        s.advance_many(steps)
    e1.record()
    torch.cuda.synchronize()
    ms_seq = max_over_ranks(e0.elapsed_time(e1), pg, red)
    pts = sum(costs)
    return {"workload": f"{n} seeded cases (seed {seed}): {{256, 384, 512}} x 256 cells at h 0.01, 3 levels, "
                        "cylinders D ~ U[0.5, 1.5] or plates at AoA ~ U[0, 45] deg, Re ~ U[50, 300], dt 0.002, FP32",
            "ranks": world, "cases_per_rank": [len(p) for p in parts], "batched_groups": groups,
            "setup_s": t_setup, "steps": steps, "case_steps_per_s": n * steps / (ms_conc / 1000.0),
            "grid_point_updates_per_s": pts * steps / (ms_conc / 1000.0), "ms_per_ensemble_step": ms_conc / steps,
            "sequential_case_steps_per_s": n * steps / (ms_seq / 1000.0), "speedup_vs_sequential": ms_seq / ms_conc,
            "forces_finite": bool(np.isfinite(forces).all()),
            "timing": "CUDA events on the current stream around the call, slowest rank; cases sharded by cost, "
                      "forces gathered"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    ib = load_package()
    threads = os.cpu_count() or 1
    # the GPU arm's own steps and warm-up (a CPU step of the full case takes a
    # fraction of a second on all host threads); capped so the run stays within minutes
    steps = max(1, min(args.steps, 200))
    warm = max(1, min(args.warmup, 20))
    v, used = cpu_time_oracle(ib, steps, warm, threads)
    line = {"metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus, "steps": steps, "warmup": warm,
            "ms_per_step": 1000.0 / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded vorticity noise, seed 12345)", "impl": "reference",
            "config": {"workload": WORKLOAD, "parallelism": "cpu"},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": used, "kind": "port",
                             "sample": f"{steps} steps of the full 1024^2 x 5 case after {warm} warm-up steps; "
                                       "CPU FP64 restatement of the reference (Julia is not installed); B^-1 "
                                       "setup skipped (timing only)"},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    # the pass-shape autotuner times its candidates at setup; its choices are in the JSON line
    os.environ.setdefault("IBPM_TUNE", "1")
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-chosen", action="store_true", help="skip the mixed-precision engine")
    ap.add_argument("--no-learned", action="store_true", help="skip the moving-body CG warm-start comparison")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 128-case ensemble measurement")
    ap.add_argument("--no-tensor-core", action="store_true",
                    help="skip the tensor-core B rebuild measurement")
    ap.add_argument("--ensemble-only", action="store_true",
                    help="time only the 128-case ensemble (one JSON line) and exit")
    ap.add_argument("--direct-start-only", action="store_true",
                    help="time only the moving-body direct CG start (one JSON line) and exit")
    ap.add_argument("--direct-start-points", type=int, default=101,
                    help="plate points of --direct-start-only (B has twice as many columns)")
    ap.add_argument("--rebuild-products", type=int, default=0, choices=[0, 1, 3],
                    help="--direct-start-only: assemble B on the tensor cores with 1 or 3 BF16 products "
                         "(the preconditioned mode rebuilt every step)")
    args = ap.parse_args()
    world, rank, local = dist_init()
    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.ensemble_only:
        import torch

        torch.cuda.set_device(local)
        line = ensemble_report(load_package(), local)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    if args.direct_start_only:
        ib = load_package()
        line = direct_start_run(ib, local, args.steps, args.warmup, args.direct_start_points, args.rebuild_products)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return

    import torch

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    ib = load_package()
    warm = max(3, args.warmup)
    prob = ib.configs.cylinder_re100_1024()
    st = ib.configs.seed_vorticity(ib.State(prob))
    solver = ib.GpuCnabSolver(st, device=local)
    stream = torch.cuda.ExternalStream(solver.stream_handle())
    L = prob.grid.nlevel
    nx, ny = prob.grid.base.n
    launches0 = solver.kernel_launches()

    # warm-up
    solver.advance_many(warm)
    torch.cuda.synchronize()

    # timed region: K steps with device-resident state (inputs 0.5 GB > L2, no flush needed)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    launches_a = solver.kernel_launches()
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("timed")
        ev0.record(stream)
        solver.advance_many(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    launches = solver.kernel_launches() - launches_a
    ms = max_over_ranks(ev0.elapsed_time(ev1), pg, "cuda")
    ms_step = ms / args.steps
    value = whole_job_rate(world, args.steps, ms)

    # end to end through the public API: per step, params host->device and fb device->host
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(3, min(args.steps, 20))
    e0.record(stream)
    for _ in range(e2e_steps):
        solver.advance_()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), pg, "cuda")
    e2e_value = whole_job_rate(world, e2e_steps, e2e_ms)
    h2d = 8 * 8  # StepDev: freestream (2) + grid motion (6) doubles
    d2h = 8 * 2 * prob.bodies.npanel  # fb

    # per-kernel device times: a profiled pass (CUDA events around every launch of
    # the pass kernels, eager launches) of a few steps after the timed region
    prof_steps = max(2, min(args.steps, 10))
    solver.profile(True)
    solver.advance_many(prof_steps)
    kern = {k: solver.profile_read(k) for k in ("ypass", "xpass", "nonlinear", "curl", "xtrial", "ytrial")}
    solver.profile(False)

    peak, peak_kind = read_peaks()
    # the dominant kernel: the class with the largest device time per step; its
    # achieved bandwidth is the algorithmic bytes of all its launches over their time
    names = {"ypass": "ypass_kernel (DST along y, multiply by scale/Λ, DST along y)",
             "xpass": "xpass_kernel (DST along x of row pairs, with the solves' prologues and epilogues)",
             "nonlinear": "nonlinear_kernel", "curl": "curl_kernel", "xtrial": "xpass_trial_kernel",
             "ytrial": "ypass_trial_kernel"}
    dom_key = max(kern, key=lambda k: kern[k][1])
    n_d, ms_d, b_d = kern[dom_key]
    achieved = b_d / (ms_d / 1000.0) / 1e9 if n_d else None
    traffic = NCU_TRAFFIC.get(dom_key)
    step_bytes = step_bytes_model(nx, ny, L, prob.bodies.npanel)
    n_y, ms_y, b_y = kern["ypass"]
    roofline = {"kernel": names[dom_key], "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None, "traffic": traffic,
                "traffic_source": traffic and NCU_TRAFFIC_RUN.get(dom_key),
                "peak_source": peak_kind,
                "launches_per_step": n_d / prof_steps if n_d else None,
                "algorithmic_bytes_per_launch": b_d / n_d if n_d else None,
                "launch_ms": ms_d / n_d if n_d else None,
                "kernel_ms_per_step": {k: v[1] / prof_steps for k, v in kern.items()},
                "single_level_ypass": {"achieved": (b_y / n_y) / ((ms_y / n_y) / 1000.0) / 1e9 if n_y else None,
                                       "launch_ms": ms_y / n_y if n_y else None},
                "timing": f"CUDA events around each launch during {prof_steps} profiled steps (eager launches) "
                          "after the timed region",
                "step": {"algorithmic_bytes": step_bytes, "achieved": step_bytes / (ms_step / 1000.0) / 1e9,
                         "frac": step_bytes / (ms_step / 1000.0) / 1e9 / peak, "unit": "GB/s",
                         "model": "one read + one write of each field per pass; 3 passes per 2D solve"}}

    # the mixed-precision engine on the same case, stepped to the same index
    chosen = None
    if not args.no_chosen:
        st32 = ib.configs.seed_vorticity(ib.State(prob))
        s32 = ib.GpuCnabSolver(st32, device=local, precision="mixed")
        s32.advance_many(warm)
        torch.cuda.synchronize()
        stream32 = torch.cuda.ExternalStream(s32.stream_handle())
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream32)
        s32.advance_many(args.steps)
        c1.record(stream32)
        torch.cuda.synchronize()
        ms32 = c0.elapsed_time(c1)
        s32.advance_many(st.index - st32.index)
        st64 = solver.getstate()
        st32 = s32.getstate()
        f64, f32 = solver.total_force(), s32.total_force()
        dC = float(np.abs(2 * f64 - 2 * f32).max())  # C = 2F / (U^2 D), U = D = 1
        vort = float(np.linalg.norm(st32.Gamma - st64.Gamma) / np.linalg.norm(st64.Gamma))
        v32 = world * args.steps / (ms32 / 1000.0)
        chosen = {"precision": "mixed by level: level 1 (the body's) in fp64 fields and transforms, levels 2..5 "
                               "in fp32; fp64 scans, force sums, B^-1",
                  "value": v32, "unit": "steps/s", "ms_per_step": ms32 / args.steps, "ratio_vs_fp64": v32 / value,
                  "max_abs_dCD_dCL_vs_fp64": dC, "vorticity_rel_l2_vs_fp64": vort, "compared_at_step": st.index,
                  "bar": "|dC_D|,|dC_L| <= 1e-4 and vorticity rel-L2 <= 1e-5 vs FP64",
                  "meets_bar": bool(dC <= 1e-4 and vort <= 1e-5)}

    plate32 = None if args.no_chosen else mixed_precision_plate_report(ib, local)
    learned = None if args.no_learned else warm_start_report(ib, local)
    tcore = None if args.no_tensor_core else tensor_core_rebuild_report(ib, local)
    ensemble = None if args.no_ensemble else ensemble_report(ib, local, pg, rank, world)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            v, used = cpu_time_oracle(ib, 3, 1, threads)
            v1, _ = cpu_time_oracle(ib, 1, 0, 1)
            cpu = {"value": v, "unit": "steps/s", "cores": used, "kind": "port",
                   "sample": "3 steps of the same 1024^2 x 5 case after 1 warm-up step, all host threads; "
                             "CPU FP64 restatement of the reference (Julia is not installed); B^-1 setup skipped",
                   "single_thread": {"value": v1, "unit": "steps/s", "cores": 1, "sample": "1 step, no warm-up"}}
        except Exception as e:  # the baseline is reported, not required
            cpu = {"value": None, "error": str(e)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": warm, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded vorticity noise, seed 12345)",
                "config": {"workload": WORKLOAD, "nx": nx, "ny": ny, "nlevel": L, "npanel": prob.bodies.npanel,
                           "precision": "fp64 (plain drop-in path)", "parallelism": f"replicas x{world}",
                           "l2": "working set 0.5 GB > 126 MB L2; no flush",
                           "grid_point_updates_per_s": value * L * nx * ny},
                "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "steps": e2e_steps, "api": "GpuCnabSolver.advance_ (ctypes -> ibpm_advance + ibpm_get_forces)"},
                "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk.summary(),
                "chosen_form": chosen, "chosen_form_plate_aoa30": plate32, "learned_warm_start": learned,
                "tensor_core_rebuild": tcore, "ensemble": ensemble,
                "autotune": {"table": ib._abi.tune_table(),
                             "what": "Y-pass line pairs per block chosen by timing per (GPU, transform length, "
                                     "precision, batch bucket); every choice gives the same bits"}}
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
