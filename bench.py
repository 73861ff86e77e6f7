#!/usr/bin/env python3
"""Benchmark: PE grid-point updates/s of the split-step Pade range march on B200.

Workload (default): the deep-water Munk batch - 4096 rays, per-ray frequency
U[50,200] Hz and source depth U[50,1000] m, Munk sound speed with seeded
Gaussian perturbations (sigma 2 m/s, 1 km correlation) every 5 km, flat 5000 m
bottom, rmax 50 km, dr 25 m, dz 1 m, np 6, TL line output.  A "step" is one
complete march of that batch (self-starter + all range steps of all rays).

One grid-point update = one interior depth point of one ray advanced one range
step with all np Pade terms; the count is sum_rays nz * nr (self-starter
excluded).

value : device time of the march (CUDA events on the engine's stream), inputs
        already resident in HBM.
e2e   : the same march through the C ABI calls a user makes for a batch, with
        host buffers, every step: cr_create (validation, device Pade sets,
        tiling, device memory from the engine pool), cr_run (H2D of the batch's
        inputs, the march, D2H of the TL / CP lines into pinned host memory)
        and cr_destroy; host wall clock around the calls.  e2e_resident: cr_run
        alone on an engine created beforehand.

Other configurations (--config):
  pekeris   - Pekeris waveguide, one ray: 50 Hz, zs = zr = 50 m, 100 m water
              over a 1700 m/s bottom, rmax 10 km, dr 2 m, dz 0.25 m, np 8, TL
              line and TL grid (ndr 1, ndz 4)
  wedge     - uneven wedge batch, 10,000 rays: per-ray slope, bottom,
              frequency (log-U[25,500] Hz), rmax U[5,40] km, np U{4..8},
              dr = lambda/4, dz = lambda/8
  precision - the Munk batch at 16,384 rays with a coarse TL grid (ndr 20,
              ndz 100): TL errors of the chosen form against complex128 over
              the line and the grid, cells with TL < 100 dB
  surrogate - the learned surrogate: 200,000 training marches of seeded
              environments, an ensemble of 4 MLPs (4 layers, width 512, BF16,
              FP32 accumulation) trained by the package's kernels, 65,536
              served requests with fallback to the march above 1 dB of
              ensemble spread, march reruns of a 1 % sample as the judge;
              value = march grid-point updates the served requests stand for
              per second of serving

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--form plain|chosen|fast]
                       [--config munk|pekeris|wedge|precision|surrogate|gemm|peaks]
                       [--rays N] [--rmax M] [--seed S] [--no-chosen] [--no-cpu-baseline]
       python bench.py --config surrogate [--train N] [--infer N] [--epochs E]
       python bench.py --impl reference ...   (CPU restatement on host cores)
Multi-GPU: launch with torch.distributed.run; every rank marches its own
seeded batch of the same size (weak scaling, no collective on the data path).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "PE grid-point updates/s (1 B200) plain vs chosen form at ≤0.1 dB TL RMS error"
UNIT = "grid-point updates/s"
B_ALG = {"plain": 72.0, "chosen": 52.0, "fast": 52.0, "refined": 52.0}  # algorithmic bytes per grid-point update


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--form", choices=["plain", "chosen", "fast", "refined"], default="plain")
    ap.add_argument("--config", choices=["munk", "pekeris", "wedge", "precision", "surrogate", "gemm", "peaks"],
                    default="munk")
    ap.add_argument("--train", type=int, default=200_000, help="surrogate: training marches")
    ap.add_argument("--infer", type=int, default=65_536, help="surrogate: served requests")
    ap.add_argument("--epochs", type=int, default=60, help="surrogate: training epochs per member")
    ap.add_argument("--rays", type=int, default=0, help="rays per GPU (0: the configuration's own count)")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-chosen", action="store_true", help="skip the chosen-form comparison")
    ap.add_argument("--cpu-rays", type=int, default=0, help="rays in the CPU sample (0: one per core)")
    ap.add_argument("--rmax", type=float, default=50000.0,
                    help="march range (m); shorter values are for profiler captures only")
    ap.add_argument("--depth", type=float, default=5000.0,
                    help="water depth (m); shallower values are for profiler captures only")
    return ap.parse_args()


def max_over_ranks(pg, values, device="cuda"):
    """Element-wise maximum of per-rank timings over all ranks (the job lasts as long as its slowest rank)."""
    if pg is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def sum_over_ranks(pg, value, device="cuda"):
    """Sum of a per-rank quantity over all ranks."""
    if pg is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def whole_job_rate(updates_all_ranks, steps, t_ms):
    """Grid-point updates per second of the whole job: every rank marches its own seeded batch of the same
    number of rays (weak scaling), all of them within the slowest rank's time."""
    return updates_all_ranks * steps / (t_ms * 1e-3)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


DEFAULT_RAYS = {"munk": 4096, "pekeris": 1, "wedge": 10000, "precision": 16384}


def workload(a, rank):
    """(batch, config dict) of the selected configuration for this rank."""
    from cupyram_b200 import workloads
    n = a.rays or DEFAULT_RAYS[a.config]
    seed = a.seed + 1000 * rank
    if a.config == "pekeris":
        batch = workloads.build(*workloads.pekeris(), compute_grids=True)
        desc = ("Pekeris waveguide, one ray: 50 Hz, zs = zr = 50 m, 100 m water (1500 m/s) over a "
                "1700 m/s, 1.5 g/cm3, 0.5 dB/lambda bottom to 300 m + 10 lambda layer, rmax 10 km, "
                "dr 2 m, dz 0.25 m, np 8, ns 1, TL line + TL grid (ndr 1, ndz 4)")
        l2 = "working set < L2 (one ray); no flush: every step rewrites the same columns"
    elif a.config == "wedge":
        batch = workloads.build(*workloads.wedge_batch(n, seed=seed), compute_grids=False)
        desc = (f"uneven wedge batch, {n} rays per GPU: depth U[50,400] m -> U[50,400] m, "
                "cb U[1550,1800], rhob U[1.3,2.0], attn U[0.2,1.0], f log-U[25,500] Hz, rmax U[5,40] km, "
                "dr = lambda/4, dz = lambda/8, np U{4..8}, TL line")
        l2 = "working set > L2; no flush needed"
    else:
        grids = a.config == "precision"
        args, kw = workloads.munk_batch(n, seed=seed, rmax=a.rmax, depth=a.depth)
        if grids:
            kw.update(ndr=20, ndz=100)
        batch = workloads.build(args, kw, compute_grids=grids)
        desc = (f"Munk deep-water batch, {n} rays per GPU, per-ray f U[50,200] Hz, "
                "zs U[50,1000] m, SSP updates every 5 km (sigma 2 m/s, 1 km corr.), "
                f"{a.depth:g} m flat, rmax {a.rmax / 1000:g} km, dr 25 m, dz 1 m, np 6, zr 500 m, TL line"
                + (" + TL grid (ndr 20, ndz 100)" if grids else ""))
        l2 = "working set > L2 (column arrays ~4 GB per 1000 rays); no flush needed"
    r = batch.rays
    cfg = {"workload": desc, "config": a.config, "rays_per_gpu": int(batch.n_rays), "form": a.form,
           "seed": seed, "point_updates_per_gpu": batch.point_updates,
           "nz_range": [int(r["nz"].min()), int(r["nz"].max())],
           "steps_per_ray_range": [int(r["nr"].min()), int(r["nr"].max())],
           "np_range": [int(r["np"].min()), int(r["np"].max())], "l2": l2}
    return batch, cfg


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
        self.f.close()
        path = Path(self.f.name)
        self._summary = parse_clocks(path.read_text())
        path.unlink(missing_ok=True)

    def summary(self):
        return self._summary


def parse_clocks(text):
    """Median SM clock, max clock and active throttle reasons from nvidia-smi
    CSV rows (no header, no units) of ClockSampler.Q."""
    rows = []
    for line in text.splitlines():
        parts = [x.strip() for x in line.split(",")]
        if len(parts) < 9:
            continue
        try:
            rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
        except ValueError:
            continue
    if not rows:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
    return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": rows[0][1],
            "reasons": reasons, "samples": len(rows)}


def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


def profiled_traffic(form):
    """DRAM bytes per grid-point update of the march kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "march_traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        return float(d[form]["dram_bytes_per_point_update"])
    except (KeyError, ValueError, TypeError):
        return None


def cpu_sample(batch, n_rays, seed, mode):
    """Time the CPU restatement on a sample of the batch (one ray per core)."""
    from oracle import oracle  # the CPU restatement; test/benchmark infrastructure only
    rng = np.random.default_rng(seed)
    cores = os.cpu_count() or 1
    n = n_rays or cores
    n = max(1, min(n, batch.n_rays))
    pick = np.sort(rng.choice(batch.n_rays, size=n, replace=False))
    work = float(np.sum(batch.rays["nz"][pick].astype(np.float64) * batch.rays["nr"][pick]))
    t0 = time.perf_counter()
    ref = oracle.run(batch, mode, threads=min(cores, n), rays=pick)
    dt = time.perf_counter() - t0
    return work / dt, dt, n, min(cores, n), pick, ref


def sample_parity(batch, pick, ref, tll):
    """TL-line differences (dB) between a march's output `tll` and the oracle's
    lines `ref` of the sampled rays `pick` (same ragged layout): max and RMS
    over every output of those rays, plus the number of outputs compared."""
    r = batch.rays[pick]
    d = np.concatenate([np.abs(np.asarray(tll)[o:o + n] - ref["tll"][o:o + n])
                        for o, n in zip(r["line_off"].tolist(), r["nvr"].tolist())])
    if d.size == 0:
        return {"rays": int(len(pick)), "outputs": 0, "max_db": None, "rms_db": None}
    return {"rays": int(len(pick)), "outputs": int(d.size), "max_db": float(d.max()),
            "rms_db": float(np.sqrt(np.mean(d * d)))}


def tl_errors(tl_ref, tl):
    """Max and RMS |dTL| (dB) over cells where the FP64 reference has TL < 100 dB."""
    m = np.isfinite(tl_ref) & (tl_ref < 100.0)
    d = np.abs(np.asarray(tl)[m] - np.asarray(tl_ref)[m])
    return float(d.max()) if d.size else 0.0, float(np.sqrt(np.mean(d * d))) if d.size else 0.0


FORM_DESC = {"chosen": "complex64 factors and workspace, FP32 sweeps, FP64 term combination and field",
             "fast": "complex64 factors and workspace, FP32 inner loop (sweeps, couplings, M u and term "
                     "combination in FP32); FP64 factorisation and field",
             "refined": "the chosen form plus one iterative-refinement step per Pade term and range step: "
                        "FP64 residual, correction solved with the same complex64 factors (two passes a step)"}


def chosen_form(a, batch, out_plain, torch, world, pg, barrier, peak, form="chosen"):
    """Time a reduced-precision form on the same batch; TL errors against the plain run.
    Returns the bench record of the form and its TL line."""
    from cupyram_b200.engine import Engine
    refs = {k: out_plain[k].numpy().copy() for k in ("tll", "tlg") if k in out_plain}
    eng = Engine(batch, precision=form)
    out = alloc_pinned(batch, torch)
    for _ in range(a.warmup):
        eng.run(out)
    barrier()
    ms = []
    for _ in range(a.steps):
        eng.run(out)
        ms.append(eng.stats()["march_ms"])
    barrier()
    t = max_over_ranks(pg, [float(np.sum(ms))])[0]
    emax, erms = tl_errors(refs["tll"], out["tll"].numpy())
    errs = {"tl_err_max_db": emax, "tl_err_rms_db": erms, "tl_err_cells": "TL line, cells with TL < 100 dB"}
    if "tlg" in refs:
        gmax, grms = tl_errors(refs["tlg"], out["tlg"].numpy())
        errs.update(tl_grid_err_max_db=gmax, tl_grid_err_rms_db=grms,
                    tl_grid_cells=int(np.sum(np.isfinite(refs["tlg"]) & (refs["tlg"] < 100.0))))
    eng.close()
    tll_chosen = out["tll"].numpy().copy()
    pu = batch.point_updates
    value = whole_job_rate(sum_over_ranks(pg, pu), a.steps, t)
    per_launch_s = float(np.mean(ms)) * 1e-3
    achieved = pu * B_ALG["chosen"] / per_launch_s / 1e9
    tpp = profiled_traffic(form) if a.config == "munk" else None
    return {"form": FORM_DESC[form], "precision": form,
            "value": value, "unit": UNIT, "ms_per_step": t / a.steps, **errs,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "bytes_per_point_update": B_ALG["chosen"],
                         "traffic": (tpp * pu) if tpp else None,
                         "traffic_gbs": (tpp * pu / per_launch_s / 1e9) if tpp else None,
                         "traffic_frac": (tpp * pu / per_launch_s / 1e9 / peak) if tpp else None}}, tll_chosen


def alloc_pinned(batch, torch):
    """Pinned host output buffers of a batch (the end-to-end path's destination)."""
    out = {"tll": torch.empty(max(batch.line_len, 1), dtype=torch.float64, pin_memory=True),
           "cpl": torch.empty(max(batch.line_len, 1), dtype=torch.complex128, pin_memory=True)}
    if batch.compute_grids:
        out["tlg"] = torch.empty(max(batch.grid_len, 1), dtype=torch.float64, pin_memory=True)
        out["cpg"] = torch.empty(max(batch.grid_len, 1), dtype=torch.complex128, pin_memory=True)
    return out


def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    batch, cfg = workload(a, 0)
    vals = []
    for k in range(a.warmup + a.steps):
        v, dt, n, cores, _, _ = cpu_sample(batch, a.cpu_rays, a.seed + k, "ref")
        if k >= a.warmup:
            vals.append((v, dt))
    value = float(np.mean([v for v, _ in vals]))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": float(np.mean([dt for _, dt in vals]) * 1e3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
            "data": "synthetic", "impl": "reference", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{n} rays of the batch per step, one ray per core, full march "
                                       "each (the reference has no CPU path of its own: its kernels "
                                       "are Numba CUDA; this is the C restatement in oracle/ "
                                       "with the reference's float32/complex64 storage)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_surrogate(a):
    """The learned surrogate's pipeline on one GPU (rank 0 only under torchrun)."""
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    import torch
    torch.cuda.set_device(local)
    from cupyram_b200 import surrogate as S
    logs = []
    with ClockSampler(local) as clk:
        res = S.pipeline(n_train=a.train, n_infer=a.infer, epochs=a.epochs, seed=a.seed,
                         log=lambda m: (logs.append(m), print(m, file=sys.stderr, flush=True)))
    value = res["equivalent_updates_per_s"]
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 0,
            "ms_per_step": (res["net_seconds"] + res["fallback_march_seconds"]) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16 (network), complex128 (fallback march)",
            "data": "synthetic (seeded environments; training fields computed by the march)",
            "config": {"workload": f"learned surrogate: {a.train} training marches, {a.infer} served requests, "
                                   "ensemble of 4 MLPs 128-512-512-512-8192, TL on 128 ranges x 64 depths "
                                   "(0-20 km, 0-D0), fallback above 1 dB spread, 1 % judged by march reruns",
                       "config": "surrogate", "seed": a.seed},
            "e2e": {"value": res["equivalent_updates_per_s_wall"], "unit": UNIT,
                    "h2d_bytes_per_step": int(a.infer * S.D_IN * 2),
                    "d2h_bytes_per_step": int(a.infer * S.NZ_OUT * S.NR_OUT * 4)},
            "surrogate": res, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def measured_peak_bf16():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["bf16_tflops"]), "measured"
        except (KeyError, ValueError):
            pass
    return 1590.0, "fallback"


def run_peaks(a, iters=1 << 16):
    """FP64 and FP32 FMA throughput of the device (cr_peak_fma): the ALU roofline
    beside the HBM one.  Best of `steps` timed launches after the warm-up."""
    import ctypes
    import torch
    from cupyram_b200 import _lib
    torch.cuda.set_device(0)
    lib = _lib.load()
    res = {}
    with ClockSampler(0) as clk:
        for name, fp64 in (("fp64", 1), ("fp32", 0)):
            best = 0.0
            for _ in range(max(1, a.steps)):
                t, ms = ctypes.c_double(), ctypes.c_double()
                rc = lib.cr_peak_fma(fp64, iters, ctypes.byref(t), ctypes.byref(ms))
                if rc:
                    raise RuntimeError(f"cr_peak_fma failed with status {rc}")
                best = max(best, t.value)
            res[name] = best
    line = {"metric": "FMA throughput (2 flops per FMA)", "value": res["fp64"], "unit": "TFLOP/s", "n_gpus": 1,
            "steps": a.steps, "warmup": 1, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic (register-only FMA chains)",
            "config": {"workload": f"8 FMA chains per thread x {iters} iterations, 8 CTAs of 256 threads per SM",
                       "config": "peaks"},
            "fp64_tflops": res["fp64"], "fp32_tflops": res["fp32"], "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def run_gemm(a):
    """The surrogate's contraction on its inference shape (8192 x 8192 x 512, the last layer of a batch of
    8192 requests), tcgen05 and mma.sync kernels, TFLOP/s against the measured bf16 peak."""
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    import torch
    torch.cuda.set_device(local)
    from cupyram_b200 import surrogate as S
    M, N, K = 8192, 8192, 512
    g = torch.Generator(device="cuda").manual_seed(a.seed)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.zeros(N, device="cuda")
    out = torch.empty(M, N, device="cuda")
    flop = 2.0 * M * N * K
    peak, kind = measured_peak_bf16()
    res = {}
    for name, tc, feed in (("tcgen05 (TMA-fed)", True, ""),
                           ("tcgen05 persistent (TMA-fed, overlapped epilogue)", True, "persistent"),
                           ("tcgen05 (cp.async-fed)", True, "cp"), ("mma.sync", False, "cp")):
        os.environ["CUPYRAM_B200_GEMM"] = feed
        for _ in range(a.warmup):
            S.gemm(S.EPI_BIAS_F32, A, B, out, bias=bias, tc=tc)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(a.steps):
            S.gemm(S.EPI_BIAS_F32, A, B, out, bias=bias, tc=tc)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.steps
        res[name] = {"ms": ms, "tflops": flop / ms * 1e-9}
    assert int(S.tc_error_flag().item()) == 0
    os.environ.pop("CUPYRAM_B200_GEMM", None)
    t = res["tcgen05 (TMA-fed)"]["tflops"]
    line = {"metric": "surrogate GEMM TFLOP/s (bf16 x bf16 -> f32, 8192 x 8192 x 512)", "value": t,
            "unit": "TFLOP/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": res["tcgen05 (TMA-fed)"]["ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16", "data": "synthetic (random matrices)",
            "config": {"workload": "surrogate last-layer contraction, batch of 8192 requests", "config": "gemm",
                       "l2": "operands 16 MB (L2-resident); output 268 MB"},
            "roofline": {"bound": "tensor", "achieved": t, "peak": peak, "unit": "TFLOP/s", "frac": t / peak,
                         "peak_source": kind, "traffic": None},
            "kernels": res}
    print(json.dumps(line), flush=True)
    return 0


def main():
    a = parse()
    if a.config == "surrogate":
        return run_surrogate(a)
    if a.config == "gemm":
        return run_gemm(a)
    if a.config == "peaks":
        return run_peaks(a)
    if a.impl == "reference":
        return run_reference(a)
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        pg = dist
    from cupyram_b200.engine import Engine
    batch, cfg = workload(a, rank)
    out = alloc_pinned(batch, torch)  # pinned host output buffers for the end-to-end path

    def barrier():
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()

    # Every step is the whole C-ABI call sequence a user makes for a batch:
    # cr_create (validation, device Pade sets, tiling, device memory),
    # cr_run (upload of the host batch, march, download of the TL / CP lines
    # into pinned host buffers) and cr_destroy.  The march alone is timed on
    # the device by CUDA events inside cr_march.
    for _ in range(a.warmup):
        with Engine(batch, precision=a.form) as eng:
            eng.run(out)
    barrier()
    march_ms, e2e_ms, run_ms, create_ms, h2d_b, d2h_b, launches = [], [], [], [], 0, 0, 0
    with ClockSampler(local) as clk:
        for _ in range(a.steps):
            t0 = time.perf_counter()
            eng = Engine(batch, precision=a.form)
            t1 = time.perf_counter()
            eng.run(out)
            t2 = time.perf_counter()
            st = eng.stats()
            eng.close()
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
            run_ms.append((t2 - t1) * 1e3)
            create_ms.append((t1 - t0) * 1e3)
            march_ms.append(st["march_ms"])
            h2d_b, d2h_b = st["h2d_bytes"], st["d2h_bytes"]
            launches += st["kernel_launches"] + 1  # + the Pade launch of cr_create
    barrier()
    t_march, t_e2e, t_run = max_over_ranks(pg, [float(np.sum(march_ms)), float(np.sum(e2e_ms)),
                                                float(np.sum(run_ms))])
    pu = batch.point_updates
    pu_all = sum_over_ranks(pg, pu)
    value = whole_job_rate(pu_all, a.steps, t_march)
    e2e = whole_job_rate(pu_all, a.steps, t_e2e)
    e2e_resident = whole_job_rate(pu_all, a.steps, t_run)
    # sanity: every ray's line is finite
    tl = out["tll"].numpy()
    if not np.all(np.isfinite(tl)):
        raise RuntimeError("non-finite TL in the benchmark output")
    peak, peak_kind = measured_peak_hbm()
    reduced = {}  # form -> (bench record, TL line)
    if a.form == "plain" and not a.no_chosen:  # every rank takes part (max-over-ranks timing)
        for form in ("chosen", "fast", "refined"):
            reduced[form] = chosen_form(a, batch, out, torch, world, pg, barrier, peak, form)
    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return 0
    per_launch_s = float(np.mean(march_ms)) * 1e-3
    achieved = pu * B_ALG[a.form] / per_launch_s / 1e9
    tpp = profiled_traffic(a.form) if a.config == "munk" else None
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": t_march / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "complex128" if a.form == "plain" else "complex64",
            "data": "synthetic", "config": cfg,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "bytes_per_point_update": B_ALG[a.form],
                         "traffic": (tpp * pu) if tpp else None,
                         "traffic_gbs": (tpp * pu / per_launch_s / 1e9) if tpp else None,
                         "traffic_frac": (tpp * pu / per_launch_s / 1e9 / peak) if tpp else None},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d_b),
                    "d2h_bytes_per_step": int(d2h_b),
                    "calls": "cr_create + cr_run (upload, march, download to pinned host buffers) + cr_destroy",
                    "create_ms_per_step": float(np.mean(create_ms))},
            "e2e_resident": {"value": e2e_resident, "unit": UNIT,
                             "calls": "cr_run on an engine already created (upload, march, download)"},
            "gpu_launches": int(launches), "clocks": clk.summary(),
            "schedule": {"column_rays": int(st["column_rays"]), "column_launches": int(st["column_launches"]),
                         "queue_ctas": int(st["queue_ctas"]), "tuner_row_step_s": st["tuner_row_step_s"],
                         "tuner_updates_per_s": st["tuner_updates_per_s"], "tuner_slots": st["tuner_slots"],
                         "create_ms": st["create_ms"], "pade_ms": st["pade_ms"]}}
    for form, (rec, _) in reduced.items():
        line[form] = rec
    if world == 1 and not a.no_cpu_baseline:
        v, dt, n, cores, pick, ref = cpu_sample(batch, a.cpu_rays, a.seed, "plain")
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": f"{n} of the {batch.n_rays} rays, full march each, one ray "
                                          f"per core, {dt:.1f} s (C restatement in oracle/, FP64)"}
        # the timed sample doubles as a parity check of this very batch: the
        # march's TL lines of the sampled rays against the oracle's
        line["parity"] = {"plain_vs_oracle": dict(sample_parity(batch, pick, ref, tl), bar_max_db=1e-3),
                          "oracle": "plain complex128 C restatement, same rays, full range"}
        for form, (_, tll_form) in reduced.items():
            line["parity"][f"{form}_vs_oracle"] = dict(sample_parity(batch, pick, ref, tll_form), bar_rms_db=0.1)
    print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
