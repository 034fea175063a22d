#!/usr/bin/env python
"""Benchmark of the uniform-grid LLG hot path on B200: cell-steps/s of FP32 RK45.

Workload (one film per GPU): 1024x1024x1 cells of 2x2x2 nm, Ms 5.8e5 A/m,
A 1.5e-11 J/m, perpendicular Ku 8e5 J/m^3, interfacial DMI 3e-3 J/m^2,
alpha 0.3, demag on (open boundaries), seeded random initial m
(init_random), Dormand-Prince RK45 with max_err 1e-5.  A step is one
accepted RK45 step of the whole film (six field evaluations, FSAL).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun each rank advances its own film (weak scaling, no data-path
collective: films are independent); times are the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "llg-sim_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

WORKLOAD = dict(nx=1024, ny=1024, dx=2e-9, dy=2e-9, dz=2e-9, ms=5.8e5, a_ex=1.5e-11, k_u=8e5,
                easy=(0.0, 0.0, 1.0), dmi=3e-3, alpha=0.3, seed=1, max_err=1e-5, headroom=0.8, dt0=1e-13,
                dt_min=1e-18, dt_max=1e-11, b_ext=(0.0, 0.0, 0.0))
GAMMA = 1.76085963023e11
# Algorithmic HBM bytes per cell per accepted FP32 RK45 step (six evaluations):
# per evaluation m_s 12 + k_s 12 + m0 12 + spectral round trips 96 + kernel 16 = 148,
# plus 12 B per previous torque in the stage combinations, the error-norm reads
# and the accepted state: 6*148 + 240 + 60 + 12 = 1200.
BYTES_PER_CELL_STEP = 1200
METRIC = "cell-steps/s FP32 vs FP64 at 1e-4 <m>; relax wall-time learned vs plain start"
UNIT = "cell-steps/s"


def workload_desc():
    w = WORKLOAD
    return (f"{w['nx']}x{w['ny']}x1 film, {w['dx']*1e9:.0f}x{w['dy']*1e9:.0f}x{w['dz']*1e9:.0f} nm cells, "
            f"Ms {w['ms']:.2e}, A {w['a_ex']:.2e}, Ku {w['k_u']:.0e} (+z), D {w['dmi']:.0e}, alpha {w['alpha']}, "
            f"demag on, random m0 (seed {w['seed']}), RK45 max_err {w['max_err']:.0e}")


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dist_env():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), int(
        os.environ.get("LOCAL_RANK", "0"))


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons during a timed region.  NVML is read from a
    thread every 5 ms (read-only queries; a region of a few milliseconds still gets
    samples, and one sample is taken at start and at stop); without NVML,
    nvidia-smi is polled every 200 ms."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None
        self.nvml = None
        self.thread = None

    def _nvml_sample(self):
        nv, h = self.nvml
        try:
            self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
            mask = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
            for name, bit in self.REASONS:
                if mask & bit:
                    self.reasons.add(name)
        except Exception:
            pass

    def start(self):
        self.sm, self.reasons, self.smax = [], set(), None
        try:
            import threading

            import pynvml as nv

            nv.nvmlInit()
            h = None
            try:   # the CUDA device's own PCI address (CUDA and NVML number devices differently)
                import torch

                pr = torch.cuda.get_device_properties(self.dev)
                h = nv.nvmlDeviceGetHandleByPciBusId(
                    f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0")
            except Exception:
                h = nv.nvmlDeviceGetHandleByIndex(self.dev)
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.nvml = (nv, h)
            self.stop_flag = threading.Event()
            self._nvml_sample()

            def loop():
                while not self.stop_flag.wait(0.005):
                    self._nvml_sample()

            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.nvml is not None:
            self._nvml_sample()
            self.stop_flag.set()
            self.thread.join(timeout=5)
            return {"sm_mhz": float(np.median(self.sm)) if self.sm else None, "sm_max_mhz": self.smax,
                    "samples": len(self.sm), "reasons": sorted(self.reasons), "source": "nvml"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], None, set()
        names = [n for n, _ in self.REASONS]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons), "source": "nvidia-smi"}


# ---------------------------------------------------------------------------
# CPU baseline: the FP64 oracle (C++ restatement of the reference path)
# ---------------------------------------------------------------------------
CPU_VARIANTS = {
    "reference-threading": "demag FFT loops OpenMP-parallel on all threads, local terms / torques / RK "
                           "combinations serial (the reference's rayon structure, demag_fft_uniform.rs:110-133)",
    "fully-parallel": "demag FFT loops and the per-cell local-term / torque / RK-combination loops "
                      "OpenMP-parallel on all threads",
}


def cpu_host_info():
    """Threads available to this process and the CPU model."""
    try:
        aff = len(os.sched_getaffinity(0))
    except AttributeError:
        aff = os.cpu_count() or 1
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"threads": aff, "logical_cpus": os.cpu_count(), "cpu_model": model,
            "omp_proc_bind": os.environ.get("OMP_PROC_BIND", "unset"), "omp_places": os.environ.get("OMP_PLACES", "unset")}


def cpu_leg(variant, warmup_steps, max_steps, budget_s):
    """Accepted FP64 RK45 steps of the benchmark film on the host cores: the oracle with
    all threads this process may use, `variant` selecting the threading structure.
    Returns (cell-steps/s, accepted, rejected, seconds, threads)."""
    import oracle as O

    w = WORKLOAD
    threads = cpu_host_info()["threads"]
    O.set_threads(threads)
    O.set_parallel_local(variant == "fully-parallel")
    n = w["nx"] * w["ny"]
    g = O.make_grid(w["nx"], w["ny"], w["dx"], w["dy"], w["dz"])
    s = O.Solver(g, O.make_material(w["ms"], w["a_ex"], w["k_u"], w["easy"], w["dmi"], True))
    m = O.init_random(n, w["seed"])
    p = O.make_params(GAMMA, w["alpha"], w["dt0"], w["b_ext"])
    s.build_h_eff(m, w["b_ext"], 2)  # builds the cached demag operator (untimed: the reference caches it)
    sargs = (2, w["max_err"], w["headroom"], w["dt_min"], w["dt_max"])
    for _ in range(warmup_steps):
        s.step_rk45(m, p, *sargs)
    acc = rej = 0
    t0 = time.perf_counter()
    while acc < max_steps:
        _, a, _ = s.step_rk45(m, p, *sargs)
        acc += a
        rej += not a
        if acc >= 1 and time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return n * acc / el, acc, rej, el, threads


def cpu_baseline_fresh(warmup_steps, max_steps, budget_s):
    """Both CPU variants, each timed in a fresh process (no GPU context, no torch
    threads, no sampler running), so the figure does not depend on what ran before."""
    out = {}
    for variant in CPU_VARIANTS:
        cmd = [sys.executable, os.path.abspath(__file__), "--cpu-leg", variant, "--warmup", str(warmup_steps),
               "--steps", str(max_steps), "--cpu-budget", str(budget_s)]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=budget_s * 3 + 300)
        if r.returncode != 0:
            out[variant] = {"error": r.stderr.strip().splitlines()[-1:] or ["failed"]}
            continue
        out[variant] = json.loads(r.stdout.strip().splitlines()[-1])
    ref = out.get("reference-threading", {})
    par = out.get("fully-parallel", {})
    info = cpu_host_info()
    if "value" not in ref:
        return {"value": None, "unit": UNIT, "cores": info["threads"], "kind": "port", "sample": str(out)}
    return {"value": ref["value"], "unit": UNIT, "cores": ref["threads"], "kind": "port",
            "sample": f"{ref['accepted']} accepted (+{ref['rejected']} rejected) FP64 RK45 steps of the full "
                      f"{WORKLOAD['nx']}x{WORKLOAD['ny']} film after {warmup_steps} warm-up steps, oracle C++ "
                      f"restatement, {CPU_VARIANTS['reference-threading']}, fresh process",
            "fully_parallel": {"value": par.get("value"), "accepted": par.get("accepted"),
                               "note": CPU_VARIANTS["fully-parallel"]},
            "host": info}


def run_cpu_leg(args):
    value, acc, rej, el, threads = cpu_leg(args.cpu_leg, args.warmup, args.steps, args.cpu_budget)
    print(json.dumps({"value": value, "accepted": acc, "rejected": rej, "seconds": el, "threads": threads}))
    return 0


def config_dict(world):
    """The `config` object of both arms (identical keys and values)."""
    w = WORKLOAD
    n = w["nx"] * w["ny"]
    return {"workload": workload_desc(), "cells_per_gpu": n, "global_cells": n * world,
            "parallelism": f"independent films, 1 per GPU x{world}",
            "l2": "inputs larger than L2: ~190 MB per film working set (m, 7 torques, stage states, 25 MB "
                  "spectrum, 16 MB kernel) vs 126 MB L2"}


def run_reference(args):
    """The reference arm: the reference's CPU path (the oracle restatement with the
    reference's threading structure) on all host threads, same workload, same
    warm-up and step counts as the GPU arm, each step a full-film accepted step."""
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    budget = 150.0
    value, acc, rej, el, threads = cpu_leg("reference-threading", args.warmup, args.steps, budget)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": acc, "warmup": args.warmup, "ms_per_step": 1e3 * el / acc, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{acc} accepted (+{rej} rejected) FP64 RK45 steps of the full film after "
                                       f"{args.warmup} warm-up steps (bounded to ~{budget:.0f} s); oracle C++ "
                                       f"restatement (the Rust reference cannot be compiled here), "
                                       f"{CPU_VARIANTS['reference-threading']}",
                             "host": cpu_host_info()},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def make_solver(L, precision):
    w = WORKLOAD
    g = L.Grid2D(w["nx"], w["ny"], w["dx"], w["dy"], w["dz"])
    mat = L.Material(w["ms"], w["a_ex"], w["k_u"], w["easy"], w["dmi"], True)
    return L.Solver(g, mat, precision)


def params(L):
    w = WORKLOAD
    return L.LLGParams(GAMMA, w["alpha"], w["dt0"], w["b_ext"])


def batch_leg(L, torch, stream, world, rank, max_over_ranks, sum_over_ranks):
    """Mixed-size batch: 256 films (nx 64..256, ny 32..128), FP32 RK45 for 1 ns each,
    per-film dt, one engine per GPU; with N ranks the films are partitioned across
    them by transform cost (strong scaling, no collective while stepping).  Whole-
    batch cell-steps/s: the cell-steps of all ranks over the slowest rank's device time."""
    import workloads as W

    films_all, run = W.mixed_film_batch(256)
    mine = W.partition_films(films_all, world, rank)
    films = [films_all[i] for i in mine]
    b = L.Batch([f.grid(L) for f in films], [f.material(L) for f in films], L.FP32)
    b.set_stream(stream.cuda_stream)

    def reset():
        for k, i in enumerate(mine):
            f = films_all[i]
            b.set_state(k, L.init_uniform_with_noise(f.n, (1.0, 0.0, 0.0), run["noise"], 1000 + i))
        return [L.LLGParams(GAMMA, f.alpha, run["dt0"], f.b_ext) for f in films]

    ctl = (run["max_err"], run["headroom"], run["dt_min"], run["dt_max"])
    b.run_rk45(reset(), L.FULL, *ctl, n_accepted=3)   # graphs and kernels warm
    P = reset()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    acc, rej, t = b.run_rk45(P, L.FULL, *ctl, t_end=run["t_total"])
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1))
    cells = np.array([f.n for f in films], dtype=np.float64)
    cell_steps = sum_over_ranks(float((cells * acc).sum()))
    b.close()
    return {"workload": "256 films, nx in {64,96,128,192,256} x ny in {32,64,128}, 4x4x3 nm, Ms U[6e5,9e5], "
                        "A U[1e-11,1.5e-11], alpha 0.02, 0-50 mT in-plane, FP32 RK45 max_err 1e-5, 1 ns each",
            "scaling": "strong (films partitioned across ranks by transform cost)",
            "value": cell_steps / (ms * 1e-3), "unit": UNIT, "ms": ms, "films_this_rank": len(films),
            "cells_this_rank": int(cells.sum()), "accepted_mean": float(acc.mean()), "accepted_max": int(acc.max()),
            "rejected": int(rej.sum()), "t_sim_min": float(t.min())}


def flow_leg(L, torch, stream):
    """128x32 film: relax (SP4 settings) then 1 ns at 20 mT in 10 ps windows, FP32 and FP64 wall times."""
    import workloads as W

    f, rx, run = W.film_128x32_relax_then_field()
    out = {"workload": "128x32x1 film 4x4x3 nm, relax to max|m x B| 1e-4 T then 1 ns RK45 at 20 mT, <m> every "
                       "10 ps"}
    means = {}
    for prec, name in ((L.FP64, "fp64"), (L.FP32, "fp32")):
        sv = L.Solver(f.grid(L), f.material(L), prec)
        sv.set_stream(stream.cuda_stream)
        sv.set_state(f.m0)
        t0 = time.perf_counter()
        p = L.LLGParams(GAMMA, rx["alpha"], rx["dt0"], (0.0, 0.0, 0.0))
        st = L.RelaxSettings.default(**{k: v for k, v in rx.items() if k not in ("alpha", "dt0")})
        rep = sv.relax(p, L.FULL, st)
        t1 = time.perf_counter()
        p = L.LLGParams(GAMMA, run["alpha"], run["dt0"], f.b_ext)
        acc = 0
        for _ in range(int(round(run["t_total"] / run["dt_out"]))):
            a, _, _ = sv.run_rk45(p, L.FULL, run["max_err"], run["headroom"], run["dt_min"], run["dt_max"],
                                  t_end=run["dt_out"])
            acc += a
            sv.mean_m()
        t2 = time.perf_counter()
        means[name] = sv.mean_m()
        out[name] = {"relax_s": t1 - t0, "relax_steps": int(rep.accepted_steps), "run_s": t2 - t1,
                     "run_steps": int(acc), "mean_m": [float(x) for x in means[name]]}
        sv.close()
    out["mean_m_max_abs_diff"] = float(np.abs(means["fp32"] - means["fp64"]).max())
    return out


def warmstart_leg(L, torch, stream, max_over_ranks, n_films=16, size=256, torque=1e-6, fp32_torque=1e-3,
                  max_steps=60000, fp64_steps=2000, weights=None):
    """c5: holey films (0-6 holes, D U[0,2e-3], 0-30 mT), random m0, relaxed in two
    stages: the batched FP32 device relax to `fp32_torque` (near the FP32 field
    round-off floor), then the FP64 device relax from the FP32 state toward `torque`
    (1e-6 T) within `fp64_steps` accepted steps.  Arms: plain start, and the learned
    proposal (network on the tensor cores) then the same two stages.  Device-clock wall
    time per stage and arm (the FP32 -> FP64 hand-over through host memory included in
    the FP64 stage).  Per film: final max torque and FP64 energy of both arms; a learned
    film whose energy differs from the plain one by more than 1e-6 relative falls back
    to the plain start, and the fallback's cost (the plain pipeline re-run for those
    films) is added to the learned arm."""
    import workloads as W

    wpath = weights or os.path.join(ROOT, "llg-sim_b200", "weights", "warmstart_holey128.npy")
    net = L.WarmStartNet(np.load(wpath))
    films, rx = W.holey_film_batch(n_films, size, seed=77)
    m0 = []
    for i, f in enumerate(films):
        m = L.init_random(f.n, 900000 + i)
        m[f.mask == 0] = 0.0
        m0.append(m)
    s32 = dict(torque_threshold=fp32_torque, max_err=rx["max_err"], headroom=rx["headroom"], dt_min=rx["dt_min"],
               dt_max=rx["dt_max"], max_accepted_steps=max_steps)
    s64 = dict(s32, torque_threshold=torque, max_accepted_steps=fp64_steps)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def arm(idx, learned):
        fs = [films[i] for i in idx]
        grids = [f.grid(L) for f in fs]
        mats = [f.material(L) for f in fs]
        msk = [f.mask for f in fs]
        bex = [f.b_ext for f in fs]
        b32 = L.Batch(grids, mats, L.FP32, masks=msk)
        b64 = L.Batch(grids, mats, L.FP64, masks=msk)
        for b in (b32, b64):
            b.set_stream(stream.cuda_stream)
        for k, i in enumerate(idx):
            b32.set_state(k, m0[i])
        torch.cuda.synchronize()
        e0, e1, e2 = ev(), ev(), ev()
        e0.record(stream)
        if learned:
            b32.warm_start(net, bex)
        r32 = b32.relax([L.LLGParams(GAMMA, f.alpha, rx["dt0"], f.b_ext) for f in fs], L.FULL,
                        L.RelaxSettings.default(**s32))
        e1.record(stream)
        for k in range(len(fs)):
            b64.set_state(k, b32.get_state(k))
        r64 = b64.relax([L.LLGParams(GAMMA, f.alpha, rx["dt0"], f.b_ext) for f in fs], L.FULL,
                        L.RelaxSettings.default(**s64))
        e2.record(stream)
        torch.cuda.synchronize()
        t32 = max_over_ranks(e0.elapsed_time(e1)) * 1e-3
        tot = max_over_ranks(e0.elapsed_time(e2)) * 1e-3
        en32 = np.array([e.total() for e in b32.compute_energy(bex)])
        en = np.array([e.total() for e in b64.compute_energy(bex)])
        # final max |m x B| of every film in FP64 (the relax stops at its step budget
        # without a final check), after the timed region
        tq = np.empty(len(fs))
        for k, f in enumerate(fs):
            sv = L.Solver(grids[k], mats[k], L.FP64, geom_mask=msk[k])
            sv.set_state(b64.get_state(k))
            tq[k] = sv.torque_metric(L.LLGParams(GAMMA, f.alpha, rx["dt0"], f.b_ext), L.FULL, L.TORQUE_MAX)
            sv.close()
        out = {"wall_s": tot, "fp32_stage_s": t32, "fp64_stage_s": tot - t32,
               "fp32_steps_mean": float(np.mean([r.accepted_steps for r in r32])),
               "fp32_at_cap": int(sum(r.accepted_steps >= max_steps for r in r32)),
               "fp64_steps_mean": float(np.mean([r.accepted_steps for r in r64])),
               "final_torque_T": {"median": float(np.median(tq)), "max": float(tq.max())},
               "reached_torque": int((tq <= torque).sum())}
        b32.close()
        b64.close()
        return out, en, en32, tq, np.array([r.accepted_steps for r in r32])

    all_idx = list(range(n_films))
    plain, e_plain, e32_plain, t_plain, s_plain = arm(all_idx, False)
    learned, e_learn, e32_learn, t_learn, s_learn = arm(all_idx, True)
    rel = np.abs(e_learn - e_plain) / np.abs(e_plain)
    rel32 = np.abs(e32_learn - e32_plain) / np.abs(e32_plain)
    differ = [i for i in all_idx if not rel[i] <= 1e-6]
    fallback = {"films": len(differ), "wall_s": 0.0}
    if differ:
        fb = arm(differ, False)[0]
        fallback["wall_s"] = fb["wall_s"]
    net.close()
    return {"workload": f"{n_films} films {size}x{size}, 4x4x3 nm, 0-6 holes r 8-24 cells, D U[0,2e-3], 0-30 mT "
                        f"in-plane, alpha 0.5, random m0; FP32 device relax (RK23) to max|m x B| {fp32_torque:.0e} T "
                        f"(at most {max_steps} steps), then FP64 device relax toward {torque:.0e} T within "
                        f"{fp64_steps} steps",
            "weights": os.path.relpath(wpath, ROOT), "plain": plain, "learned": learned,
            "speedup_fp32_stage": plain["fp32_stage_s"] / learned["fp32_stage_s"],
            "speedup_total": plain["wall_s"] / learned["wall_s"],
            "fallback": fallback, "learned_with_fallback_s": learned["wall_s"] + fallback["wall_s"],
            "speedup_with_fallback": plain["wall_s"] / (learned["wall_s"] + fallback["wall_s"]),
            "films_same_energy_1e-6": int((rel <= 1e-6).sum()),
            "energy_rel_diff_fp64": {"median": float(np.median(rel)), "max": float(rel.max()),
                                     "learned_lower": int(((e_learn < e_plain) & (rel > 1e-6)).sum()),
                                     "learned_higher": int(((e_learn > e_plain) & (rel > 1e-6)).sum())},
            "energy_rel_diff_fp32_stage": {"median": float(np.median(rel32)), "max": float(rel32.max())},
            "films": [{"film": i, "film_cells_frac": round(float(np.mean(films[i].mask != 0)), 3), "b_ext_mT": [round(1e3 * b, 2) for b in films[i].b_ext],
                       "fp32_steps_plain": int(s_plain[i]), "fp32_steps_learned": int(s_learn[i]),
                       "final_torque_T_plain": float(t_plain[i]), "final_torque_T_learned": float(t_learn[i]),
                       "energy_J_plain": float(e_plain[i]), "energy_J_learned": float(e_learn[i]),
                       "energy_rel_diff": float(rel[i]), "fallback": bool(i in differ)} for i in all_idx]}


def amr_leg(L, reps=5):
    """The AMR consumers of the uniform FFT demag through the public API (host arrays in
    and out, wall clock per call after a warm-up call): compute_coarse_fft_demag on a
    192x192 base film refined by 7 patches (ratio 2/4/8) and the AllFft demag of the
    same film at 8x resolution (1536x1536, FP64 FFT of 3072x3072), the sizes
    coarse_fft_demag.rs:28-31 quotes (all_fft ~29 s, coarse_fft 0.3-0.5 s + 0.1 s on
    the reference's CPU).  The FP64 oracle times the coarse-FFT evaluation on the host
    (operator cached, as the reference caches it)."""
    import time
    import workloads as W

    nx = ny = 192
    dx = dy = 4e-9
    dz = 3e-9
    ms = 8.0e5
    mc, specs = W.amr_vortex_hierarchy(nx, ny, dx, dy, dz)
    patches = [L.AmrPatch(p.i0, p.j0, p.cnx, p.cny, p.ratio, p.ghost, p.m) for p in specs]
    mat = L.Material(ms, 1.3e-11, demag=True)
    out = {"workload": "vortex, 192x192 base of 4x4x3 nm cells, Ms 8e5; patches: four 38x38 ratio 2, two 19x19 "
                       "ratio 4, one 12x12 ratio 8 (ghost 2); AllFft on the 1536x1536 fine grid",
           "patch_cells": int(sum(p.pnx * p.pny for p in patches))}
    t0 = time.perf_counter()
    h = L.AmrDemag(L.Grid2D(nx, ny, dx, dy, dz))
    out["coarse_build_s"] = time.perf_counter() - t0
    h.compute(mat, mc, patches)
    t0 = time.perf_counter()
    for _ in range(reps):
        bc, bp = h.compute(mat, mc, patches)
    out["coarse_fft_ms"] = (time.perf_counter() - t0) / reps * 1e3
    h.close()
    h2 = L.AmrDemag(L.Grid2D(nx, ny, dx, dy, dz), coarsen_ratio=2)
    h2.compute(mat, mc, patches)
    t0 = time.perf_counter()
    for _ in range(reps):
        h2.compute(mat, mc, patches)
    out["coarse_fft_r2_ms"] = (time.perf_counter() - t0) / reps * 1e3
    h2.close()
    fg = L.Grid2D(8 * nx, 8 * ny, dx / 8, dy / 8, dz)
    t0 = time.perf_counter()
    op = L.DemagOp(fg)
    out["allfft_build_s"] = time.perf_counter() - t0
    mf = W.amr_fine_vortex(8 * nx, 8 * ny, dx / 8, dy / 8)
    bg = L.Grid2D(nx, ny, dx, dy, dz)
    L.allfft_demag(op, mat, mf, None, bg)
    t0 = time.perf_counter()
    for _ in range(reps):
        L.allfft_demag(op, mat, mf, None, bg)
    out["allfft_ms"] = (time.perf_counter() - t0) / reps * 1e3
    out["allfft_io_bytes"] = int(mf.nbytes * 2 + nx * ny * 24)
    # the same on resident device arrays (an AMR code that keeps its hierarchy on the GPU)
    import torch

    d_m = torch.from_numpy(np.ascontiguousarray(mf)).cuda()
    d_bf = torch.empty_like(d_m)
    d_bc = torch.empty((nx * ny, 3), dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream()
    L.allfft_demag_device(op, mat, d_m.data_ptr(), 0, bg, d_bf.data_ptr(), d_bc.data_ptr(), st.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        L.allfft_demag_device(op, mat, d_m.data_ptr(), 0, bg, d_bf.data_ptr(), d_bc.data_ptr(), st.cuda_stream)
    e1.record(st)
    torch.cuda.synchronize()
    out["allfft_device_ms"] = e0.elapsed_time(e1) / reps
    op.close()
    try:
        import oracle as O

        og = O.make_grid(nx, ny, dx, dy, dz)
        om = O.make_material(ms, 1.3e-11, demag=True)
        O.coarse_fft_demag(og, om, mc, specs)          # builds and caches the operator
        t0 = time.perf_counter()
        oc, _ = O.coarse_fft_demag(og, om, mc, specs)
        out["cpu_coarse_fft_ms"] = (time.perf_counter() - t0) * 1e3
        out["cpu_threads"] = O.get_threads()
        out["coarse_max_rel_diff_vs_fp64_oracle"] = float(np.abs(bc - oc).max() / np.abs(oc).max())
    except Exception as exc:   # the oracle library is optional where the benchmark runs
        out["cpu_coarse_fft_ms"] = f"unavailable: {exc}"
    return out


def minimize_leg(L, torch, stream, iters=300):
    """minimize_damping_only on the 1024x1024 film of the main workload (FP32 and FP64,
    random m0), a fixed number of iterations (threshold and dM stop out of reach),
    device-clock time per iteration; the FP64 oracle times three iterations on the host.
    An iteration is one field build plus the update: m in, spectrum out and back, kernel
    planes, m' out = 148 B per cell as one RK stage evaluation."""
    import time

    w = WORKLOAD
    n = w["nx"] * w["ny"]
    g = L.Grid2D(w["nx"], w["ny"], w["dx"], w["dy"], w["dz"])
    mat = L.Material(w["ms"], w["a_ex"], w["k_u"], w["easy"], w["dmi"], True)
    p = L.LLGParams(GAMMA, w["alpha"], w["dt0"], w["b_ext"])
    st = L.MinimizeSettings.default(max_iters=iters, torque_threshold=0.0, dm_stop=None, stall_iters=10 ** 9)
    pk, _ = peaks()
    out = {"workload": workload_desc().split(", RK45")[0] + f", {iters} minimiser iterations (lambda0 2e-2)"}
    for name, prec in (("fp32", L.FP32), ("fp64", L.FP64)):
        s = L.Solver(g, mat, prec)
        s.set_stream(stream.cuda_stream)
        s.set_state(L.init_random(n, w["seed"]))
        s.minimize(p, L.FULL, L.MinimizeSettings.default(max_iters=3, torque_threshold=0.0, dm_stop=None))
        s.set_state(L.init_random(n, w["seed"]))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = s.minimize(p, L.FULL, st)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        it = max(int(r.iters), 1)
        out[name] = {"iters": int(r.iters), "ms_per_iter": ms / it, "cell_iters_per_s": n * it / (ms * 1e-3),
                     "achieved_gbs": 148.0 * n * it / (ms * 1e-3) / 1e9, "final_torque": r.final_torque,
                     "final_tmean": r.final_tmean, "final_lambda": r.final_lambda}
        out[name]["hbm_frac"] = out[name]["achieved_gbs"] / pk
        s.close()
    try:
        import oracle as O

        O.set_threads(os.cpu_count() or 1)
        og = O.make_grid(w["nx"], w["ny"], w["dx"], w["dy"], w["dz"])
        osv = O.Solver(og, O.make_material(w["ms"], w["a_ex"], w["k_u"], w["easy"], w["dmi"], True))
        m = O.init_random(n, w["seed"])
        op = O.make_params(GAMMA, w["alpha"], w["dt0"], w["b_ext"])
        osv.build_h_eff(m, w["b_ext"], 2)            # kernel built outside the timed region
        t0 = time.perf_counter()
        osv.minimize(m, op, 2, O.default_minimize_settings(max_iters=3, torque_threshold=0.0, dm_stop=None))
        el = time.perf_counter() - t0
        out["cpu_oracle"] = {"ms_per_iter": el / 3 * 1e3, "cell_iters_per_s": n * 3 / el, "threads": O.get_threads()}
    except Exception as exc:   # the oracle library is optional where the benchmark runs
        out["cpu_oracle"] = f"unavailable: {exc}"
    return out


def sp4_leg(L):
    """The µMAG SP4 driver flow (st_problems/sp4.rs) end to end through the public API:
    relax, then 1 ns of RK45 under field a with 10 ps samples, table.csv and the text
    OVF snapshots written to a temporary directory; wall clock per precision."""
    import tempfile
    import time

    import sp4

    out = {"workload": "SP4a: 200x50x1 cells of 2.5x2.5x3 nm, relax to max|m x B| 1e-4 T, 1 ns RK45 at "
                       "(-24.6, 4.3, 0) mT, table every 10 ps, OVF every 100 ps"}
    for name, prec in (("fp32", L.FP32), ("fp64", L.FP64)):
        with tempfile.TemporaryDirectory() as d:
            t0 = time.perf_counter()
            r = sp4.run_sp4("a", d, precision=prec, log=lambda *a: None)
            wall = time.perf_counter() - t0
        out[name] = {"wall_s": wall, "relax_steps": int(r["relax_accepted"]), "run_steps": r["run_accepted"],
                     "run_rejected": r["run_rejected"], "crossover_t_s": r["crossover_t"],
                     "mean_m_final": [float(x) for x in r["rows"][-1][1:]], "ovf_snapshots": r["snapshots"]}
    return out


def reduce_over_ranks(dist, x, op, device):
    """x reduced over the process group (op "max" or "sum"); x itself without one."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def _r(x, nd=4):
    """Round floats for the one-line record (3-4 significant digits)."""
    if isinstance(x, float):
        return float(f"{x:.{nd}g}")
    if isinstance(x, dict):
        return {k: _r(v, nd) for k, v in x.items()}
    if isinstance(x, list):
        return [_r(v, nd) for v in x]
    return x


def compact_legs(batch, flow, warm, amr, sp4r, mini):
    """Short per-leg summaries for the bench line (the full records go to --detail)."""
    out = {}
    if batch:
        out["batch_c3"] = _r({"value": batch["value"], "ms": batch["ms"], "accepted_mean": batch["accepted_mean"],
                              "rejected": batch["rejected"]})
    if flow:
        out["flow_c1"] = _r({"fp64_relax_s": flow["fp64"]["relax_s"], "fp32_relax_s": flow["fp32"]["relax_s"],
                             "fp64_run_s": flow["fp64"]["run_s"], "fp32_run_s": flow["fp32"]["run_s"],
                             "mean_m_max_abs_diff": flow["mean_m_max_abs_diff"]})
    if warm:
        out["warm_start_c5"] = _r({k: warm[k] for k in warm if k not in ("workload", "weights", "films")})
    if amr:
        out["amr_demag"] = _r({"coarse_fft_ms": amr["coarse_fft_ms"], "allfft_ms": amr["allfft_ms"],
                               "allfft_device_ms": amr.get("allfft_device_ms"),
                               "cpu_coarse_fft_ms": amr.get("cpu_coarse_fft_ms")})
    if sp4r:
        out["sp4"] = _r({"fp32_wall_s": sp4r["fp32"]["wall_s"], "fp64_wall_s": sp4r["fp64"]["wall_s"],
                         "crossover_t_s": sp4r["fp32"]["crossover_t_s"]})
    if mini:
        out["minimize"] = _r({"fp32_ms_per_iter": mini["fp32"]["ms_per_iter"],
                              "fp64_ms_per_iter": mini["fp64"]["ms_per_iter"],
                              "fp32_hbm_frac": mini["fp32"]["hbm_frac"]})
    return out


def run_gpu(args):
    import torch

    import llg_b200 as L

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        return reduce_over_ranks(dist, x, "max", "cuda")

    def sum_over_ranks(x):
        return reduce_over_ranks(dist, x, "sum", "cuda")

    w = WORKLOAD
    n = w["nx"] * w["ny"]
    fm = L.FULL
    ctl = (w["max_err"], w["headroom"], w["dt_min"], w["dt_max"])
    m0 = L.init_random(n, w["seed"] + rank)
    stream = torch.cuda.Stream()
    s = make_solver(L, L.FP32)
    s.set_stream(stream.cuda_stream)
    s.set_state(m0)
    p = params(L)
    # warm-up (graph capture, clocks) — untimed
    s.run_rk45(p, fm, *ctl, n_accepted=args.warmup)
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = s.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier()
    e0.record(stream)
    acc, rej, t_adv = s.run_rk45(p, fm, *ctl, n_accepted=args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_local = e0.elapsed_time(e1)
    clk = clocks.stop()
    launches = s.launch_count() - launches0
    ms = max_over_ranks(ms_local)
    value = n * acc * world / (ms * 1e-3)
    step_ms = ms / acc
    peak, peak_kind = peaks()

    # per-kernel roofline of one RK45 stage (same state, CUDA events per pass).  An
    # accepted FSAL step launches the row-forward pass once (stage 2), the column
    # pass six times, the fused row pass five times (stages 2->3 .. 6->7) and the
    # row-inverse pass once (stage 7, with the error norm); the dominant kernel is
    # the one with the largest share of the step's device time.
    prof = s.profile_stage(p, fm, reps=30)
    row_plan, col_plan = s.fft_plans()
    K1 = w["nx"] + 1
    x_bytes = 3 * K1 * w["ny"] * 8
    khat_bytes = K1 * (w["ny"] + 1) * 16
    plane = 3 * n * 4
    names = ["k_row_forward", "k_column", "k_row_inverse", "k_row_fused"]
    bytes_pass = {"k_row_forward": plane * (1 + 3 + 1) + x_bytes,      # m0 + 3 torques + m_s out + X out
                  "k_column": 2 * x_bytes + khat_bytes,               # X in/out + kernel planes
                  "k_row_inverse": x_bytes + 2 * plane,               # X in + m_s in + k out
                  "k_row_fused": 2 * x_bytes + plane * (1 + 1 + 1 + 3 + 1)}   # X in/out, m_s, k_s, m0, 3 k, m_next
    per_step = {"k_row_forward": 1, "k_column": 6, "k_row_inverse": 1, "k_row_fused": 5}
    if prof[3] <= 0.0:   # no fused pass on this path: every stage runs the three passes
        per_step = {"k_row_forward": 6, "k_column": 6, "k_row_inverse": 6, "k_row_fused": 0}
    live = [k for k in names if per_step[k] > 0]
    share = {k: per_step[k] * float(prof[names.index(k)]) for k in live}
    dom = max(live, key=lambda k: share[k])
    dom_ms = float(prof[names.index(dom)])
    achieved = bytes_pass[dom] / (dom_ms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if os.path.exists(tpath):
        for line in open(tpath):
            if line.startswith(dom + " "):
                try:
                    traffic = float(line.split()[1])
                except ValueError:
                    pass
    roofline = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                "bytes_per_launch": bytes_pass[dom], "ms_per_launch": dom_ms,
                "launches_per_step": {k: per_step[k] for k in live},
                "fft_plans": {"row": row_plan, "column": col_plan},
                "per_pass_ms": {k: _r(float(prof[names.index(k)])) for k in live},
                "per_pass_frac": {k: _r(bytes_pass[k] / (float(prof[names.index(k)]) * 1e-3) / 1e9 / peak)
                                  for k in live}}
    step_ach = BYTES_PER_CELL_STEP * n * acc / (ms_local * 1e-3) / 1e9
    roofline_step = {"bound": "hbm", "achieved": step_ach, "peak": peak, "unit": "GB/s", "frac": step_ach / peak,
                     "bytes_per_cell_step": BYTES_PER_CELL_STEP, "peak_source": peak_kind}

    # end to end through the reference-facing calls with host buffers.  e2e: the
    # drop-in binding of step(&mut m, ...) (llg.rs:795): every accepted step uploads
    # the caller's AoS f64 m from pinned memory (llg_set_state), runs llg_step_rk45
    # attempts (params in, eps / accepted / dt out) and reads m back (llg_get_state).
    # e2e_resident: the state stays on the GPU between steps (set once, read once).
    e2e = e2e_res = None
    if not args.no_e2e:
        host_m = torch.from_numpy(m0.copy()).pin_memory()
        state_bytes = n * 3 * 8   # AoS f64 m; per attempt 64 B of llg_params in, 32 B of results out

        def timed(per_step_copies, k):
            s2 = make_solver(L, L.FP32)
            s2.set_stream(stream.cuda_stream)
            host_m.copy_(torch.from_numpy(m0))
            s2.set_state_ptr(host_m.data_ptr())
            p2 = params(L)
            s2.run_rk45(p2, fm, *ctl, n_accepted=args.warmup)  # graphs and clocks warm
            s2.get_state_ptr(host_m.data_ptr())
            p2 = params(L)
            torch.cuda.synchronize()
            barrier()
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            f0.record(stream)
            acc2 = calls = 0
            if not per_step_copies:
                s2.set_state_ptr(host_m.data_ptr())
            while acc2 < k:
                if per_step_copies:
                    s2.set_state_ptr(host_m.data_ptr())
                a = 0
                while not a:
                    _, a, _ = s2.step_rk45(p2, fm, *ctl)
                    calls += 1
                acc2 += 1
                if per_step_copies:
                    s2.get_state_ptr(host_m.data_ptr())
            if not per_step_copies:
                s2.get_state_ptr(host_m.data_ptr())
            f1.record(stream)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            s2.close()
            ms_e = max_over_ranks(max(f0.elapsed_time(f1), wall * 1e3))
            nsets = acc2 if per_step_copies else 1
            return {"value": n * acc2 * world / (ms_e * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": (state_bytes * nsets + 64 * calls) / acc2,
                    "d2h_bytes_per_step": (state_bytes * nsets + 32 * calls) / acc2, "steps": acc2,
                    "attempts": calls, "ms_per_step": ms_e / acc2}

        k_e2e = max(1, min(args.steps, 100))
        e2e = timed(True, k_e2e)
        e2e["path"] = ("per accepted step: llg_set_state (pinned AoS f64 m in) + llg_step_rk45 attempts + "
                       "llg_get_state (m out), as a binding of step(&mut m, ...) does")
        e2e_res = timed(False, k_e2e)
        e2e_res["path"] = "llg_set_state once + llg_step_rk45 per attempt + llg_get_state once"

    # FP32 vs FP64 at matched simulated time from the same initial state
    fp64 = None
    if not args.no_fp64:
        k64 = max(1, args.fp64_steps)
        a32 = make_solver(L, L.FP32)
        a64 = make_solver(L, L.FP64)
        for sv in (a32, a64):
            sv.set_stream(stream.cuda_stream)
            sv.set_state(m0)
        pa = params(L)
        acc32, _, t32 = a32.run_rk45(pa, fm, *ctl, n_accepted=k64)
        pb = params(L)
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        acc64, rej64, t64 = a64.run_rk45(pb, fm, *ctl, t_end=t32)
        g1.record(stream)
        torch.cuda.synchronize()
        ms64 = g0.elapsed_time(g1)
        # FP32 to the same time (its own dt sequence), compare <m>
        a32.set_state(m0)
        pa = params(L)
        a32.run_rk45(pa, fm, *ctl, t_end=t32)
        d = np.abs(a32.mean_m() - a64.mean_m()).max()
        fp64 = {"value": n * acc64 * world / (ms64 * 1e-3), "unit": UNIT, "accepted": acc64, "rejected": rej64,
                "t_sim": t64, "mean_m_max_abs_diff_vs_fp32": float(d), "tolerance": 1e-4}
        a32.close()
        a64.close()

    batch = None
    if not args.no_batch:
        batch = batch_leg(L, torch, stream, world, rank, max_over_ranks, sum_over_ranks)
    flow = None
    if not args.no_flow:
        flow = flow_leg(L, torch, stream)
    warm = None
    if not args.no_warmstart:
        warm = warmstart_leg(L, torch, stream, max_over_ranks, n_films=args.warm_films, weights=args.warm_weights)
    amr = None
    if not args.no_amr and world == 1:
        amr = amr_leg(L)
    sp4r = None
    if not args.no_sp4 and world == 1:
        sp4r = sp4_leg(L)
    mini = None
    if not args.no_minimize and world == 1:
        mini = minimize_leg(L, torch, stream)

    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline_fresh(min(args.warmup, 2), args.steps, args.cpu_budget)

    if rank == 0:
        cfg = config_dict(world)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": acc, "warmup": args.warmup,
                "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "config": cfg,
                "rejected_steps": rej, "t_sim_s": t_adv,
                "clocks": clk, "gpu_launches": launches, "roofline": roofline, "roofline_step": roofline_step,
                "cpu_baseline": cpu, "e2e": e2e, "e2e_resident": e2e_res,
                "legs": compact_legs(batch, flow, warm, amr, sp4r, mini),
                "fp64": fp64}
        if args.detail:
            with open(args.detail, "w") as fh:
                json.dump({"batch": batch, "flow": flow, "warm_start": warm, "amr_demag": amr, "sp4": sp4r,
                           "minimize": mini, "line": line}, fh, indent=1)
        print(json.dumps(line), flush=True)
    s.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--fp64-steps", type=int, default=2000)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-flow", action="store_true")
    ap.add_argument("--no-warmstart", action="store_true")
    ap.add_argument("--no-amr", action="store_true")
    ap.add_argument("--no-sp4", action="store_true")
    ap.add_argument("--no-minimize", action="store_true")
    ap.add_argument("--warm-films", type=int, default=16, help="films of the learned-warm-start leg (c5: 256)")
    ap.add_argument("--warm-weights", default=None, help="network parameters (.npy) of the warm-start leg")
    ap.add_argument("--detail", default=None, help="also write every leg's full record to this JSON file")
    ap.add_argument("--cpu-leg", default=None, choices=sorted(CPU_VARIANTS), help=argparse.SUPPRESS)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.cpu_leg:
        return run_cpu_leg(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
