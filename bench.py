"""Benchmark: cell-updates/s of the structured SSP-RK2 step on B200.

Workload (per GPU): the 4096 x 4096 wet/dry configuration - dx = dy = 5 m, a
bed of 32 seeded Gaussians (amplitudes U[-4, 12] m, widths U[50, 500] m), a
0.5 m / 200 m hump at the centre, Manning n = 0.025, walls - advanced through
librakali.so.  One "step" is one full SSP-RK2 step of the grid.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--precision 64|32] [--one-form]

The headline line is the FP64 depth form (the reference's arithmetic); the
FP32 surface form is timed on the same handle right after and reported under
"forms" with its free-surface error against the FP64 step after 50 .. 1000
steps, beside the FP64 step's own drift under 1e-7 and 1e-15 relative
perturbations of h (the conditioning floors of this flow).  The same line
carries the CPU baseline (the oracle on every host core, 20 steps of the
full workload), the parity of the FP64 step with that oracle run
(`parity_4096`), the lake-at-rest variant over 1000 steps in both forms
(`lake_at_rest_4096`), the batched ensemble, the adjoint and the batched
FP32 forward + adjoint of 64 x 2048^2 grids (`adjoint_fp32_batched`).

N > 1 runs N independent replicas (one per rank, launched by torchrun): the
step does not exchange data between instances, so scaling is weak and no
collective sits on the data path; the ranks only meet for the barrier and
the max-over-ranks of the timed region.

Timing: W untimed steps, then K steps bracketed by CUDA events recorded on
the simulation's own stream (rkb_time_steps), max over ranks.  Each field is
16.8 M cells x 8 B = 134 MB (FP64) or 67 MB (FP32), so every step streams
more than L2 holds.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from rakali_b200 import replicas as rp  # noqa: E402  (after the path setup)

N_CELLS_SIDE = 4096
METRIC = "cell-updates/s on 1 B200: FP64 plain vs FP32, batched, fwd+adjoint, at stated err"
# algorithmic bytes per cell-update of the two fused stage kernels (FP64):
# stage 1 reads h, hu, hv, b and writes h*, hu*, hv* (7 words); stage 2 reads
# h*, hu*, hv*, b, h^n, hu^n, hv^n and writes h^{n+1}, hu^{n+1}, hv^{n+1} (10).
BYTES_STAGE1 = 7 * 8
BYTES_STAGE2 = 10 * 8
BYTES_PER_CELL_UPDATE = BYTES_STAGE1 + BYTES_STAGE2
# FP32 surface form: eta, hu, hv are 4-byte words, the bed stays 8 bytes:
# stage 1 reads 3 x 4 + 8 and writes 3 x 4 (32 B); stage 2 reads 3 x 4 + 8 +
# 3 x 4 and writes 3 x 4 (44 B): 76 B per cell-update.
BYTES_STAGE1_32 = 3 * 4 + 8 + 3 * 4
BYTES_STAGE2_32 = 3 * 4 + 8 + 3 * 4 + 3 * 4
BYTES_PER_CELL_UPDATE_32 = BYTES_STAGE1_32 + BYTES_STAGE2_32


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.is_file():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "1", "yes"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def traffic_per_launch(n_cells: int, precision: int = 64):
    """DRAM bytes per stage-2 launch from the committed ncu summary, scaled by cells."""
    p = ROOT / "profiles" / f"stage2_fp{precision}_ncu.json"
    if not p.is_file():
        return None
    d = json.loads(p.read_text())
    return d["dram_bytes_per_launch"] * n_cells / d["cells"]


# Issue capacity of a B200: 148 SMs x 4 schedulers x 1 warp instruction per
# clock at 1965 MHz, in thread instructions per second.
ISSUE_THREAD_INST_PER_S = 148 * 4 * 32 * 1965e6


def issue_bound(value: float, precision: int):
    """The instruction-issue roofline beside the HBM one: warp instructions
    per cell of the two stage kernels from the committed ncu capture, the
    cell-update rate full issue would give, and the fraction reached."""
    p = ROOT / "profiles" / f"stage2_fp{precision}_ncu.json"
    if not p.is_file():
        return None
    d = json.loads(p.read_text())
    w = d.get("warp_inst_per_cell")
    if not w:
        return None
    per_update = 32.0 * (w["stage1"] + w["stage2"])
    bound = ISSUE_THREAD_INST_PER_S / per_update
    return {"thread_inst_per_cell_update": per_update, "bound_cell_updates_per_s": bound,
            "frac": value / bound, "source": d.get("inst_source", "")}


def oracle_run(b, h, n, threads: int, steps: int):
    """The oracle (OpenMP over `threads` host threads) stepped `steps` times
    from the workload's initial state; returns (oracle, threads used, seconds)."""
    from oracle import oracle as orc
    from rakali_b200 import workloads as wl
    used = orc.set_threads(threads)
    o = orc.OracleSim.from_config(dict(nx=n, ny=n, **wl.CONFIG2_KW), bathymetry=b, initial_h=h)
    t0 = time.perf_counter()
    o.step(steps)
    return o, used, time.perf_counter() - t0


def cpu_baseline_and_parity(b, h, n, steps=20):
    """The CPU baseline on the full workload (the oracle on every host core,
    `steps` SSP-RK2 steps from the initial state) and, from the same run, the
    parity check of the FP64 step at full size: a fresh simulation stepped as
    many times on the device, compared with the oracle bit for bit (ghosts
    included)."""
    from rakali_b200 import Rakali
    from rakali_b200 import workloads as wl
    o, used, secs = oracle_run(b, h, n, os.cpu_count() or 1, steps)
    base = {"value": n * n * steps / secs, "unit": "cell-updates/s", "cores": used,
            "kind": "port",
            "sample": f"{steps} SSP-RK2 steps of the full {n}x{n} workload from its initial "
                      f"state, FP64, {used} OpenMP threads ({secs:.1f} s)"}
    s = Rakali(defer_init=True, nx=n, ny=n, **wl.CONFIG2_KW)
    s.set_bathymetry(b)
    s.set_initial_h(h)
    s.finalize()
    s.step(steps)
    diff = {}
    for name in ("h", "hu", "hv"):
        got, want = getattr(s, name), o.arrays[name]
        diff[name] = {"max_abs_diff": float(np.max(np.abs(got - want))),
                      "cells_differing": int(np.sum(got != want))}
    parity = {"workload": f"{n}x{n}, the benchmark workload, FP64", "steps": steps,
              "bit_identical": all(d["cells_differing"] == 0 for d in diff.values()),
              "time_equal": s.time == o.time, "dt_equal": s.dt == o.dt, "fields": diff,
              "tolerance": "0 (bit-identical; the required bar is 1e-12 relative)"}
    s.close()
    del o
    return base, parity


FORM_DESC = {64: "FP64 depth form (the reference's arithmetic, bit-identical to the oracle)",
             32: "FP32 surface form (FP64 bed differences, wet/dry tests and mass sums)"}


def arm_config(n: int, world: int, precision: int) -> dict:
    """The `config` of the JSON line, shared by both arms."""
    return {"workload": f"structured SSP-RK2 wet/dry step, {n}x{n} per GPU, dx=5 m, "
                        "32-Gaussian bed, 0.5 m hump, Manning 0.025, walls, " + FORM_DESC[precision],
            "cells_per_gpu": n * n, "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (every field >= 67 MB, 7+ fields per stage)"}


def run_reference(args, rank, world):
    """CPU implementation of the path (the oracle port), all host threads, on
    the benchmark workload itself (4096^2) while K + W steps take well under
    a minute; beyond that each step is a window of the workload (said in the
    line's config and sample)."""
    if rank != 0:
        return 0
    from oracle import oracle as orc
    from rakali_b200 import workloads as wl
    threads = os.cpu_count() or 1
    used = orc.set_threads(threads)
    side = N_CELLS_SIDE if args.steps + args.warmup <= 40 else 1024
    b, h = wl.config2(n=side, seed=2024)
    cfg = dict(nx=side, ny=side, **wl.CONFIG2_KW)
    o = orc.OracleSim.from_config(cfg, bathymetry=b, initial_h=h)
    o.step(args.warmup)
    t0 = time.perf_counter()
    o.step(args.steps)
    elapsed = time.perf_counter() - t0
    value = side * side * args.steps / elapsed
    if side == N_CELLS_SIDE:
        sample = (f"each step: one SSP-RK2 step of the full {side}x{side} workload, FP64, "
                  f"{used} OpenMP threads")
    else:
        sample = (f"each step: one SSP-RK2 step of a {side}x{side} window of the "
                  f"{N_CELLS_SIDE}^2 workload (same bed family), FP64, {used} OpenMP threads")
    config = arm_config(side, world, 64)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config,
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": used,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _form_numbers(sim, args, world, local_rank, dist, cells, inputs):
    """Time one arithmetic form on the current state: device time of K steps,
    per-kernel events and the end-to-end run through the public API."""
    import ctypes

    import torch

    lib = sim._lib

    def device_steps(k):
        ms = ctypes.c_double()
        rc = lib.rkb_time_steps(sim._handle, int(k), ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError(f"rkb_time_steps failed rc={rc}: {lib.rki_last_error()}")
        return ms.value

    device_steps(max(args.warmup, 3))
    rp.barrier(dist)
    torch.cuda.synchronize()
    with ClockSampler(rp.visible_gpu_index(local_rank)) as clk:
        ms = device_steps(args.steps)
    torch.cuda.synchronize()
    ms = rp.max_over_ranks(ms, dist)
    rp.barrier(dist)
    value = rp.weak_value(world, cells, args.steps, ms)

    # per-kernel device times (events between launches, same stream)
    prof = (ctypes.c_double * 5)()
    if lib.rkb_profile_steps(sim._handle, 5, prof) != 0:
        raise RuntimeError("rkb_profile_steps failed")

    # end to end through the public API with host buffers: the inputs (the
    # workload's initial h, hu, hv in host memory) go up through the setters,
    # K steps run, the result (h) comes back through its zero-copy view -
    # wall clock around all of it.  The setters send the interiors straight
    # to the device; the view brings home h alone, ghosts included.
    state = [np.asfortranarray(a) for a in inputs]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim.set_h(state[0])
    sim.set_hu(state[1])
    sim.set_hv(state[2])
    sim.step(args.steps)
    h_back = sim.h_phys
    _ = float(h_back[0, 0])
    e2e_s = rp.max_over_ranks(time.perf_counter() - t0, dist)
    n = int(round(cells ** 0.5))
    nxt = n + 2 * sim.nghost
    e2e = {"value": world * cells * args.steps / e2e_s, "unit": "cell-updates/s",
           "h2d_bytes_per_step": 3 * 8 * cells / args.steps,   # interior h, hu, hv
           "d2h_bytes_per_step": 8 * nxt * nxt / args.steps,   # h with its ghosts
           "flow": "set_h/set_hu/set_hv from host arrays, K steps, h read through its view"}
    return {"value": value, "ms": ms, "e2e": e2e, "clocks": clk.summary(),
            "stage_ms": {"bc_stage1": prof[0], "stage1": prof[1], "bc_stage2": prof[2],
                         "stage2": prof[3]},
            "launches_per_step": int(prof[4])}


def _roofline(form, precision, cells, world, tile):
    hbm, peak_kind = peaks()
    f32 = precision == 32
    b_s2 = BYTES_STAGE2_32 if f32 else BYTES_STAGE2
    b_cell = BYTES_PER_CELL_UPDATE_32 if f32 else BYTES_PER_CELL_UPDATE
    achieved = b_s2 * cells / (form["stage_ms"]["stage2"] * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "traffic": traffic_per_launch(cells, precision),
            "kernel": ("k_sweep<stage 2> (FP32 surface form: flux + update + RK2 average)"
                       if f32 else "k_stage_tma<16,15, stage 2> (TMA-staged tiles: fused flux + "
                       "update + RK2 average)" if tile == 10
                       else "k_stage<stage 2> (fused flux + update + RK2 average)"),
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
            if peak_kind == "measured" else "fallback 6650 GB/s",
            "stage_ms": form["stage_ms"], "bytes_per_cell_update": b_cell,
            "step_frac_of_hbm": b_cell * form["value"] / world / 1e9 / hbm,
            "issue": issue_bound(form["value"] / world, precision)}


def _accuracy(b, h, n, steps):
    """Free-surface error of the FP32 form against the FP64 step (which the
    parity tests hold bit-identical to the oracle) after 50 .. `steps` steps
    from the same state, beside two floors of the FP64 step against itself:
    h perturbed by 1e-7 relative noise (FP32 round-off) and by 1e-15 (FP64
    round-off).  The second floor is the error any arithmetic other than the
    reference's own would show on this flow.  Also the domain volume drift of
    each run (closed walls: the volume is conserved)."""
    from rakali_b200 import Rakali
    from rakali_b200 import workloads as wl

    marks = sorted({k for k in (50, 100, 200, 500) if k < steps} | {steps})

    def run(hh, prec, sink):
        s = Rakali(defer_init=True, nx=n, ny=n, **wl.CONFIG2_KW)
        s.set_bathymetry(b)
        s.set_initial_h(hh)
        s.finalize()
        s.set_precision(prec)
        v0 = float(np.sum(s.h_phys))
        done = 0
        for k in marks:
            s.step(k - done)
            done = k
            sink(k, s.h_phys)
        v1 = float(np.sum(s.h_phys))
        s.close()
        return (v1 - v0) / v0

    ref = {}
    drift = {"fp64": run(h, 64, lambda k, a: ref.__setitem__(k, a.copy()))}
    err32, floor7, floor15 = {}, {}, {}

    def stats(store):
        def put(k, a):
            d = a - ref[k]
            store[k] = (float(np.abs(d).max()), float(np.sqrt(np.mean(d * d))))
        return put

    drift["fp32"] = run(h, 32, stats(err32))
    rng = np.random.default_rng(17)
    noise = rng.standard_normal(h.shape)
    drift["fp64_1e-7"] = run(np.asfortranarray(h * (1.0 + 1.0e-7 * noise)), 64, stats(floor7))
    drift["fp64_1e-15"] = run(np.asfortranarray(h * (1.0 + 1.0e-15 * noise)), 64, stats(floor15))
    by = {str(k): {"max": err32[k][0], "rms": err32[k][1],
                   "fp64_floor_1e-7_max": floor7[k][0], "fp64_floor_1e-7_rms": floor7[k][1],
                   "fp64_floor_1e-15_max": floor15[k][0], "fp64_floor_1e-15_rms": floor15[k][1]}
          for k in marks}
    return {"steps": steps, "unit": "m", "max": err32[steps][0], "rms": err32[steps][1],
            "fp64_floor_max": floor15[steps][0], "fp64_floor_rms": floor15[steps][1],
            "by_steps": by, "volume_drift_rel": drift,
            "note": "free surface vs the FP64 step; floors = the FP64 step vs itself from h x "
                    "(1 + eps noise), eps = 1e-7 (FP32 round-off) and 1e-15 (FP64 round-off)"}


def _lake_at_rest(n, steps):
    """The workload's bed with a flat surface (eta = 0, emergent islands):
    after `steps` steps in each form, max |eta| over wet cells, max |hu|,
    |hv| and the domain volume drift."""
    from rakali_b200 import Rakali
    from rakali_b200 import workloads as wl
    b, h = wl.config2(n=n, seed=2024, hump=False)
    out = {"workload": f"{n}x{n}, the benchmark bed, eta = 0, no hump", "steps": steps}
    for prec in (64, 32):
        s = Rakali(defer_init=True, nx=n, ny=n, **wl.CONFIG2_KW)
        s.set_bathymetry(b)
        s.set_initial_h(h)
        s.finalize()
        s.set_precision(prec)
        s.step(steps)
        hh = s.h_phys
        wet = hh > 0
        out[f"fp{prec}"] = {
            "eta_max_abs": float(np.abs((hh + b)[wet]).max()),
            "momentum_max_abs": max(float(np.abs(s.hu_phys).max()),
                                    float(np.abs(s.hv_phys).max())),
            "state_unchanged": bool(np.array_equal(hh, h)),
            "volume_drift_rel": (float(np.sum(hh)) - float(np.sum(h))) / float(np.sum(h))}
        s.close()
    hmax = float(h.max())
    out["bound"] = {"eta_m": 1e-13, "momentum_m2_s": 1e-12 * hmax * float(np.sqrt(9.80665 * hmax)),
                    "source": "|eta| <= 1e-13 m; momentum 1e-12 H sqrt(gH) with H the deepest "
                              "water (the reference's test_c_property.F90:97-104 scaling)"}
    return out


def run_ensemble(args, world, local_rank, dist):
    """The batched ensemble: 256 members of uneven sizes (U[64, 1024] cells a
    side, planar bed -20 m -> +2 m, M2 tide at the west edge with seeded
    amplitude and phase, walls, n = 0.02), autotuned, then timed over
    `ensemble_steps` steps in each form."""
    import torch

    from rakali_b200 import workloads as wl
    from rakali_b200.ensemble import Ensemble

    torch.cuda.set_device(local_rank)
    rank = int(os.environ.get("RANK", "0"))
    t_setup = time.perf_counter()
    members = wl.ensemble_members(n_inst=args.ensemble_members, seed=rp.replica_seed(7, rank))
    sims = [wl.build_member(m) for m in members]
    cells = sum(s.nx * s.ny for s in sims)
    setup_s = time.perf_counter() - t_setup
    out = {"workload": f"{len(sims)} independent members, {cells} cells in total "
                       "(nx, ny ~ U[64, 1024], dx = 10 m, planar bed -20 -> +2 m, M2 tide "
                       "west with seeded amplitude/phase, walls, n = 0.02)",
           "members": len(sims), "cells_per_gpu": cells, "setup_s": setup_s, "forms": {}}
    for prec in (64, 32):
        with Ensemble(sims, precision=prec) as ens:
            best = ens.autotune(trial_steps=3)
            ens.step(max(args.warmup, 3))
            rp.barrier(dist)
            with ClockSampler(rp.visible_gpu_index(local_rank)) as clk:
                ms = ens.time_steps(args.ensemble_steps)
            ms = rp.max_over_ranks(ms, dist)
            # the same steps launch by launch, with events between the phases:
            # what the six launches of a step cost beyond their kernels
            phases = ens.profile_steps(20)
            kernel_sum = sum(phases[k] for k in ("bc_stage1", "stage1", "bc_stage2", "stage2"))
            graph_ms = ms / args.ensemble_steps
            out["forms"][f"fp{prec}"] = {
                "value": rp.weak_value(world, cells, args.ensemble_steps, ms),
                "unit": "cell-updates/s", "steps": args.ensemble_steps,
                "ms_per_step": graph_ms, "variant": list(ens.variant),
                "autotune_best_ms_per_step": best, "clocks": clk.summary(),
                "launches_per_step": 7 if prec == 64 else 6,  # FP64: + the step close
                "phases_ms_per_step": phases,
                "launch_overhead": {"kernel_sum_ms": kernel_sum, "graph_ms_per_step": graph_ms,
                                    "share_outside_kernels": (graph_ms - kernel_sum) / graph_ms}}
    for s in sims:
        s.close()
    return out


def run_adjoint(args):
    """Gauge-misfit gradient w.r.t. bed and Manning n at 1024^2 over 500 steps:
    device time of the forward and of forward + adjoint (sqrt(N) checkpoints
    and recomputation, and beside it every state kept in device memory),
    the production FP64 forward of the same grid, and central differences on
    random directions."""
    from rakali_b200 import Rakali
    from rakali_b200 import workloads as wl
    from rakali_b200.adjoint import GaugeMisfit

    n, steps = args.adjoint_side, args.adjoint_steps
    w = wl.adjoint_problem(n=n, steps=steps)
    p = GaugeMisfit(n, n, w["dx"], w["dx"], w["h"], w["gauges"], steps)
    b, nf = w["b"], w["n"]
    p.record_dt(b, nf)
    _, obs = p.forward(b + w["noise"], nf)
    p.set_observations(obs)
    J, _ = p.forward(b, nf)
    fwd_ms = p.last_ms
    J, gb, gn = p.gradient(b, nf)
    grad_ms = p.last_ms
    interval = p.checkpoint_interval
    # every state kept in device memory (12.7 GB here): no segment recompute
    p.set_state_budget(None)
    Jk, gbk, gnk = p.gradient(b, nf)
    kept_ms = p.last_ms
    kept = p.checkpoint_interval == 1
    same_bits = bool(Jk == J and np.array_equal(gbk, gb) and np.array_equal(gnk, gn))
    p.set_state_budget(0)  # frees them
    # the production FP64 step on the same grid and dt sequence
    sim = Rakali(defer_init=True, nx=n, ny=n, dx=w["dx"], dy=w["dx"], nghost=2, t_end=1e9,
                 cfl=0.45, manning_n=0.025)
    sim.set_bathymetry(b)
    sim.set_initial_h(w["h"])
    sim.finalize()
    import ctypes
    ms = ctypes.c_double()
    sim._lib.rkb_time_steps(sim._handle, steps, ctypes.byref(ms))
    prod_ms = ms.value
    sim.close()
    def fd_errors(prob, gb_, gn_, n_dirs, eps=1e-6):
        rng = np.random.default_rng(5)
        errs = []
        for k in range(n_dirs):
            db = wl.gaussian_bed(n, n, w["dx"], w["dx"], 3, 500 + k, base=0.0, amp=(-1.0, 1.0),
                                 width=(200.0, 1500.0))
            dn = np.asfortranarray(0.005 * rng.standard_normal((n, n)))
            Jp, _ = prob.forward(b + eps * db, nf + eps * dn)
            Jm, _ = prob.forward(b - eps * db, nf - eps * dn)
            fd = (Jp - Jm) / (2 * eps)
            ad = float(np.sum(gb_ * db) + np.sum(gn_ * dn))
            errs.append(abs(fd - ad) / max(abs(fd), 1e-300))
        return errs

    # Finite differences validate the derivative where J is smooth at the
    # scale of the step: the same problem over the first fd_steps steps.
    # Over all 500 steps J crosses limiter / wet-dry kinks densely at any
    # finite step (secant slopes scatter by 1e-3..1e-1 for eps = 1e-5..1e-10),
    # so that run is reported but is not a check.
    short = GaugeMisfit(n, n, w["dx"], w["dx"], w["h"], w["gauges"], args.adjoint_fd_steps)
    short.set_dt(p.dt[:args.adjoint_fd_steps])
    short.set_observations(obs[:args.adjoint_fd_steps])
    _, gbs, gns = short.gradient(b, nf)
    errs = fd_errors(short, gbs, gns, args.adjoint_fd)
    short.close()
    errs_full = fd_errors(p, gb, gn, 3)
    out = {"workload": f"{n}x{n}, dx = {w['dx']} m, 16-Gaussian bed, 0.5 m hump on a smooth "
                       f"surface undulation, Manning n field 0.025, walls, FP64, {steps} steps, "
                       f"{len(w['gauges'])} gauges; observations from the bed + 0.2 m smooth noise",
           "J": J, "checkpoint_interval": interval,
           "forward_ms": fwd_ms, "forward_plus_adjoint_ms": grad_ms,
           "cost_multiple_of_forward": grad_ms / fwd_ms,
           "production_forward_ms": prod_ms,
           "cost_multiple_of_production_forward": grad_ms / prod_ms,
           "kept_states": {"note": "every state U^0..U^N kept in device memory instead of "
                                   "sqrt(N) checkpoints + segment recompute "
                                   "(rkb_adjoint_set_state_budget)",
                           "used": kept, "forward_plus_adjoint_ms": kept_ms,
                           "cost_multiple_of_production_forward": kept_ms / prod_ms,
                           "same_bits_as_checkpointed": same_bits},
           "fd_check": {"steps": args.adjoint_fd_steps, "directions": len(errs), "eps": 1e-6,
                        "max_rel_err": max(errs) if errs else None,
                        "median_rel_err": float(np.median(errs)) if errs else None},
           "fd_scatter_all_steps": {"steps": steps, "directions": len(errs_full), "eps": 1e-6,
                                    "rel_err": errs_full,
                                    "note": "J is not smooth at the scale of any finite step "
                                            "over all steps; not a check"}}
    p.close()
    return out


def run_config5(args):
    """FP32 forward + FP32 adjoint of 64 independent 2048^2 gradient problems
    (the 1024^2 gradient workload's family at 2048^2, one seed per member),
    500 steps, batched: every kernel launch covers a group of members sized to
    the free device memory.  Reports throughput of the forward and of forward +
    adjoint, the cost multiple, the FP64 mass drift of the FP32 forward, and
    member 0's J and gradient against the FP64 adjoint of the same member on
    the same dt sequence and observations, beside the FP64 gradient's own
    sensitivity to a 1e-7 |b|max bed perturbation."""
    import torch

    from rakali_b200 import workloads as wl
    from rakali_b200.adjoint import GaugeMisfitBatch

    nm, n, steps = args.c5_members, args.c5_side, args.c5_steps
    dx = 10.0
    pitch = (n + 4 + 31) // 32 * 32
    per_member = 4 * pitch * (n + 4) * 240  # bytes: ~240 FP32 fields (states, tapes, checkpoints)
    free, _ = torch.cuda.mem_get_info()
    group = nm
    while group > 1 and group * per_member > 0.7 * free:
        group //= 2
    fwd_ms = grad_ms = 0.0
    drift = 0.0
    ref = None
    for g0 in range(0, nm, group):
        ms = list(range(g0, min(nm, g0 + group)))
        probs = [wl.adjoint_problem(n=n, steps=steps, dx=dx, seed=1000 + m) for m in ms]
        b = np.array([p["b"] for p in probs])
        h = np.array([p["h"] for p in probs])
        nf = np.array([p["n"] for p in probs])
        noise = np.array([p["noise"] for p in probs])
        gauges = [p["gauges"] for p in probs]
        del probs
        with GaugeMisfitBatch(len(ms), n, n, dx, dx, h, gauges, steps, precision=32) as pb:
            pb.record_dt(b, nf)
            _, obs = pb.forward(b + noise, nf)
            pb.set_observations(obs)
            J, _ = pb.forward(b, nf)
            fwd_ms += pb.last_ms
            mass = pb.mass
            drift = max(drift, float(np.max(np.abs(mass[1] - mass[0]) / mass[0])))
            _, gb, gn = pb.gradient(b, nf)
            grad_ms += pb.last_ms
            if ref is None:
                ref = dict(b=b[0], h=h[0], n=nf[0], gauges=gauges[0], dt=pb.dt[0], obs=obs[:, 0, :],
                           J=float(J[0]), gb=gb[0], gn=gn[0],
                           checkpoint_interval=pb.checkpoint_interval)
        del b, h, nf, noise, gb, gn
    cells = nm * n * n * steps
    # member 0 in FP64 on the same dt sequence and observations
    shape = (1, n, n)
    with GaugeMisfitBatch(1, n, n, dx, dx, ref["h"][None], [ref["gauges"]], steps,
                          precision=64) as p64:
        p64.set_dt(ref["dt"][None])
        p64.set_observations(ref["obs"][:, None, :])
        J64, gb64, gn64 = p64.gradient(ref["b"][None], ref["n"][None])
        rng = np.random.default_rng(9)
        pert = 1e-7 * float(np.abs(ref["b"]).max()) * rng.standard_normal(shape)
        _, gbf, gnf = p64.gradient(ref["b"][None] + pert, ref["n"][None])

    def rel(a, r):
        return float(np.linalg.norm(a - r) / np.linalg.norm(r))

    # Cells whose FP64 gradient does not move under the 1e-7 bed perturbation
    # (away from limiter / wet-dry kinks and thin films, where the gradient
    # jumps or is dominated by the 1/h of near-dry velocities): the FP32
    # arithmetic error is measured there.
    def regular(g, gf):
        return np.abs(gf - g) <= 1e-3 * np.abs(g) + 1e-9 * np.abs(g).max()

    reg_b, reg_n = regular(gb64[0], gbf[0]), regular(gn64[0], gnf[0])

    def rel_on(a, r, m):
        return float(np.linalg.norm((a - r)[m]) / np.linalg.norm(r[m]))

    dd, dd_floor = [], []
    for k in range(8):
        db = wl.gaussian_bed(n, n, dx, dx, 3, 700 + k, base=0.0, amp=(-1.0, 1.0),
                             width=(200.0, 1500.0))
        dn = wl.gaussian_bed(n, n, dx, dx, 3, 800 + k, base=0.0, amp=(-0.01, 0.01),
                             width=(200.0, 1500.0))
        d64 = float(np.sum(gb64[0] * db) + np.sum(gn64[0] * dn))
        d32 = float(np.sum(ref["gb"] * db) + np.sum(ref["gn"] * dn))
        dfl = float(np.sum(gbf[0] * db) + np.sum(gnf[0] * dn))
        dd.append(abs(d32 - d64) / abs(d64))
        dd_floor.append(abs(dfl - d64) / abs(d64))
    # The same comparison over the first steps only, where J is smooth at the
    # scale of FP32 rounding (over all 500 steps the gradient of either
    # precision moves by O(1) under the 1e-7 bed perturbation above).
    ks = min(args.c5_cmp_steps, steps)
    short = {}
    for prec in (32, 64):
        with GaugeMisfitBatch(1, n, n, dx, dx, ref["h"][None], [ref["gauges"]], ks,
                              precision=prec) as ps:
            ps.set_dt(ref["dt"][None, :ks])
            ps.set_observations(ref["obs"][:ks, None, :])
            Js, gbs, gns = ps.gradient(ref["b"][None], ref["n"][None])
            short[prec] = (float(Js[0]), gbs[0], gns[0])
            if prec == 64:
                _, gbsf, gnsf = ps.gradient(ref["b"][None] + pert, ref["n"][None])
    sd, sd_floor = [], []
    for k in range(8):
        db = wl.gaussian_bed(n, n, dx, dx, 3, 700 + k, base=0.0, amp=(-1.0, 1.0),
                             width=(200.0, 1500.0))
        dn = wl.gaussian_bed(n, n, dx, dx, 3, 800 + k, base=0.0, amp=(-0.01, 0.01),
                             width=(200.0, 1500.0))
        d64 = float(np.sum(short[64][1] * db) + np.sum(short[64][2] * dn))
        d32 = float(np.sum(short[32][1] * db) + np.sum(short[32][2] * dn))
        dfl = float(np.sum(gbsf[0] * db) + np.sum(gnsf[0] * dn))
        sd.append(abs(d32 - d64) / abs(d64))
        sd_floor.append(abs(dfl - d64) / abs(d64))
    first_steps = {
        "steps": ks,
        "J_rel_err": abs(short[32][0] - short[64][0]) / abs(short[64][0]),
        "grad_b_rel_l2": rel(short[32][1], short[64][1]),
        "grad_n_rel_l2": rel(short[32][2], short[64][2]),
        "directional_rel_err_median": float(np.median(sd)),
        "directional_rel_err_max": float(np.max(sd)),
        "fp64_floor": {"grad_b_rel_l2": rel(gbsf[0], short[64][1]),
                       "grad_n_rel_l2": rel(gnsf[0], short[64][2]),
                       "directional_rel_err_median": float(np.median(sd_floor)),
                       "directional_rel_err_max": float(np.max(sd_floor))}}
    # Frozen-slope gradients of member 0 over the whole window: the limited
    # slopes held constant, which removes the limiter's branch sensitivity.
    # Both gradients are also set against central-difference secants of the
    # FP64 J along the same directions (step eps: 1 mm of bed at the
    # directions' 1 m amplitude).
    eps = 1e-3
    frozen = {}
    secant = []
    for prec in (32, 64):
        with GaugeMisfitBatch(1, n, n, dx, dx, ref["h"][None], [ref["gauges"]], steps,
                              precision=prec) as pz:
            pz.set_dt(ref["dt"][None])
            pz.set_observations(ref["obs"][:, None, :])
            pz.set_frozen_slopes(True)
            _, gbz, gnz = pz.gradient(ref["b"][None], ref["n"][None])
            frozen[prec] = (gbz[0], gnz[0])
            if prec == 64:
                _, gbzf, gnzf = pz.gradient(ref["b"][None] + pert, ref["n"][None])
                for k in range(8):
                    db = wl.gaussian_bed(n, n, dx, dx, 3, 700 + k, base=0.0, amp=(-1.0, 1.0),
                                         width=(200.0, 1500.0))
                    dn = wl.gaussian_bed(n, n, dx, dx, 3, 800 + k, base=0.0,
                                         amp=(-0.01, 0.01), width=(200.0, 1500.0))
                    Jp, _ = pz.forward(ref["b"][None] + eps * db[None],
                                       ref["n"][None] + eps * dn[None])
                    Jm, _ = pz.forward(ref["b"][None] - eps * db[None],
                                       ref["n"][None] - eps * dn[None])
                    secant.append(float(Jp[0] - Jm[0]) / (2.0 * eps))
    fd, fd_floor, sec_frozen, sec_exact = [], [], [], []
    for k in range(8):
        db = wl.gaussian_bed(n, n, dx, dx, 3, 700 + k, base=0.0, amp=(-1.0, 1.0),
                             width=(200.0, 1500.0))
        dn = wl.gaussian_bed(n, n, dx, dx, 3, 800 + k, base=0.0, amp=(-0.01, 0.01),
                             width=(200.0, 1500.0))
        d64 = float(np.sum(frozen[64][0] * db) + np.sum(frozen[64][1] * dn))
        d32 = float(np.sum(frozen[32][0] * db) + np.sum(frozen[32][1] * dn))
        dfl = float(np.sum(gbzf[0] * db) + np.sum(gnzf[0] * dn))
        dex = float(np.sum(gb64[0] * db) + np.sum(gn64[0] * dn))
        fd.append(abs(d32 - d64) / abs(d64))
        fd_floor.append(abs(dfl - d64) / abs(d64))
        sec_frozen.append(abs(d64 - secant[k]) / abs(secant[k]))
        sec_exact.append(abs(dex - secant[k]) / abs(secant[k]))
    # the production FP32 step (surface-form sweep) on member 0's grid, for
    # the cost of the gradient in forward steps; all members take the same work
    from rakali_b200 import Rakali
    import ctypes
    psim = Rakali(defer_init=True, nx=n, ny=n, dx=dx, dy=dx, nghost=2, t_end=1e9, cfl=0.45,
                  manning_n=float(ref["n"].flat[0]))
    psim.set_bathymetry(ref["b"])
    psim.set_initial_h(ref["h"])
    psim.finalize()
    psim.set_precision(32)
    pms = ctypes.c_double()
    psim._lib.rkb_time_steps(psim._handle, 5, ctypes.byref(pms))
    if psim._lib.rkb_time_steps(psim._handle, steps, ctypes.byref(pms)) != 0:
        raise RuntimeError("production forward timing failed")
    prod_ms = pms.value * nm
    psim.close()
    frozen_slopes = {
        "steps": steps,
        "grad_b_rel_l2": rel(frozen[32][0], frozen[64][0]),
        "grad_n_rel_l2": rel(frozen[32][1], frozen[64][1]),
        "directional_rel_err_median": float(np.median(fd)),
        "directional_rel_err_max": float(np.max(fd)),
        "fp64_floor": {"grad_b_rel_l2": rel(gbzf[0], frozen[64][0]),
                       "grad_n_rel_l2": rel(gnzf[0], frozen[64][1]),
                       "directional_rel_err_median": float(np.median(fd_floor)),
                       "directional_rel_err_max": float(np.max(fd_floor))},
        "vs_fp64_secants": {"eps": eps,
                            "frozen_rel_err_median": float(np.median(sec_frozen)),
                            "frozen_rel_err_max": float(np.max(sec_frozen)),
                            "exact_rel_err_median": float(np.median(sec_exact)),
                            "exact_rel_err_max": float(np.max(sec_exact))}}
    return {
        "workload": f"{nm} members x {n}x{n}, dx = {dx} m, 16-Gaussian bed per member "
                    f"(seeds 1000..{1000 + nm - 1}), 0.5 m hump on a smooth undulation, "
                    f"Manning n field 0.025, walls, {steps} steps, 64 gauges per member; "
                    "FP32 forward + FP32 adjoint, FP64 misfit and mass sums",
        "members_per_launch": group,
        "checkpoint_interval": ref["checkpoint_interval"],
        "forward_ms": fwd_ms, "forward_plus_adjoint_ms": grad_ms,
        "forward_cell_updates_per_s": cells / (fwd_ms * 1e-3),
        "forward_plus_adjoint_cell_updates_per_s": cells / (grad_ms * 1e-3),
        "cost_multiple_of_forward": grad_ms / fwd_ms,
        "production_forward_ms": prod_ms,
        "cost_multiple_of_production_forward": grad_ms / prod_ms,
        "production_forward_note": "FP32 surface-form sweep on member 0's grid, "
                                   f"{steps} CFL steps, times {nm} members",
        "mass_drift_rel_max": drift,
        "vs_fp64_member0_first_steps": first_steps,
        "vs_fp64_member0_frozen_slopes": frozen_slopes,
        "vs_fp64_member0": {
            "J_rel_err": abs(ref["J"] - float(J64[0])) / abs(float(J64[0])),
            "grad_b_rel_l2": rel(ref["gb"], gb64[0]), "grad_n_rel_l2": rel(ref["gn"], gn64[0]),
            "directional_rel_err_median": float(np.median(dd)),
            "directional_rel_err_max": float(np.max(dd)),
            "regular_cells": {"note": "cells whose FP64 gradient moves by < 1e-3 relative under "
                                      "the 1e-7 bed perturbation",
                              "fraction_b": float(reg_b.mean()), "fraction_n": float(reg_n.mean()),
                              "grad_b_rel_l2": rel_on(ref["gb"], gb64[0], reg_b),
                              "grad_n_rel_l2": rel_on(ref["gn"], gn64[0], reg_n)},
            "fp64_floor": {"bed_noise_rel": 1e-7,
                           "grad_b_rel_l2": rel(gbf[0], gb64[0]),
                           "grad_n_rel_l2": rel(gnf[0], gn64[0]),
                           "directional_rel_err_median": float(np.median(dd_floor)),
                           "directional_rel_err_max": float(np.max(dd_floor))}},
    }


def run_b200(args, rank, world, local_rank, dist):
    import torch

    from rakali_b200 import Rakali
    from rakali_b200 import workloads as wl

    torch.cuda.set_device(local_rank)
    n = args.side
    b, h = wl.config2(n=n, seed=2024 + rank)
    sim = Rakali(defer_init=True, nx=n, ny=n, **wl.CONFIG2_KW)
    sim.set_bathymetry(b)
    sim.set_initial_h(h)
    sim.finalize()
    sim.set_tile(args.tile)
    sim.set_sweep(args.sweep_cols, args.sweep_rows)
    cells = n * n

    # the headline form first, then the other one on the same handle
    head = args.precision
    other = 32 if head == 64 else 64
    forms = {}
    for prec in (head, other) if args.both_forms else (head,):
        sim.set_precision(prec)
        # the inputs of the end-to-end leg: the initial state in ordinary
        # (written, so resident) host arrays
        zeros = np.full(h.shape, 0.0, order="F")
        forms[prec] = _form_numbers(sim, args, world, local_rank, dist, cells,
                                    (h, zeros, zeros.copy(order="F")))
        forms[prec]["roofline"] = _roofline(forms[prec], prec, cells, world, args.tile)
    sim.close()
    ens = run_ensemble(args, world, local_rank, dist) if args.ensemble_steps > 0 else None
    err = lake = None
    if args.both_forms and rank == 0 and not args.no_accuracy:
        err = _accuracy(b, h, n, args.accuracy_steps)
        lake = _lake_at_rest(n, args.accuracy_steps)
    if rank != 0:
        return 0

    f = forms[head]
    desc = FORM_DESC
    line = {
        "metric": METRIC, "value": f["value"], "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": f["ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if head == 32 else "f64", "data": "synthetic",
        "config": arm_config(n, world, head),
        "e2e": f["e2e"],
        "gpu_launches": f["launches_per_step"] * args.steps,
        "roofline": f["roofline"],
        "clocks": f["clocks"],
    }
    if len(forms) > 1:
        line["forms"] = {}
        for prec, fm in forms.items():
            entry = {"dtype": "f32" if prec == 32 else "f64", "form": desc[prec],
                     "value": fm["value"], "ms_per_step": fm["ms"] / args.steps,
                     "e2e": fm["e2e"]["value"], "roofline_frac": fm["roofline"]["frac"],
                     "roofline_achieved_gbs": fm["roofline"]["achieved"],
                     "stage_ms": fm["stage_ms"], "clocks": fm["clocks"]}
            if prec == 32 and err is not None:
                entry["error_vs_fp64"] = err
            line["forms"][f"fp{prec}"] = entry
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"], line["parity_4096"] = cpu_baseline_and_parity(b, h, n)
    if lake is not None:
        line["lake_at_rest_4096"] = lake
    if args.ensemble_steps > 0:
        line["ensemble"] = ens
    if world == 1 and args.adjoint_steps > 0:
        line["adjoint"] = run_adjoint(args)
    if world == 1 and args.config5:
        line["adjoint_fp32_batched"] = run_config5(args)
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tile", type=int, default=10,
                    help="stage-kernel variant (rkb_set_tile): 0-3 shared-memory tiles "
                         "32x8, 32x16, 64x4, 16x16, "
                         "4/5 marching strips of 64/32 rows, 6/7 tiles 32x8 / 32x12 with two "
                         "extra warps, 8 tiles 16x15, 9 tiles 32x7 with one extra warp, 10 16x15 "
                         "tiles loaded by TMA (the default, the fastest measured)")
    ap.add_argument("--precision", type=int, choices=(32, 64), default=64,
                    help="headline form: 64 = FP64 depth form (reference arithmetic), "
                         "32 = FP32 surface form")
    ap.add_argument("--one-form", dest="both_forms", action="store_false",
                    help="time only the headline form (default: both, the other under 'forms')")
    ap.add_argument("--ensemble-steps", type=int, default=2000,
                    help="steps of the batched 256-member ensemble run after the single-grid "
                         "forms (0 skips it)")
    ap.add_argument("--ensemble-members", type=int, default=256)
    ap.add_argument("--adjoint-steps", type=int, default=500,
                    help="steps of the gauge-misfit gradient run (0 skips it)")
    ap.add_argument("--adjoint-side", type=int, default=1024)
    ap.add_argument("--adjoint-fd", type=int, default=20,
                    help="random directions of the finite-difference check")
    ap.add_argument("--adjoint-fd-steps", type=int, default=100,
                    help="steps of the finite-difference check (the gradient's first steps)")
    ap.add_argument("--no-config5", dest="config5", action="store_false",
                    help="skip the batched FP32 forward + adjoint (64 x 2048^2, 500 steps; "
                         "about a minute, run by default on one GPU)")
    ap.add_argument("--c5-members", type=int, default=64)
    ap.add_argument("--c5-side", type=int, default=2048)
    ap.add_argument("--c5-steps", type=int, default=500)
    ap.add_argument("--c5-cmp-steps", type=int, default=50,
                    help="steps of the FP32-vs-FP64 gradient comparison on member 0")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the FP32-vs-FP64 error and lake-at-rest measurements")
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="steps of the FP32-vs-FP64 error and lake-at-rest runs")
    ap.add_argument("--sweep-cols", type=int, choices=(0, 2, 4), default=0,
                    help="FP32 form: columns per lane of the sweep kernel (0 = default)")
    ap.add_argument("--sweep-rows", type=int, default=0,
                    help="FP32 form: rows per warp sweep (0 = automatic)")
    ap.add_argument("--side", type=int, default=N_CELLS_SIDE,
                    help="grid side (smaller sides are for profiler captures only)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1 and args.impl == "b200":
        import datetime

        import torch
        import torch.distributed as td
        torch.cuda.set_device(local_rank)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = td
    try:
        if args.impl == "reference":
            return run_reference(args, rank, world)
        return run_b200(args, rank, world, local_rank, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
