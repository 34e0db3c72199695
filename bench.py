"""Benchmark of the B200 finite-rate chemistry path; prints ONE JSON line (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl tiger|reference]

Workloads (seeded synthetic states, built like the reference's init_flow tool; the GRI-Mech
3.0 workloads run the reference's 36-species / 422-slot grimech30F stand-in):

  gri-surrogate    (default) one chemistry substep of 2,097,152 cells (a 128^3 grid) through
                   the learned surrogate with fallback to the implicit solve: smooth seeded
                   mixture-fraction field, CH4 / air at 300 K, progress c ~ Beta(2,2) mapped to
                   T in [300, 2400] K, minor species log-uniform in [1e-10, 1e-3], per-cell dt
                   log-uniform in [1e-7, 1e-5] s, P = 1 atm. The plain implicit GPU solve of the
                   same cells (a strided subsample) is timed beside it and is the accuracy
                   reference (max relative T error, max |dY| / max Y).
  gri-substep      the plain implicit substep (BDF/Newton, persistent work-stealing kernel in a
                   CUDA graph, FP64 LU) of the same 2,097,152-cell batch.
  gri-substep-mixed the same with the rate-constant exponentials on the FP32 unit (precision split).
  h2-substep       the plain implicit substep of the hydrogen mechanism on 32^3 cells, dt = 1e-6 s.
  gri-rates        production-rate evaluation only (finitechem_compute_rhs + PRODRATES),
                   128^3 cells, FP64.
  gri-rates-mixed  the same in mixed precision (FP32 log-space rates, FP64 reverse exponents).
  gri-transport    the mixture transport properties around the substep (finitechem_viscosity +
                   finitechem_diffusivity fused: Wilke viscosity, lambda/Cp per species) of the
                   128^3 rate-evaluation states (Y, T), FP64.
  gri-density      the equation of state (finitechem_density + finitechem_W) of the same cells.
  dme-sweep        the DME39 mechanism on a 256x192x192 temporal mixing layer (DME at 400 K above air
                   at 300 K, tanh mixture-fraction profile plus seeded Fourier perturbations of
                   amplitude 0.1, seeded burning fraction), 100 consecutive substeps of dt = 2e-6 s
                   with the state resident on the device, through the surrogate with fallback;
                   reports the hit rate, the fallback cost and the p50/p99 substep latency, and the
                   accuracy after all substeps against the plain solve of a strided subsample.

A step is one pass of the hot path over the whole batch, starting every time from the same
initial state (restored outside the timed interval). `value` is device-timed with CUDA events
on the library's stream, inputs resident in HBM (every batch is larger than the 126 MB L2);
`e2e` is the same metric through the C-ABI with pinned host buffers, host<->device copies
inside the timed region. Multi-GPU: every rank owns its own batch (cells are independent, no
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

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

import numpy as np  # noqa: E402

P_ATM = 101325.0
MODELS = os.path.join(REPO, "tiger_nga_b200", "models")
WORKLOADS = {
    "gri-surrogate": {"kind": "surrogate", "mech": "grimech30", "side": 128, "precision": "fp64",
                      "metric": "GRI-3.0 substep cells/s: surrogate+fallback vs plain GPU at ≤1% ΔT error",
                      "desc": "GRI-Mech 3.0 stand-in (36 sp) substep, 128^3 cells, per-cell dt 1e-7..1e-5 s, "
                              "surrogate (tcgen05 BF16 MLP) + implicit fallback", "steps": 5, "ref_sample": 2048},
    "dme-sweep": {"kind": "sweep", "mech": "dme39", "shape": (256, 192, 192), "precision": "fp64",
                  "metric": "DME39 mixing-layer sweep cell-substeps/s (surrogate+fallback, 100 substeps resident)",
                  "desc": "DME39 temporal mixing layer 256x192x192, dt = 2e-6 s, 100 consecutive substeps on the "
                          "device through the surrogate with implicit fallback", "steps": 100, "ref_sample": 2048,
                  "weights": "dme39.tngs"},
    "gri-substep": {"kind": "substep", "mech": "grimech30", "side": 128, "precision": "fp64",
                    "metric": "GRI-3.0 (36-sp stand-in) implicit substep cells/s",
                    "desc": "GRI-Mech 3.0 stand-in (36 sp) implicit substep, 128^3 cells, per-cell dt 1e-7..1e-5 s",
                    "steps": 1, "ref_sample": 2048},
    "gri-substep-mixed": {"kind": "substep", "mech": "grimech30", "side": 128, "precision": "mixed",
                          "metric": "GRI-3.0 (36-sp stand-in) implicit substep cells/s",
                          "desc": "GRI-Mech 3.0 stand-in implicit substep, 128^3 cells, per-cell dt 1e-7..1e-5 s, "
                                  "rate-constant exponentials in FP32 (exponents, LU, Newton in FP64)",
                          "steps": 1, "ref_sample": 2048},
    "h2-substep": {"kind": "substep", "mech": "hydrogen", "side": 32, "precision": "fp64",
                   "metric": "H2 implicit substep cells/s",
                   "desc": "hydrogen (9 sp) implicit substep, 32^3 cells, dt = 1e-6 s", "steps": 20,
                   "ref_sample": 16384},
    "gri-rates": {"kind": "rates", "mech": "grimech30", "side": 128, "precision": "fp64",
                  "metric": "GRI-3.0 (36-sp stand-in) rate evaluation cells/s",
                  "desc": "GRI-Mech 3.0 stand-in (36 sp, 422 slots) rates, 128^3 cells, FP64", "steps": 400,
                  "ref_sample": 131072},
    "gri-rates-mixed": {"kind": "rates", "mech": "grimech30", "side": 128, "precision": "mixed",
                        "metric": "GRI-3.0 (36-sp stand-in) rate evaluation cells/s",
                        "desc": "GRI-Mech 3.0 stand-in (36 sp, 422 slots) rates, 128^3 cells, mixed FP32/FP64",
                        "steps": 400, "ref_sample": 131072},
    "gri-transport": {"kind": "props", "what": "transport", "mech": "grimech30", "side": 128, "precision": "fp64",
                      "metric": "GRI-3.0 (36-sp stand-in) mixture transport properties cells/s",
                      "desc": "finitechem_viscosity + finitechem_diffusivity in one pass (Wilke viscosity, "
                              "conductivity, lambda/Cp per species), 128^3 cells, FP64", "steps": 200,
                      "ref_sample": 2048},
    "gri-density": {"kind": "props", "what": "density", "mech": "grimech30", "side": 128, "precision": "fp64",
                    "metric": "GRI-3.0 (36-sp stand-in) density (equation of state) cells/s",
                    "desc": "finitechem_density + finitechem_W, 128^3 cells, FP64", "steps": 400,
                    "ref_sample": 262144},
}
# kernels of this library launched per step (counted from the host code of each path)
# surrogate step: judge-sample gather, 2 ensemble inferences, post-processing, fallback gather,
# list fill, solver graph (counter reset + solver), statistics, fallback scatter, judge compare
LAUNCHES = {"rates": 1, "substep": 3, "surrogate": 11, "sweep": 11, "props": 1}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", self.gpu_id], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def read_profile_value(profile: str, key: str):
    """A number recorded in a committed ncu summary (line '<key>: X')."""
    path = os.path.join(REPO, "profiles", profile)
    if not os.path.exists(path):
        return None
    for ln in open(path):
        if ln.startswith(key + ":"):
            return float(ln.split(":", 1)[1])
    return None


def make_state(wl, rank):
    """Seeded host state (N+1, n) and per-cell dt (or a scalar) of a workload."""
    from tiger_nga_b200 import states
    from tiger_nga_b200.mechanism import load

    mech = load(wl["mech"])
    seed = 20261204 + rank
    if wl["kind"] == "sweep":
        sol, _ = states.mixing_layer(mech, shape=wl["shape"], seed=20261205 + rank)
        return sol, 2e-6
    n = wl["side"] ** 3
    if wl["mech"] == "hydrogen":
        sol, _ = states.h2_cube(mech, wl["side"], seed)
        return sol, 1e-6
    if wl["kind"] == "rates":
        sol, _ = states.chem_state(mech, n, seed, "CH4", grid=(wl["side"],) * 3)
        return sol, None
    if wl["kind"] == "props":
        # the solver's scalars [Y_1..Y_N, T] of the rate-evaluation states
        sol, _ = states.chem_state(mech, n, seed, "CH4", grid=(wl["side"],) * 3)
        rho = sol[:mech.ns].sum(0)
        return np.ascontiguousarray(sol / rho), None
    from tiger_nga_b200.train_surrogate import state_batch

    return state_batch(wl["mech"], n, seed, side=wl["side"])


# ---- host-core baselines (the oracle / transliterated reference; never the product path) ----
def cpu_rates_runner(mech):
    """The reference's own rate arithmetic on the host cores: the transliterated Fortran
    (oracle/_ref) when it was built, else the table-driven oracle port."""
    from oracle.oracle import REF_LIB, Oracle, Reference

    if os.path.exists(REF_LIB):
        return "reference", Reference(mech)
    return "port", Oracle(mech)


def cpu_step(wl, impl, sol, dts, lo, m, nthreads, stride=1):
    """One bounded sample of the workload on the host cores: cells lo, lo + stride, ... (m of
    them, wrapping). With stride = ncells / m the sample spans the whole batch, so that it sees
    the batch's mix of easy and stiff cells. Returns (cells, seconds of the compute call);
    gathering the sample is not timed."""
    n = sol.shape[1]
    idx = (lo + stride * np.arange(m)) % n
    sub = np.ascontiguousarray(sol[:, idx])
    d = None if dts is None or np.ndim(dts) == 0 else np.ascontiguousarray(dts[idx])
    y, t = (np.ascontiguousarray(sub[:-1]), np.ascontiguousarray(sub[-1])) if wl["kind"] == "props" else (None, None)
    t0 = time.perf_counter()
    if wl["kind"] == "rates":
        impl.rhs_batch(sub, P_ATM, nthreads)
    elif wl["kind"] == "props":
        what = ("visc", "diff") if wl["what"] == "transport" else ("wmix", "rho")
        impl.props_batch(y, t, p_thermo=P_ATM, what=what, nthreads=nthreads)
    else:
        impl.substep_batch(sub, dts if d is None else d, P_ATM, nthreads=nthreads)
    return m, time.perf_counter() - t0


def cpu_impl(wl):
    if wl["kind"] in ("rates", "props"):
        return cpu_rates_runner(wl["mech"])
    from oracle.oracle import Oracle

    return "port", Oracle(wl["mech"])


def time_cpu(wl, sol, dts, seconds: float, nthreads: int):
    kind, impl = cpu_impl(wl)
    m = min(wl["ref_sample"], sol.shape[1])
    stride = max(1, sol.shape[1] // m)
    cpu_step(wl, impl, sol, dts, 0, min(m, 256), nthreads, stride)  # warm-up
    done, el, i = 0, 0.0, 0
    while el < seconds:
        c, s = cpu_step(wl, impl, sol, dts, (1 + i * 7919) % stride, m, nthreads, stride)
        done, el, i = done + c, el + s, i + 1
    return kind, done / el, done, el


def cpu_what(wl, kind):
    src = "transliterated reference Fortran" if kind == "reference" else "oracle port"
    if wl["kind"] == "rates":
        return f"rate evaluation ({src})"
    if wl["kind"] == "props":
        r = "finitechem_viscosity + finitechem_diffusivity" if wl["what"] == "transport" else "finitechem_density"
        return f"{r} ({'the reference routines restated over its transliterated getters' if kind == 'reference' else src})"
    return "implicit BDF/Newton substep (oracle port: the reference's CVODE is not buildable here)"


def reference_arm(args, wl, config, metric, unit):
    """The reference's CPU implementation of the path on the host cores (rank 0 only)."""
    sol, dts = make_state(wl, 0)
    nthreads = os.cpu_count() or 1
    kind, impl = cpu_impl(wl)
    m = min(wl["ref_sample"], sol.shape[1])
    stride = max(1, sol.shape[1] // m)
    for w in range(args.warmup):
        cpu_step(wl, impl, sol, dts, (104729 * (w + 1)) % stride, m, nthreads, stride)
    el = sum(cpu_step(wl, impl, sol, dts, (1 + k * 7919) % stride, m, nthreads, stride)[1] for k in range(args.steps))
    val = m * args.steps / el
    what = cpu_what(wl, kind)
    sample = (f"{m} cells of the workload per step (every {stride}th cell of the batch, a new offset per step), "
              f"{what}, OpenMP over cells")
    print(json.dumps({"impl": "reference", "metric": metric, "value": val, "unit": unit, "n_gpus": args.gpus,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                      "data": "synthetic", "config": config,
                      "cpu_baseline": {"value": val, "unit": unit, "cores": nthreads, "kind": kind, "sample": sample},
                      "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        pk = json.load(open(path))
        return pk["hbm_gbs"], pk.get("bf16_tflops"), "measured"
    return 6650.0, 1590.0, "fallback"


def max_over_ranks(pg, dev, v):
    if not pg:
        return v
    import torch

    t = torch.tensor([v], device=dev, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def solver_flops(mech, st):
    """FP64 flops of the implicit solve that can be counted exactly from its statistics: one
    reference-formulation RHS per Newton iteration, the LU factorisation (2/3 n^3) per Jacobian
    and the two triangular solves (2 n^2) per Newton iteration. Jacobian assembly, error tests
    and the Nordsieck history are left out, so this is a lower bound of the work done."""
    from tiger_nga_b200.workcount import rhs_work

    nv = mech.ns + 1
    rf = rhs_work(mech)["flops"]
    return st["newton_iters"] * (rf + 2 * nv * nv) + st["jacobians"] * (2.0 / 3.0) * nv ** 3


def run_sweep(args, wl, config, metric, unit, ws, rank, local, dev, pg):
    """K consecutive substeps of a resident state through the surrogate with fallback."""
    import torch

    from tiger_nga_b200 import capi
    from tiger_nga_b200.mechanism import load

    mech = load(wl["mech"])
    sol, dt = make_state(wl, rank)
    ncells = sol.shape[1]
    chem = capi.FiniteChem(wl["mech"], wl["precision"], device=local)
    st = chem.torch_stream()
    if not os.path.exists(args.surrogate):
        raise FileNotFoundError(f"trained surrogate weights not found: {args.surrogate}")
    sur = capi.Surrogate(chem)
    sur.load(args.surrogate)
    x0 = torch.from_numpy(sol).to(dev)
    work = x0.clone()
    for _ in range(args.warmup):
        sur.substep(work, dt, P_ATM)
    work.copy_(x0)
    torch.cuda.synchronize(dev)
    if pg:
        pg.barrier()
    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    clocks = ClockSampler(uuid if uuid.startswith("GPU-") else f"GPU-{uuid}")
    clocks.start()
    time.sleep(0.3)
    per, acc, fb, fb_ms, inf_ms, post_ms, judgeT, judgeY = [], 0, 0, 0.0, 0.0, 0.0, 0.0, 0.0
    solver_tot = {"steps": 0, "newton_iters": 0, "jacobians": 0, "cells": 0}
    solver_ms = 0.0
    t_wall = time.perf_counter()
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        r = sur.substep(work, dt, P_ATM)
        e1.record(st)
        e1.synchronize()
        per.append(e0.elapsed_time(e1))
        acc += r["accepted"]
        fb += r["fallback"]["cells"]
        fb_ms += r["ms_fallback"]
        inf_ms += r["ms_infer"]
        post_ms += r["ms_post"]
        judgeT = max(judgeT, r["judge_max_rel_dT"])
        judgeY = max(judgeY, r["judge_max_dY"])
        for k in solver_tot:
            solver_tot[k] += r["fallback"][k]
        solver_ms += r["fallback"]["ms"]
    t_wall = time.perf_counter() - t_wall
    torch.cuda.synchronize(dev)
    if pg:
        pg.barrier()
    clk = clocks.stop()
    ms_total = max_over_ranks(pg, dev, sum(per))
    ms_step = ms_total / args.steps
    value = ncells * ws / (ms_step * 1e-3)
    if not bool(torch.isfinite(work).all()):
        raise RuntimeError("non-finite values after the sweep")
    # accuracy after all substeps: the plain implicit solve of a strided subsample, substep by substep
    m = min(16384, ncells)
    idx = torch.arange(0, ncells, max(1, ncells // m), device=dev)[:m]
    ref = x0[:, idx].contiguous()
    for _ in range(args.steps):
        chem.substep(ref, dt, P_ATM, stats=False)
    torch.cuda.synchronize(dev)
    got = work[:, idx]
    ns = mech.ns
    rg, rr = got[:ns].sum(0), ref[:ns].sum(0)
    errT = ((got[ns] / rg - ref[ns] / rr).abs() / (ref[ns] / rr))
    errY = ((got[:ns] / rg - ref[:ns] / rr).abs().amax(0) / (ref[:ns] / rr).amax(0))
    pa = np.array(per)
    extra = {
        "substep_latency_ms": {"p50": float(np.percentile(pa, 50)), "p99": float(np.percentile(pa, 99)),
                               "max": float(pa.max()), "min": float(pa.min())},
        "surrogate": {"hit_rate": acc / (ncells * args.steps), "fallback_cells_per_substep": fb / args.steps,
                      "fallback_ms_per_substep": fb_ms / args.steps, "infer_ms_per_substep": inf_ms / args.steps,
                      "post_ms_per_substep": post_ms / args.steps, "fallback_share_of_time": fb_ms / sum(per),
                      "judge_max_rel_dT": judgeT, "judge_max_dY": judgeY,
                      "weights": os.path.relpath(args.surrogate, REPO)},
        "accuracy_vs_plain_gpu_after_all_substeps": {
            "cells": m, "substeps": args.steps, "max_rel_T": float(errT.max()),
            "p99_rel_T": float(torch.quantile(errT.float(), 0.99)), "max_dY_over_maxY": float(errY.max()),
            "p99_dY_over_maxY": float(torch.quantile(errY.float(), 0.99))},
        "solver": dict(solver_tot, ms=solver_ms),
    }
    hbm_peak, bf16_peak, peak_src = peaks()
    roof = None
    flops = solver_flops(mech, solver_tot) if solver_tot["newton_iters"] else None
    if flops and solver_ms > 0:
        fp64_peak = capi.fp64_peak_tflops(local)
        ach = flops / (solver_ms * 1e-3) / 1e12
        nbytes = 2 * (mech.ns + 1) * 8 * solver_tot["cells"]
        roof = {"bound": "hbm", "achieved": nbytes / (solver_ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                "frac": nbytes / (solver_ms * 1e-3) / 1e9 / hbm_peak, "traffic": None, "peak_source": peak_src,
                "kernel": "k_bdf",
                "fp64_pipe": {"achieved_tflops": ach, "peak_tflops_measured": fp64_peak, "frac": ach / fp64_peak,
                              "counted_flops": flops}}
    if inf_ms > 0 and bf16_peak:
        ach = 2.0 * sur.nparam * ncells * args.steps / (inf_ms * 1e-3) / 1e12
        extra["inference_roofline"] = {"bound": "tensor", "achieved": ach, "peak": bf16_peak, "unit": "TFLOP/s",
                                       "frac": ach / bf16_peak, "peak_source": peak_src, "kernel": "k_mlp_infer"}
    # e2e: substeps through the host-pointer call (state copied in and out every substep)
    e2e_steps = args.e2e_steps if args.e2e_steps > 0 else 1
    hin = torch.from_numpy(sol).pin_memory()
    hbuf = hin.clone().pin_memory()
    sur.substep(hbuf.numpy(), dt, P_ATM)  # warm-up
    hbuf.copy_(hin)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sur.substep(hbuf.numpy(), dt, P_ATM)
    e2e_s = max_over_ranks(pg, dev, (time.perf_counter() - t0) / e2e_steps)
    e2e = {"value": ncells * ws / e2e_s, "unit": unit, "h2d_bytes_per_step": sol.nbytes * ws,
           "d2h_bytes_per_step": sol.nbytes * ws, "steps": e2e_steps}
    cpu = None
    if rank == 0 and ws == 1 and args.cpu_seconds > 0:
        kind, cval, cdone, cel = time_cpu(wl, sol, dt, args.cpu_seconds, os.cpu_count() or 1)
        cpu = {"value": cval, "unit": unit, "cores": os.cpu_count() or 1, "kind": kind,
               "sample": f"{cdone} cells ({cel:.1f} s) of the initial mixing layer in strided samples spanning "
                         "the layer, one implicit BDF/Newton substep each (no surrogate), OpenMP over cells"}
    if rank == 0:
        line = {"metric": metric, "value": value, "unit": unit, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "bf16/f32 (network), f64 (conservation, fallback solve)",
                "data": "synthetic (seeded DME/air temporal mixing layer)", "config": config, "e2e": e2e,
                "gpu_launches": LAUNCHES["sweep"] * args.steps, "roofline": roof, "cpu_baseline": cpu,
                "clocks": clk, "wall_s": t_wall}
        line.update(extra)
        print(json.dumps(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    sur.close()
    chem.close()
    return 0


def props_work(mech, what):
    """Algorithmic bytes and FP64 flops per cell of one properties launch. Bytes: the N+1 scalars
    read, and for transport the viscosity plus N+1 diffusivities written (density: rho and W_mix).
    Flops (transport): Wilke's pair sum as three FMAs per ordered pair j != k, plus per species
    the collision-integral fit (7 FMAs), the NASA cp polynomial (5 FMAs + 1 multiply), the
    conductivity and the mixture sums (~8)."""
    ns = mech.ns
    if what == "transport":
        return {"bytes": 8 * (ns + 1) + 8 * (1 + ns + 1), "flops": 6 * ns * (ns - 1) + ns * (14 + 11 + 8)}
    return {"bytes": 8 * (ns + 1) + 16, "flops": 4 * ns}


def run_props(args, wl, config, metric, unit, ws, rank, local, dev, pg):
    """Mixture properties (tng_chem_transport / tng_chem_density) of a resident batch: K launches
    back to back between one event pair; e2e through the Fortran-array C-ABI with host arrays."""
    import ctypes

    import torch

    from tiger_nga_b200 import capi

    mech = load_mech(wl["mech"])
    sol, _ = make_state(wl, rank)
    n = sol.shape[1]
    ns = mech.ns
    chem = capi.FiniteChem(wl["mech"], wl["precision"], device=local)
    st = chem.torch_stream()
    x0 = torch.from_numpy(sol).to(dev)
    transport = wl["what"] == "transport"
    outs = {"visc": torch.empty(n, dtype=torch.float64, device=dev),
            "diff": torch.empty((ns + 1, n), dtype=torch.float64, device=dev)} if transport else \
        {"rho": torch.empty(n, dtype=torch.float64, device=dev), "wmix": torch.empty(n, dtype=torch.float64, device=dev)}
    ext = capi.batch_extent(n, ns)
    lib, h = chem.lib, chem.h

    def launch():
        if transport:
            rc = lib.tng_chem_transport(h, outs["visc"].data_ptr(), outs["diff"].data_ptr(), x0.data_ptr(), None,
                                        ctypes.byref(ext), None, 0, capi.TNG_DEVICE_PTRS)
        else:
            rc = lib.tng_chem_density(h, outs["rho"].data_ptr(), outs["wmix"].data_ptr(), x0.data_ptr(), None,
                                      ctypes.byref(ext), P_ATM, capi.TNG_DEVICE_PTRS)
        if rc:
            raise RuntimeError(capi.last_error())

    torch.cuda.synchronize(dev)
    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize(dev)
    if pg:
        pg.barrier()
    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    clocks = ClockSampler(uuid if uuid.startswith("GPU-") else f"GPU-{uuid}")
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        launch()
    e1.record(st)
    e1.synchronize()
    ms_total = e0.elapsed_time(e1)
    if pg:
        pg.barrier()
    clk = clocks.stop()
    ms_total = max_over_ranks(pg, dev, ms_total)
    ms_step = ms_total / args.steps
    value = n * ws / (ms_step * 1e-3)
    for v in outs.values():
        if not bool(torch.isfinite(v).all()):
            raise RuntimeError("non-finite values in the benchmark output")

    hbm_peak, _, peak_src = peaks()
    wk = props_work(mech, wl["what"])
    achieved = wk["bytes"] * n / (ms_step * 1e-3) / 1e9
    fp64_peak = capi.fp64_peak_tflops(local)
    fp64_ach = wk["flops"] * n / (ms_step * 1e-3) / 1e12
    tr = read_profile_value(f"k_props_{wl['mech']}_{wl['what']}.txt", "dram_bytes_per_cell")
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
            "traffic": tr * n if tr else None, "peak_source": peak_src, "kernel": "k_props",
            "algorithmic_bytes_per_cell": wk["bytes"],
            "fp64_pipe": {"achieved_tflops": fp64_ach, "peak_tflops_measured": fp64_peak, "frac": fp64_ach / fp64_peak,
                          "alg_flops_per_cell": wk["flops"]}}

    # e2e: the Fortran-array drop-in with host arrays (copies in and out inside the call)
    hin = torch.from_numpy(sol).pin_memory()
    SC = hin.numpy().T  # Fortran (n, N+1)
    if transport:
        hv = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
        hd = torch.empty((ns + 1, n), dtype=torch.float64).pin_memory().numpy().T
        call = lambda: chem.transport(SC, ext_dict(ext), VISC=hv, DIFF=hd)  # noqa: E731
        d2h = 8 * n * (ns + 2)
    else:
        hr = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
        hw = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
        call = lambda: chem.density(hr, SC, ext_dict(ext), P_ATM, W=hw)  # noqa: E731
        d2h = 16 * n
    e2e_steps = args.e2e_steps if args.e2e_steps > 0 else min(args.steps, 5)
    call()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        call()
    e2e_s = max_over_ranks(pg, dev, (time.perf_counter() - t0) / e2e_steps)
    e2e = {"value": n * ws / e2e_s, "unit": unit, "h2d_bytes_per_step": sol.nbytes * ws,
           "d2h_bytes_per_step": d2h * ws, "steps": e2e_steps}
    cpu = None
    if rank == 0 and ws == 1 and args.cpu_seconds > 0:
        kind, cval, cdone, cel = time_cpu(wl, sol, None, args.cpu_seconds, os.cpu_count() or 1)
        cpu = {"value": cval, "unit": unit, "cores": os.cpu_count() or 1, "kind": kind,
               "sample": f"{cdone} cells ({cel:.1f} s) of the same workload in strided samples spanning the "
                         f"batch, {cpu_what(wl, kind)}, OpenMP over cells"}
    if rank == 0:
        print(json.dumps({"metric": metric, "value": value, "unit": unit, "n_gpus": ws, "steps": args.steps,
                          "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded CH4/air states)",
                          "config": config, "e2e": e2e, "gpu_launches": LAUNCHES["props"] * args.steps,
                          "roofline": roof, "cpu_baseline": cpu, "clocks": clk}))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    chem.close()
    return 0


def ext_dict(e):
    return {f: getattr(e, f) for f, _ in e._fields_}


def load_mech(name):
    from tiger_nga_b200.mechanism import load

    return load(name)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=0, help="timed steps (0: the workload's default)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="gri-surrogate", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="tiger", choices=["tiger", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--e2e-steps", type=int, default=0, help="e2e steps (0: the timed steps of `value`)")
    ap.add_argument("--plain-cells", type=int, default=0,
                    help="gri-surrogate: cells of the strided subsample solved by the plain GPU path (0 = all)")
    ap.add_argument("--side", type=int, default=0, help="cube side override (small profiling cases)")
    ap.add_argument("--surrogate", default="", help="weights file (default: the workload's trained model)")
    ap.add_argument("--tune", type=int, default=1, help="run the autotuner before timing (substep, rates)")
    args = ap.parse_args()
    ws, rank, local = dist_env()
    wl = dict(WORKLOADS[args.workload])
    if args.side:
        if wl["kind"] == "sweep":
            wl["shape"] = (args.side, args.side * 3 // 4, args.side * 3 // 4)
        else:
            wl["side"] = args.side
    if not args.surrogate:
        args.surrogate = os.path.join(MODELS, wl.get("weights", "grimech30.tngs"))
    if args.steps <= 0:
        args.steps = wl["steps"]
    args.warmup = max(args.warmup, 3)
    from tiger_nga_b200.mechanism import load

    mech = load(wl["mech"])
    ncells = int(np.prod(wl["shape"])) if wl["kind"] == "sweep" else wl["side"] ** 3
    config = {"workload": args.workload, "desc": wl["desc"], "mechanism": wl["mech"], "cells_per_gpu": ncells,
              "pressure_pa": P_ATM, "precision": wl["precision"],
              "l2": "inputs larger than L2 (no flush needed)" if ncells * (mech.ns + 1) * 8 > 126e6 else
              "inputs smaller than L2 (state restored from a copy before every step)",
              "parallelism": f"cells sharded, {ws} independent GPU(s)"}
    metric, unit = wl["metric"], "cells/s"

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args, wl, config, metric, unit)
        return 0

    import torch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
        pg = dist
    from tiger_nga_b200 import capi

    if wl["kind"] == "sweep":
        return run_sweep(args, wl, config, metric, unit, ws, rank, local, dev, pg)
    if wl["kind"] == "props":
        return run_props(args, wl, config, metric, unit, ws, rank, local, dev, pg)
    sol, dts = make_state(wl, rank)
    chem = capi.FiniteChem(wl["mech"], wl["precision"], device=local)
    st = chem.torch_stream()
    x0 = torch.from_numpy(sol).to(dev)
    d_dev = torch.from_numpy(dts).to(dev) if dts is not None and np.ndim(dts) else dts
    extra = {}
    sur = None
    if wl["kind"] == "surrogate":
        if not os.path.exists(args.surrogate):
            raise FileNotFoundError(f"trained surrogate weights not found: {args.surrogate}")
        sur = capi.Surrogate(chem)
        sur.load(args.surrogate)

    if args.tune and wl["kind"] in ("substep", "rates"):
        # the project's autotuner picks the launch configuration on these cells (untimed set-up)
        t = chem.autotune(x0, d_dev, P_ATM, kind=wl["kind"], sample=65536)
        config["tuned"] = {"best": t["best"], "candidates": len(t["candidates"])}
    work = torch.empty_like(x0)
    out = torch.empty_like(x0)
    stats_last = {}

    def step():
        """One timed pass; returns its device time in ms (events on the library stream)."""
        if wl["kind"] != "rates":
            work.copy_(x0)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        if wl["kind"] == "rates":
            chem.launch_rhs(x0.data_ptr(), out.data_ptr(), ncells, ncells, P_ATM)
        elif wl["kind"] == "substep":
            r = chem.substep(work, d_dev, P_ATM, stats=True)
            stats_last.update(r)
        else:
            r = sur.substep(work, d_dev, P_ATM)
            stats_last.update(r)
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1)

    for _ in range(args.warmup):
        step()
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    clocks = ClockSampler(uuid if uuid.startswith("GPU-") else f"GPU-{uuid}")
    clocks.start()
    time.sleep(0.3)
    if wl["kind"] == "rates":
        # back-to-back launches, one event pair around all K (the kernel is ~1 ms)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(st)
        for _ in range(args.steps):
            chem.launch_rhs(x0.data_ptr(), out.data_ptr(), ncells, ncells, P_ATM)
        e1.record(st)
        e1.synchronize()
        ms_total = e0.elapsed_time(e1)
    else:
        ms_total = sum(step() for _ in range(args.steps))
    torch.cuda.synchronize(dev)
    if pg:
        pg.barrier()
    clk = clocks.stop()
    ms_total = max_over_ranks(pg, dev, ms_total)
    ms_step = ms_total / args.steps
    value = ncells * ws / (ms_step * 1e-3)
    res = out if wl["kind"] == "rates" else work
    if not bool(torch.isfinite(res).all()):
        raise RuntimeError("non-finite values in the benchmark output")

    hbm_peak, bf16_peak, peak_src = peaks()
    roof = None
    if wl["kind"] == "rates":
        from tiger_nga_b200.workcount import rhs_work

        work_c = rhs_work(mech)
        achieved = work_c["bytes"] * ncells / (ms_step * 1e-3) / 1e9
        fp64_peak = capi.fp64_peak_tflops(local)
        fp64_ach = work_c["flops"] * ncells / (ms_step * 1e-3) / 1e12
        tr = read_profile_value(f"k_rhs_{wl['mech']}_{wl['precision']}.txt", "dram_bytes_per_cell")
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                "traffic": tr * ncells if tr else None, "peak_source": peak_src,
                "kernel": "k_rhs", "algorithmic_bytes_per_cell": work_c["bytes"],
                "fp64_pipe": {"achieved_tflops": fp64_ach, "peak_tflops_measured": fp64_peak,
                              "frac": fp64_ach / fp64_peak, "alg_flops_per_cell": work_c["flops"],
                              "transcendentals_per_cell": work_c["transcendentals"],
                              "note": "reference-formulation flops (transcendentals counted separately); the "
                                      "kernel is FP64-pipe bound, the HBM figure is reported per schema"}}
    else:
        # dominant kernel: the implicit solver (k_bdf) -- the whole substep, or the fallback cells
        sst = stats_last if wl["kind"] == "substep" else stats_last["fallback"]
        ms_solver = sst["ms"]
        flops = solver_flops(mech, sst) if sst.get("newton_iters") else None
        fp64_peak = capi.fp64_peak_tflops(local)
        nbytes = 2 * (mech.ns + 1) * 8 * (sst["cells"] or 0)
        if flops and ms_solver > 0:
            # the solver is bound by the latency of a warp's dependent FP64 chains, not by HBM: its
            # roofline is the FP64 pipe (counted flops over the measured FP64 FMA peak), with the
            # profile's issue and occupancy figures beside it
            ach = flops / (ms_solver * 1e-3) / 1e12
            prof = f"k_bdf_{wl['mech']}.txt"
            roof = {"bound": "fp64/latency", "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s",
                    "frac": ach / fp64_peak,
                    "traffic": (lambda v: v * sst["cells"] if v else None)(
                        read_profile_value(prof, "dram_bytes_per_cell")),
                    "peak_source": "measured (the library's FP64 FMA probe on this GPU; MEASURED_PEAKS has no FP64)",
                    "kernel": "k_bdf", "counted_flops_per_launch": flops,
                    "issue_active_frac": read_profile_value(prof, "issue_active_frac"),
                    "warps_active_frac": read_profile_value(prof, "warps_active_frac"),
                    "hbm": {"algorithmic_bytes": nbytes, "achieved_gbs": nbytes / (ms_solver * 1e-3) / 1e9,
                            "peak_gbs": hbm_peak},
                    "note": "counted flops are a lower bound (one reference-formulation RHS per Newton iteration, "
                            "2/3 n^3 per LU, two triangular solves per iteration); the kernel is latency bound"}
        extra["solver"] = {k: sst.get(k) for k in ("cells", "cells_failed", "steps", "newton_iters", "jacobians",
                                                   "max_steps_cell", "max_newton_cell", "passes", "ms")}

    if wl["kind"] == "surrogate":
        # the plain implicit GPU solve of a strided subsample: speed and the accuracy reference
        m = ncells if args.plain_cells <= 0 else min(args.plain_cells, ncells)
        idx = torch.arange(0, ncells, max(1, ncells // m), device=dev)[:m]
        ref = x0[:, idx].contiguous()
        dsub = d_dev[idx].contiguous()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        pst = chem.substep(ref, dsub, P_ATM, stats=True)
        e1.record(st)
        e1.synchronize()
        ms_plain = e0.elapsed_time(e1)
        plain_cps = m / (ms_plain * 1e-3)
        got = work[:, idx]
        ns = mech.ns
        rg, rr = got[:ns].sum(0), ref[:ns].sum(0)
        errT = ((got[ns] / rg - ref[ns] / rr).abs() / (ref[ns] / rr))
        errY = ((got[:ns] / rg - ref[:ns] / rr).abs().amax(0) / (ref[:ns] / rr).amax(0))
        extra["plain_gpu"] = {"value": plain_cps, "unit": unit, "cells": m, "ms": ms_plain,
                              "steps": pst["steps"], "newton_iters": pst["newton_iters"]}
        extra["speedup_vs_plain_gpu"] = value / ws / plain_cps
        extra["accuracy_vs_plain_gpu"] = {
            "cells": m, "max_rel_T": float(errT.max()), "p99_rel_T": float(torch.quantile(errT.float(), 0.99)),
            "max_dY_over_maxY": float(errY.max()), "p99_dY_over_maxY": float(torch.quantile(errY.float(), 0.99)),
            "within_1pct_T": bool(float(errT.max()) <= 0.01), "within_1e-3_dY": bool(float(errY.max()) <= 1e-3)}
        extra["surrogate"] = {k: stats_last[k] for k in ("accepted", "fallback_ood", "fallback_consistency",
                                                         "fallback_clip", "fallback_ensemble", "judged",
                                                         "judge_max_rel_dT",
                                                         "judge_max_dY", "ms_infer", "ms_post", "ms_fallback",
                                                         "ms_total")}
        extra["surrogate"]["fallback_fraction"] = 1.0 - stats_last["accepted"] / ncells
        extra["surrogate"]["weights"] = os.path.relpath(args.surrogate, REPO)
        # tensor roofline of the inference chain (reported beside the dominant solver kernel):
        # algorithmic flops = 2 x (weights of the unpadded layers) per cell, summed over the
        # networks of the launch (the ensemble members and the error gate, whose two outputs are
        # the predicted errors); ms_infer covers the one launch that evaluates all of them
        has_gate = sur.gate_info()[0]
        H, nh = sur.cfg.hidden, sur.cfg.layers
        gate_w = (sur.n_in * H + (nh - 1) * H * H + H * 2) if has_gate else 0
        alg = 2.0 * (sur.weights_unpadded * sur.members + gate_w)
        t_inf = stats_last["ms_infer"] * 1e-3
        if t_inf > 0 and bf16_peak:
            ach = alg * ncells / t_inf / 1e12
            extra["inference_roofline"] = {"bound": "tensor", "achieved": ach, "peak": bf16_peak, "unit": "TFLOP/s",
                                           "frac": ach / bf16_peak, "peak_source": peak_src,
                                           "kernel": "k_mlp_infer", "networks": sur.members + (1 if has_gate else 0),
                                           "alg_flops_per_cell": alg,
                                           "alg_flops_per_cell_per_member": 2.0 * sur.weights_unpadded,
                                           "alg_flops_per_cell_gate": 2.0 * gate_w,
                                           "executed_flops_per_cell_per_member": 2.0 * sur.weights_padded}

    # ---- e2e through the C-ABI with pinned host buffers -----------------------------------------
    e2e_steps = args.e2e_steps if args.e2e_steps > 0 else args.steps
    hin = torch.from_numpy(sol).pin_memory()
    hbuf = torch.empty_like(hin).pin_memory()
    hd = torch.from_numpy(np.ascontiguousarray(dts)).pin_memory().numpy() if dts is not None and np.ndim(dts) else dts
    h2d = sol.nbytes + (hd.nbytes if isinstance(hd, np.ndarray) else 0)
    if wl["kind"] == "rates":
        d2h = sol.nbytes
    else:
        d2h = sol.nbytes

    def e2e_step():
        if wl["kind"] == "rates":
            chem.compute_rhs(hin.numpy(), P_ATM, out=hbuf.numpy())
        else:
            hbuf.copy_(hin)  # host restore of the initial state (outside the timed call below)
            t0 = time.perf_counter()
            if wl["kind"] == "substep":
                chem.substep(hbuf.numpy(), hd, P_ATM, stats=False)
            else:
                sur.substep(hbuf.numpy(), hd, P_ATM)
            return time.perf_counter() - t0
        return None

    e2e_step()  # warm-up (staging buffers)
    if pg:
        pg.barrier()
    if wl["kind"] == "rates":
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        e2e_s = (time.perf_counter() - t0) / e2e_steps
    else:
        e2e_s = sum(e2e_step() for _ in range(e2e_steps)) / e2e_steps
    e2e_s = max_over_ranks(pg, dev, e2e_s)
    e2e = {"value": ncells * ws / e2e_s, "unit": unit, "h2d_bytes_per_step": h2d * ws, "d2h_bytes_per_step": d2h * ws,
           "steps": e2e_steps}

    # ---- CPU baseline (rank 0, N = 1 only) ------------------------------------------------------
    cpu = None
    if rank == 0 and ws == 1 and args.cpu_seconds > 0:
        kind, cval, cdone, cel = time_cpu(wl, sol, dts, args.cpu_seconds, os.cpu_count() or 1)
        what = cpu_what(wl, kind) if wl["kind"] in ("rates", "props") else "implicit BDF/Newton substep (no surrogate)"
        cpu = {"value": cval, "unit": unit, "cores": os.cpu_count() or 1, "kind": kind,
               "sample": f"{cdone} cells ({cel:.1f} s) of the same workload in strided samples of "
                         f"{min(wl['ref_sample'], ncells)} cells spanning the batch, {what}, OpenMP over cells"}
    if rank == 0:
        line = {"metric": metric, "value": value, "unit": unit, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if wl["precision"] == "fp64" else "f32/f64",
                "data": "synthetic (seeded CH4/air or H2/air states, reference init_flow recipe)", "config": config,
                "e2e": e2e, "gpu_launches": LAUNCHES[wl["kind"]] * args.steps, "roofline": roof,
                "cpu_baseline": cpu, "clocks": clk}
        if wl["kind"] == "surrogate":
            line["dtype"] = "bf16/f32 (network), f64 (conservation, fallback solve)"
        line.update(extra)
        print(json.dumps(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if sur is not None:
        sur.close()
    chem.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
