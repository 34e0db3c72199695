"""Benchmark of the B200 finite-rate chemistry path; prints ONE JSON line (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl tiger|reference]

Workloads (seeded synthetic states, built like the reference's init_flow tool):
  gri-rates        GRI-Mech 3.0 C/H/O subset (36 species, 422 slots -- the reference's grimech30F
                   stand-in for the 53/325 mechanism), production-rate evaluation only
                   (finitechem_compute_rhs + PRODRATES), 128^3 = 2,097,152 cells, FP64, P = 1 atm.
  gri-rates-mixed  the same in mixed precision (FP32 log-space rates, FP64 reverse exponents).

A step is one pass of the hot path over the whole batch. `value` is device-timed with CUDA
events on the library's stream, inputs resident in HBM (1.24 GB per pass > 126 MB L2, so no
L2 flush is needed); `e2e` is the same metric through the C-ABI with pinned host buffers,
host<->device copies inside the timed region. Multi-GPU: every rank owns its own batch
(cells are independent, no collective on the data path); the step time is the max over ranks.
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

WORKLOADS = {
    "gri-rates": {"mech": "grimech30", "n": 128, "precision": "fp64", "fuel": "CH4",
                  "desc": "GRI-Mech 3.0 C/H/O subset (36 sp, 422 slots) rates, 128^3 cells, FP64"},
    "gri-rates-mixed": {"mech": "grimech30", "n": 128, "precision": "mixed", "fuel": "CH4",
                        "desc": "GRI-Mech 3.0 C/H/O subset (36 sp, 422 slots) rates, 128^3 cells, mixed FP32/FP64"},
}
P_ATM = 101325.0


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


def read_traffic(profile: str):
    """DRAM bytes per cell recorded in a committed ncu summary (line 'dram_bytes_per_cell: X')."""
    path = os.path.join(REPO, "profiles", profile)
    if not os.path.exists(path):
        return None
    for ln in open(path):
        if ln.startswith("dram_bytes_per_cell:"):
            return float(ln.split(":", 1)[1])
    return None


def cpu_rhs_runner():
    """The reference's own rate arithmetic on the host cores: the transliterated Fortran
    (oracle/_ref) when it was built, else the table-driven oracle port."""
    from oracle.oracle import REF_LIB, Oracle, Reference

    def make(mech):
        if os.path.exists(REF_LIB):
            return "reference", Reference(mech)
        return "port", Oracle(mech)

    return make


def time_cpu(mech, sol, seconds: float, nthreads: int):
    kind, impl = cpu_rhs_runner()(mech)
    n = sol.shape[1]
    chunk = min(n, 131072)
    impl.rhs_batch(np.ascontiguousarray(sol[:, :1024]), P_ATM, nthreads)  # warm-up
    done, t0, i = 0, time.perf_counter(), 0
    while True:
        lo = (i * chunk) % n
        sub = np.ascontiguousarray(sol[:, lo:lo + chunk])
        impl.rhs_batch(sub, P_ATM, nthreads)
        done += sub.shape[1]
        i += 1
        el = time.perf_counter() - t0
        if el >= seconds or done >= 8 * n:
            break
    return kind, done / el, done, el


def e2e_run(chem, sol, steps, pg, dev, ncells, ws, unit):
    """Same metric through the C-ABI host-pointer call: pinned host state in, rates out."""
    import torch

    hin = torch.from_numpy(sol).pin_memory().numpy()
    hout = torch.empty(sol.shape, dtype=torch.float64).pin_memory().numpy()
    chem.compute_rhs(hin, P_ATM, out=hout)  # warm-up (staging buffers)
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        chem.compute_rhs(hin, P_ATM, out=hout)
    e2e_s = (time.perf_counter() - t0) / steps
    if pg:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_s = float(t.item())
    return {"value": ncells * ws / e2e_s, "unit": unit, "h2d_bytes_per_step": sol.nbytes * ws,
            "d2h_bytes_per_step": sol.nbytes * ws}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="gri-rates", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="tiger", choices=["tiger", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--n", type=int, default=0, help="cube side override (small profiling cases)")
    args = ap.parse_args()
    ws, rank, local = dist_env()
    wl = dict(WORKLOADS[args.workload])
    if args.n:
        wl["n"] = args.n
    from tiger_nga_b200 import states
    from tiger_nga_b200.mechanism import load
    from tiger_nga_b200.workcount import rhs_work

    mech = load(wl["mech"])
    work = rhs_work(mech)
    ncells = wl["n"] ** 3
    config = {"workload": args.workload, "desc": wl["desc"], "mechanism": wl["mech"], "cells_per_gpu": ncells,
              "pressure_pa": P_ATM, "precision": wl["precision"], "l2": "inputs larger than L2 (1.24 GB/pass)",
              "parallelism": f"cells sharded, {ws} independent GPU(s)"}
    metric = "GRI-3.0 (36-sp stand-in) rate evaluation cells/s"
    unit = "cells/s"

    if args.impl == "reference":
        if rank != 0:
            return 0
        sol, _ = states.chem_state(mech, ncells, 20261204 + rank, wl["fuel"], grid=(wl["n"],) * 3)
        nthreads = os.cpu_count() or 1
        kind, impl = cpu_rhs_runner()(wl["mech"])
        chunk = 131072
        for w in range(args.warmup):
            impl.rhs_batch(np.ascontiguousarray(sol[:, :chunk]), P_ATM, nthreads)
        t0 = time.perf_counter()
        for k in range(args.steps):
            lo = (k * chunk) % ncells
            impl.rhs_batch(np.ascontiguousarray(sol[:, lo:lo + chunk]), P_ATM, nthreads)
        el = time.perf_counter() - t0
        val = chunk * args.steps / el
        sample = f"{chunk} cells of the workload per step"
        print(json.dumps({"impl": "reference", "metric": metric, "value": val, "unit": unit, "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic", "config": config,
                          "cpu_baseline": {"value": val, "unit": unit, "cores": nthreads, "kind": kind,
                                           "sample": sample},
                          "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return 0

    import torch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    from tiger_nga_b200 import capi

    sol, _ = states.chem_state(mech, ncells, 20261204 + rank, wl["fuel"], grid=(wl["n"],) * 3)
    chem = capi.FiniteChem(wl["mech"], wl["precision"], device=local)
    x = torch.from_numpy(sol).to(dev)
    y = torch.empty_like(x)
    st = chem.torch_stream()
    torch.cuda.synchronize()
    for _ in range(max(args.warmup, 3)):
        chem.launch_rhs(x.data_ptr(), y.data_ptr(), ncells, ncells, P_ATM)
    chem.sync()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    clocks = ClockSampler(uuid if uuid.startswith("GPU-") else f"GPU-{uuid}")
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        chem.launch_rhs(x.data_ptr(), y.data_ptr(), ncells, ncells, P_ATM)
    e1.record(st)
    e1.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if pg:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = ncells * ws / (ms_step * 1e-3)
    if not bool(torch.isfinite(y).all()):
        raise RuntimeError("non-finite rates in the benchmark output")

    # ---- e2e through the C-ABI with pinned host buffers -------------------------------------
    e2e = None
    nbytes = sol.nbytes
    if args.e2e_steps > 0:
        e2e = e2e_run(chem, sol, args.e2e_steps, pg, dev, ncells, ws, unit)

    # ---- roofline of the rate kernel ----------------------------------------------------------
    hout = torch.empty(sol.shape, dtype=torch.float64).pin_memory().numpy()
    peaks_path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peaks = json.load(open(peaks_path))
        hbm_peak, src = peaks["hbm_gbs"], "measured"
    else:
        hbm_peak, src = 6650.0, "fallback"
    alg_bytes = work["bytes"] * ncells
    achieved = alg_bytes / (ms_step * 1e-3) / 1e9
    fp64_peak = capi.fp64_peak_tflops(local)
    alg_flops = work["flops"] * ncells
    fp64_ach = alg_flops / (ms_step * 1e-3) / 1e12
    tr = read_traffic(f"k_rhs_{wl['mech']}_{wl['precision']}.txt")
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
            "traffic": tr * ncells if tr else None, "peak_source": src,
            "algorithmic_bytes_per_cell": work["bytes"],
            "fp64_pipe": {"achieved_tflops": fp64_ach, "peak_tflops_measured": fp64_peak,
                          "frac": fp64_ach / fp64_peak, "alg_flops_per_cell": work["flops"],
                          "transcendentals_per_cell": work["transcendentals"],
                          "note": "reference-formulation flops (transcendentals counted separately); "
                                  "the kernel is FP64-pipe bound, the HBM figure is reported per schema"}}

    # ---- CPU baseline (rank 0, N = 1 only) ---------------------------------------------------
    cpu = None
    if rank == 0 and ws == 1 and args.cpu_seconds > 0:
        kind, cval, cdone, cel = time_cpu(wl["mech"], sol, args.cpu_seconds, os.cpu_count() or 1)
        cpu = {"value": cval, "unit": unit, "cores": os.cpu_count() or 1, "kind": kind,
               "sample": f"{cdone} cells ({cel:.1f} s) of the same workload, OpenMP over cells"}
    if rank == 0:
        out = {"metric": metric, "value": value, "unit": unit, "n_gpus": ws, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64" if wl["precision"] == "fp64" else "f32/f64",
               "data": "synthetic (seeded CH4/air states, reference init_flow recipe)", "config": config,
               "e2e": e2e,
               "gpu_launches": args.steps, "roofline": roof, "cpu_baseline": cpu, "clocks": clk}
        print(json.dumps(out))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    chem.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
