"""Train the learned substep of a mechanism on pairs from the plain implicit GPU solver.

    python -m tiger_nga_b200.train_surrogate --mech grimech30 --pairs 8388608 \\
        --out tiger_nga_b200/models/grimech30.tngs

With --gate-only MODEL the ensemble of a trained surrogate is kept and only its error gate is
trained again (on --gate-pairs held-out pairs) and recalibrated, then saved to --out.

Pairs (--dist uneven, the default): seeded states of the uneven-stiffness batch -- 128^3 grids
of a smooth Fourier-mode mixture-fraction field (CH4 fuel / air at 300 K for GRI-Mech, DME at
400 K for DME39),
progress c ~ Beta(2,2) mapped to T in [300, 2400] K, minor species log-uniform in
[1e-10, 1e-3], dt log-uniform in [1e-7, 1e-5] s per cell, P = 1 atm -- each advanced by
tng_substep_batch. With --dist mixing-layer the pairs are taken along 100-substep
(dt = 2e-6 s) trajectories of temporal mixing layers (fuel above air, seeded burning fraction)
instead; with --onpolicy MODEL part of them come from the states MODEL's own sweep visits
(targets from the implicit solve), so the network also sees its own drift. The network is trained by the library's own CUDA kernels
(tng_surrogate_train: FP32 forward/backward, Adam, cosine learning rate), then evaluated
on fresh cells against the plain solve (accepted fraction, max relative error of T, max
species error over max Y). Writes the weights file and a JSON log beside it.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import capi, states
from .mechanism import load

FUEL = {"grimech30": ("CH4", 300.0), "dme39": ("CH3OCH3", 400.0), "hydrogen": ("H2", 300.0)}
P_ATM = 101325.0


def state_batch(mech_name: str, n: int, seed: int, side: int = 128):
    """Seeded (state (N+1, n), dt (n,)) of the uneven-stiffness distribution, on the host."""
    m = load(mech_name)
    fuel, t_fuel = FUEL[mech_name]
    grid = (side, side, side) if side ** 3 == n else (n, 1, 1)
    sol, _ = states.chem_state(m, n, seed, fuel, T_fuel=t_fuel, progress="beta22", T_range=(300.0, 2400.0), grid=grid)
    rng = np.random.default_rng(seed + 104729)
    dts = 10.0 ** rng.uniform(-7.0, -5.0, n)
    return sol, dts


def make_pairs(chem, n_pairs: int, seed: int, chunk: int = 1 << 21):
    """(s0, s1, dt) device tensors of n_pairs cells; s1 = plain implicit solve of s0 over dt."""
    import torch

    nv = chem.nspecies + 1
    s0 = torch.empty((nv, n_pairs), dtype=torch.float64, device="cuda")
    s1 = torch.empty_like(s0)
    d = torch.empty(n_pairs, dtype=torch.float64, device="cuda")
    done, k, solve_s = 0, 0, 0.0
    while done < n_pairs:
        m = min(chunk, n_pairs - done)
        sol, dts = state_batch(chem.mechanism, m, seed + 1000 * k, side=128 if m == 1 << 21 else 0)
        s0[:, done:done + m].copy_(torch.from_numpy(sol))
        d[done:done + m].copy_(torch.from_numpy(dts))
        x = s0[:, done:done + m].clone()  # a copy: s0 keeps the initial states (a view of all of s0 would be s0)
        t0 = time.perf_counter()
        chem.substep(x, d[done:done + m], P_ATM)
        torch.cuda.synchronize()
        solve_s += time.perf_counter() - t0
        s1[:, done:done + m].copy_(x)
        done += m
        k += 1
    return s0, s1, d, solve_s


def make_trajectory_pairs(chem, n_pairs: int, seed: int, dt: float = 2e-6, substeps: int = 100,
                          shape=(64, 48, 48), grids: int = 2):
    """(s0, s1, dt) pairs along implicit-solver trajectories of temporal mixing layers.

    Each of ``grids`` seeded mixing layers (fuel above air, seeded burning fraction) is advanced
    ``substeps`` times by dt with tng_substep_batch; every substep contributes a random subset of
    its cells, so the pairs cover the states a 100-substep run visits, not only the first.
    """
    import torch

    m = load(chem.mechanism)
    fuel, t_fuel = FUEL[chem.mechanism]
    nv = chem.nspecies + 1
    per = -(-n_pairs // (grids * substeps))
    s0 = torch.empty((nv, n_pairs), dtype=torch.float64, device="cuda")
    s1 = torch.empty_like(s0)
    done, solve_s = 0, 0.0
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    for g in range(grids):
        sol, _ = states.mixing_layer(m, shape=shape, seed=seed + 7 * g, fuel=fuel, T_fuel=t_fuel)
        x = torch.from_numpy(sol).cuda()
        for k in range(substeps):
            take = min(per, n_pairs - done, x.shape[1])
            if take <= 0:
                break
            idx = torch.randperm(x.shape[1], device="cuda", generator=gen)[:take]
            s0[:, done:done + take] = x[:, idx]
            t0 = time.perf_counter()
            chem.substep(x, dt, P_ATM)
            torch.cuda.synchronize()
            solve_s += time.perf_counter() - t0
            s1[:, done:done + take] = x[:, idx]
            done += take
    d = torch.full((done,), dt, dtype=torch.float64, device="cuda")
    return s0[:, :done].contiguous(), s1[:, :done].contiguous(), d, solve_s


def make_onpolicy_pairs(chem, sur, n_pairs: int, seed: int, dt: float = 2e-6, substeps: int = 100,
                        shape=(64, 48, 48)):
    """Pairs from the states a surrogate-with-fallback sweep itself visits (its own errors
    included): a seeded mixing layer is advanced ``substeps`` times by ``sur``; at every substep a
    random subset of its cells is also advanced by the implicit solve, which gives the targets."""
    import torch

    m = load(chem.mechanism)
    fuel, t_fuel = FUEL[chem.mechanism]
    nv = chem.nspecies + 1
    per = -(-n_pairs // substeps)
    s0 = torch.empty((nv, n_pairs), dtype=torch.float64, device="cuda")
    s1 = torch.empty_like(s0)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    sol, _ = states.mixing_layer(m, shape=shape, seed=seed, fuel=fuel, T_fuel=t_fuel)
    x = torch.from_numpy(sol).cuda()
    done = 0
    for _ in range(substeps):
        take = min(per, n_pairs - done, x.shape[1])
        if take <= 0:
            break
        idx = torch.randperm(x.shape[1], device="cuda", generator=gen)[:take]
        a = x[:, idx].contiguous()
        b = a.clone()
        chem.substep(b, dt, P_ATM, stats=False)
        s0[:, done:done + take] = a
        s1[:, done:done + take] = b
        done += take
        sur.substep(x, dt, P_ATM)
    d = torch.full((done,), dt, dtype=torch.float64, device="cuda")
    return s0[:, :done].contiguous(), s1[:, :done].contiguous(), d


def errors_vs(chem, y, ref):
    """Per-cell errors of states y against ref relative to the bars: (|dT|/T) / 1e-2 and
    (max |dY| / max Y) / 1e-3, as numpy arrays."""
    ns = chem.nspecies
    ry, rr = y[:ns].sum(0), ref[:ns].sum(0)
    eT = ((y[ns] / ry - ref[ns] / rr).abs() / (ref[ns] / rr)) / 1e-2
    eY = ((y[:ns] / ry - ref[:ns] / rr).abs().amax(0) / (ref[:ns] / rr).amax(0)) / 1e-3
    return eT.cpu().numpy(), eY.cpu().numpy()


def calibrate_gate(chem, sur, s0, d, ref, margin: float = 0.7):
    """The gate threshold on held-out cells: the largest tolerance (fraction of the bars) at which
    every cell the surrogate accepts has both errors within ``margin`` of the bars. Returns
    (tol, accepted fraction at tol, max error ratio of the accepted cells)."""
    pred, reason, ind = sur.predict(s0, d, P_ATM)
    eT, eY = errors_vs(chem, pred, ref)
    r = np.maximum(eT, eY)
    reason = reason.cpu().numpy()
    g = np.maximum(ind[:, 3].cpu().numpy(), ind[:, 4].cpu().numpy())
    other = (reason == 0) | (reason == 5)  # accepted apart from the gate
    viol = other & ~(r <= margin)
    t = float(g[viol].min()) - 1e-6 if viol.any() else float(g[other].max())
    acc = other & (g <= t)
    return 10.0 ** t, float(acc.mean()), float(r[acc].max()) if acc.any() else 0.0


def evaluate(chem, sur, n: int, seed: int, tolerances=(2.0, 5.0), ens_K=(0.5, 1.0, 2.0, 4.0),
             ens_Y=(1e-4, 2e-4, 5e-4, 1e-3), dist: str = "uneven"):
    """The surrogate against the plain solve on n fresh cells.

    Returns the timed surrogate-with-fallback substep (stats, speed-up over the plain solve) and,
    from the fallback-free prediction of every cell, the error of the cells each consistency
    tolerance (K) and ensemble-spread tolerances (K, mass fraction) would accept, with the plain
    solver's share of steps those cells leave to the fallback. Per-cell arrays (errors,
    indicators, reason, T0, dt, steps) are returned as well.
    """
    import torch

    if dist == "mixing-layer":
        fuel, t_fuel = FUEL[chem.mechanism]
        sol, _ = states.mixing_layer(load(chem.mechanism), shape=(64, 48, 48), seed=seed, fuel=fuel, T_fuel=t_fuel)
        dts = np.full(sol.shape[1], 2e-6)
        n = sol.shape[1]
    else:
        sol, dts = state_batch(chem.mechanism, n, seed, side=128 if n == 1 << 21 else 0)
    s0 = torch.from_numpy(sol).cuda()
    d = torch.from_numpy(dts).cuda()
    ref = s0.clone()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, cnt = chem.substep(ref, d, P_ATM, cell_counts=True)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    x = s0.clone()
    t0 = time.perf_counter()
    st = sur.substep(x, d, P_ATM)
    torch.cuda.synchronize()
    t_sur = time.perf_counter() - t0
    ns = chem.nspecies

    def errors(y):
        ry, rr = y[:ns].sum(0), ref[:ns].sum(0)
        eT = ((y[ns] / ry - ref[ns] / rr).abs() / (ref[ns] / rr))
        eY = ((y[:ns] / ry - ref[:ns] / rr).abs().amax(0) / (ref[:ns] / rr).amax(0))
        return eT.cpu().numpy(), eY.cpu().numpy()

    errT_run, errY_run = errors(x)
    pred, reason, ind = sur.predict(s0, d, P_ATM)
    eT, eY = errors(pred)
    reason = reason.cpu().numpy()
    ind = ind.cpu().numpy()
    nst = cnt["nst"].cpu().numpy().astype(np.float64)
    hard = (reason == 1) | (reason == 3)
    curve = []
    for tol in tolerances:
        for ek in ens_K:
            for ey in ens_Y:
                acc = (~hard) & (ind[:, 0] <= tol) & (ind[:, 1] <= ek) & (ind[:, 2] <= ey)
                curve.append({"tol_K": tol, "ens_tol_K": ek, "ens_tol_Y": ey, "accepted": float(acc.mean()),
                              "max_rel_T": float(eT[acc].max()) if acc.any() else 0.0,
                              "max_dY_over_maxY": float(eY[acc].max()) if acc.any() else 0.0,
                              "fallback_step_share": float(nst[~acc].sum() / max(nst.sum(), 1.0))})
    T0 = (s0[ns] / s0[:ns].sum(0)).cpu().numpy()
    summary = {
        "cells": n, "plain_s": t_plain, "surrogate_s": t_sur, "speedup": t_plain / t_sur,
        "accepted": st["accepted"], "fallback": st["fallback"]["cells"], "fallback_ood": st["fallback_ood"],
        "fallback_consistency": st["fallback_consistency"], "fallback_clip": st["fallback_clip"],
        "fallback_ensemble": st["fallback_ensemble"], "fallback_gate": st["fallback_gate"],
        "max_rel_T": float(errT_run.max()), "p99_rel_T": float(np.quantile(errT_run, 0.99)),
        "max_dY_over_maxY": float(errY_run.max()), "p99_dY_over_maxY": float(np.quantile(errY_run, 0.99)),
        "judge_max_rel_dT": st["judge_max_rel_dT"], "judge_max_dY": st["judge_max_dY"],
        "ms_infer": st["ms_infer"], "ms_post": st["ms_post"], "ms_fallback": st["ms_fallback"],
        "prediction_max_rel_T": float(eT.max()), "prediction_p99_rel_T": float(np.quantile(eT, 0.99)),
        "tolerance_curve": curve,
    }
    cells = {"errT": eT.astype(np.float32), "errY": eY.astype(np.float32), "ind": ind[:, 0].astype(np.float32),
             "ensT": ind[:, 1].astype(np.float32), "ensY": ind[:, 2].astype(np.float32),
             "reason": reason.astype(np.int8), "T0": T0.astype(np.float32), "dt": dts.astype(np.float32),
             "nst": nst.astype(np.int32)}
    return summary, cells


def train_and_calibrate_gate(a, chem, sur):
    """The error gate: trained on the ensemble's errors on pairs the ensemble was not trained on,
    its threshold calibrated on further held-out cells against the plain solve (pairs of the same
    distribution: the uneven batch, or mixing-layer trajectories of other seeds)."""
    import torch

    t0 = time.perf_counter()
    gseed = a.gate_seed or a.seed + 50021
    if a.dist == "mixing-layer":
        g0, g1, gd, _ = make_trajectory_pairs(chem, a.gate_pairs, gseed)
    else:
        g0, g1, gd, _ = make_pairs(chem, a.gate_pairs, gseed)
    n_hard = 0
    if a.gate_boost > 1:
        # the pairs whose ensemble error is near or above the bars are repeated gate_boost times:
        # the calibrated threshold is set by the lowest-scored of those, so the gate's ranking of
        # them matters more than its fit of the bulk
        r = []
        for lo in range(0, g0.shape[1], 1 << 21):
            hi = min(lo + (1 << 21), g0.shape[1])
            pred, _, _ = sur.predict(g0[:, lo:hi], gd[lo:hi], P_ATM)
            eT, eY = errors_vs(chem, pred, g1[:, lo:hi])
            r.append(np.maximum(eT, eY))
            del pred
        hard = torch.from_numpy(np.nonzero(np.concatenate(r) > a.gate_boost_min)[0]).to(g0.device)
        n_hard = int(hard.numel())
        if n_hard:
            rep = hard.repeat(int(a.gate_boost) - 1)
            g0, g1, gd = torch.cat([g0, g0[:, rep]], 1), torch.cat([g1, g1[:, rep]], 1), torch.cat([gd, gd[rep]])
    gl = sur.train_gate(g0, g1, gd, P_ATM, epochs=a.gate_epochs, batch=a.batch, lr=a.lr, under=a.gate_under)
    del g0, g1, gd
    if a.dist == "mixing-layer":
        c0, c1, cd, _ = make_trajectory_pairs(chem, a.calib_cells, a.seed + 70001)
    else:
        c0, c1, cd, _ = make_pairs(chem, a.calib_cells, a.seed + 70001)
    tol, acc, rmax = calibrate_gate(chem, sur, c0, cd, c1, margin=a.calib_margin)
    sur.set_gate_tol(tol)
    del c0, c1, cd
    torch.cuda.empty_cache()
    return {"pairs": a.gate_pairs, "seed": gseed, "epochs": a.gate_epochs, "under": a.gate_under,
            "boost": a.gate_boost, "boost_min": a.gate_boost_min, "boosted_pairs": n_hard,
            "losses": [float(v) for v in gl], "calib_cells": a.calib_cells, "calib_margin": a.calib_margin,
            "tol": tol, "calib_accepted": acc, "calib_max_err_ratio": rmax, "s": time.perf_counter() - t0}


def retrain_gate(a, chem):
    """--gate-only: the ensemble of a.gate_only kept, its error gate trained and calibrated again;
    the log of the original training is kept in the new JSON log with the new gate and evaluation."""
    sur = capi.Surrogate(chem, members=a.members)
    sur.load(a.gate_only)
    gate = train_and_calibrate_gate(a, chem, sur)
    sur.save(a.out)
    ev, cells = evaluate(chem, sur, a.eval_cells, a.seed + 99991, dist=a.dist)
    if a.cells_out:
        np.savez_compressed(a.cells_out, **cells)
    try:
        with open(a.gate_only + ".json") as f:
            log = json.load(f)
    except OSError:
        log = {"mechanism": a.mech}
    log["gate"], log["eval"], log["gate_retrained_from"] = gate, ev, a.gate_only
    with open(a.out + ".json", "w") as f:
        json.dump(log, f, indent=1)
    print(json.dumps({"gate": gate, "eval": ev}))
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--mech", default="grimech30")
    ap.add_argument("--dist", default="uneven", choices=["uneven", "mixing-layer"],
                    help="pairs from the uneven-stiffness batch, or along 100-substep mixing-layer trajectories")
    ap.add_argument("--pairs", type=int, default=1 << 23)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--eval-cells", type=int, default=1 << 21)
    ap.add_argument("--target-mode", type=int, default=1)
    ap.add_argument("--post-mode", type=int, default=1)
    ap.add_argument("--members", type=int, default=2)
    ap.add_argument("--loss-T-weight", type=float, default=2.0)
    ap.add_argument("--consist-tol", type=float, default=5.0)
    ap.add_argument("--out", required=True)
    ap.add_argument("--cells-out", default="", help="write the per-cell evaluation arrays (.npz) here")
    ap.add_argument("--onpolicy", default="", help="a trained surrogate: part of the pairs come from the states "
                    "its own sweep visits (mixing-layer distribution)")
    ap.add_argument("--onpolicy-frac", type=float, default=0.5)
    ap.add_argument("--refine-epochs", type=int, default=20, help="hard-example refinement epochs (0: none)")
    ap.add_argument("--refine-lr", type=float, default=5e-4)
    ap.add_argument("--boost", type=float, default=4.0, help="refinement: extra copies per unit of error/bar")
    ap.add_argument("--gate-pairs", type=int, default=1 << 22, help="held-out pairs the error gate is trained on "
                    "(0: no gate)")
    ap.add_argument("--gate-epochs", type=int, default=30)
    ap.add_argument("--gate-under", type=float, default=4.0)
    ap.add_argument("--calib-cells", type=int, default=1 << 21, help="held-out cells that calibrate the gate")
    ap.add_argument("--calib-margin", type=float, default=0.7, help="accepted cells stay within this fraction of "
                    "the bars on the calibration cells")
    ap.add_argument("--gate-only", default="", help="a trained surrogate: keep its ensemble, train and calibrate "
                    "its error gate again")
    ap.add_argument("--gate-boost", type=float, default=1.0, help="copies of the gate pairs whose ensemble error "
                    "exceeds --gate-boost-min of the bars")
    ap.add_argument("--gate-boost-min", type=float, default=0.3)
    ap.add_argument("--gate-seed", type=int, default=0, help="seed of the gate's training pairs (0: derived from "
                    "--seed)")
    a = ap.parse_args(argv)
    chem = capi.FiniteChem(a.mech, "fp64")
    if a.gate_only:
        return retrain_gate(a, chem)
    t0 = time.perf_counter()
    if a.dist == "mixing-layer":
        n_on = int(a.pairs * a.onpolicy_frac) if a.onpolicy else 0
        s0, s1, d, solve_s = make_trajectory_pairs(chem, a.pairs - n_on, a.seed)
        if n_on:
            import torch

            prev = capi.Surrogate(chem, members=a.members)
            prev.load(a.onpolicy)
            o0, o1, od = make_onpolicy_pairs(chem, prev, n_on, a.seed + 31337)
            prev.close()
            s0, s1, d = torch.cat([s0, o0], 1), torch.cat([s1, o1], 1), torch.cat([d, od])
            del o0, o1, od
    else:
        s0, s1, d, solve_s = make_pairs(chem, a.pairs, a.seed)
    t_pairs = time.perf_counter() - t0
    sur = capi.Surrogate(chem, target_mode=a.target_mode, post_mode=a.post_mode, loss_T_weight=a.loss_T_weight,
                         consist_tol_K=a.consist_tol, members=a.members)
    t0 = time.perf_counter()
    losses = sur.train(s0, s1, d, P_ATM, epochs=a.epochs, batch=a.batch, lr=a.lr)
    t_train = time.perf_counter() - t0
    refine = {}
    if a.refine_epochs > 0:
        t0 = time.perf_counter()
        rl, pop = sur.refine(s0, s1, d, P_ATM, epochs=a.refine_epochs, batch=a.batch, lr=a.refine_lr, boost=a.boost)
        refine = {"epochs": a.refine_epochs, "lr": a.refine_lr, "boost": a.boost, "population": pop,
                  "losses": [float(v) for v in rl], "s": time.perf_counter() - t0}
    del s0, s1, d
    gate = train_and_calibrate_gate(a, chem, sur) if a.gate_pairs > 0 else {}
    sur.save(a.out)
    ev, cells = evaluate(chem, sur, a.eval_cells, a.seed + 99991, dist=a.dist)
    if a.cells_out:
        np.savez_compressed(a.cells_out, **cells)
    log = {"mechanism": a.mech, "dist": a.dist, "pairs": a.pairs, "onpolicy": a.onpolicy,
           "onpolicy_frac": a.onpolicy_frac if a.onpolicy else 0.0, "epochs": a.epochs, "batch": a.batch, "lr": a.lr, "seed": a.seed,
           "target_mode": a.target_mode, "post_mode": a.post_mode, "loss_T_weight": a.loss_T_weight,
           "members": a.members,
           "consist_tol_K": a.consist_tol,
           "pairs_s": t_pairs, "plain_solve_s": solve_s, "train_s": t_train,
           "losses": [float(v) for v in losses], "refine": refine, "gate": gate, "eval": ev}
    with open(a.out + ".json", "w") as f:
        json.dump(log, f, indent=1)
    print(json.dumps(log))


if __name__ == "__main__":
    main()
