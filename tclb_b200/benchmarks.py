"""Runners for the benchmark configurations other than the headline one.

Each returns a dict that bench.py prints as one JSON line. All inputs are
seeded synthetic cases (tclb_b200.cases); timings use CUDA events on the
lattice's stream or, for the batch and serving loops whose work spans several
streams, synchronised wall-clock time around the whole run.
"""
from __future__ import annotations

import json
import math
import os
import time
from typing import Dict, List

import numpy as np

from . import cases
from . import models as M
from .batch import Batch, CaseSpec, autotune
from .lattice import Lattice
from .serve import Request, Server

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def hbm_peak() -> float:
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        return 6650.0


def _events(torch, stream):
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    return a, b


# ---------------------------------------------------------------------------
# Configuration 1: d2q9 channel with a disc, FP64 (and FP32), 10k iterations
# ---------------------------------------------------------------------------
def config1(iterations: int = 10000, log_every: int = 100, precision: str = "fp64") -> dict:
    import torch

    nx, ny = 1024, 256
    lat = Lattice("d2q9", nx, ny, precision=precision)
    lat.set_flags(cases.channel_disc_d2q9(nx, ny, r=16, cx=256, cy=128))
    for kind, name, v in cases.channel_disc_settings(ux=0.01, nu=0.02, bgk=True):
        lat.set_zone_setting(name, v) if kind == "zone" else lat.SetSetting(name, v)
    lat.Init()
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    lat.Iterate(log_every, M.ITER_NORM | M.ITER_LASTGLOB, stream=sp)  # warm-up, graph capture
    lat.Init()
    log = []
    a, b = _events(torch, stream)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(iterations // log_every):
        lat.Iterate(log_every, M.ITER_NORM | M.ITER_LASTGLOB, stream=sp)
        log.append(lat.globals.tolist())
    b.record(stream)
    torch.cuda.synchronize()
    t = a.elapsed_time(b) / 1e3
    mlups = lat.N * iterations / t / 1e6
    g = lat.globals_dict()
    u = lat.GetQuantity("U")
    lat.close()
    bpu = 2 * 9 * (8 if precision == "fp64" else 4) + 2
    return {"config": "1: d2q9 channel 1024x256, disc r=16 at (256,128), Zou-He inlet Ux=0.01 / outlet rho=1, "
                      f"BGK nu=0.02, {iterations} iterations, Globals every {log_every}",
            "precision": precision, "MLUPS": mlups, "time_s": t,
            "hbm_roofline_frac": mlups * 1e6 * bpu / (hbm_peak() * 1e9),
            "note": "lattice (2 x 18.9 MB) is L2-resident: the HBM roofline is not the bound; "
                    "plain iterations replay CUDA graphs of 32",
            "globals_final": g, "max_u": float(np.abs(u).max()), "log_rows": len(log)}


# ---------------------------------------------------------------------------
# Configuration 3: d3q19 porous channel, storage precision study
# ---------------------------------------------------------------------------
def config3(iterations: int = 5000, storages=("fp64", "fp32", "fp16s", "bf16s"), n=(384, 192, 192)) -> dict:
    import torch

    nx, ny, nz = n
    fl = cases.porous_channel_d3q19(nx, ny, nz, p=0.08, band=4, seed=0)
    out = {"config": f"3: d3q19 MRT {nx}x{ny}x{nz} channel, body force Fx=1e-6, nu=0.01, Bernoulli(0.08) "
                     f"solids (seed 0, 4-node wall band free), periodic x, walls y/z, {iterations} iterations",
           "runs": {}}
    ref_u, ref_g = None, None
    for st in storages:
        prec = "fp64" if st == "fp64" else "fp32"
        storage = "same" if st in ("fp64", "fp32") else st
        lat = Lattice("d3q19", nx, ny, nz, precision=prec, storage=storage)
        lat.set_flags(fl)
        lat.SetSetting("nu", 0.01)
        lat.SetSetting("ForceX", 1e-6)
        lat.Init()
        stream = torch.cuda.Stream()
        sp = stream.cuda_stream
        lat.Iterate(64, M.ITER_NORM, stream=sp)  # warm-up
        lat.Init()
        a, b = _events(torch, stream)
        torch.cuda.synchronize()
        a.record(stream)
        lat.Iterate(iterations, M.ITER_NORM | M.ITER_LASTGLOB, stream=sp)
        b.record(stream)
        torch.cuda.synchronize()
        t = a.elapsed_time(b) / 1e3
        mlups = lat.N * iterations / t / 1e6
        u = lat.GetQuantity("U").astype(np.float64)
        g = lat.globals_dict()
        r = {"MLUPS": mlups, "bytes_per_update": lat.bytes_per_update,
             "hbm_roofline_frac": mlups * 1e6 * lat.bytes_per_update / (hbm_peak() * 1e9),
             "VOLvx": g["VOLvx"], "MaxV": g["MaxV"]}
        if st == "fp64":
            ref_u, ref_g = u, g
        else:
            r["u_rel_l2_vs_fp64"] = float(np.linalg.norm(u - ref_u) / np.linalg.norm(ref_u))
            r["flux_rel_err_vs_fp64"] = float(abs(g["VOLvx"] - ref_g["VOLvx"]) / abs(ref_g["VOLvx"]))
        out["runs"][st] = r
        lat.close()
    if "fp32" in out["runs"] and "fp16s" in out["runs"]:
        out["fp16s_speedup_vs_fp32"] = out["runs"]["fp16s"]["MLUPS"] / out["runs"]["fp32"]["MLUPS"]
    out["reference_for_errors"] = ("the GPU FP64 path of this library, which matches the CPU FP64 oracle to "
                                   "1e-12 in the parity tests (a CPU FP64 run of this size takes about an hour)")
    return out


# ---------------------------------------------------------------------------
# Configuration 4: 512 batched d2q9 cases
# ---------------------------------------------------------------------------
def batch_specs(n_cases=512, seed=0, iterations=2000) -> List[CaseSpec]:
    specs, _clamps = [], 0
    lst, clamps = cases.batch_cases_d2q9(n_cases, seed=seed)
    for c in lst:
        fl = cases.disc_channel_flags(c["W"], c["H"], c["r"], c["cx"], c["cy"])
        specs.append(CaseSpec(fl, {"Viscosity": c["nu"]}, {0: {"VelocityX": c["ux"]}, 1: {"VelocityX": c["ux"]}},
                              iterations))
    return specs, clamps


def single_large_mlups(model="d2q9", shape=(1, 1024, 4096), precision="fp32", storage="same", iters=200) -> float:
    import torch

    nz, ny, nx = shape
    lat = Lattice(model, nx, ny, nz, precision=precision, storage=storage)
    if model == "d2q9":
        lat.set_flags(cases.disc_channel_flags(nx, ny, ny / 8, nx / 4, ny / 2))
        lat.SetSetting("Viscosity", 0.02)
        lat.set_zone_setting("VelocityX", 0.02)
    else:
        lat.set_flags(cases.porous_channel_d3q19(nx, ny, nz, p=0.08, band=2, seed=1))
        lat.SetSetting("nu", 0.02)
    lat.Init()
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    lat.Iterate(64, stream=sp)
    a, b = _events(torch, stream)
    torch.cuda.synchronize()
    a.record(stream)
    lat.Iterate(iters, stream=sp)
    b.record(stream)
    torch.cuda.synchronize()
    t = a.elapsed_time(b) / 1e3
    n = lat.N
    lat.close()
    return n * iters / t / 1e6


def aggregate_batch(reps, updates: float, seconds: float, ncases: int, single: float) -> dict:
    """Whole-job figures of a batch run whose cases are shared out over the
    ranks: the work of all ranks over the slowest rank's time, and the
    fraction of N times the single-large-case rate (the ranks' mean)."""
    t = reps.reduce_max(seconds)
    u = reps.reduce_sum(updates)
    c = reps.reduce_sum(ncases)
    single_mean = reps.reduce_sum(single) / reps.world
    mlups = u / t / 1e6 if t > 0 else 0.0
    return {"MLUPS": mlups, "cases_per_s": c / t if t > 0 else 0.0, "time_s": t,
            "single_large_case_MLUPS": single_mean, "fraction_of_single": mlups / (reps.world * single_mean)}


def config4(n_cases=512, iterations=2000, storages=("same", "fp16s"), tune=True, reps=None, launch=None) -> dict:
    """With reps over N > 1 ranks (one GPU each) the cases are shared out by
    work (replicas.partition_cases), with no exchange between the ranks.
    launch = (bx, by, K), or a dict of them by storage, fixes the launch shape
    instead of autotuning."""
    from .replicas import Replicas, partition_cases

    reps = reps or Replicas("gloo")
    specs, clamps = batch_specs(n_cases, iterations=iterations)
    nodes = sum(int(np.prod(s.shape)) for s in specs)
    mine = partition_cases([float(np.prod(s.shape)) for s in specs], reps.world)[reps.rank]
    specs = [specs[i] for i in mine]
    my_nodes = sum(int(np.prod(s.shape)) for s in specs)
    out = {"config": f"4: {n_cases} d2q9 BGK-like cases, W log-uniform 64..2048 (H=W/4), one disc each, "
                     f"Ux=0.02, Re U[20,200], {iterations} iterations each, persistent graph-captured launches",
           "nodes_total": nodes, "omega_clamps": clamps, "gpus": reps.world, "runs": {}}
    for st in storages:
        tuned = None
        if tune:
            sample = specs[:: max(1, len(specs) // 64)]
            tuned = autotune("d2q9", sample, precision="fp32", storage=st, trial_iters=64, globals_at_end=True)
        b = Batch("d2q9", "fp32", storage=st, budget_bytes=100 << 30, max_cases=max(1, len(specs)))
        b.set_paths(globals_at_end=True)  # Globals of each case's last iteration only
        fixed = launch.get(st) if isinstance(launch, dict) else launch
        if tuned:
            b.set_launch(tuned["bx"], tuned["by"], tuned["K"])
        elif fixed:
            b.set_launch(*fixed)
        t_add = time.perf_counter()
        ids = [b.add_case(s) for s in specs]
        t_add = time.perf_counter() - t_add
        b.sync()
        reps.barrier()
        t0 = time.perf_counter()
        steps = b.run_to_completion()
        t = time.perf_counter() - t0
        single = single_large_mlups(storage=st)
        r = aggregate_batch(reps, float(my_nodes) * iterations, t, len(ids), single)
        r.update({"replays": steps, "admission_s": t_add, "launch": dict(zip(("bx", "by", "K"), b.get_launch()))})
        if tuned:
            r["autotune_table"] = tuned["table"]
        out["runs"][st] = r
        b.close()
    return out


# ---------------------------------------------------------------------------
# Configuration 5: serving a Poisson stream of mixed requests
# ---------------------------------------------------------------------------
def serve_requests(n_requests=120, rate=6.0, seed=0, d3_edge=(64, 256), iters=(500, 5000)) -> List[Request]:
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    d2, _ = cases.batch_cases_d2q9(n_requests, seed=seed + 1)
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate)
        n_it = int(rng.integers(iters[0], iters[1] + 1))
        if rng.random() < 0.7:
            c = d2[i]
            fl = cases.disc_channel_flags(c["W"], c["H"], c["r"], c["cx"], c["cy"])
            spec = CaseSpec(fl, {"Viscosity": c["nu"]}, {0: {"VelocityX": c["ux"]}, 1: {"VelocityX": c["ux"]}}, n_it)
            out.append(Request(i, "d2q9", spec, t))
        else:
            e = int(rng.integers(d3_edge[0], d3_edge[1] + 1))
            e = max(32, cases.pad_nx(e) if e % 32 else e)
            p = float(rng.uniform(0.02, 0.15))
            fl = cases.porous_channel_d3q19(e, e, e, p=p, band=2, seed=1000 + i)
            spec = CaseSpec(fl, {"nu": 0.02, "ForceX": 1e-5}, {}, n_it)
            out.append(Request(i, "d3q19", spec, t))
    return out


def aggregate_serving(reps, rep: dict, tts: list, updates: float, ideal_s: float) -> dict:
    """Whole-job serving figures over the ranks (each serving its share of
    the requests on its own GPU): requests and updates of all ranks over the
    longest wall time, time-to-solution percentiles over all requests, and
    the efficiency as the ideal single-large-case time of all served updates
    over the GPU-seconds the servers had work in flight."""
    parts = reps.gather({"tts": list(tts), "updates": float(updates), "ideal": float(ideal_s),
                         "busy": float(rep["busy_s"]), "wall": float(rep["wall_s"]), "rounds": int(rep["rounds"]),
                         "pending": int(rep["pending"])})
    all_tts = np.array([t for p in parts for t in p["tts"]]) if any(p["tts"] for p in parts) else np.zeros(1)
    n = sum(len(p["tts"]) for p in parts)
    upd = sum(p["updates"] for p in parts)
    busy = sum(p["busy"] for p in parts)
    wall = max(p["wall"] for p in parts)
    ideal = sum(p["ideal"] for p in parts)
    return {"requests": n, "wall_s": wall, "cases_per_s": n / wall if wall else 0.0,
            "mlups": upd / wall / 1e6 if wall else 0.0, "busy_s": busy,
            "busy_mlups": upd / busy / 1e6 * reps.world if busy else 0.0,
            "p50_s": float(np.percentile(all_tts, 50)), "p99_s": float(np.percentile(all_tts, 99)),
            "rounds": sum(p["rounds"] for p in parts), "pending": sum(p["pending"] for p in parts),
            "fraction_of_single": ideal / busy if busy else 0.0, "gpus": reps.world}


def config5(n_requests=120, rate=6.0, storages=("same", "fp16s"), budget_gb=150, reps=None,
            solo_nodes=None) -> dict:
    """With reps over N > 1 ranks the requests are dealt out round-robin in
    arrival order (request i to rank i mod N), each rank serving its share on
    its own GPU with no exchange; the figures are aggregated over the ranks.
    solo_nodes: requests of at least that many nodes run as lattices of their own (a number, or a dict
    by storage). Default: 10M nodes in FP32 storage, where batched and one-lattice kernels are both
    close to the HBM roofline and only the largest boxes gain from running alone; 4M nodes in 16-bit
    storage, where the batch's tile-staged kernel falls further behind the one-lattice kernels."""
    if solo_nodes is None:
        solo_nodes = {"same": 10_000_000, "fp16s": 4_000_000}
    from .replicas import Replicas

    reps = reps or Replicas("gloo")
    out = {"config": f"5: serving, Poisson arrivals (rate {rate}/s, seed 0), 70% d2q9 obstacle channels (config-4 "
                     "sizes), 30% d3q19 porous boxes (edge U[64,256], p U[0.02,0.15]), iterations U[500,5000], "
                     f"admission by footprint under {budget_gb} GB (pools of 4 + 24 GiB set aside at start-up), resident "
                     f"lattices, continuous batching; requests of at least {solo_nodes} nodes as lattices of their own",
           "gpus": reps.world, "runs": {}}
    for st in storages:
        reqs = serve_requests(n_requests, rate)[reps.rank::reps.world]
        # pools set aside at start-up, above the peak of the admitted footprints (9-11 GB): the first
        # admissions then take memory like those of a running server instead of growing the pools
        srv = Server(("d2q9", "d3q19"), "fp32", st, budget_bytes=budget_gb << 30,
                     launch={"d2q9": (64, 64, 64), "d3q19": (64, 16, 16) if st == "same" else (64, 64, 16)},
                     reserve={"d2q9": 4 << 30, "d3q19": 24 << 30},
                     solo_nodes=solo_nodes.get(st) if isinstance(solo_nodes, dict) else solo_nodes)
        reps.barrier()
        rep = srv.run(reqs)
        done = srv.done
        srv.close()
        # Efficiency against one large case of each model: the time the served
        # updates would take at each model's single-large-case rate, over the
        # time the server had GPU work in flight.
        single = {"d2q9": single_large_mlups("d2q9", storage=st),
                  "d3q19": single_large_mlups("d3q19", (256, 256, 256), storage=st, iters=100)}
        t_ideal = sum(r.updates / (single[r.model] * 1e6) for r in done)
        agg = aggregate_serving(reps, rep, [r.finished - r.arrival for r in done], sum(r.updates for r in done),
                                t_ideal)
        agg["single_large_case_MLUPS"] = single
        if reps.world == 1:  # where the busy time went (one server)
            agg["busy_by_model_s"] = rep["busy_by_model_s"]
            agg["busy_all_models_s"] = rep["busy_all_models_s"]
            agg["model_mlups_while_in_flight"] = {
                m: rep["updates_by_model"][m] / t / 1e6 for m, t in rep["busy_by_model_s"].items() if t > 0}
        out["runs"][st] = agg
    return out


# ---------------------------------------------------------------------------
# Configuration 2 accuracy: the Taylor-Green vortex of the throughput lines
# run in each storage next to an FP64 run of the same case; relative L2 error
# of the velocity field and relative errors of the kinetic energy and
# enstrophy after the given iterations.
# ---------------------------------------------------------------------------
TGV_NU = {"d3q27_cumulant": 1e-3, "d3q19": 1e-2}


def config2_accuracy(models=("d3q27_cumulant", "d3q19"), n=256, iterations=2000,
                     storages=("fp32", "fp16s", "bf16s")) -> dict:
    out = {"config": f"2 (accuracy): Taylor-Green vortex {n}^3, u0 = 0.05, {iterations} iterations, each storage "
                     "against an FP64 run of the same case", "runs": {}}
    for model in models:
        res, ref_u, ref_ee = {}, None, None
        for st in ("fp64",) + tuple(storages):
            prec = "fp64" if st == "fp64" else "fp32"
            storage = "same" if st in ("fp64", "fp32") else st
            lat = Lattice(model, n, n, n, precision=prec, storage=storage)
            lat.set_flags(cases.tgv_flags(model, n))
            lat.SetSetting("nu", TGV_NU[model])
            rho, u = cases.tgv_fields(n, u0=0.05, dtype=lat.real)
            lat.init_equilibrium(rho, u)
            lat.Iterate(iterations)
            u = lat.GetQuantity("U").astype(np.float64)
            ee = lat.energy_enstrophy()
            path = lat.launch_path()
            lat.close()
            if st == "fp64":
                ref_u, ref_ee = u, ee
                res[st] = {"kinetic_energy": ee[0], "enstrophy": ee[1]}
                continue
            res[st] = {"u_rel_l2_vs_fp64": float(np.linalg.norm(u - ref_u) / np.linalg.norm(ref_u)),
                       "energy_rel_err": abs(ee[0] - ref_ee[0]) / abs(ref_ee[0]),
                       "enstrophy_rel_err": abs(ee[1] - ref_ee[1]) / abs(ref_ee[1]),
                       "path": "tma" if path["tma"] else ("pairs" if path["pairs"] else "one")}
            del u
        out["runs"][model] = res
    return out


def sphere_drag_accuracy(shape=(128, 128, 256), r=12, cx=64, iterations=2000, u_in=0.02, nu=0.02,
                         storages=("fp32", "fp16s", "bf16s")) -> dict:
    """d3q27_cumulant flow past a Body-flagged sphere (cases.sphere_channel_d3q27)
    in each storage next to FP64: relative error of the Drag Global at the
    last iteration, relative L2 error of the velocity field, and the rate
    (MLUPS, CUDA events around the whole run of plain iterations and the
    final Globals one) with the kernel path taken."""
    import torch

    nz, ny, nx = shape
    fl, zones = cases.sphere_channel_d3q27(nx, ny, nz, r=r, cx=cx)
    res, ref_u, ref_drag = {}, None, None
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    for st in ("fp64",) + tuple(storages):
        prec = "fp64" if st == "fp64" else "fp32"
        storage = "same" if st in ("fp64", "fp32") else st
        lat = Lattice("d3q27_cumulant", nx, ny, nz, precision=prec, storage=storage)
        lat.set_flags(fl)
        lat.SetSetting("nu", nu)
        lat.set_zone_setting("Velocity", u_in, zones["Inlet"])
        lat.Init()
        lat.Iterate(8, stream=sp)  # graph capture, warm-up
        lat.Init()
        a, b = _events(torch, stream)
        torch.cuda.synchronize()
        a.record(stream)
        lat.Iterate(iterations - 1, M.ITER_NORM, stream=sp)
        lat.Iterate(1, M.ITER_NORM | M.ITER_LASTGLOB, stream=sp)
        b.record(stream)
        torch.cuda.synchronize()
        mlups = lat.N * iterations / (a.elapsed_time(b) / 1e3) / 1e6
        drag = lat.globals_dict()["Drag"]
        u = lat.GetQuantity("U").astype(np.float64)
        path = lat.launch_path()
        lat.close()
        if st == "fp64":
            ref_u, ref_drag = u, drag
            res[st] = {"drag": drag, "MLUPS": mlups}
            continue
        res[st] = {"drag": drag, "drag_rel_err": abs(drag - ref_drag) / abs(ref_drag),
                   "u_rel_l2_vs_fp64": float(np.linalg.norm(u - ref_u) / np.linalg.norm(ref_u)), "MLUPS": mlups,
                   "path": "tma" if path["tma"] else ("pairs" if path["pairs"] else "one")}
    if "fp32" in res:
        for st in storages:
            if st != "fp32":
                res[st]["speedup_vs_fp32"] = res[st]["MLUPS"] / res["fp32"]["MLUPS"]
    return {"config": f"d3q27_cumulant sphere (r = {r}, Body-flagged walls) in a {nx}x{ny}x{nz} duct, inlet "
                      f"u = {u_in}, nu = {nu}, {iterations} iterations", "runs": res}


# ---------------------------------------------------------------------------
# Profiling workloads: one porous d3q19 box (p = 0.08, 2-node wall band, seed
# 1), n^3 nodes, advanced through a batch (its kernel path chosen by the
# batch's paths) or through a single lattice. Small enough for an ncu capture.
# ---------------------------------------------------------------------------
def porous_box_batch(n=128, storage="fp16s", replays=3, K=8, bx=64, by=64, use_tma=True) -> dict:
    import torch

    b = Batch("d3q19", "fp32", storage=storage, budget_bytes=8 << 30, max_cases=2)
    b.set_launch(bx, by, K)
    b.set_paths(use_tma=use_tma)
    fl = cases.porous_channel_d3q19(n, n, n, p=0.08, band=2, seed=1)
    b.add_case(CaseSpec(fl, {"nu": 0.02, "ForceX": 1e-5}, {}, 1 << 20))
    staged, pairs = b.uses_tma(), b.uses_pairs()
    for _ in range(replays):
        b.step()
    b.sync()
    torch.cuda.synchronize()
    b.close()
    return {"workload": f"batch, one d3q19 porous box {n}^3, {storage}", "replays": replays, "K": K,
            "tile_staged": staged, "pairs": pairs}


def porous_box_single(n=128, storage="fp16s", iters=24) -> dict:
    import torch

    lat = Lattice("d3q19", n, n, n, precision="fp32", storage=storage)
    lat.set_flags(cases.porous_channel_d3q19(n, n, n, p=0.08, band=2, seed=1))
    lat.SetSetting("nu", 0.02)
    lat.SetSetting("ForceX", 1e-5)
    lat.Init()
    lat.Iterate(iters)
    torch.cuda.synchronize()
    path = lat.launch_path()
    lat.close()
    return {"workload": f"single lattice, d3q19 porous box {n}^3, {storage}", "iterations": iters, "path": path}


def config4_replays(n_cases=512, storage="same", bx=32, by=32, K=64, replays=2) -> dict:
    """The config-4 cases in one batch at a fixed launch shape, a few replays
    (profiling workload: no autotuning, no single-case reference)."""
    import torch

    specs, _ = batch_specs(n_cases, iterations=1 << 20)
    b = Batch("d2q9", "fp32", storage=storage, budget_bytes=100 << 30, max_cases=n_cases)
    b.set_paths(globals_at_end=True)
    b.set_launch(bx, by, K)
    for s_ in specs:
        b.add_case(s_)
    for _ in range(replays):
        b.step()
    b.sync()
    torch.cuda.synchronize()
    info = b.info()
    b.close()
    return {"workload": f"config-4 batch, {n_cases} d2q9 cases, {storage}, tiles {bx}x{by}, K={K}",
            "replays": replays, "tiles": info["tiles"], "nodes": sum(int(np.prod(x.shape)) for x in specs)}


def main(argv=None):
    import argparse

    p = argparse.ArgumentParser(description="profiling workloads (one JSON line)")
    p.add_argument("what", choices=["porous-box-batch", "porous-box-single", "config4-replays"])
    p.add_argument("--n", type=int, default=128)
    p.add_argument("--cases", type=int, default=512)
    p.add_argument("--storage", default="fp16s")
    p.add_argument("--no-tma", action="store_true")
    a = p.parse_args(argv)
    if a.what == "porous-box-batch":
        r = porous_box_batch(a.n, a.storage, use_tma=not a.no_tma)
    elif a.what == "porous-box-single":
        r = porous_box_single(a.n, a.storage)
    else:
        r = config4_replays(a.cases, a.storage)
    print(json.dumps(r))


if __name__ == "__main__":
    main()
