#!/usr/bin/env python
"""Benchmark of the lattice-Boltzmann hot path on B200.

Workload (N=1 line): d3q27_cumulant, FP32, triply periodic Taylor-Green vortex
on 256^3 nodes (u0=0.05, rho0=1, nu=1e-3), Globals, kinetic energy and
enstrophy every 50 iterations -- the configuration the MLUPS metric is quoted
on. A *step* is one logging interval: 49 plain iterations, one iteration that
integrates the Globals (ITER_LASTGLOB) and reads them back, and the kinetic
energy / enstrophy reduction read back. ``value`` is MLUPS over K steps with
the lattice resident in HBM; ``e2e`` is the same metric through the C ABI from
host buffers: each e2e step uploads the initial snapshot from pinned host
memory, runs the full 2000-iteration case with the same diagnostics every 50,
and reads the velocity field back.

At N=1 the line also carries ``storage_variants``: the same workload with
FP16-shift storage (the tile-staged kernel) and in FP64, each timed on the
device like the headline (MLUPS, the iteration kernel's fraction of the
measured HBM bandwidth, the ratio to the FP32 line), and each storage's
relative L2 velocity error against the FP64 run after 2000 iterations from the
same initial state. It also carries ``other_configs``: configuration 3 (the
d3q19 porous channel in four storages, with their errors against FP64) and
configuration 4 (512 batched d2q9 cases, FP32 and FP16-shift).

Multi-GPU (torchrun, one rank per GPU): independent replicas, weak scaling, no
data-path collective (the case does not shard across GPUs here).

``--impl reference`` times the reference's CPU path on the host cores on a
bounded slab of the same workload, K steps: TCLB's own d3q27_cumulant node
code (CollisionMRT compiled from its source into oracle/_ref) in a pull-stream
loop when that library is built, else the oracle (the CPU restatement; TCLB as
a whole cannot be built without R/polyAlgebra/MPI).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "MLUPS"
UNIT = "MLUPS"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=40)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=256, help="edge of the cubic lattice")
    p.add_argument("--model", default="d3q27_cumulant")
    p.add_argument("--precision", default="fp32")
    p.add_argument("--storage", default="same")
    p.add_argument("--log-every", type=int, default=50)
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--e2e-iters", type=int, default=2000)
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--cpu-slab", type=int, default=16, help="z extent of the CPU-baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--variants", default="fp16s,fp64",
                   help="N=1: storage variants timed after the headline on the same workload "
                        "(comma list of fp16s, bf16s, fp64; empty for none)")
    p.add_argument("--variant-steps", type=int, default=10)
    p.add_argument("--no-configs", action="store_true",
                   help="N=1: skip the configuration-3 and configuration-4 runs added to the line")
    p.add_argument("--accuracy-iters", type=int, default=2000,
                   help="iterations of the accuracy run of each variant (and FP32) against FP64; 0 for none")
    p.add_argument("--rate", type=float, default=6.0, help="config 5: Poisson arrival rate (requests/s)")
    p.add_argument("--path", default="auto", choices=["auto", "tma", "pairs", "one"],
                   help="16-bit storage kernel for plain iterations: auto (tile-staged TMA where it "
                        "applies and is the faster choice, else two nodes per thread), tma, pairs, one "
                        "(one node per thread)")
    p.add_argument("--case", default="tgv", choices=["tgv", "porous"],
                   help="timed lattice: the Taylor-Green vortex (the headline) or, with --shape, the d3q19 porous "
                        "channel of configuration 3 (Bernoulli(0.08) solids, ForceX 1e-6, nu 0.01) for profiling")
    p.add_argument("--shape", default="", help="nx,ny,nz of a --case porous lattice (default 384,192,192)")
    p.add_argument("--porosity", type=float, default=0.08, help="solid fraction of a --case porous lattice")
    p.add_argument("--config", type=int, default=2,
                   help="2 = the headline Taylor-Green line; 1, 3, 4, 5 = the other configurations (one JSON line)")
    p.add_argument("--accuracy", action="store_true",
                   help="with --config 2: velocity, energy and enstrophy errors of each storage against FP64")
    return p.parse_args()


def dist_env():
    from tclb_b200.replicas import env

    return env()


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "of measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "of fallback"


def profiled_traffic(kernel, model, precision, storage, n):
    """DRAM bytes per launch of the iteration kernel from the committed ncu
    summary of this kernel and workload, if one exists
    (profiles/<kernel>_<model>_<precision>_<storage>_<n>.md, line
    'traffic_bytes_per_launch: X')."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{model}_{precision}_{storage}_{n}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1])
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------
# Taylor-Green viscosity per model: 1e-3 is the d3q27_cumulant configuration;
# the d3q19 MRT (omega = 1.988 at nu = 1e-3) diverges on this under-resolved
# flow, so its throughput lines run the stable nu = 1e-2.
TGV_NU = {"d3q27_cumulant": 1e-3, "d3q19": 1e-2, "d2q9": 1e-2}


def tgv_setup(lat, n, u0=0.05, nu=None):
    from tclb_b200 import cases

    if nu is None:
        nu = TGV_NU[lat.model.name]

    lat.set_flags(cases.tgv_flags(lat.model, n, nz=lat.nz))
    lat.SetSetting("nu", nu)
    rho, u = cases.tgv_fields(n, u0=u0, nz=lat.nz, dtype=lat.real)
    lat.init_equilibrium(rho, u)


def case_lattice(args, precision=None, storage=None):
    """The timed lattice of --case, set up and resident on the current device."""
    from tclb_b200 import cases
    from tclb_b200.lattice import Lattice

    precision, storage = precision or args.precision, storage or args.storage
    if args.case == "tgv":
        n = args.n
        lat = Lattice(args.model, n, n, n, precision=precision, storage=storage)
        tgv_setup(lat, n)
        return lat
    nx, ny, nz = (int(v) for v in (args.shape or "384,192,192").split(","))
    lat = Lattice("d3q19", nx, ny, nz, precision=precision, storage=storage)
    lat.set_flags(cases.porous_channel_d3q19(nx, ny, nz, p=args.porosity, band=4, seed=0))
    lat.SetSetting("nu", 0.01)
    lat.SetSetting("ForceX", 1e-6)
    lat.Init()
    return lat


def ref_cpu_baseline(args, seconds, threads=None):
    """TCLB's own d3q27_cumulant node code (CollisionMRT, models/flow/d3q27_cumulant/Dynamics.c.Rt:309-519,
    compiled from the reference's source into oracle/_ref by oracle/make_ref.py) in a pull-stream loop over a
    slab of the workload (256 x 256 x cpu_slab nodes, periodic, OpenMP over rows); None if that library is
    not on this machine."""
    try:
        from oracle import make_ref, ref
        if not os.path.exists(make_ref.LIB):
            return None
        cores = ref.threads(threads or os.cpu_count() or 1)
    except Exception:
        return None
    from tclb_b200 import cases
    from tclb_b200 import models as M

    n, nz = args.n, args.cpu_slab
    dt = np.float64 if args.precision == "fp64" else np.float32
    m = M.get("d3q27_cumulant")
    rho, u = cases.tgv_fields(n, u0=0.05, nz=nz, dtype=np.float64)
    J = rho[..., None] * u
    e = np.array(m.velocities, float)
    w = np.array(m.weights)
    eu = np.einsum("qd,zyxd->qzyx", e, J)
    a = np.ascontiguousarray(w[:, None, None, None] * (rho + 3 * eu + 4.5 * eu ** 2 / rho - 1.5 * (J ** 2).sum(-1) / rho),
                             dtype=dt)
    b = np.empty_like(a)
    S = {"nu": TGV_NU["d3q27_cumulant"]}
    ref.d3q27c_iterate(a, b, S)
    done, t0 = 0, time.perf_counter()
    while True:
        ref.d3q27c_iterate(a, b, S)
        a, b = b, a
        done += 1
        el = time.perf_counter() - t0
        if el >= seconds and done >= 2:
            break
    return {"value": n * n * nz * done / el / 1e6, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"d3q27_cumulant TGV slab {n}x{n}x{nz}, {done} iterations in {el:.1f} s, {args.precision}: "
                      "TCLB's CollisionMRT compiled from its source (oracle/make_ref.py) in a pull-stream loop, "
                      "OpenMP over rows (TCLB's own build needs R+polyAlgebra, autoconf, MPI)"}


def cpu_baseline(args, model_name, seconds, threads=None):
    """The reference's CPU path on a slab of the workload: TCLB's own node code (oracle/_ref) for
    d3q27_cumulant when it is built here, else the oracle (CPU restatement of the path): 256 x 256 x
    cpu_slab nodes, periodic, same settings."""
    if model_name == "d3q27_cumulant":
        r = ref_cpu_baseline(args, seconds, threads)
        if r is not None:
            return r
    import oracle
    from tclb_b200 import cases
    from tclb_b200 import models as M

    cores = oracle.set_threads(threads or os.cpu_count() or 1)
    n, nz = args.n, args.cpu_slab
    o = oracle.OracleLattice(model_name, n, n, nz, precision=args.precision if args.precision == "fp64" else "fp32")
    o.set_flags(cases.tgv_flags(model_name, n, nz=nz))
    o.set_setting("nu", TGV_NU[model_name])
    m = M.get(model_name)
    rho, u = cases.tgv_fields(n, u0=0.05, nz=nz, dtype=np.float64)
    J = rho[..., None] * u
    e = np.array(m.velocities, float)
    w = np.array(m.weights)
    eu = np.einsum("qd,zyxd->qzyx", e, J)
    f = w[:, None, None, None] * (rho + 3 * eu + 4.5 * eu ** 2 / rho - 1.5 * (J ** 2).sum(-1) / rho)
    o.set_densities(f)
    del f, eu, J
    o.iterate(1)
    done, t0 = 0, time.perf_counter()
    while True:
        o.iterate(1)
        done += 1
        el = time.perf_counter() - t0
        if el >= seconds and done >= 2:
            break
    mlups = n * n * nz * done / el / 1e6
    return {"value": mlups, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{model_name} TGV slab {n}x{n}x{nz}, {done} iterations in {el:.1f} s, {args.precision}, "
                      f"OpenMP over nodes (TCLB CPU build unavailable: needs R+polyAlgebra, autoconf, MPI)"}


# ---------------------------------------------------------------------------
def workload_config(args, world: int) -> dict:
    """The workload both arms report (the reference arm times bounded samples of it)."""
    from tclb_b200 import models as M

    if args.case == "porous":
        nx, ny, nz = (int(v) for v in (args.shape or "384,192,192").split(","))
        return {"workload": f"d3q19 porous channel {nx}x{ny}x{nz}, Bernoulli({args.porosity:g}) solids, ForceX=1e-6, "
                            "nu=0.01",
                "model": "d3q19", "lattice": [nx, ny, nz], "precision": args.precision, "storage": args.storage,
                "iterations_per_step": args.log_every, "parallelism": f"replicas x{world}"}
    m = M.get(args.model)
    n = args.n
    elem = 8 if args.precision == "fp64" else (4 if args.storage == "same" else 2)
    snap_gb = m.Q * elem * n ** 3 / 1e9
    return {"workload": f"{args.model} Taylor-Green vortex {n}^3 periodic, u0=0.05, nu={TGV_NU[args.model]:g}",
            "model": args.model, "lattice": [n, n, n], "precision": args.precision, "storage": args.storage,
            "iterations_per_step": args.log_every, "globals_every": args.log_every,
            "energy_enstrophy_every": args.log_every,
            "l2": "inputs larger than L2 (2 x %.2f GB snapshots)" % snap_gb, "parallelism": f"replicas x{world}"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    # K steps, each a bounded sample of the workload (at most cpu_seconds / 4, and 120 s over all steps)
    per = max(0.5, min(args.cpu_seconds / 4, 120.0 / max(1, args.steps)))
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_baseline(args, args.model, 0.5)
    vals = []
    t_all = time.perf_counter()
    for _ in range(args.steps):
        r = cpu_baseline(args, args.model, per)
        vals.append(r["value"])
    el = time.perf_counter() - t_all
    v = float(np.mean(vals))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": len(vals),
            "warmup": args.warmup, "ms_per_step": el / len(vals) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
            "impl": "reference",
            "config": workload_config(args, world),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "gpu_launches": 0}
    print(json.dumps(line), flush=True)
    return 0


def timed_steps(lat, steps, I, stream):
    """K logging steps (I-1 plain iterations, one with Globals, the energy/enstrophy reduction) timed with
    CUDA events on the launching stream: (total seconds, mean plain-iteration seconds, last energy)."""
    import torch

    from tclb_b200 import models as M

    sp = stream.cuda_stream
    pairs = []
    energy = (0.0, 0.0)
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        lat.Iterate(I - 1, M.ITER_NORM, stream=sp)
        b.record(stream)
        lat.Iterate(1, M.ITER_NORM | M.ITER_LASTGLOB, stream=sp)
        energy = lat.energy_enstrophy(stream=sp)
        pairs.append((a, b))
    e_end.record(stream)
    torch.cuda.synchronize()
    t = e_start.elapsed_time(e_end) / 1e3
    kern = sum(a.elapsed_time(b) for a, b in pairs) / 1e3 / (steps * (I - 1))
    return t, kern, energy


def kernel_name(path) -> str:
    return "k_iterate_tma" if path["tma"] else ("k_iterate_pair" if path["pairs"] else "k_iterate")


def storage_variants(args, stream, fp32_value, fp32_kern):
    """The headline workload with other storage: FP16-shift (tile-staged kernel), BF16-shift, FP64.
    Each: MLUPS over --variant-steps logging steps (lattice resident), its plain-iteration kernel's
    fraction of the measured HBM bandwidth, the ratio to the FP32 line; then the relative L2 velocity
    error of each storage (and of FP32) against FP64 after --accuracy-iters iterations."""
    import torch

    from tclb_b200 import models as M
    from tclb_b200.lattice import Lattice

    n, I = args.n, args.log_every
    peaks, _ = measured_peaks()
    names = [v for v in args.variants.split(",") if v]
    out = {}
    for v in names:
        prec, sto = ("fp64", "same") if v == "fp64" else ("fp32", v)
        lat = Lattice(args.model, n, n, n, precision=prec, storage=sto)
        tgv_setup(lat, n)
        for _ in range(3):
            timed_steps(lat, 1, I, stream)
        clocks = ClockSampler(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0])
        clocks.start()
        time.sleep(0.2)
        t, kern, _ = timed_steps(lat, args.variant_steps, I, stream)
        clk = clocks.stop()
        bpu = lat.bytes_per_update
        value = lat.N * I * args.variant_steps / t / 1e6
        out[v] = {"precision": prec, "storage": sto, "value": value, "unit": UNIT,
                  "kernel": kernel_name(lat.launch_path()), "kernel_mlups": lat.N / kern / 1e6,
                  "bytes_per_update": bpu, "frac": bpu * lat.N / kern / 1e9 / peaks["hbm_gbs"],
                  "ratio_vs_fp32": value / fp32_value, "kernel_ratio_vs_fp32": fp32_kern / kern,
                  "steps": args.variant_steps, "sm_mhz": clk.get("sm_mhz"), "clock_reasons": clk.get("reasons")}
        lat.close()
    if args.accuracy_iters > 0:
        u = {}
        for v in ["fp64", "fp32"] + [x for x in names if x != "fp64"]:
            prec, sto = ("fp64", "same") if v == "fp64" else ("fp32", "same" if v == "fp32" else v)
            lat = Lattice(args.model, n, n, n, precision=prec, storage=sto)
            tgv_setup(lat, n)
            lat.Iterate(args.accuracy_iters, M.ITER_NORM, stream=stream.cuda_stream)
            u[v] = lat.GetQuantity("U", stream=stream.cuda_stream).astype(np.float64)
            lat.close()
        ref = u["fp64"]
        nrm = float(np.linalg.norm(ref))
        for v, uv in u.items():
            if v == "fp64":
                continue
            err = float(np.linalg.norm(uv - ref) / nrm)
            out.setdefault(v, {})["velocity_rel_l2_vs_fp64"] = err
        out["accuracy_run"] = f"{args.accuracy_iters} iterations from the same initial state, U against FP64"
    torch.cuda.synchronize()
    return out


def other_configs() -> dict:
    """Configurations 3 and 4 in the N=1 line, so their rates are recorded with the headline:
    configuration 3 (d3q19 porous channel 384x192x192, 5000 iterations, FP64 / FP32 / FP16-shift /
    BF16-shift, each storage's velocity and flux error against the FP64 run) and configuration 4
    (512 batched d2q9 cases, 2000 iterations each, FP32 and FP16-shift, 64 iterations per replay and
    tiles of 64 x 32 (FP32) and 64 x 64 (FP16-shift), the fastest in a sweep of tile shapes on B200,
    fixed here to keep the run short; tiles 64 wide let the 16-bit cases not staged in shared memory
    take the two-nodes-per-thread kernel)."""
    from tclb_b200 import benchmarks as BM

    c3 = BM.config3()
    c4 = BM.config4(tune=False, launch={"same": (64, 32, 64), "fp16s": (64, 64, 64)})
    keep = ("MLUPS", "hbm_roofline_frac", "u_rel_l2_vs_fp64", "flux_rel_err_vs_fp64")
    out = {"config3": {"workload": c3["config"], "fp16s_speedup_vs_fp32": c3.get("fp16s_speedup_vs_fp32"),
                       "runs": {k: {x: v[x] for x in keep if x in v} for k, v in c3["runs"].items()}},
           "config4": {"workload": c4["config"],
                       "runs": {k: {x: v[x] for x in ("MLUPS", "cases_per_s", "fraction_of_single",
                                                      "single_large_case_MLUPS", "launch") if x in v}
                                for k, v in c4["runs"].items()}}}
    return out


def run_ours(args):
    import torch

    from tclb_b200.replicas import Replicas

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    # replicas only: one lattice per GPU, host coordination over NCCL
    reps = Replicas("nccl")
    barrier, reduce_max = reps.barrier, reps.reduce_max

    from tclb_b200 import models as M
    from tclb_b200.lattice import Lattice

    n, I = args.n, args.log_every
    # CPU baseline first (rank 0, N=1): host-only work before the GPU is busy
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, args.model, args.cpu_seconds)

    lat = case_lattice(args)
    if args.path != "auto":
        lat.set_launch(128 if lat.nx >= 128 else 32, 2 if lat.nx >= 128 else 8, use_graphs=True,
                       use_pairs=args.path in ("pairs", "tma"), use_tma=args.path == "tma",
                       tma_always=args.path == "tma")
    path = lat.launch_path()
    # a dedicated (non-default) stream: the library launches on it, the CUDA
    # events below are recorded on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    assert sp != 0
    N = lat.N
    bpu = lat.bytes_per_update

    for _ in range(args.warmup):
        lat.Iterate(I - 1, M.ITER_NORM, stream=sp)
        lat.Iterate(1, M.ITER_NORM | M.ITER_LASTGLOB, stream=sp)
    barrier()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    phys = vis.split(",")[local] if vis and len(vis.split(",")) > local else str(local)
    clocks = ClockSampler(phys)
    clocks.start()
    time.sleep(0.3)
    t_wall0 = time.perf_counter()
    barrier()
    # kinetic energy and enstrophy every I iterations
    t, kern, energy = timed_steps(lat, args.steps, I, stream)
    barrier()
    wall = time.perf_counter() - t_wall0
    clk = clocks.stop()
    kern = reduce_max(kern)
    glob = lat.globals_dict()
    updates = N * I * args.steps
    value, t_max = reps.whole_job_rate(updates / 1e6, t)

    peaks, peak_src = measured_peaks()
    achieved = bpu * N / kern / 1e9
    kernel = kernel_name(path)
    traffic = profiled_traffic(kernel, args.model, args.precision, args.storage, n) if args.case == "tgv" else None
    roof = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "peak_source": peak_src,
            "kernel": kernel + (" (no-Globals variant)" if kernel == "k_iterate" else ""), "bytes_per_update": bpu,
            "kernel_ms": kern * 1e3, "kernel_mlups": N / kern / 1e6}

    # ---- end to end through the C ABI from pinned host buffers -------------
    e2e = None
    if not args.no_e2e and args.e2e_steps > 0:
        snap = torch.empty(lat.snapshot_bytes(), dtype=torch.uint8, pin_memory=True)
        lat.save(snap.data_ptr(), stream=sp)
        ubuf = torch.empty(N * 3, dtype=torch.float32 if args.precision == "fp32" else torch.float64,
                           pin_memory=True)
        uview = ubuf.numpy()
        nlog = args.e2e_iters // I
        gl_bytes = len(lat.model.globals) * 8
        barrier()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(args.e2e_steps):
            lat.load(snap.data_ptr(), stream=sp)
            for _ in range(nlog):
                lat.Iterate(I - 1, M.ITER_NORM, stream=sp)
                lat.Iterate(1, M.ITER_NORM | M.ITER_LASTGLOB, stream=sp)
                lat.energy_enstrophy(stream=sp)
            lat.GetQuantity("U", out=uview, stream=sp)
        s1.record(stream)
        torch.cuda.synchronize()
        te = reduce_max(s0.elapsed_time(s1) / 1e3)
        e2e = {"value": N * nlog * I * args.e2e_steps * world / te / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": int(snap.numel()),
               "d2h_bytes_per_step": int(ubuf.numel() * ubuf.element_size() + nlog * (gl_bytes + 16)),
               "steps": args.e2e_steps, "iterations_per_step": nlog * I,
               "step": "upload snapshot (pinned), full case with Globals, kinetic energy and enstrophy every "
                       "50 iterations, read U back"}

    lat.close()
    variants = None
    if world == 1 and args.variants and args.storage == "same" and args.precision == "fp32" and args.case == "tgv":
        variants = storage_variants(args, stream, value, kern)
    configs = None
    if world == 1 and not args.no_configs and args.case == "tgv" and args.storage == "same":
        configs = other_configs()

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
                "config": workload_config(args, world),
                "kernel_path": "tma" if path["tma"] else ("pairs" if path["pairs"] else "one"),
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
                "gpu_launches": args.steps * (I + 2), "wall_s": wall, "storage_variants": variants,
                "other_configs": configs,
                "globals_last": dict({k: float(v) for k, v in glob.items()}, KineticEnergy=energy[0],
                                     Enstrophy=energy[1])}
        print(json.dumps(line), flush=True)
    reps.close()
    return 0


def run_config(args):
    import torch

    from tclb_b200 import benchmarks as BM

    from tclb_b200.replicas import Replicas

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if args.config in (4, 5):
        # independent cases / requests shared out over the ranks, no exchange
        reps = Replicas("nccl" if world > 1 else "gloo")
        res = BM.config4(reps=reps) if args.config == 4 else BM.config5(rate=args.rate, reps=reps)
        reps.close()
    elif rank != 0:  # one case: rank 0 alone runs it
        return 0
    elif args.config == 2:  # --accuracy
        res = BM.config2_accuracy(n=args.n)
        res["drag"] = BM.sphere_drag_accuracy()
    else:
        res = {1: BM.config1, 3: BM.config3}[args.config]()
    if rank == 0:
        print(json.dumps({"metric": METRIC, "unit": UNIT, "config_id": args.config, "data": "synthetic", **res}),
              flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.config != 2 or args.accuracy:
        return run_config(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
