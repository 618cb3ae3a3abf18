"""Benchmark: time to relative residual 1e-8 per 3D Helmholtz solve.

Workload (default): the 128^3 heterogeneous medium (1500 -> 3000 m/s linear
depth gradient along y, three seeded Gaussian anomalies of +-20 %, radius
8-15 h), h = 10 m, 12-point PML on every face, 8 points per minimum
wavelength, a seeded Gaussian point source; the 7-point PML operator solved
by FGMRES(20) to ||f - A u|| / ||f|| <= 1e-8, preconditioned by the FFT-z /
per-kz block LU (complex shift 0.25).  Inputs are synthetic (seeded
splitmix64), no dataset is read.

One step = one complete solve: set-up + block LU factor of all 128 kz
systems + FGMRES iterations to 1e-8.  `value` is seconds per solve with the
medium and the right-hand side resident on the device, timed with CUDA
events on the solver's stream; the headline path factors and applies the
preconditioner in complex64 (outer loop complex128); the plain complex128
path is timed beside it (`fp64_plain`).  `e2e` repeats the headline solve
through the C ABI with host buffers (medium and RHS copied in, solution
copied out inside the timed region).

    python bench.py [--steps K] [--warmup W] [--impl ours|reference] [--n 128]
    torchrun --nproc-per-node N bench.py --gpus N     (N independent replicas)
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(REPO, "iterative-helmholtz-solver-with-pardiso_b200")
for _p in (REPO, PKG_DIR):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "time to 1e-8 residual per 3D solve: FP32-precond/batched vs plain FP64 GPU"
TOL = 1e-8
RESTART = 20
BETA_PREC = 0.25
# FGMRES iterations the complex128 path needs at the 128^3 workload (measured
# on a B200 with this bench); the CPU port times a sample of iterations and
# scales to this count.
ITERS_128 = None


def workload(n: int):
    from oracle import media
    p = media.config_c2(n=n, pml=12, seed=2024)
    return p


def read_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sms.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        finally:
            os.unlink(self.path)
        out["sm_mhz"] = statistics.median(sms) if sms else None
        out["sm_max_mhz"] = mx
        out["reasons"] = sorted(reasons)
        out["samples"] = len(sms)
        return out


# ---------------------------------------------------------------- GPU arm
def run_ours(args, rank, world, dist):
    import torch

    import helm3d

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    p = workload(args.n)
    f_host = p.rhs(0)
    s2_host = np.ascontiguousarray(p.s2)
    grid = helm3d.grid_mode_n(p.nx, p.ny, p.nz, p.h, p.pml, p.omega)
    N = p.nx * p.ny * p.nz
    # a dedicated stream: the solver's launches and the timing events share it
    stream = torch.cuda.Stream(dev)

    f_dev = torch.from_numpy(f_host).to(dev)
    s2_dev = torch.from_numpy(s2_host).to(dev)
    u_dev = torch.empty_like(f_dev)

    def make(prec, zt=0):
        o = helm3d.default_opts(precision=prec, restart=RESTART, tol=TOL, beta_prec=BETA_PREC, max_iter=20000,
                                device=dev.index, z_transform=zt)
        s = helm3d.Solver(grid, s2_dev, o)
        s.set_stream(stream)
        return s

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed_solves(s, steps, warmup):
        its = []
        for _ in range(warmup):
            s.set_medium(s2_dev)
            s.solve(f_dev, u=u_dev, allow_not_converged=True)
        barrier()
        launches0 = s.kernel_launches
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            s.set_medium(s2_dev)
            s.solve(f_dev, u=u_dev, allow_not_converged=True)
            its.append(s.last_stats.iterations)
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1)
        return max_over_ranks(ms) / steps, its, s.kernel_launches - launches0, s.last_stats

    # headline: complex64 preconditioner
    s32 = make(helm3d.PREC_C64)
    clocks = Clocks(dev.index)
    clocks.start()
    ms32, its32, launches32, st32 = timed_solves(s32, args.steps, args.warmup)
    clk = clocks.stop()

    # profile pass: per-kernel-family device time of one solve
    s32.profile(True)
    s32.set_medium(s2_dev)
    s32.solve(f_dev, u=u_dev, allow_not_converged=True)
    prof = s32.profile_read()
    s32.profile(False)
    relres32 = s32.last_stats.relres

    # e2e through the C ABI with host buffers (pinned)
    f_pin = torch.from_numpy(f_host).pin_memory()
    s2_pin = torch.from_numpy(s2_host).pin_memory()
    u_pin = torch.empty_like(f_pin).pin_memory()
    for _ in range(1):
        s32.set_medium(s2_pin)
        s32.solve(f_pin, u=u_pin, allow_not_converged=True)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s32.set_medium(s2_pin)
        s32.solve(f_pin, u=u_pin, allow_not_converged=True)
    e1.record(stream)
    barrier()
    e2e_s = max_over_ranks(e0.elapsed_time(e1) / 1e3 / args.steps)
    # error of the FP32-preconditioned solution against the FP64 path
    u32 = u_dev.clone()
    s32.close()

    # plain complex128 path
    s64 = make(helm3d.PREC_C128)
    ms64, its64, launches64, st64 = timed_solves(s64, max(1, args.steps // 2), 1)
    u64 = u_dev.clone()
    relerr_vs_fp64 = float(torch.linalg.vector_norm(u32 - u64) / torch.linalg.vector_norm(u64))
    relres64 = s64.last_stats.relres
    s64.close()

    # the same solve with the PML-eigenbasis z-transform (c64 and c128)
    zeig = {}
    for prec, key in ((helm3d.PREC_C64, "c64"), (helm3d.PREC_C128, "c128")):
        sz = make(prec, helm3d.ZT_PML_EIGEN)
        msz, itsz, _, _ = timed_solves(sz, args.steps, 1)
        sz.profile(True)
        sz.set_medium(s2_dev)
        sz.solve(f_dev, u=u_dev, allow_not_converged=True)
        pz = sz.profile_read()
        uz = u_dev.clone()
        zeig[key] = {"value": msz / 1e3 / world, "unit": "s", "iterations": itsz[-1] if itsz else None,
                     "relres": sz.last_stats.relres,
                     "relerr_vs_fft_fp64_path": float(torch.linalg.vector_norm(uz - u64) / torch.linalg.vector_norm(u64)),
                     "kernel_ms_per_solve": {k: round(v[0], 3) for k, v in pz.items()}}
        sz.close()

    if rank != 0:
        return None

    # roofline of the dominant kernel (the block sweep): G^T read twice per
    # launch plus the planes read/written forward and backward
    e = 8
    sweep_ms, sweep_n = prof["sweep"]
    sweep_bytes = 2.0 * p.nz * p.ny * p.nx * p.nx * e + 4.0 * N * e
    sweep_avg_s = (sweep_ms / max(1, sweep_n)) / 1e3
    achieved = sweep_bytes / sweep_avg_s / 1e9 if sweep_avg_s > 0 else None
    peak, peak_kind = read_peaks()
    total_prof = sum(v[0] for v in prof.values())
    line = {
        "metric": METRIC,
        "value": ms32 / 1e3 / world,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms32,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c64 preconditioner / c128 outer",
        "data": "synthetic (seeded splitmix64 media and sources)",
        "config": {
            "workload": f"{p.nx}^3 heterogeneous medium, PML 12, 8 ppw, Gaussian source; "
                        f"one step = set-up + block LU factor + FGMRES({RESTART}) to 1e-8",
            "n": p.nx, "pml": p.pml, "restart": RESTART, "tol": TOL, "beta_prec": BETA_PREC,
            "l2": "inputs larger than L2 (factor 2.1 GB c64 / 4.3 GB c128, Krylov basis 0.7 GB)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        },
        "iterations": its32[-1] if its32 else None,
        "relres": relres32,
        "relerr_vs_fp64_path": relerr_vs_fp64,
        "fp64_plain": {"value": ms64 / 1e3 / world, "unit": "s", "iterations": its64[-1] if its64 else None,
                       "relres": relres64},
        "speedup_vs_fp64_plain": (ms64 / ms32) if ms32 > 0 else None,
        "zpml_eigen": zeig,
        "e2e": {"value": e2e_s / world, "unit": "s", "h2d_bytes_per_step": N * 8 + N * 16,
                "d2h_bytes_per_step": N * 16},
        "gpu_launches": int(launches32 / max(1, args.steps)) * args.steps,
        "roofline": {"bound": "hbm", "kernel": "sweep", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                     "bytes_per_launch": sweep_bytes, "traffic": None},
        "kernel_ms_per_solve": {k: round(v[0], 3) for k, v in prof.items()},
        "kernel_share": {k: round(v[0] / total_prof, 4) for k, v in prof.items()} if total_prof > 0 else None,
        "clocks": clk,
    }
    return line, its64[-1] if its64 else None


# ------------------------------------------------------------ CPU baseline
def cpu_port_sample(n: int, iters: int | None, cores: int, budget_iters: int = 2):
    """Time the oracle port (SciPy SuperLU per kz + NumPy FFT + NumPy stencil,
    FP64, `cores` threads) on a bounded sample of the workload and scale to
    one full solve: factor of a subset of kz systems scaled to all nz, plus a
    few preconditioned FGMRES iterations scaled to `iters`."""
    from concurrent.futures import ThreadPoolExecutor

    import scipy.sparse.linalg as spla

    from oracle import mode_n
    from oracle.mode_r import assemble_2d

    p = workload(n)
    st = mode_n.setup(p, beta_prec=BETA_PREC, factor=False)
    nz = p.nz
    kf = min(nz, max(2 * cores, 8))
    ks = list(range(0, nz, max(1, nz // kf)))[:kf]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(cores) as ex:
        lus = list(ex.map(lambda k: spla.splu(assemble_2d(st.g, st.shifts[k])), ks))
    t_factor = (time.perf_counter() - t0) * nz / len(ks)
    # one preconditioner apply: FFT, nz 2D solves (sampled kz, scaled), iFFT
    f = p.rhs(0)
    rng = np.random.default_rng(0)
    v = (rng.standard_normal(p.shape) + 1j * rng.standard_normal(p.shape))
    t0 = time.perf_counter()
    vh = np.fft.fft(v, axis=0)
    t_fft = time.perf_counter() - t0
    t0 = time.perf_counter()
    with ThreadPoolExecutor(cores) as ex:
        list(ex.map(lambda q: lus[q].solve(vh[ks[q]].ravel()), range(len(ks))))
    t_solves = (time.perf_counter() - t0) * nz / len(ks)
    t0 = time.perf_counter()
    w = st.apply_a(v)
    t_stencil = time.perf_counter() - t0
    # CGS2 against RESTART/2 basis vectors on average
    nv = RESTART // 2
    V = np.stack([v.ravel()] * nv)
    t0 = time.perf_counter()
    for _ in range(2):
        h = V.conj() @ w.ravel()
        wv = w.ravel() - V.T @ h
    t_cgs = time.perf_counter() - t0
    per_it = 2 * t_fft + t_solves + t_stencil + t_cgs
    its = iters if iters else 0
    return {
        "value": t_factor + per_it * its,
        "unit": "s",
        "cores": cores,
        "kind": "port",
        "sample": f"splu factor of {len(ks)} of {nz} kz systems and one preconditioned FGMRES iteration "
                  f"(FFT, {len(ks)} 2D solves, stencil, CGS2 on {nv} vectors) on the {n}^3 workload, "
                  f"scaled to {nz} systems and {its} iterations",
        "factor_s": t_factor,
        "per_iteration_s": per_it,
    }


def run_reference(args, rank):
    if rank != 0:
        return None
    cores = os.cpu_count() or 1
    iters = ITERS_128 if args.n == 128 else None
    vals = []
    for _ in range(args.warmup):
        cpu_port_sample(args.n, iters, cores)
    for _ in range(args.steps):
        vals.append(cpu_port_sample(args.n, iters, cores))
    v = statistics.median(x["value"] for x in vals)
    base = vals[-1]
    base["value"] = v
    p = workload(args.n)
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": "s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "higher_is_better": False,
        "dtype": "c128",
        "data": "synthetic (seeded splitmix64 media and sources)",
        "config": {"workload": f"{p.nx}^3 heterogeneous medium, PML 12, 8 ppw, Gaussian source; FGMRES({RESTART}) "
                               f"to 1e-8", "n": p.nx},
        "cpu_baseline": base,
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist

    if args.impl == "reference":
        out = run_reference(args, rank)
        if rank == 0 and out is not None:
            print(json.dumps(out))
    else:
        res = run_ours(args, rank, world, dist)
        if rank == 0 and res is not None:
            line, its64 = res
            if world == 1 and not args.no_cpu_baseline:
                line["cpu_baseline"] = cpu_port_sample(args.n, its64, os.cpu_count() or 1)
            print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
