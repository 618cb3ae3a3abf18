"""Benchmark: time to relative residual 1e-8 per 3D Helmholtz solve.

Workload (default): the 128^3 heterogeneous medium (1500 -> 3000 m/s linear
depth gradient along y, three seeded Gaussian anomalies of +-20 %, radius
8-15 h), h = 10 m, 12-point PML on every face, 8 points per minimum
wavelength, 16 seeded Gaussian point sources; the 7-point PML operator
solved by FGMRES(20) to ||f - A u|| / ||f|| <= 1e-8 for every source.
Inputs are synthetic (seeded splitmix64), no dataset is read.

One step = one medium: set-up + block LU factor of all kz systems + one
lockstep batched FGMRES over the 16 sources, with the preconditioner in
complex64 and the z-transform in the PML eigenbasis (outer loop, operator
and Gram-Schmidt in complex128).  `value` is seconds per source-solve (step
time / 16) with the medium and the sources resident on the device, timed
with CUDA events on the solver's stream.  Beside it: the same preconditioner
with one source per step, the FFT-z preconditioner (the reference's method)
in complex64, and the plain complex128 FFT-z path with one source per step
(`fp64_plain`, the drop-in baseline).  `e2e` repeats the headline step
through the C ABI with pinned host buffers (medium and sources copied in,
solutions copied out inside the timed region).

    python bench.py [--steps K] [--warmup W] [--impl ours|reference] [--grid 128]
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
BATCH = 16
# FGMRES iterations the complex128 FFT-z path needs at the 128^3 workload
# (measured on a B200 with this bench: 513); the CPU port times a sample of
# iterations and scales to this count.
ITERS_128 = 513


def workload(n: int, nsrc: int = 1):
    """The 128^3 heterogeneous medium recipe at size n with nsrc seeded
    sources (the medium does not depend on nsrc; source 0 is the same)."""
    from helm3d import media
    p = media.layered_medium(n, n, n, 10.0, 12, 2024, ppw=8.0, n_sources=nsrc)
    p.meta["config"] = "C2"
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


def dist_max(dist, x: float, device=None) -> float:
    """Max of a per-rank float over all ranks (identity without a process group)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def init_dist(world: int):
    """One process per GPU over NCCL (gloo where no GPU is visible), with a
    short timeout so that ranks waiting on a dead peer end with an error."""
    if world <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as tdist
    if torch.cuda.is_available():
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        backend = "nccl"
    else:
        backend = "gloo"
    tdist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return tdist


# ---------------------------------------------------------------- GPU arm
def run_ours(args, rank, world, dist):
    import torch

    import helm3d

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    p = workload(args.n, BATCH)
    F_host = np.stack([p.rhs(i) for i in range(BATCH)])
    s2_host = np.ascontiguousarray(p.s2)
    grid = helm3d.grid_mode_n(p.nx, p.ny, p.nz, p.h, p.pml, p.omega)
    N = p.nx * p.ny * p.nz
    # a dedicated stream: the solver's launches and the timing events share it
    stream = torch.cuda.Stream(dev)

    F_dev = torch.from_numpy(F_host).to(dev)
    s2_dev = torch.from_numpy(s2_host).to(dev)
    U_dev = torch.empty_like(F_dev)

    def make(prec, zt):
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
        return dist_max(dist, x, dev)

    def step(s, nrhs, s2=s2_dev, F=F_dev, U=U_dev):
        s.set_medium(s2)
        s.solve(F[:nrhs], nrhs=nrhs, u=U[:nrhs], allow_not_converged=True)

    def timed_steps(s, nrhs, steps, warmup):
        """ms per step (max over ranks), iterations per source of the last
        step, launches in the timed region, last stats."""
        for _ in range(warmup):
            step(s, nrhs)
        barrier()
        launches0 = s.kernel_launches
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step(s, nrhs)
        e1.record(stream)
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1) / steps)
        st = s.last_stats
        return ms, st.iterations / nrhs, s.kernel_launches - launches0, st

    def profiled(s, nrhs):
        s.profile(True)
        step(s, nrhs)
        prof = s.profile_read()
        s.profile(False)
        return prof

    # headline: eigenbasis z-transform, complex64 preconditioner, 16 sources per step
    sh = make(helm3d.PREC_C64, helm3d.ZT_PML_EIGEN)
    clocks = Clocks(dev.index)
    clocks.start()
    time.sleep(1.5)   # let the sampler start up before the timed region
    ms_h, its_h, launches_h, st_h = timed_steps(sh, BATCH, args.steps, args.warmup)
    clk = clocks.stop()
    prof = profiled(sh, BATCH)
    relres_h = sh.last_stats.relres
    U_h = U_dev.clone()

    # e2e through the C ABI with host buffers (pinned): medium and sources in,
    # solutions out, every step
    F_pin = torch.from_numpy(F_host).pin_memory()
    s2_pin = torch.from_numpy(s2_host).pin_memory()
    U_pin = torch.empty_like(F_pin).pin_memory()
    step(sh, BATCH, s2_pin, F_pin, U_pin)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step(sh, BATCH, s2_pin, F_pin, U_pin)
    e1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    # the same preconditioner, one source per step
    ms_1, its_1, _, _ = timed_steps(sh, 1, args.steps, 1)
    sh.close()

    # the reference's method (FFT-z) with the complex64 preconditioner, one source
    sf = make(helm3d.PREC_C64, helm3d.ZT_FFT)
    ms_f, its_f, _, st_f = timed_steps(sf, 1, max(1, args.steps // 2), 1)
    relres_f = st_f.relres
    sf.close()

    # plain complex128 FFT-z path, one source per step
    s64 = make(helm3d.PREC_C128, helm3d.ZT_FFT)
    ms64, its64, _, st64 = timed_steps(s64, 1, max(1, args.steps // 2), 1)
    u64 = U_dev[0].clone()
    relres64 = st64.relres
    s64.close()
    relerr = float(torch.linalg.vector_norm(U_h[0] - u64) / torch.linalg.vector_norm(u64))

    if rank != 0:
        return None

    # roofline of the dominant single kernel of the headline step (the
    # preconditioner kernels; the Krylov family is several kernels)
    e = 8
    nbytes = {
        # G^T read in both passes, planes of all sources read + written in both
        "sweep": 2.0 * p.nz * p.ny * p.nx * p.nx * e + 4.0 * N * e * BATCH,
        # x (complex128) in, planes (complex64) out; W from L2
        "fft_fwd": (16.0 + e) * N * BATCH,
        "fft_inv": (16.0 + e) * N * BATCH,
        "stencil": (16.0 * 2 + 8.0) * N * BATCH,
    }
    top = max(nbytes, key=lambda k: prof[k][0])
    # DRAM read + write of one launch of the tensor-core sweep on this
    # workload (128^3, 16 sources), measured with ncu (dram__bytes_read.sum
    # + dram__bytes_write.sum of one captured launch)
    traffic = 5.273e9 if (top == "sweep" and p.nx == 128 and BATCH == 16) else None
    k_ms, k_n = prof[top]
    avg_s = (k_ms / max(1, k_n)) / 1e3
    achieved = nbytes[top] / avg_s / 1e9 if avg_s > 0 else None
    peak, peak_kind = read_peaks()
    total_prof = sum(v[0] for v in prof.values())
    per_src = ms_h / BATCH
    line = {
        "metric": METRIC,
        "value": per_src / 1e3 / world,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_h,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c64 preconditioner / c128 outer",
        "data": "synthetic (seeded splitmix64 medium and sources)",
        "config": {
            "workload": f"{p.nx}^3 heterogeneous medium, PML 12, 8 ppw, {BATCH} Gaussian sources; one step = "
                        f"set-up + block LU factor + batched FGMRES({RESTART}) to 1e-8 for all sources; "
                        f"value = step time / {BATCH}",
            "n": p.nx, "pml": p.pml, "sources_per_step": BATCH, "restart": RESTART, "tol": TOL,
            "beta_prec": BETA_PREC, "z_transform": "PML eigenbasis",
            "l2": "inputs larger than L2 (factor 2.1 GB, sources 0.54 GB, Krylov bases 22 GB)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        },
        "solves_per_s": world * 1e3 / per_src,
        "iterations_per_source": its_h,
        "relres": relres_h,
        "relerr_vs_fp64_plain": relerr,
        "single_source": {"value": ms_1 / 1e3 / world, "unit": "s", "iterations": its_1},
        "fft_z_c64_single": {"value": ms_f / 1e3 / world, "unit": "s", "iterations": its_f, "relres": relres_f},
        "fp64_plain": {"value": ms64 / 1e3 / world, "unit": "s", "iterations": its64, "relres": relres64},
        "speedup_vs_fp64_plain": (ms64 / per_src) if per_src > 0 else None,
        "e2e": {"value": e2e_ms / BATCH / 1e3 / world, "unit": "s",
                "h2d_bytes_per_step": N * 8 + BATCH * N * 16, "d2h_bytes_per_step": BATCH * N * 16},
        "gpu_launches": int(launches_h),
        "roofline": {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                     "bytes_per_launch": nbytes[top], "traffic": traffic},
        "kernel_ms_per_step": {k: round(v[0], 3) for k, v in prof.items()},
        "kernel_launches_per_step": {k: int(v[1]) for k, v in prof.items()},
        "kernel_share": {k: round(v[0] / total_prof, 4) for k, v in prof.items()} if total_prof > 0 else None,
        "clocks": clk,
    }
    return line, round(its64) if its64 else None


# ------------------------------------------------------ kernel microbench
def run_kernels(args):
    """Per-kernel device times of one batched FGMRES(1) iteration (one
    preconditioner apply and one operator apply for all 16 sources, plus the
    Gram-Schmidt and residual kernels) on the headline workload, with the
    algorithmic bytes and HBM fraction of each kernel family.  The solver
    holds only two Krylov vectors per source (about 4 GB on the device at
    128^3), which keeps profiler captures of these kernels small."""
    import torch

    import helm3d

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    p = workload(args.n, BATCH)
    F = torch.from_numpy(np.stack([p.rhs(i) for i in range(BATCH)])).to(dev)
    U = torch.empty_like(F)
    grid = helm3d.grid_mode_n(p.nx, p.ny, p.nz, p.h, p.pml, p.omega)
    o = helm3d.default_opts(precision=helm3d.PREC_C64, restart=1, tol=TOL, beta_prec=BETA_PREC, max_iter=1,
                            device=0, z_transform=helm3d.ZT_PML_EIGEN)
    s = helm3d.Solver(grid, torch.from_numpy(np.ascontiguousarray(p.s2)).to(dev), o)
    for _ in range(args.warmup):
        s.solve(F, nrhs=BATCH, u=U, allow_not_converged=True)
    torch.cuda.synchronize()
    s.profile(True)
    for _ in range(args.steps):
        s.solve(F, nrhs=BATCH, u=U, allow_not_converged=True)
    prof = s.profile_read()
    s.close()
    N = p.nx * p.ny * p.nz
    e = 8
    nbytes = {
        "sweep": 2.0 * p.nz * p.ny * p.nx * p.nx * e + 4.0 * N * e * BATCH,
        "fft_fwd": (16.0 + e) * N * BATCH,
        "fft_inv": (16.0 + e) * N * BATCH,
    }
    peak, peak_kind = read_peaks()
    out = {"mode": "kernels", "workload": f"{p.nx}^3, {BATCH} sources, c64 preconditioner, PML eigenbasis",
           "steps": args.steps, "peak_gbs": peak, "peak_source": peak_kind, "kernels": {}}
    for k, (ms, n) in prof.items():
        d = {"ms_total": round(ms, 4), "launches": int(n)}
        if n and k in nbytes:
            avg = ms / n / 1e3
            d["bytes_per_launch"] = nbytes[k]
            d["achieved_gbs"] = nbytes[k] / avg / 1e9
            d["frac"] = d["achieved_gbs"] / peak
        out["kernels"][k] = d
    return out


# ------------------------------------------------- the other configurations
def _solver(helm3d, p, s2, prec, zt, restart=RESTART, tol=TOL, stream=None):
    g = helm3d.grid_mode_n(p.nx, p.ny, p.nz, p.h, p.pml, p.omega)
    o = helm3d.default_opts(precision=prec, restart=restart, tol=tol, beta_prec=BETA_PREC, max_iter=20000,
                            device=0, z_transform=zt)
    s = helm3d.Solver(g, s2, o)
    if stream is not None:
        s.set_stream(stream)
    return s


def _events_ms(stream, fn, steps):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def run_large(args, n: int, restart: int, label: str):
    """One n^3 heterogeneous medium (the 128^3 recipe at size n): time per
    source-solve of the batched complex64 preconditioner (16 sources, PML
    eigenbasis), of one source with it, and of the plain complex128 FFT-z path
    with one source; each step includes set-up and factor.  The complex64
    solutions' error is measured against the complex128 solution."""
    import torch

    import helm3d
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    p = helm3d_media().layered_medium(n, n, n, 10.0, 12 if n < 200 else 16, 2024, ppw=8.0, n_sources=BATCH)
    F = torch.from_numpy(np.stack([p.rhs(i) for i in range(BATCH)])).to(dev)
    s2 = torch.from_numpy(np.ascontiguousarray(p.s2)).to(dev)
    U = torch.empty_like(F)
    out = {"mode": label, "workload": f"{n}^3 heterogeneous medium (1500->3000 m/s depth gradient, three +-20 % "
                                      f"anomalies), PML {p.pml}, 8 ppw; FGMRES({restart}) to {TOL}; each step "
                                      f"= set-up + factor + solve", "n": n}
    res = {}
    for name, prec, zt, nrhs in (("batched16_c64_eigen", helm3d.PREC_C64, helm3d.ZT_PML_EIGEN, BATCH),
                                 ("single_c64_eigen", helm3d.PREC_C64, helm3d.ZT_PML_EIGEN, 1),
                                 ("fp64_plain", helm3d.PREC_C128, helm3d.ZT_FFT, 1)):
        s = _solver(helm3d, p, s2, prec, zt, restart=restart, stream=stream)

        def step():
            s.set_medium(s2)
            s.solve(F[:nrhs], nrhs=nrhs, u=U[:nrhs], allow_not_converged=True)
        for _ in range(args.warmup):
            step()
        ms = _events_ms(stream, step, args.steps)
        st = s.last_stats
        res[name] = {"s_per_solve": ms / 1e3 / nrhs, "ms_per_step": ms, "sources": nrhs,
                     "iterations_per_source": st.iterations / nrhs, "relres": st.relres}
        if name == "batched16_c64_eigen":
            Ub = U.clone()
        s.close()
    u64 = U[0]
    res["batched16_c64_eigen"]["relerr_vs_fp64"] = float(torch.linalg.vector_norm(Ub[0] - u64) /
                                                         torch.linalg.vector_norm(u64))
    out["results"] = res
    out["speedup_batched_vs_fp64_plain"] = res["fp64_plain"]["s_per_solve"] / res["batched16_c64_eigen"]["s_per_solve"]
    out["speedup_single_vs_fp64_plain"] = res["fp64_plain"]["s_per_solve"] / res["single_c64_eigen"]["s_per_solve"]
    return out


def run_group(args):
    """16 sources on a 96^3 medium plus 8 uneven grids with one source each,
    every grid its own medium: set-up and factor of all nine contexts, then
    one grouped FGMRES (restart cycles of all grids in one CUDA graph),
    against the same contexts solved one after another."""
    import torch

    import helm3d
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    probs = helm3d_media().config_c4()
    Fs = [torch.from_numpy(np.stack([p.rhs(i) for i in range(len(p.sources))])).to(dev) for p in probs]
    S2 = [torch.from_numpy(np.ascontiguousarray(p.s2)).to(dev) for p in probs]
    Us = [torch.empty_like(f) for f in Fs]
    ss = [_solver(helm3d, p, s2, helm3d.PREC_C64, helm3d.ZT_PML_EIGEN, stream=stream) for p, s2 in zip(probs, S2)]
    nsol = sum(int(f.shape[0]) for f in Fs)

    def setup():
        for s, s2 in zip(ss, S2):
            s.set_medium(s2)

    def grouped():
        setup()
        helm3d.solve_group(ss, Fs, us=Us, allow_not_converged=True)

    def one_by_one():
        setup()
        for s, f, u in zip(ss, Fs, Us):
            s.solve(f, nrhs=int(f.shape[0]), u=u, allow_not_converged=True)

    out = {"mode": "group", "workload": "16 sources on 96^3 + 8 uneven grids (" +
           ", ".join(f"{p.nx}x{p.ny}x{p.nz}" for p in probs[1:]) + "), one source each, own media, PML 8; "
           f"c64 preconditioner (PML eigenbasis), FGMRES({RESTART}) to {TOL}; step = set-up + factor of all "
           "grids + solve", "solves_per_step": nsol}
    for name, fn in (("grouped", grouped), ("one_by_one", one_by_one)):
        for _ in range(args.warmup):
            fn()
        ms = _events_ms(stream, fn, args.steps)
        out[name] = {"ms_per_step": ms, "s_per_solve": ms / 1e3 / nsol,
                     "iterations": [s.last_stats.iterations for s in ss],
                     "relres_max": max(s.last_stats.relres for s in ss)}
    for s in ss:
        s.close()
    return out


def run_gradient(args):
    """The misfit gradient on the 200^3 configuration (PML 16, 8 sources,
    50 x 50 receivers at the top of the interior, data from a model with
    +-10 % anomalies, gradient at the smooth starting model): time of one
    helm3d_misfit_grad (forward solves, adjoint solves, gradient kernel; the
    factor of the starting model is set-up), and central finite differences
    of the misfit on 20 seeded interior cells.  J(s2 +- d e_c) is evaluated
    exactly from the base solutions by the rank-one update of A (Sherman-
    Morrison: u' = u - k w u_c / (1 + k w_c), w = A^{-1} e_c, k = omega^2
    (1 + i beta) d), one extra solve per cell and no refactorization, so
    that the difference is free of the solver's tolerance."""
    import torch

    import helm3d
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    start, true, recv = helm3d_media().config_c5(n=args.n if args.n != 128 else 200)
    ns = len(true.sources)
    F = torch.from_numpy(np.stack([true.rhs(i) for i in range(ns)])).to(dev)
    rec = torch.from_numpy(recv).to(dev)
    tol = 1e-10
    # data from the true model
    st_ = _solver(helm3d, true, torch.from_numpy(np.ascontiguousarray(true.s2)).to(dev), helm3d.PREC_C64,
                  helm3d.ZT_PML_EIGEN, restart=30, tol=tol, stream=stream)
    Ut = st_.solve(F, nrhs=ns)
    data = Ut.reshape(ns, -1)[:, rec].contiguous()
    st_.close()
    del Ut
    s2 = torch.from_numpy(np.ascontiguousarray(start.s2)).to(dev)
    s = _solver(helm3d, start, s2, helm3d.PREC_C64, helm3d.ZT_PML_EIGEN, restart=30, tol=tol, stream=stream)
    for _ in range(args.warmup):
        s.misfit_grad(F, rec, data)
    box = {}

    def grad_step():
        box["J"], box["g"] = s.misfit_grad(F, rec, data)
    ms = _events_ms(stream, grad_step, args.steps)
    its = s.last_stats.iterations
    J, g = box["J"], box["g"].reshape(-1)
    # base solutions and the finite differences
    U = s.solve(F, nrhs=ns).reshape(ns, -1)
    rng = helm3d_media().SplitMix64(77)
    nz, ny, nx = start.shape
    pm = start.pml + 4
    cells = []
    while len(cells) < 20:
        i, j, k = (rng.randint(pm, nx - 1 - pm), rng.randint(pm, ny // 2), rng.randint(pm, nz - 1 - pm))
        cells.append((k * ny + j) * nx + i)
    E = torch.zeros((len(cells), nz * ny * nx), dtype=torch.complex128, device=dev)
    for q, c in enumerate(cells):
        E[q, c] = 1.0
    W = torch.empty_like(E)
    for q0 in range(0, len(cells), BATCH):
        q1 = min(len(cells), q0 + BATCH)
        s.solve(E[q0:q1], nrhs=q1 - q0, u=W[q0:q1])
    resid = U[:, rec] - data                                   # (ns, nrecv)
    kap0 = start.omega ** 2 * complex(1.0, start.beta_phys)
    fd, ad = [], []
    for q, c in enumerate(cells):
        delta = 1e-3 * float(s2.reshape(-1)[c])
        dJ = []
        for sgn in (1.0, -1.0):
            kap = kap0 * sgn * delta
            wc = W[q, c]
            du = -kap * W[q, rec][None, :] * (U[:, c][:, None] / (1.0 + kap * wc))   # P (u' - u)
            dJ.append(float((torch.real(torch.conj(resid) * du)).sum() + 0.5 * (du.abs() ** 2).sum()))
        fd.append((dJ[0] - dJ[1]) / (2 * delta))
        ad.append(float(g[c]))
    fd, ad = np.array(fd), np.array(ad)
    relerr = np.abs(fd - ad) / np.maximum(np.abs(fd), 1e-300)
    s.close()
    return {"mode": "gradient", "workload": f"{nx}^3 (PML {start.pml}), {ns} sources, {len(recv)} receivers; "
            f"gradient of 0.5||P u - d||^2 w.r.t. s^2 at the smooth starting model; c64 preconditioner, "
            f"FGMRES(30) to {tol}", "ms_per_gradient": ms, "iterations": its, "misfit": J,
            "fd_cells": len(cells), "fd_relerr_max": float(relerr.max()), "fd_relerr_median": float(np.median(relerr)),
            "fd_step": "1e-3 s^2 at the cell (central)"}


def helm3d_media():
    from helm3d import media
    return media


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
        "config": {"workload": f"{p.nx}^3 heterogeneous medium, PML 12, 8 ppw, Gaussian source; the reference's "
                               f"method (FFT-z + per-kz sparse LU, FGMRES({RESTART}) to 1e-8, complex128) per "
                               f"source-solve", "n": p.nx},
        "cpu_baseline": base,
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", dest="n", type=int, default=128, help="grid points per axis")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--kernels", action="store_true",
                    help="per-kernel microbench: batched FGMRES(1) iterations instead of full solves")
    ap.add_argument("--workload", default="headline", choices=["headline", "c3", "c4", "c5", "n200"],
                    help="c3: 160^3 mixed precision, FGMRES(30); c4: 96^3 x 16 sources + 8 uneven grids as one "
                         "group; c5: 200^3 misfit gradient with finite-difference check; n200: 200^3 batched "
                         "complex64 vs plain complex128")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.kernels:
        print(json.dumps(run_kernels(args)))
        return
    if args.workload != "headline" and args.impl == "ours":
        if args.workload == "c3":
            out = run_large(args, 160, 30, "c3")
        elif args.workload == "n200":
            out = run_large(args, 200, RESTART, "n200")
        elif args.workload == "c4":
            out = run_group(args)
        else:
            out = run_gradient(args)
        print(json.dumps(out))
        return
    if args.impl == "reference":
        # the CPU reference runs on rank 0 only; the other ranks exit at once
        out = run_reference(args, rank)
        if rank == 0 and out is not None:
            print(json.dumps(out))
        return
    dist = init_dist(world)
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
