"""Benchmark: time to relative residual 1e-8 per 3D Helmholtz solve.

Workload (default): the 200^3 heterogeneous medium (1500 -> 3000 m/s linear
depth gradient along y, three seeded Gaussian anomalies of +-20 %, radius
8-15 h), h = 10 m, 16-point PML on every face, 8 points per minimum
wavelength, 16 seeded Gaussian point sources; the 7-point PML operator
solved by FGMRES(20) to ||f - A u|| / ||f|| <= 1e-8 for every source.
Inputs are synthetic (seeded splitmix64), no dataset is read.  `--grid 128`
selects the 128^3 medium of the same recipe with a 12-point PML.

One step = one medium: set-up + block LU factor of all kz systems + one
lockstep batched FGMRES over the 16 sources, with the preconditioner in
complex64 and the z-transform in the PML eigenbasis (outer loop, operator
and Gram-Schmidt in complex128).  `value` is seconds per source-solve (step
time / 16) with the medium and the sources resident on the device, timed
with CUDA events on the solver's stream.  Both call the C ABI's
helm3d_solve_medium (medium, factor and solve in one call).  `e2e` repeats
the headline step with pinned host buffers (medium and sources copied in,
the sources while the medium is factored, solutions copied out, all inside
the timed region).

Beside the headline, one step each (after one warm-up step) of the same
workload solved other ways, so that each stated change can be read apart:

  fp64_plain          FFT-z, complex128 preconditioner, one source per step
                      (the plain FP64 GPU drop-in of the reference's method)
  fft_z_c64_single    FFT-z, complex64 preconditioner, one source
  fft_z_c64_batched   FFT-z, complex64 preconditioner, 16 sources in lockstep
  eigen_c128_single   PML eigenbasis, complex128 preconditioner, one source
  single_source       PML eigenbasis, complex64 preconditioner, one source
  kz_skip_5           the headline with the reference's SAVE_MEM skipping at
                      its ratio 5 (a further method change, not the headline)

The eigenbasis arms use the preconditioner shift beta_prec = 0.01, the FFT-z
arms 0.25 (see BETA_PREC_EIGEN).

Every arm's source-0 solution is compared with the FP64 oracle's solution
of the same source (tests/golden/port_*_n<grid>.npz, a strided sample).

    python bench.py [--steps K] [--warmup W] [--impl ours|reference] [--grid 200]
    torchrun --nproc-per-node N bench.py --gpus N     (N independent replicas)

`--impl reference` times the CPU port of the reference's method (oracle.port:
FFT-z + one SuperLU factor per kz + FGMRES(20) in complex128 on every host
core) on the same workload; see run_reference.
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
GOLDEN = os.path.join(REPO, "tests", "golden")
for _p in (REPO, PKG_DIR):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "time to 1e-8 residual per 3D solve: FP32-precond/batched vs plain FP64 GPU"
TOL = 1e-8
RESTART = 20
# the preconditioner's complex shift: the FFT-z preconditioner needs damping
# (the FFT does not represent the z PML; 0.25 from the 64^3 oracle runs); the
# PML-eigenbasis one is exact along z, and a small shift takes the 200^3
# workload from 32.7 iterations per source at 0.25 to 8 at 0.01 (7 at 0; 128^3
# 22.4 -> 7-8, 160^3 27.7 -> 8.2 at 0.02), 0.01 keeping a margin of damping
BETA_PREC = 0.25
BETA_PREC_EIGEN = 0.01
BATCH = 16
SAMPLE_STRIDE = 8


def beta_for(zt) -> float:
    import helm3d
    return BETA_PREC_EIGEN if zt == helm3d.ZT_PML_EIGEN else BETA_PREC


def pml_for(n: int) -> int:
    return 16 if n >= 200 else 12


def workload(n: int, nsrc: int = BATCH):
    """The heterogeneous medium recipe at size n with nsrc seeded sources
    (the medium does not depend on nsrc; source 0 is the same)."""
    from helm3d import media   # pure Python: loads no native library
    p = media.layered_medium(n, n, n, 10.0, pml_for(n), 2024, ppw=8.0, n_sources=nsrc)
    p.meta["config"] = "C5-forward" if n == 200 else "C2"
    return p


def workload_config(n: int) -> dict:
    """The `config` object of both arms' lines: what is solved, not how."""
    return {
        "workload": f"{n}^3 heterogeneous medium (1500->3000 m/s depth gradient, three +-20 % Gaussian "
                    f"anomalies), h = 10 m, PML {pml_for(n)} on all faces, 8 ppw, {BATCH} seeded Gaussian "
                    f"sources; 7-point PML operator solved to ||f - A u|| / ||f|| <= {TOL} per source; "
                    f"value = seconds per source-solve including set-up and factor",
        "n": n, "pml": pml_for(n), "sources": BATCH, "tol": TOL, "restart": RESTART,
        "l2": "inputs larger than L2 (Krylov bases and factor tens of GB; sources alone 2 GB at 200^3)",
    }


def oracle_record(n: int, kind: str):
    """The oracle port's full solve of source 0 at grid n (kind "fftz": the
    reference's method to 1e-8; "eigen": to 1e-12), or None."""
    path = os.path.join(GOLDEN, f"port_{kind}_n{n}.npz")
    if not os.path.exists(path):
        return None
    d = np.load(path)
    return {k: d[k] for k in d.files}


def sample_err(u0, rec):
    """Relative error of a source-0 solution (torch or NumPy, (nz, ny, nx))
    against the oracle's strided sample."""
    if rec is None:
        return None
    s = int(rec["stride"])
    a = u0[::s, ::s, ::s]
    a = a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)
    ref = rec["sample"]
    return float(np.linalg.norm(a - ref) / np.linalg.norm(ref))


def read_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return d, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def native_libs_loaded():
    """In-tree shared objects mapped into this process (Linux)."""
    out = set()
    try:
        with open("/proc/self/maps") as fh:
            for line in fh:
                path = line.rsplit(None, 1)[-1]
                if path.endswith(".so") and path.startswith(REPO):
                    out.add(os.path.relpath(path, REPO))
    except OSError:
        pass
    return sorted(out)


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


# ---------------------------------------------------------------- GPU arm
def family_bytes_flops(p, its_per_source: float, nsrc: int, e: int = 8):
    """Algorithmic bytes (HBM families) or flops (factor) per launch of each
    kernel family on the headline step; Krylov is per step (its launches
    differ in size), from the mean Arnoldi step over a restart cycle."""
    N = p.nx * p.ny * p.nz
    R = nsrc
    # DCGS2 step j of a restart cycle moves (2j + 5) 16 N bytes per source: a
    # cycle of L steps sum_j (2j + 5) = L^2 + 4 L; k iterations = full cycles
    # of RESTART steps and a last one of the rest
    k = float(its_per_source)
    full = math.floor(k / RESTART)
    rest = k - full * RESTART
    krylov_step = 16.0 * N * R * (full * (RESTART * RESTART + 4 * RESTART) + rest * rest + 4 * rest)
    return {
        # G^T read forward and backward + the planes of all sources read and written in both passes
        "sweep": ("hbm", 2.0 * p.nz * p.ny * p.nx * p.nx * e + 4.0 * N * e * R),
        # complex128 x in, planes out (forward); planes in, FGMRES's Z_j out,
        # complex64 with the complex64 preconditioner (inverse)
        "fft_fwd": ("hbm", (16.0 + e) * N * R),
        "fft_inv": ("hbm", (e + e) * N * R),
        # Z_j (complex64) read, w (complex128) written per source, s2 once
        # per z chunk (source-minor order)
        "stencil": ("hbm", (e + 16.0) * N * R + 8.0 * N),
        # 8 nx^3 real flops per (kz, y-line) block, per step (the family's
        # second launch, the blocks' power-of-two scales, takes ~1 %)
        "factor": ("tensor_per_step", 8.0 * p.nx ** 3 * p.ny * p.nz),
        "krylov": ("hbm_per_step", krylov_step),
    }


def roofline_table(p, prof, its_per_source, nsrc, peaks):
    fam = family_bytes_flops(p, its_per_source, nsrc)
    hbm = float(peaks["hbm_gbs"])
    tc = float(peaks.get("bf16_tflops_sustained") or peaks["bf16_tflops"])
    out = {}
    for k, (ms, n) in prof.items():
        if not n or k not in fam:
            continue
        kind, amount = fam[k]
        if kind == "hbm_per_step":
            t = ms / 1e3
            ach = amount / t / 1e9
            out[k] = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                      "bytes_per_step": amount, "ms_per_step": ms, "launches": int(n)}
            continue
        if kind == "tensor_per_step":
            t = ms / 1e3
            ach = amount / t / 1e12
            out[k] = {"bound": "tensor", "achieved": ach, "peak": tc, "unit": "TFLOP/s", "frac": ach / tc,
                      "flops_per_step": amount, "ms_per_step": ms, "launches": int(n)}
            continue
        t = ms / n / 1e3
        if kind == "hbm":
            ach = amount / t / 1e9
            out[k] = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                      "bytes_per_launch": amount, "ms_per_launch": ms / n, "launches": int(n)}
        else:
            ach = amount / t / 1e12
            out[k] = {"bound": "tensor", "achieved": ach, "peak": tc, "unit": "TFLOP/s", "frac": ach / tc,
                      "flops_per_launch": amount, "ms_per_launch": ms / n, "launches": int(n)}
    return out


# DRAM read + write of one launch (ncu: dram__bytes_read.sum +
# dram__bytes_write.sum of one captured launch), per (family, grid, sources)
TRAFFIC = {
    ("sweep", 128, 16): 5.273e9,
    # the 200 x 200 x 32 capture of the packed sweep (4.825 GB) scaled by the kz chains, 200 / 32
    ("sweep", 200, 16): 30.16e9,
}


def run_ours(args, rank, world, dist):
    import torch

    import helm3d

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    n = args.n
    p = workload(n, BATCH)
    F_host = np.stack([p.rhs(i) for i in range(BATCH)])
    s2_host = np.ascontiguousarray(p.s2)
    grid = helm3d.grid_mode_n(p.nx, p.ny, p.nz, p.h, p.pml, p.omega)
    N = p.nx * p.ny * p.nz
    # a dedicated stream: the solver's launches and the timing events share it
    stream = torch.cuda.Stream(dev)

    F_dev = torch.from_numpy(F_host).to(dev)
    s2_dev = torch.from_numpy(s2_host).to(dev)
    U_dev = torch.empty_like(F_dev)
    rec_eig = oracle_record(n, "eigen")
    rec_fft = oracle_record(n, "fftz")

    def make(prec, zt, skip=0.0):
        o = helm3d.default_opts(precision=prec, restart=RESTART, tol=TOL, beta_prec=beta_for(zt), max_iter=20000,
                                device=dev.index, z_transform=zt, kz_skip_ratio=skip)
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
        # helm3d_solve_medium: set-up, factor and solve in one call (with host
        # buffers the sources are copied in while the medium is factored)
        s.solve_medium(s2, F[:nrhs], nrhs=nrhs, u=U[:nrhs], allow_not_converged=True)

    def timed_steps(s, nrhs, steps, warmup, s2=s2_dev, F=F_dev, U=U_dev):
        """ms per step (max over ranks), iterations per source of the last
        step, launches in the timed region, last stats."""
        for _ in range(warmup):
            step(s, nrhs, s2, F, U)
        barrier()
        launches0 = s.kernel_launches
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step(s, nrhs, s2, F, U)
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
    relres_h = st_h.relres
    err_h = sample_err(U_dev[0], rec_eig)
    prof = profiled(sh, BATCH)

    # e2e through the C ABI with host buffers (pinned): medium and sources in,
    # solutions out, every step
    F_pin = torch.from_numpy(F_host).pin_memory()
    s2_pin = torch.from_numpy(s2_host).pin_memory()
    U_pin = torch.empty_like(F_pin).pin_memory()
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    e2e_ms, _, _, _ = timed_steps(sh, BATCH, e2e_steps, 1, s2_pin, F_pin, U_pin)
    del F_pin, U_pin, s2_pin
    sh.close()

    # the same workload solved other ways, one step each after a warm-up step
    # kz_skip_5: the headline with the reference's SAVE_MEM option at its
    # ratio (5): modes with kz^2 >= 5 k^2 not factored, solved by their
    # diagonal (a stated method change, so not the headline itself)
    arms = {}
    for name, prec, zt, nrhs, skip in (("single_source", helm3d.PREC_C64, helm3d.ZT_PML_EIGEN, 1, 0.0),
                                       ("kz_skip_5", helm3d.PREC_C64, helm3d.ZT_PML_EIGEN, BATCH, 5.0),
                                       ("fft_z_c64_batched", helm3d.PREC_C64, helm3d.ZT_FFT, BATCH, 0.0),
                                       ("fft_z_c64_single", helm3d.PREC_C64, helm3d.ZT_FFT, 1, 0.0),
                                       ("eigen_c128_single", helm3d.PREC_C128, helm3d.ZT_PML_EIGEN, 1, 0.0),
                                       ("fp64_plain", helm3d.PREC_C128, helm3d.ZT_FFT, 1, 0.0)):
        if name in args.skip_arms:
            continue
        s = make(prec, zt, skip)
        ms, its, _, st = timed_steps(s, nrhs, args.arm_steps, 1)
        arms[name] = {"value": ms / nrhs / 1e3 / world, "unit": "s", "ms_per_step": ms, "sources_per_step": nrhs,
                      "iterations_per_source": its, "relres": st.relres,
                      "relerr_vs_fp64_oracle": sample_err(U_dev[0], rec_eig),
                      "precision": "c64" if prec == helm3d.PREC_C64 else "c128",
                      "z_transform": "fft" if zt == helm3d.ZT_FFT else "PML eigenbasis"}
        if skip > 0:
            arms[name]["kz_skip_ratio"] = skip
        s.close()

    if rank != 0:
        return None

    peaks, peak_kind = read_peaks()
    table = roofline_table(p, prof, its_h, BATCH, peaks)
    # the dominant single kernel: the family with the largest device time
    # whose launches are one kernel each (Krylov is several kernels per step)
    single = {k: v for k, v in prof.items() if k in table and k != "krylov"}
    top = max(single, key=lambda k: single[k][0])
    r = dict(table[top])
    r["kernel"] = top
    r["peak_source"] = peak_kind
    r["traffic"] = TRAFFIC.get((top, n, BATCH))
    total_prof = sum(v[0] for v in prof.values())
    per_src = ms_h / BATCH

    def ratio(a, b):
        return (a / b) if (a and b) else None

    fp = arms.get("fp64_plain", {}).get("value")
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
        "config": dict(workload_config(n), parallelism=f"replicas x{world}" if world > 1 else "single GPU"),
        "method": f"PML-eigenbasis z-transform, complex64 preconditioner (tcgen05 sweep and z-transforms), "
                  f"complex128 FGMRES({RESTART}) with DCGS2, {BATCH} sources in lockstep, beta_prec {BETA_PREC_EIGEN} "
                  f"(FFT-z arms {BETA_PREC})",
        "solves_per_s": world * 1e3 / per_src,
        "iterations_per_source": its_h,
        "relres": relres_h,
        "relerr_vs_fp64_oracle": err_h,
        "oracle": {"eigen": f"tests/golden/port_eigen_n{n}.npz" if rec_eig is not None else None,
                   "fftz": f"tests/golden/port_fftz_n{n}.npz" if rec_fft is not None else None,
                   "compared_on": f"source 0, every {SAMPLE_STRIDE}th point per axis"},
        **arms,
        "speedup_vs_fp64_plain": ratio(fp, per_src / 1e3 / world),
        "forms_apart": {
            "precision_and_batching_under_fft_z": ratio(fp, arms.get("fft_z_c64_batched", {}).get("value")),
            "precision_alone_under_fft_z": ratio(fp, arms.get("fft_z_c64_single", {}).get("value")),
            "precision_and_batching_under_eigenbasis": ratio(arms.get("eigen_c128_single", {}).get("value"),
                                                             per_src / 1e3 / world),
            "z_transform_alone_c128": ratio(fp, arms.get("eigen_c128_single", {}).get("value")),
        },
        "e2e": {"value": e2e_ms / BATCH / 1e3 / world, "unit": "s", "steps": e2e_steps,
                "h2d_bytes_per_step": N * 8 + BATCH * N * 16, "d2h_bytes_per_step": BATCH * N * 16},
        "gpu_launches": int(launches_h),
        "roofline": r,
        "roofline_by_family": table,
        "kernel_ms_per_step": {k: round(v[0], 3) for k, v in prof.items()},
        "kernel_launches_per_step": {k: int(v[1]) for k, v in prof.items()},
        "kernel_share": {k: round(v[0] / total_prof, 4) for k, v in prof.items()} if total_prof > 0 else None,
        "clocks": clk,
    }
    if rec_fft is not None:
        line["oracle"]["fftz_iterations"] = int(rec_fft["iterations"])
    return line


def run_kernels(args):
    """Per-kernel device times of one batched FGMRES(1) iteration (one
    preconditioner apply and one operator apply for all 16 sources, plus the
    Gram-Schmidt and residual kernels) on the headline workload, with the
    algorithmic bytes and HBM fraction of each kernel family.  The solver
    holds only two Krylov vectors per source (about 4 GB on the device at
    128^3), which keeps profiler captures of these kernels small.  --nz
    shortens the z axis (fewer kz chains, the same block size) for captures
    of a single kernel."""
    import torch

    import helm3d

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    if args.nz and args.nz != args.n:
        from helm3d import media
        p = media.layered_medium(args.n, args.n, args.nz, 10.0, pml_for(min(args.n, args.nz)), 2024, ppw=8.0,
                                 n_sources=BATCH)
    else:
        p = workload(args.n, BATCH)
    F = torch.from_numpy(np.stack([p.rhs(i) for i in range(BATCH)])).to(dev)
    U = torch.empty_like(F)
    grid = helm3d.grid_mode_n(p.nx, p.ny, p.nz, p.h, p.pml, p.omega)
    o = helm3d.default_opts(precision=helm3d.PREC_C64, restart=1, tol=TOL, beta_prec=BETA_PREC_EIGEN, max_iter=1,
                            device=0, z_transform=helm3d.ZT_PML_EIGEN)
    s = helm3d.Solver(grid, torch.from_numpy(np.ascontiguousarray(p.s2)).to(dev), o)
    def one():
        if args.prec_applies:
            s.apply_prec_batch(F)   # launched one by one (no graph): profiler captures see each kernel
        else:
            s.solve(F, nrhs=BATCH, u=U, allow_not_converged=True)
    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    s.profile(True)
    for _ in range(args.steps):
        one()
    prof = s.profile_read()
    s.close()
    N = p.nx * p.ny * p.nz
    e = 8
    nbytes = {
        "sweep": 2.0 * p.nz * p.ny * p.nx * p.nx * e + 4.0 * N * e * BATCH,
        "fft_fwd": (16.0 + e) * N * BATCH,
        "fft_inv": (16.0 + e) * N * BATCH,
    }
    peaks, peak_kind = read_peaks()
    peak = float(peaks["hbm_gbs"])
    out = {"mode": "kernels" + (" (preconditioner applies)" if args.prec_applies else ""),
           "workload": f"{p.nx}x{p.ny}x{p.nz}, {BATCH} sources, c64 preconditioner, PML eigenbasis",
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
    o = helm3d.default_opts(precision=prec, restart=restart, tol=tol, beta_prec=beta_for(zt), max_iter=20000,
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


# ------------------------------------------------------------ CPU baseline
def port_iterations(n: int, workers: int):
    """FGMRES iterations the CPU port of the reference's method needs on
    source 0 of the n^3 workload: from its recorded full solve
    (tests/golden/port_fftz_n<n>.npz, made by `python -m oracle.port`), or,
    for small grids, from a full solve run here.  Never from a GPU run."""
    rec = oracle_record(n, "fftz")
    if rec is not None:
        return int(rec["iterations"]), f"the port's recorded full solve (tests/golden/port_fftz_n{n}.npz)"
    if n > 64:
        return None, f"no recorded full solve of the port at {n}^3"
    from oracle import port
    p = workload(n, 1)
    with port.PortPreconditioner(p, beta_prec=BETA_PREC, workers=workers) as pre:
        pre.factor()
        op = port.PortOperator(p, threads=workers)
        _, its, _, _, _ = port.fgmres(op, pre.apply, p.rhs(0), tol=TOL, m=RESTART, max_iter=20000)
    return its, "a full solve of the port run here"


class PortSample:
    """The CPU port of the reference's method on the workload: the factor of
    every kz system (timed in full) and real FGMRES(20) iterations of source
    0 from a zero start (each timed), with the host's cores."""

    def __init__(self, n: int, workers: int):
        from oracle import port
        self.port = port
        self.n = n
        self.workers = workers
        self.p = workload(n, 1)
        self.pre = port.PortPreconditioner(self.p, beta_prec=BETA_PREC, workers=workers)
        self.factor_s = self.pre.factor()
        self.op = port.PortOperator(self.p, threads=workers)
        f = self.p.rhs(0)
        t0 = time.perf_counter()
        r = f - self.op(np.zeros_like(f))
        np.linalg.norm(r)
        self.residual_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        self.pre.apply(f)
        self.apply_s = time.perf_counter() - t0

    def iterations(self, count: int):
        """Seconds of each of the first `count` FGMRES iterations."""
        _, _, _, _, times = self.port.fgmres(self.op, self.pre.apply, self.p.rhs(0), tol=TOL, m=RESTART,
                                             max_iter=count, max_cycles_iters=count)
        return times

    def close(self):
        self.pre.close()


def cpu_port_value(ps: PortSample, per_it: float, iters: int):
    restarts = max(1, math.ceil(iters / RESTART))
    return ps.factor_s + per_it * iters + (restarts + 1) * ps.residual_s


def cpu_port_sample(n: int, cores: int, sample_iters: int = RESTART):
    """cpu_baseline of the GPU line: the port's factor of all kz systems and
    its first restart cycle of FGMRES iterations on the workload (the
    Gram-Schmidt work grows along a cycle), scaled to the port's own
    iteration count."""
    iters, src = port_iterations(n, cores)
    if iters is None:
        return {"value": None, "unit": "s", "cores": cores, "kind": "port", "sample": src}
    ps = PortSample(n, cores)
    try:
        times = ps.iterations(sample_iters)
    finally:
        ps.close()
    per_it = statistics.mean(times)
    return {
        "value": cpu_port_value(ps, per_it, iters),
        "unit": "s",
        "cores": cores,
        "kind": "port",
        "sample": f"SuperLU factor of all {ps.p.nz} kz systems ({ps.factor_s:.1f} s) and the first "
                  f"{len(times)} FGMRES({RESTART}) iterations of source 0 ({per_it:.2f} s each: FFT-z, {ps.p.nz} 2D "
                  f"solves, 7-point operator, CGS2) on the {n}^3 workload, scaled to {iters} iterations "
                  f"({src}) plus one true residual per restart",
        "factor_s": ps.factor_s,
        "per_iteration_s": per_it,
        "iterations": iters,
    }


def run_reference(args, rank):
    """The reference's method on the host cores: the CPU port (oracle.port,
    the restatement of Source/FGMRES.cpp:464-684 with Solve3DSparseUsingFT_CSR,
    Source/functions.cpp:5837-6061: FFT-z, a SuperLU factor per kz in place
    of PARDISO, complex128) on the same workload and `config` as the GPU arm.
    Set-up factors all kz systems (timed in full, part of every solve); each
    step is one real FGMRES(20) iteration of source 0 from a zero start
    (warm-up iterations first), so that K steps sample the cost of an
    iteration across the restart cycle.  value = factor + mean iteration x
    the port's own iteration count for this workload + one true residual
    per restart.  Loads none of this repository's native code."""
    if rank != 0:
        return None
    cores = os.cpu_count() or 1
    iters, src = port_iterations(args.n, cores)
    base = {"impl": "reference", "metric": METRIC, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False, "dtype": "c128",
            "data": "synthetic (seeded splitmix64 medium and sources)", "config": workload_config(args.n)}
    if iters is None:
        return dict(base, unavailable=src)
    ps = PortSample(args.n, cores)
    try:
        times = ps.iterations(args.warmup + max(1, args.steps))
    finally:
        ps.close()
    timed = times[args.warmup:] or times
    per_it = statistics.mean(timed)
    v = cpu_port_value(ps, per_it, iters)
    # the reference applies L0^{-1} three times per iteration
    # (Source/FGMRES.cpp:503,579,601); the port once
    t_apply_extra = 2.0 * ps.apply_s
    line = dict(base)
    line.update({
        "value": v,
        "method": f"FFT-z preconditioner, SuperLU per kz (PARDISO in the reference), complex128 FGMRES({RESTART}) "
                  f"with CGS2, one source per solve as the reference's main loop",
        "iterations": iters,
        "iterations_source": src,
        "cpu_baseline": {"value": v, "unit": "s", "cores": cores, "kind": "port",
                         "sample": f"set-up: SuperLU factor of all {ps.p.nz} kz systems ({ps.factor_s:.1f} s); "
                                   f"each step one FGMRES({RESTART}) iteration of source 0 ({len(timed)} timed after "
                                   f"{args.warmup} warm-up, mean {per_it:.2f} s); scaled to {iters} iterations",
                         "factor_s": ps.factor_s, "per_iteration_s": per_it},
        "reference_structure_estimate": {
            "value": ps.factor_s + (per_it + t_apply_extra) * iters,
            "note": f"three preconditioner applies per iteration as Source/FGMRES.cpp:503,579,601 "
                    f"(one apply timed: {ps.apply_s:.2f} s)"},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "native_libs_loaded": native_libs_loaded(),
    })
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", dest="n", type=int, default=200, help="grid points per axis")
    ap.add_argument("--e2e-steps", type=int, default=5, help="timed e2e steps (at most --steps)")
    ap.add_argument("--arm-steps", type=int, default=1, help="timed steps of each comparison arm")
    ap.add_argument("--skip-arms", default="", help="comma-separated comparison arms to leave out")
    ap.add_argument("--nz", type=int, default=0, help="--kernels: z points (default: the grid size)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--kernels", action="store_true",
                    help="per-kernel microbench: batched FGMRES(1) iterations instead of full solves")
    ap.add_argument("--prec-applies", action="store_true",
                    help="--kernels: batched preconditioner applies (z-transforms and sweep) instead")
    ap.add_argument("--workload", default="headline", choices=["headline", "c3", "c4", "c5", "n200"],
                    help="c3: 160^3 mixed precision, FGMRES(30); c4: 96^3 x 16 sources + 8 uneven grids as one "
                         "group; c5: 200^3 misfit gradient with finite-difference check; n200: 200^3 batched "
                         "complex64 vs plain complex128")
    args = ap.parse_args()
    args.skip_arms = set(a for a in args.skip_arms.split(",") if a)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        # the CPU reference runs on rank 0 only; the other ranks exit at once
        out = run_reference(args, rank)
        if rank == 0 and out is not None:
            print(json.dumps(out))
        return
    if args.kernels:
        print(json.dumps(run_kernels(args)))
        return
    if args.workload != "headline":
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
    dist = init_dist(world)
    line = run_ours(args, rank, world, dist)
    if rank == 0 and line is not None:
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_port_sample(args.n, os.cpu_count() or 1)
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
