"""Benchmark: CG-SENSE reconstructions per second on one or more B200s.

Workload (default): 2D radial CG-SENSE, 256x256 image, 16 coils with smooth
polynomial maps, 96 golden-angle spokes x 512 samples, 40 dB noise,
lambda 0.01, 30 CG iterations, Toeplitz normal operator, automatic data
scaling -- ``bart pics -l2 -r0.01 -i30 -t traj ksp sens out``. One step is
one full reconstruction from device-resident trajectory, maps and k-space:
model set-up (trajectory upload, PSF on the device), adjoint, scaling, CG.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU (torchrun, one rank per GPU): every rank reconstructs its own
independent problems (no collective on the data path; replicas, weak
scaling); the time is the max over ranks. Prints one JSON line on rank 0.
"""

from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_IMG, COILS, SPOKES, READ_OS, LAM, ITERS, SNR_DB = 256, 16, 96, 2, 0.01, 30, 40.0
METRIC = "CG-SENSE recons/s (2D radial 256^2, 16 coils, 96 spokes x 512, lambda 0.01, 30 CG iters)"
WORKLOAD = "cgsense2d_256_c16_s96_i30_toeplitz"
DOMINANT = "cols_toeplitz"


def make_problem(seed: int):
    """Seeded synthetic problem (numpy, BART layout)."""
    from bart_b200 import synth
    rng = np.random.default_rng(seed)
    traj = synth.radial_traj(N_IMG, SPOKES, os=READ_OS)
    truth = synth.ellipse_phantom(N_IMG, 20, rng)
    sens = synth.coil_maps(N_IMG, COILS, rng)
    return traj, truth, sens, rng


def simulate_ksp(traj, truth, sens, rng):
    """k-space of the SENSE model on the GPU (NUFFT of truth * maps) + noise."""
    from bart_b200.nufft import NufftConf, nufft_create2
    cim = (truth.reshape(N_IMG, N_IMG, 1, 1) * sens).astype(np.complex64)
    kd = [1, traj.shape[1], traj.shape[2], COILS]
    op = nufft_create2(kd, list(cim.shape), list(traj.shape), traj, conf=NufftConf(toeplitz=False))
    y = np.asarray(op.forward(cim)).reshape(kd, order="F")
    op.free()
    from bart_b200 import synth
    return synth.add_noise(y, SNR_DB, rng)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def reference_pics_seconds(traj, sens, ksp, iters=ITERS, threads=None):
    """Wall time of the reference's own CPU ``pics`` (built from its sources
    into oracle/_ref) on this workload, or None if it is not built."""
    exe = os.path.join(ROOT, "oracle", "_ref", "bin", "pics")
    if not os.path.exists(exe):
        return None
    from bart_b200.cfl import writecfl
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(threads or os.cpu_count())
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "t"), traj)
        writecfl(os.path.join(d, "s"), sens)
        writecfl(os.path.join(d, "k"), ksp)
        t0 = time.perf_counter()
        r = subprocess.run([exe, "-l2", f"-r{LAM}", f"-i{iters}", "-t", "t", "k", "s", "o"], cwd=d, env=env,
                           capture_output=True, text=True)
        dt = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError("reference pics failed: " + r.stderr[-500:])
    return dt


def oracle_pics_seconds(traj, sens, ksp):
    from oracle import nufft_oracle as orc
    t0 = time.perf_counter()
    orc.pics_l2(traj.real.reshape(3, -1, order="F"), ksp.reshape(-1, COILS, order="F"), sens, lam=LAM, maxiter=ITERS)
    return time.perf_counter() - t0


def cpu_baseline(traj, sens, ksp):
    dt = reference_pics_seconds(traj, sens, ksp)
    if dt is not None:
        return {"value": 1.0 / dt, "unit": "recons/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "1 full recon with the reference's CPU pics (OpenMP, MKL FFT via FFTW shim), wall incl. .cfl I/O"}
    dt = oracle_pics_seconds(traj, sens, ksp)
    return {"value": 1.0 / dt, "unit": "recons/s", "cores": 1, "kind": "port",
            "sample": "1 full recon with the NumPy oracle (float64)"}


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU path on the host cores."""
    if rank != 0:
        return
    traj, truth, sens, rng = make_problem(1000)
    # k-space from the oracle's forward model (CPU; this arm uses no GPU code)
    from oracle import nufft_oracle as orc
    A = orc.SenseOracle(traj.real.reshape(3, -1, order="F"), sens)
    from bart_b200 import synth
    y = A.forward(truth.reshape(N_IMG, N_IMG, 1, 1))
    ksp = synth.add_noise(y, SNR_DB, rng).reshape(1, traj.shape[1], traj.shape[2], COILS, order="F")
    kind = "reference" if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "bin", "pics")) else "port"
    run = (lambda: reference_pics_seconds(traj, sens, ksp)) if kind == "reference" else \
        (lambda: oracle_pics_seconds(traj, sens, ksp))
    for _ in range(args.warmup):
        run()
    times = [run() for _ in range(args.steps)]
    tot = sum(times)
    value = args.steps / tot
    line = {"metric": METRIC, "value": value, "unit": "recons/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "image": N_IMG, "coils": COILS, "spokes": SPOKES, "samples": 512,
                       "iters": ITERS, "lambda": LAM, "toeplitz": True},
            "cpu_baseline": {"value": value, "unit": "recons/s", "cores": os.cpu_count() if kind == "reference" else 1,
                             "kind": kind, "sample": "full recon per step, wall time incl. .cfl I/O"},
            "e2e": {"value": value, "unit": "recons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from bart_b200 import _lib
    from bart_b200.pics import Pics, PicsConf

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    lib = _lib.load()
    traj, truth, sens, rng = make_problem(1000 + rank)
    ksp = simulate_ksp(traj, truth, sens, rng)

    def dev_tensor(a):
        return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).to(dev)

    traj_d, sens_d, ksp_d = dev_tensor(traj), dev_tensor(sens), dev_tensor(ksp)
    img_d = torch.empty(N_IMG * N_IMG, dtype=torch.complex64, device=dev)
    conf = PicsConf(lam=LAM, maxiter=ITERS, toeplitz=True)

    def step():
        p = Pics(traj_d, sens_d, ksp_dims=list(ksp.shape), conf=conf, traj_dims=list(traj.shape),
                 sens_dims=list(sens.shape))
        p.run(ksp_d, out=img_d)
        p.free()

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    stream = torch.cuda.current_stream(dev)
    l0 = lib.bnufft_launch_count()
    lib.bnufft_prof_start(DOMINANT.encode())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = lib.bnufft_launch_count() - l0
    import ctypes
    kms, kn = ctypes.c_double(), ctypes.c_long()
    lib.bnufft_prof_stop(ctypes.byref(kms), ctypes.byref(kn))

    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    ms_max = float(t.item())

    # end to end through the host API: host arrays in, host image out
    h2d = traj.nbytes + sens.nbytes + ksp.nbytes
    d2h = N_IMG * N_IMG * 8
    img_h = np.zeros((N_IMG, N_IMG, 1), dtype=np.complex64, order="F")
    e2e_steps = max(3, args.steps // 2)

    def step_host():
        p = Pics(traj, sens, ksp_dims=list(ksp.shape), conf=conf)
        p.run(ksp, out=img_h)
        p.free()

    step_host()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        step_host()
    torch.cuda.synchronize()
    e2e_s = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(e2e_s, op=dist.ReduceOp.MAX)

    # roofline of the dominant kernel: Toeplitz column pass, per launch
    # reads + writes the [2X, Y, C] row-transformed buffer and reads the PSF
    G0, G1 = 2 * N_IMG, 2 * N_IMG
    alg_bytes = 2 * (G0 * N_IMG * COILS * 8) + G0 * G1 * 8
    k_avg_s = (kms.value / 1e3) / max(1, kn.value)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = float(json.load(open(peaks_path))["hbm_gbs"])
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    achieved = alg_bytes / k_avg_s / 1e9 if k_avg_s > 0 else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(DOMINANT)

    if rank == 0:
        value = world * args.steps / (ms_max / 1e3)
        line = {"metric": METRIC, "value": value, "unit": "recons/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "image": N_IMG, "coils": COILS, "spokes": SPOKES, "samples": 512,
                           "iters": ITERS, "lambda": LAM, "toeplitz": True, "parallelism": f"replicas{world}",
                           "l2": "inputs and work buffers (~60 MB) are L2-resident; no flush between steps"},
                "e2e": {"value": world * e2e_steps / float(e2e_s.item()), "unit": "recons/s",
                        "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "gpu_launches": launches,
                "roofline": {"bound": "hbm", "kernel": DOMINANT, "achieved": achieved, "peak": peak,
                             "peak_source": peak_src, "unit": "GB/s",
                             "frac": (achieved / peak) if achieved else None,
                             "traffic": traffic, "alg_bytes": alg_bytes,
                             "avg_launch_us": k_avg_s * 1e6, "launches": kn.value},
                "clocks": clk.summary()}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(traj, sens, ksp)
        print(json.dumps(line), flush=True)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
