"""Benchmark: CG-SENSE reconstructions per second on one or more B200s.

Workload (default): 2D radial CG-SENSE, 256x256 image, 16 coils with smooth
polynomial maps, 96 golden-angle spokes x 512 samples, 40 dB noise,
lambda 0.01, Toeplitz normal operator, automatic data scaling, solved until
the relative normal-equation residual reaches 1e-4 (the problem of
``bart pics -l2 -r0.01 -t traj ksp sens out``). The headline solver is
PCG with the padded-circulant preconditioner (the Toeplitz operator's own
circulant inverted on the padded image); flexible CG with the reference's
Strang circulant preconditioner, plain CG (the reference's method) and
flexible CG with the learned correction are timed beside it.
One step is one full reconstruction from device-resident trajectory, maps
and k-space: model set-up (trajectory upload, PSF on the device), adjoint,
scaling, CG graph. L2 is flushed before every timed step. The config's
fixed 30 plain-CG iterations, Toeplitz on and off, are reported beside.

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
TOL, MAXITER = 1e-4, 300
# where the reference arm's search for the iteration count that takes its
# pics (no tolerance option) to 1e-4 on this seeded problem starts; the GPU
# plain CG needs 50 here
REF_ITERS_TO_TOL = 50
METRIC = ("CG-SENSE recons/s to 1e-4 rel. normal-equation residual "
          "(2D radial 256^2, 16 coils, 96 spokes x 512, lambda 0.01)")
WORKLOAD = "cgsense2d_256_c16_s96_tol1e-4_toeplitz"
DOMINANT = "cols_toeplitz"
# the ncu summary of the dominant kernel on this workload; its table carries
# the DRAM bytes (read + write) of one launch
DOMINANT_PROFILE = os.path.join(ROOT, "profiles", "k_cols_toe512_cgsense2d.md")
# FP32 peak of the CUDA cores (no measured figure exists for it): 148 SMs x
# 128 lanes x 2 flop (FMA) x the max SM clock 1.965 GHz
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12
L2_FLUSH_BYTES = 512 << 20     # > 126 MB L2


def make_problem(seed: int):
    """Seeded synthetic problem (numpy, BART layout)."""
    from bart_b200 import synth
    rng = np.random.default_rng(seed)
    traj = synth.radial_traj(N_IMG, SPOKES, os=READ_OS)
    truth = synth.ellipse_phantom(N_IMG, 20, rng)
    sens = synth.coil_maps(N_IMG, COILS, rng)
    return traj, truth, sens, rng


def workload_config():
    """The workload both arms measure (the same dict in both JSON lines)."""
    return {"workload": WORKLOAD, "image": N_IMG, "coils": COILS, "spokes": SPOKES, "samples": 512,
            "tol": TOL, "lambda": LAM, "toeplitz": True}


def inputs_record(traj, sens, ksp):
    """Checksums of the inputs a step reconstructs: both arms print them, so
    equal digests show the arms solved byte-identical problems."""
    import hashlib

    def h(a):
        return hashlib.sha256(np.ascontiguousarray(np.asfortranarray(a).ravel(order="F")).tobytes()).hexdigest()[:16]
    return {"traj_sha256": h(traj), "sens_sha256": h(sens), "ksp_sha256": h(ksp),
            "ksp_generator": "the library's forward NUFFT (GPU) of the seeded phantom times the maps, "
                             "plus seeded 40 dB noise, outside the timed region"}


def simulate_ksp(traj, truth, sens, rng):
    """k-space of the SENSE model on the GPU (NUFFT of truth * maps) + noise.
    Both arms of the bench simulate their input this way, so they read
    byte-identical k-space."""
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


def nufft_throughput(dev, steps=50, warmup=5):
    """NUFFT GB/s on the 2D single-coil workload: 256^2
    i.i.d. complex Gaussian image, 402 golden-angle spokes x 512 samples,
    os 2, width 6. One step = forward + adjoint on device-resident data with
    the plan reused; bytes = compulsory I/O of both directions (image, k-space,
    trajectory as 2 float32 per sample)."""
    import torch
    from bart_b200 import synth
    from bart_b200.nufft import NufftConf, nufft_create2
    rng = np.random.default_rng(1)
    t = synth.radial_traj(256, 402)
    img = synth.random_image(256, rng)
    M = t.shape[1] * t.shape[2]
    op = nufft_create2([1, t.shape[1], t.shape[2], 1], [256, 256, 1, 1], list(t.shape), t,
                       conf=NufftConf(toeplitz=False))
    x = torch.from_numpy(np.asfortranarray(img).ravel(order="F").copy()).to(dev)
    k = torch.empty(M, dtype=torch.complex64, device=dev)
    a = torch.empty(256 * 256, dtype=torch.complex64, device=dev)
    for _ in range(warmup):
        op.forward(x, k)
        op.adjoint(k, a)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        op.forward(x, k)
        op.adjoint(k, a)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    op.free()
    nbytes = 2 * (256 * 256 * 8 + M * 8 + M * 8)
    return {"workload": "nufft2d_256_r402x512_c1_fwd+adj", "value": nbytes / (ms * 1e-3) / 1e9, "unit": "GB/s",
            "us_per_fwd_adj": ms * 1e3, "bytes_per_step": nbytes}


def true_residual(dev, p, traj_d, sens_d, ksp_d, x, ksp_shape, traj_shape, scale):
    """||b - (A^H A + lambda) x|| / ||b|| with b = A^H y / scale, recomputed
    from the operators (not CG's recursive residual)."""
    import torch
    from bart_b200.nufft import NufftConf, nufft_create2
    op = nufft_create2(list(ksp_shape), [N_IMG, N_IMG, 1, COILS], list(traj_shape), traj_d,
                       conf=NufftConf(toeplitz=False))
    adj = op.adjoint(ksp_d).reshape(COILS, N_IMG * N_IMG)
    b = (torch.conj(sens_d.reshape(COILS, N_IMG * N_IMG)) * adj).sum(0) / scale
    r = b - (p.normal(x) + LAM * x)
    op.free()
    return float(torch.linalg.vector_norm(r) / torch.linalg.vector_norm(b))


def timed_steps(step, steps, flush, stream):
    """Device time (ms) of `steps` calls of step(), each bracketed by CUDA
    events on `stream` after an L2 flush (outside the bracket)."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    for e0, e1 in ev:
        flush.zero_()
        e0.record(stream)
        step()
        e1.record(stream)
    torch.cuda.synchronize()
    return sum(e0.elapsed_time(e1) for e0, e1 in ev)


def run_normal3d(dev, steps, warmup, coils=8, N=128, spokes=2000):
    """The 3D SENSE normal operator of the CG iterations (Toeplitz; 128^3,
    `coils` coils, kooshball PSF): device time per apply and per pass class
    (CUDA events per launch), against the HBM bytes of its five passes:
    rows (x + maps in, [2N, N, N, C] out), y forward ([2N, 2N, N, C] out),
    z Toeplitz (in place on it, + the (2N)^3 PSF), y inverse, rows (maps in,
    the coil-group sums out)."""
    import ctypes
    import torch
    from bart_b200 import _lib, synth
    from bart_b200.pics import Pics, PicsConf
    rng = np.random.default_rng(7)
    t = synth.kooshball_traj(N, spokes)
    sens = synth.coil_maps(N, coils, rng, ndim=3)
    cd = [N, N, N, coils]
    kd = [1, t.shape[1], t.shape[2], coils]
    t_d = torch.from_numpy(np.asfortranarray(t).ravel(order="F").copy()).to(dev)
    sens_d = torch.from_numpy(np.asfortranarray(sens).ravel(order="F").copy()).to(dev)
    p = Pics(t_d, sens_d, ksp_dims=kd, conf=PicsConf(lam=LAM, maxiter=10), traj_dims=list(t.shape), sens_dims=cd)
    x = torch.randn(N ** 3, dtype=torch.complex64, device=dev)
    y = torch.empty_like(x)
    for _ in range(max(1, warmup)):
        p.normal(x, y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        p.normal(x, y)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    lib = _lib.load()
    passes = {}
    for kind in ("rows_fwd", "cols_fwd", "cols_toeplitz", "cols_inv", "rows_inv"):
        lib.bnufft_prof_start(kind.encode())
        p.normal(x, y)
        kms, kn = ctypes.c_double(), ctypes.c_long()
        lib.bnufft_prof_stop(ctypes.byref(kms), ctypes.byref(kn))
        passes[kind] = {"ms": kms.value, "launches": kn.value}
    p.free()
    img, G = N ** 3 * 8, 2 * N
    t1, t2 = G * N * N * coils * 8, G * G * N * coils * 8
    maps = img * coils
    pass_bytes = {"rows_fwd": img + maps + t1, "cols_fwd": t1 + t2, "cols_toeplitz": 2 * t2 + G ** 3 * 8,
                  "cols_inv": t2 + t1, "rows_inv": t1 + maps + img}
    peak, peak_src = peak_hbm()
    for k, b in pass_bytes.items():
        if passes[k]["ms"] > 0:
            passes[k]["gbs"] = b / (passes[k]["ms"] * 1e-3) / 1e9
            passes[k]["hbm_frac"] = passes[k]["gbs"] / peak
    total = sum(pass_bytes.values())
    return {"workload": f"normal3d_{N}_c{coils}", "ms_per_apply": ms, "hbm_bytes_per_apply": total,
            "gbs": total / (ms * 1e-3) / 1e9, "hbm_frac": total / (ms * 1e-3) / 1e9 / peak,
            "hbm_peak_gbs": peak, "peak_source": peak_src, "passes": passes}


def run_ecalib(dev, steps, warmup, N=256, coils=16, cpu_base=True, ndim=2, slices=0):
    """ESPIRiT calibration with the reference's ecalib defaults (6 x 6
    kernel, calibration region up to 24 x 24, threshold 0.001, 2 maps, 30
    orthogonal iterations, crop 0.8) of 2D Cartesian k-space: N x N, `coils`
    coils, ellipse phantom, polynomial maps, 40 dB noise, 24 fully sampled
    centre lines and every other line outside. One step = one calibration
    from device k-space to device maps (value); e2e = from pinned host
    k-space to pinned host maps and eigenvalue maps. Per-stage device times by CUDA events;
    the per-pixel pass against the FP32 FMA peak (its arithmetic: the C x C
    matrix from 12 x-interpolation terms per entry, then 30 x maps x C^2
    complex multiply-adds of the orthogonal iteration). cpu_baseline: the
    reference's ecalib built from its sources, whole command with .cfl
    I/O, all host cores. ndim 3: an N^3 volume, 24 fully sampled centre
    lines in y and z (the reference then splits the point-wise step along
    z, src/ecalib.c:137-138)."""
    import ctypes
    import torch
    from bart_b200 import _lib, synth
    from bart_b200.espirit import ecalib
    rng = np.random.default_rng(11)
    img = synth.ellipse_phantom(N, 20, rng, ndim=ndim)
    k = synth.cartesian_ksp(img, synth.coil_maps(N, coils, rng, ndim=ndim), rng, 40.0, 24, 2)
    dims = list(k.shape)
    kt = torch.from_numpy(np.asfortranarray(k).ravel(order="F").copy()).to(dev)
    lib = _lib.load()
    for _ in range(max(3, warmup)):
        ecalib(kt, dims=dims)
    torch.cuda.synchronize()
    ev_pairs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    n0 = lib.bnufft_launch_count()
    with ClockSampler(dev.index or 0) as clk:
        torch.cuda.synchronize()
        for a, b in ev_pairs:
            a.record()
            sens, ev, info = ecalib(kt, dims=dims)
            b.record()
        torch.cuda.synchronize()
    per = sorted(a.elapsed_time(b) for a, b in ev_pairs)
    ms = float(np.mean(per))
    launches = int(lib.bnufft_launch_count() - n0)
    stages = {}
    for kind in ("ecalib_gram", "ecalib_eig", "ecalib_imgcov", "ecalib_interp", "ecalib_pixels"):
        t = []
        for _ in range(5):		# median of 5 calls
            lib.bnufft_prof_start(kind.encode())
            ecalib(kt, dims=dims)
            kms, kn = ctypes.c_double(), ctypes.c_long()
            lib.bnufft_prof_stop(ctypes.byref(kms), ctypes.byref(kn))
            t.append(kms.value)
        stages[kind] = {"ms": sorted(t)[2], "ms_min": min(t), "ms_max": max(t), "launches": kn.value}
    # end to end from pinned host k-space to pinned host maps and eigenvalue maps
    def pinned(shape):
        t = torch.empty(int(np.prod(shape)), dtype=torch.complex64, pin_memory=True)
        return t, t.numpy().reshape(shape, order="F")

    from bart_b200.espirit import output_dims
    sd, ed = output_dims(dims)
    keep = [pinned(k.shape), pinned(sd), pinned(ed)]
    k_h, s_h, e_h = (v for _, v in keep)
    k_h[...] = k
    ecalib(k_h, out=(s_h, e_h))
    t0 = time.perf_counter()
    for _ in range(steps):
        ecalib(k_h, out=(s_h, e_h))
    e2e_s = (time.perf_counter() - t0) / steps
    M, C, xh, it = 2, coils, 12, 30
    npix = N ** ndim
    flop = npix * (C * C * xh + it * M * C * C) * 8.0
    px_ms = stages["ecalib_pixels"]["ms"]
    out_bytes = npix * (C * M + M) * 8
    t_bytes = (npix // N) * xh * (C * (C + 1) // 2) * 16
    res = {"workload": f"ecalib{ndim}d_{N}_c{coils}", "metric": "ESPIRiT calibrations/s", "unit": "calibrations/s",
           "value": 1e3 / ms, "ms_per_calibration": ms, "ms_min": per[0], "ms_median": per[len(per) // 2],
           "ms_max": per[-1], "gpu_launches": launches // steps,
           "nkernels": info["nkernels"], "caldims": list(info["caldims"]),
           "e2e": {"value": 1.0 / e2e_s, "unit": "calibrations/s", "h2d_bytes_per_step": int(k.nbytes),
                   "d2h_bytes_per_step": int(npix * (C * M + M) * 8)},
           "stages": stages,
           "pixels_kernel": {"flop": flop, "tflops": flop / (px_ms * 1e-3) / 1e12 if px_ms > 0 else None,
                             "fp32_peak_tflops": FP32_PEAK_TFLOPS,
                             "fp32_frac": flop / (px_ms * 1e-3) / 1e12 / FP32_PEAK_TFLOPS if px_ms > 0 else None,
                             "hbm_bytes": out_bytes + t_bytes},
           "clocks": clk.summary()}
    if slices > 0:
        # bart -l 8192 ecalib over `slices` slices (the k-space scaled per
        # slice): one worker (one calibration after another) against four
        # (threads with their own streams), host arrays in and out
        from bart_b200.espirit import EcalibConf
        from bart_b200.loop import loop_ecalib
        ks = np.concatenate([(k * np.complex64(1.0 + 0.1 * i)).reshape(list(k.shape) + [1] * (13 - k.ndim) + [1])
                             for i in range(slices)], axis=13)
        res["slice_loop"] = {"slices": slices}
        for w in (1, 4):
            loop_ecalib(8192, ks[..., :2], EcalibConf(), workers=w)
            t0 = time.perf_counter()
            loop_ecalib(8192, ks, EcalibConf(), workers=w)
            dt = time.perf_counter() - t0
            res["slice_loop"][f"workers{w}_ms_per_slice"] = dt / slices * 1e3
    exe = os.path.join(ROOT, "oracle", "_ref", "bin", "ecalib")
    if cpu_base and os.path.exists(exe):
        from bart_b200.cfl import writecfl
        env = dict(os.environ)
        env["OMP_NUM_THREADS"] = str(os.cpu_count())
        with tempfile.TemporaryDirectory() as d:
            writecfl(os.path.join(d, "k"), k)
            t0 = time.perf_counter()
            r = subprocess.run([exe, "k", "s", "e"], cwd=d, env=env, capture_output=True, text=True)
            dt = time.perf_counter() - t0
        if r.returncode == 0:
            res["cpu_baseline"] = {"value": 1.0 / dt, "unit": "calibrations/s", "cores": os.cpu_count(),
                                   "kind": "reference", "sample": "1 calibration with the reference's CPU ecalib "
                                   "(OpenMP, MKL eigen-decomposition), wall incl. .cfl I/O"}
    return res


def run_nufft3d(dev, steps, warmup, spokes=20000):
    """3D radial kooshball NUFFT: 128^3 image, 8 coils,
    20000 spokes x 256 samples on 3D golden means (5.12 M samples per coil).
    One step = forward + adjoint of all 8 coil images, device-resident, plan
    reused. Also the time per kernel class (CUDA events per launch), the
    scatter's atomic rate, and a 10-iteration Toeplitz CG-SENSE solve (model
    reused)."""
    import ctypes
    import torch
    from bart_b200 import _lib, synth
    from bart_b200.nufft import NufftConf, nufft_create2
    from bart_b200.pics import Pics, PicsConf
    N, C, readout = 128, 8, 128
    rng = np.random.default_rng(3)
    t = synth.kooshball_traj(readout, spokes)
    M = t.shape[1] * t.shape[2]
    sens = synth.coil_maps(N, C, rng, ndim=3)
    truth = synth.ellipse_phantom(N, 20, rng, ndim=3)
    cd = [N, N, N, C]
    kd = [1, t.shape[1], t.shape[2], C]
    t_d = torch.from_numpy(np.asfortranarray(t).ravel(order="F").copy()).to(dev)
    cim = torch.from_numpy(np.asfortranarray(truth.reshape(N, N, N, 1) * sens).ravel(order="F").copy()).to(dev)
    op = nufft_create2(kd, cd, list(t.shape), t_d, conf=NufftConf(toeplitz=False))
    k = torch.empty(M * C, dtype=torch.complex64, device=dev)
    a = torch.empty(N ** 3 * C, dtype=torch.complex64, device=dev)
    for _ in range(warmup):
        op.forward(cim, k)
        op.adjoint(k, a)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        op.forward(cim, k)
        op.adjoint(k, a)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    lib = _lib.load()
    classes = {}
    for kind in ("rows_fwd", "cols_fwd", "degrid", "grid", "cols_inv", "rows_inv"):
        lib.bnufft_prof_start(kind.encode())
        op.forward(cim, k)
        op.adjoint(k, a)
        kms, kn = ctypes.c_double(), ctypes.c_long()
        lib.bnufft_prof_stop(ctypes.byref(kms), ctypes.byref(kn))
        classes[kind] = {"ms": kms.value, "launches": kn.value}
    op.free()
    nbytes = 2 * (N ** 3 * C * 8 + M * C * 8 + M * 12)
    # scatter: one float2 atomic add per tap (6^3 taps, weight-0 taps skipped)
    atomics = M * C * 216
    classes["grid"]["g_float2_atomics_per_s"] = atomics / (classes["grid"]["ms"] * 1e-3) / 1e9
    sens_d = torch.from_numpy(np.asfortranarray(sens).ravel(order="F").copy()).to(dev)
    t0 = time.perf_counter()
    p = Pics(t_d, sens_d, ksp_dims=kd, conf=PicsConf(lam=LAM, maxiter=10), traj_dims=list(t.shape), sens_dims=cd)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    x = p.run(k)
    torch.cuda.synchronize()
    e0.record()
    p.run(k, out=x)
    e1.record()
    torch.cuda.synchronize()
    cg_ms = e0.elapsed_time(e1)
    p.free()
    # to the 1e-4 tolerance: plain CG, flexible CG with the circulant
    # preconditioner, PCG with the padded one (model reused, one solve each
    # after a warm-up)
    to_tol = {}
    for name, pc in (("cg", 0), ("fcg_circulant", 1), ("fcg_padded", 3)):
        p = Pics(t_d, sens_d, ksp_dims=kd, conf=PicsConf(lam=LAM, maxiter=200, tol=TOL, precond=pc),
                 traj_dims=list(t.shape), sens_dims=cd)
        x = p.run(k)
        torch.cuda.synchronize()
        e0.record()
        p.run(k, out=x)
        e1.record()
        torch.cuda.synchronize()
        it, rr, _ = p.stats()
        to_tol[name] = {"ms": e0.elapsed_time(e1), "iterations": it, "recursive_rel_residual": rr}
        p.free()
    # roofline of the fwd+adj step: compulsory bytes (coil images in and out,
    # k-space out and in, trajectory twice), the oversampled grid's round
    # trips (written and read once per direction), and the interpolation's
    # FP32 work (a complex multiply-add per tap, sample and coil, both
    # directions) against the nominal FP32 rate at the sampled SM clock
    peak, peak_src = peak_hbm()
    G3 = (2 * N) ** 3
    grid_bytes = 2 * 2 * G3 * C * 8
    tap_flop = 2 * 4 * 216 * M * C
    fp32_peak = 148 * 128 * 2 * 1.965e9
    return {"workload": f"nufft3d_128_c8_kooshball_{spokes}x256", "nufft_fwd_adj_ms": ms, "kernel_classes": classes,
            "nufft_gbs": nbytes / (ms * 1e-3) / 1e9, "bytes_per_step": nbytes,
            "roofline": {"hbm_peak_gbs": peak, "peak_source": peak_src,
                         "compulsory_frac": nbytes / (ms * 1e-3) / 1e9 / peak,
                         "with_grid_roundtrip_frac": (nbytes + grid_bytes) / (ms * 1e-3) / 1e9 / peak,
                         "grid_roundtrip_bytes": grid_bytes,
                         "tap_tflops": tap_flop / (ms * 1e-3) / 1e12,
                         "tap_fp32_frac": tap_flop / (ms * 1e-3) / fp32_peak,
                         "fp32_peak_note": "nominal 148 SMs x 128 FP32 lanes x 2 x 1.965 GHz = 74.4 TFLOP/s"},
            "cgsense_setup_s": setup_s, "cgsense_10iter_ms": cg_ms, "cgsense_to_1e-4": to_tol}


def run_scatter(dev, steps=5, warmup=3):
    """Adjoint gridding (the scatter) alone, per kernel variant in force
    (BNUFFT_GRIDDING: default, lines, atomic, tiles), CUDA-event time per
    launch of the "grid" class on four problems: 256^2 with 16 coils and 96
    spokes x 512 (the CG-SENSE bench problem), 256^2 single-coil with 402
    spokes (config 1), the 2D PSF's periodic 1024^2 grid (2 x trajectory, one
    channel), and the 8-coil 128^3 kooshball with 20000 spokes x 256."""
    import ctypes
    import torch
    from bart_b200 import _lib, synth
    from bart_b200.nufft import NufftConf, nufft_create2
    lib = _lib.load()

    def d(a):
        return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).to(dev)

    out = {"workload": "scatter", "variant": os.environ.get("BNUFFT_GRIDDING", "default"), "unit": "us per launch"}
    for name, N, sp, C, nd, per in (("cgsense2d_256_c16_s96", 256, 96, 16, 2, 0), ("nufft2d_256_c1_s402", 256, 402, 1, 2, 0),
                                    ("psf2d_1024_periodic", 512, 96, 1, 2, 1),
                                    ("kooshball3d_128_c8_s20000", 128, 20000, 8, 3, 0)):
        t = synth.radial_traj(N, sp) if nd == 2 else synth.kooshball_traj(N, sp)
        if per:
            t = t * 2
        M = t.shape[1] * t.shape[2]
        cd = [N, N, 1 if nd == 2 else N, C]
        kd = [1, t.shape[1], t.shape[2], C]
        op = nufft_create2(kd, cd, list(t.shape), d(t), conf=NufftConf(toeplitz=False, periodic=bool(per)))
        y = torch.randn(M * C, dtype=torch.complex64, device=dev)
        a = torch.empty(int(np.prod(cd)), dtype=torch.complex64, device=dev)
        for _ in range(warmup):
            op.adjoint(y, a)
        torch.cuda.synchronize()
        lib.bnufft_prof_start(b"grid")
        for _ in range(steps):
            op.adjoint(y, a)
        ms, n = ctypes.c_double(), ctypes.c_long()
        lib.bnufft_prof_stop(ctypes.byref(ms), ctypes.byref(n))
        out[name] = ms.value * 1e3 / max(1, n.value)
        op.free()
        del y, a
        torch.cuda.empty_cache()
    return out


def toeplitz_normal_torch(x_yx, maps_cyx, P_yx):
    """S^H F^H P F S x with torch.fft (cuFFT on a GPU): x [Y, X], maps
    [C, Y, X], P the 2N x 2N PSF in DFT order, [y][x], scaled 1/npix. Pixel
    n sits at (n - N/2) mod 2N of the zero-padded grid, as in the library."""
    import torch
    C, N = maps_cyx.shape[0], x_yx.shape[0]
    h = N // 2
    cim = maps_cyx * x_yx.unsqueeze(0)
    pad = torch.zeros(C, 2 * N, 2 * N, dtype=cim.dtype, device=cim.device)
    pad[:, :h, :h] = cim[:, h:, h:]
    pad[:, :h, -h:] = cim[:, h:, :h]
    pad[:, -h:, :h] = cim[:, :h, h:]
    pad[:, -h:, -h:] = cim[:, :h, :h]
    g = torch.fft.ifft2(torch.fft.fft2(pad) * P_yx.unsqueeze(0), norm="forward")
    out = torch.empty_like(cim)
    out[:, h:, h:] = g[:, :h, :h]
    out[:, h:, :h] = g[:, :h, -h:]
    out[:, :h, h:] = g[:, -h:, :h]
    out[:, :h, :h] = g[:, -h:, -h:]
    return (torch.conj(maps_cyx) * out).sum(0)


def psf_grid_yx(psf_ref, N):
    """The reference's decomposed PSF [X, Y, 1, 4] (sub-grid s = sx + 2 sy,
    centred cell 2w + s per axis) as the 2N x 2N DFT-order grid [y][x] / npix."""
    import torch
    sub = torch.from_numpy(np.ascontiguousarray(psf_ref.reshape(N, N, 4, order="F")))
    Pc = torch.zeros(2 * N, 2 * N, dtype=torch.complex64)   # [cx][cy]
    for s_ in range(4):
        Pc[s_ & 1::2, s_ >> 1::2] = sub[:, :, s_]
    return torch.roll(Pc, shifts=(N, N), dims=(0, 1)).t().contiguous() / (N * N)


def fft_vs_cufft(dev, traj, sens, reps=50):
    """The Toeplitz normal operator S^H F^H P F S x of the bench problem
    (256^2, 16 coils, 512^2 grid), once with this library's fused FFT passes
    (Pics.normal) and once with cuFFT (torch.fft: zero-pad, 2D FFT, PSF
    multiply, inverse 2D FFT, crop, coil sum): CUDA-event time per
    application and the relative difference of the results."""
    import torch
    from bart_b200.nufft import NufftConf, nufft_create2
    from bart_b200.pics import Pics, PicsConf
    N, C = N_IMG, COILS
    td = torch.from_numpy(np.asfortranarray(traj).ravel(order="F").copy()).to(dev)
    sd = torch.from_numpy(np.asfortranarray(sens).ravel(order="F").copy()).to(dev)
    kd = [1, traj.shape[1], traj.shape[2], C]
    p = Pics(td, sd, ksp_dims=kd, conf=PicsConf(lam=0.0), traj_dims=list(traj.shape), sens_dims=list(sens.shape))
    op = nufft_create2([1, traj.shape[1], traj.shape[2], 1], [N, N, 1, 1], list(traj.shape), td,
                       conf=NufftConf(toeplitz=True))
    P = psf_grid_yx(op.psf(), N).to(dev)
    op.free()
    x = torch.randn(N * N, dtype=torch.complex64, device=dev)
    maps = sd.reshape(C, N, N)           # [c][y][x]
    res, ys = {}, {}
    for name, fn in (("bnufft", lambda: p.normal(x)), ("cufft", lambda: toeplitz_normal_torch(x.reshape(N, N), maps, P))):
        for _ in range(5):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            y = fn()
        e1.record()
        torch.cuda.synchronize()
        res[name + "_us"] = e0.elapsed_time(e1) / reps * 1e3
        ys[name] = y.reshape(N, N)
    # cuFFT's transforms alone (forward + inverse 2D FFT of the 16 padded grids)
    pad = torch.randn(C, 2 * N, 2 * N, dtype=torch.complex64, device=dev)
    for _ in range(5):
        torch.fft.ifft2(torch.fft.fft2(pad), norm="forward")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        torch.fft.ifft2(torch.fft.fft2(pad), norm="forward")
    e1.record()
    torch.cuda.synchronize()
    res["cufft_fft_pair_only_us"] = e0.elapsed_time(e1) / reps * 1e3
    res["rel_diff"] = float(torch.linalg.vector_norm(ys["bnufft"] - ys["cufft"]) / torch.linalg.vector_norm(ys["cufft"]))
    res["speedup_vs_cufft"] = res["cufft_us"] / res["bnufft_us"]
    p.free()
    return res


def batch_analysis(br, probs, dev):
    """Where the batch's time goes: the same single solves spread over 4, 8
    and 16 streams (any concurrency, without the graph), and each solve
    timed alone, summed per Toeplitz embedding size E (next power of two
    >= 2N)."""
    import torch
    main = torch.cuda.current_stream(dev)
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))   # noqa: E731
    out = {}
    for S in (4, 8, 16):
        streams = [torch.cuda.Stream(dev) for _ in range(S)]

        def spread():
            e = torch.cuda.Event()
            e.record(main)
            for s in streams:
                s.wait_event(e)
            for i, (p, k, x) in enumerate(zip(br.models, br.ksp, br.img)):
                with torch.cuda.stream(streams[i % S]):
                    p.run(k, out=x)
            for s in streams:
                e2 = torch.cuda.Event()
                e2.record(s)
                main.wait_event(e2)

        spread()
        torch.cuda.synchronize()
        e0, e1 = ev()
        e0.record()
        spread()
        e1.record()
        torch.cuda.synchronize()
        out[f"streams{S}_ms"] = e0.elapsed_time(e1)
    per = {}
    for p, k, x, pr in zip(br.models, br.ksp, br.img, probs):
        E = 1 << int(np.ceil(np.log2(2 * pr["sens"].shape[0])))
        torch.cuda.synchronize()
        e0, e1 = ev()
        e0.record()
        p.run(k, out=x)
        e1.record()
        torch.cuda.synchronize()
        d = per.setdefault(str(E), {"problems": 0, "ms": 0.0})
        d["problems"] += 1
        d["ms"] += e0.elapsed_time(e1)
    out["alone_per_embedding"] = per
    out["alone_sum_ms"] = sum(d["ms"] for d in per.values())
    return out


def run_batch(dev, steps, warmup, nprob=512, seed=4, rank=0, world=1, cpu_base=True, analysis=False):
    """Batched uneven 2D reconstructions: nprob problems,
    N ~ U{64..320} even, spokes ~ U{16..256} x 2N samples, coils ~ U{4..32},
    ellipse phantoms, polynomial maps, 20 plain-CG iterations each, lambda
    0.01, Toeplitz. One step = all reconstructions, one graph launch (the
    problems run as independent child graphs); the baseline is a loop of
    single solves on the same GPU. Gridding bins from the autotuner. The
    batch's inputs (several GB) exceed L2.

    With several ranks every rank draws the same problem list and takes the
    share that the cost-model split gives it (no exchange while solving);
    the time is the slowest rank's and the rate is all problems over it
    (strong scaling: the total work is fixed)."""
    import torch
    import torch.distributed as dist
    from bart_b200.batch import BatchRecon, autotune_bins, uneven_problems
    from bart_b200.dist import partition, problem_cost, reduce_max, reduce_sum
    iters = 20
    t0 = time.time()
    probs = uneven_problems(nprob, seed)
    gen_s = time.time() - t0
    costs = [problem_cost(p, iters) for p in probs]
    shards = partition(costs, world)
    loads = [sum(costs[i] for i in s) for s in shards]
    Ns = [p["sens"].shape[0] for p in probs]
    probs = [probs[i] for i in shards[rank]]
    table, detail = autotune_bins(dev, reps=2)
    t0 = time.time()
    br = BatchRecon(probs, dev, maxiter=iters, bins=table)
    torch.cuda.synchronize()
    setup_s = time.time() - t0
    br.build()
    for _ in range(max(3, warmup)):
        br.run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index or 0) as clk:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            br.run()
        e1.record()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    ms = reduce_max(e0.elapsed_time(e1) / steps, dev)
    launches = int(reduce_sum(br.kernels() * steps, dev))
    loop = None
    diff = None
    if world == 1:	# the loop of single solves on the same GPU, for comparison
        xb = [x.clone() for x in br.img]
        br.run_loop()
        torch.cuda.synchronize()
        e0.record()
        br.run_loop()
        e1.record()
        torch.cuda.synchronize()
        ms_loop = e0.elapsed_time(e1)
        diff = max(float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)) for a, b in zip(xb, br.img))
        loop = {"ms": ms_loop, "recons_per_s": nprob / (ms_loop / 1e3), "batch_speedup": ms_loop / ms}
    extra = batch_analysis(br, probs, dev) if (analysis and world == 1) else None
    br.free()
    return {"metric": "batched uneven CG-SENSE recons/s (20 CG iterations each)", "value": nprob / (ms / 1e3),
            "unit": "recons/s", "n_gpus": world, "steps": steps, "warmup": warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "strong", "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batch{nprob}_uneven_2d_i20", "problems": nprob, "N_range": [min(Ns), max(Ns)],
                       "spokes": [16, 256], "coils": [4, 32], "iters": iters, "lambda": 0.01,
                       "l2": "batch inputs (GBs) exceed L2",
                       "split": "cost model C (G log G + M taps) iters, LPT" if world > 1 else "one GPU",
                       "predicted_load_max_over_mean": max(loads) / (sum(loads) / world)},
            "loop_of_single_solves": loop,
            "analysis": extra,
            "max_rel_diff_batch_vs_loop": diff, "gpu_launches": launches,
            "autotuned_bins": table, "autotune_ms": detail, "gen_s": gen_s, "setup_s": setup_s,
            "clocks": clk.summary(),
            "cpu_baseline": batch_cpu_baseline() if (cpu_base and rank == 0 and world == 1) else None}


def reference_pics_seconds(traj, sens, ksp, iters=REF_ITERS_TO_TOL, threads=None, out=None):
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
        if r.returncode == 0 and out is not None:
            from bart_b200.cfl import readcfl
            out.append(readcfl(os.path.join(d, "o")))
    if r.returncode != 0:
        raise RuntimeError("reference pics failed: " + r.stderr[-500:])
    return dt


def oracle_pics_seconds(traj, sens, ksp, iters=REF_ITERS_TO_TOL):
    from oracle import nufft_oracle as orc
    t0 = time.perf_counter()
    orc.pics_l2(traj.real.reshape(3, -1, order="F"), ksp.reshape(-1, COILS, order="F"), sens, lam=LAM, maxiter=iters)
    return time.perf_counter() - t0


def cpu_baseline(traj, sens, ksp, iters):
    dt = reference_pics_seconds(traj, sens, ksp, iters=iters)
    if dt is not None:
        return {"value": 1.0 / dt, "unit": "recons/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": f"1 full recon with the reference's CPU pics -i{iters} (the GPU's iteration count to 1e-4; "
                          "OpenMP, MKL FFT via FFTW shim), wall incl. .cfl I/O"}
    dt = oracle_pics_seconds(traj, sens, ksp, iters)
    return {"value": 1.0 / dt, "unit": "recons/s", "cores": 1, "kind": "port",
            "sample": f"1 full recon of {iters} CG iterations with the NumPy oracle (float64)"}


def oracle_forward(traj, cim, kd):
    """Noiseless SENSE k-space on the host (the oracle's NUFFT), for the
    reference arm, which runs no GPU code."""
    from oracle import nufft_oracle as orc
    op = orc.NufftOracle(traj.real.reshape(3, -1, order="F"), cim.shape[:3])
    return op.forward(cim).reshape(kd, order="F")


BATCH_REF_SAMPLE = 6	# problems of the 512-problem batch the reference solves per step


def batch_reference_sample(k=BATCH_REF_SAMPLE, seed=4):
    """The first k problems of the uneven batch (the same random stream as
    the batch), k-space from the oracle's NUFFT on the host."""
    from bart_b200.batch import uneven_problems
    return uneven_problems(k, seed, forward=oracle_forward)


def batch_reference_seconds(probs, iters=20):
    """Wall time of the reference's CPU pics -i20 on ``probs``, one after
    another as its slice loop runs them; (seconds, kind, sample)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "bin", "pics")
    t = 0.0
    for p in probs:
        if os.path.exists(exe):
            t += reference_pics_seconds(p["traj"], p["sens"], p["ksp"], iters=iters)
        else:
            from oracle import nufft_oracle as orc
            C = p["sens"].shape[3]
            t0 = time.perf_counter()
            orc.pics_l2(p["traj"].real.reshape(3, -1, order="F"), p["ksp"].reshape(-1, C, order="F"), p["sens"],
                        lam=LAM, maxiter=iters)
            t += time.perf_counter() - t0
    Ns = [p["sens"].shape[0] for p in probs]
    Cs = [p["sens"].shape[3] for p in probs]
    kind = "reference" if os.path.exists(exe) else "port"
    sample = (f"first {len(probs)} of the 512 uneven problems (N {Ns}, coils {Cs}), pics -l2 -r{LAM} "
              f"-i{iters} -t each, "
              + ("the reference's CPU pics (OpenMP), wall incl. .cfl I/O" if kind == "reference"
                 else "the NumPy oracle (float64, 1 core)"))
    return t, kind, sample


def batch_cpu_baseline():
    """cpu_baseline of the batch line: the reference on the bounded sample."""
    probs = batch_reference_sample()
    dt, kind, sample = batch_reference_seconds(probs)
    return {"value": len(probs) / dt, "unit": "recons/s", "cores": os.cpu_count() if kind == "reference" else 1,
            "kind": kind, "sample": sample}


def run_reference_batch(args):
    """--impl reference --workload batch: recons/s of the reference's CPU pics
    over a bounded sample of the uneven batch."""
    probs = batch_reference_sample()
    times = []
    for i in range(args.warmup + args.steps):
        dt, kind, sample = batch_reference_seconds(probs)
        if i >= args.warmup:
            times.append(dt)
    tot = sum(times)
    value = len(probs) * len(times) / tot
    cores = os.cpu_count() if kind == "reference" else 1
    print(json.dumps({"metric": "batched uneven CG-SENSE recons/s (20 CG iterations each)", "impl": "reference",
                      "value": value, "unit": "recons/s", "n_gpus": 0, "steps": args.steps,
                      "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True,
                      "scaling": "strong", "dtype": "f32", "data": "synthetic",
                      "config": {"workload": "batch512_uneven_2d_i20", "problems": 512, "iters": 20,
                                 "lambda": LAM, "sampled_problems": len(probs)},
                      "cpu_baseline": {"value": value, "unit": "recons/s", "cores": cores, "kind": kind,
                                       "sample": sample},
                      "e2e": {"value": value, "unit": "recons/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}), flush=True)


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU path on the host cores."""
    if rank != 0:
        return
    if args.workload == "batch":
        run_reference_batch(args)
        return
    traj, truth, sens, rng = make_problem(1000)
    # the same input bytes as the other arm: its k-space simulation (the
    # library's forward NUFFT on the GPU, outside the timed region); the timed
    # path below is the reference's own pics alone
    from oracle import nufft_oracle as orc
    A = orc.SenseOracle(traj.real.reshape(3, -1, order="F"), sens)
    try:
        ksp = simulate_ksp(traj, truth, sens, rng)
        inputs = inputs_record(traj, sens, ksp)
    except Exception as e:      # no usable GPU here: the oracle's forward model instead
        y = A.forward(truth.reshape(N_IMG, N_IMG, 1, 1))
        from bart_b200 import synth
        ksp = synth.add_noise(y, SNR_DB, rng).reshape(1, traj.shape[1], traj.shape[2], COILS, order="F")
        inputs = dict(inputs_record(traj, sens, ksp), ksp_generator=f"the oracle's forward model ({e})")
    kind = "reference" if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "bin", "pics")) else "port"
    # pics has no tolerance option: the iteration count that takes the
    # reference's own CG on these inputs to the 1e-4 true normal-equation
    # residual (checked against the FP64 oracle), found before timing
    yk = ksp.reshape(-1, COILS, order="F")
    adj = A.adjoint(yk)
    b_rhs = adj / orc.estimate_scaling_norm(adj)
    iters, true_res = REF_ITERS_TO_TOL, None
    if kind == "reference":
        while True:
            outs = []
            reference_pics_seconds(traj, sens, ksp, iters=iters, out=outs)
            x = outs[-1].astype(np.complex128).reshape(adj.shape, order="F")
            true_res = float(orc.normal_residual(A, x, b_rhs, LAM))
            if true_res <= TOL or iters >= 2 * REF_ITERS_TO_TOL:
                break
            iters += 2
    run = (lambda: reference_pics_seconds(traj, sens, ksp, iters=iters)) if kind == "reference" else \
        (lambda: oracle_pics_seconds(traj, sens, ksp, iters=iters))
    for _ in range(args.warmup):
        run()
    times = [run() for _ in range(args.steps)]
    tot = sum(times)
    value = args.steps / tot
    line = {"metric": METRIC, "value": value, "unit": "recons/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": workload_config(),
            "solver": {"method": "the reference's pics: plain CG", "iters": iters,
                       "why": "pics has no tolerance option: the fewest iterations (from 50 in steps of 2) "
                              "whose true normal-equation residual is <= 1e-4 on these inputs, found before timing"},
            "inputs": inputs,
            "true_rel_residual": true_res,
            "cpu_baseline": {"value": value, "unit": "recons/s", "cores": os.cpu_count() if kind == "reference" else 1,
                             "kind": kind, "sample": f"full recon per step (pics -l2 -r{LAM} -i{iters}), "
                                                     "wall time incl. .cfl I/O"},
            "e2e": {"value": value, "unit": "recons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def profiled_traffic(path):
    """DRAM bytes (read + write) of one launch from a committed ncu summary
    (its '| dram bytes per launch (read + write) | N |' row), or None."""
    import re
    if not os.path.exists(path):
        return None
    m = re.search(r"\|\s*dram bytes per launch \(read \+ write\)\s*\|\s*(\d+)\s*\|", open(path).read())
    return int(m.group(1)) if m else None


def peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return float(json.load(open(path))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="cgsense2d", choices=["cgsense2d", "nufft3d", "normal3d", "batch", "scatter", "ecalib"])
    ap.add_argument("--coils", type=int, default=None, help="normal3d (default 8) / ecalib (default 16): coils")
    ap.add_argument("--slices", type=int, default=0,
                    help="ecalib: also time the bart -l slice loop over this many slices, 1 and 4 workers")
    ap.add_argument("--ndim", type=int, default=None, choices=[2, 3],
                    help="ecalib: 2 (256^2, 16 coils) or 3 (128^3, 8 coils)")
    ap.add_argument("--analysis", action="store_true",
                    help="batch: also the solves spread over streams and timed alone per embedding size")
    ap.add_argument("--spokes", type=int, default=20000, help="nufft3d: kooshball spokes")
    ap.add_argument("--methods", default="fcg_padded,fcg_circulant,cg,fcg_learned",
                    help="solvers to time (cgsense2d); the first is the headline")
    ap.add_argument("--lean", action="store_true",
                    help="skip the fixed-iteration, end-to-end and NUFFT extras (for profiling runs)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import ctypes

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

    if args.workload == "nufft3d":
        if rank == 0:
            print(json.dumps(run_nufft3d(dev, args.steps, args.warmup, args.spokes)), flush=True)
        return

    if args.workload == "normal3d":
        if rank == 0:
            print(json.dumps(run_normal3d(dev, args.steps, args.warmup, args.coils or 8)), flush=True)
        return

    if args.workload == "ecalib":
        if rank == 0:
            nd = args.ndim or 2
            print(json.dumps(run_ecalib(dev, args.steps, args.warmup, N=256 if nd == 2 else 128,
                                        coils=args.coils or (16 if nd == 2 else 8), ndim=nd,
                                        cpu_base=not args.no_cpu_baseline, slices=args.slices)), flush=True)
        return

    if args.workload == "scatter":
        if rank == 0:
            print(json.dumps(run_scatter(dev, args.steps, args.warmup)), flush=True)
        return

    if args.workload == "batch":
        out = run_batch(dev, args.steps, args.warmup, rank=rank, world=world, cpu_base=not args.no_cpu_baseline,
                        analysis=args.analysis)
        if rank == 0:
            print(json.dumps(out), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    from bart_b200.dist import aggregate_rate, rank_seed, reduce_max
    traj, truth, sens, rng = make_problem(rank_seed(1000, rank))
    ksp = simulate_ksp(traj, truth, sens, rng)

    def dev_tensor(a):
        return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).to(dev)

    traj_d, sens_d, ksp_d = dev_tensor(traj), dev_tensor(sens), dev_tensor(ksp)
    img_d = torch.empty(N_IMG * N_IMG, dtype=torch.complex64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    from bart_b200.precnet import PrecNet
    net = PrecNet.load()
    # the solvers to 1e-4: the headline is the fastest, PCG with the
    # padded-circulant preconditioner; flexible CG with the reference's
    # circulant preconditioner, plain CG (the reference's method) and the
    # learned correction are measured beside it
    all_methods = {"cg": 0, "fcg_circulant": 1, "fcg_learned": 2, "fcg_padded": 3}
    names = [m for m in args.methods.split(",") if m]
    assert names and all(m in all_methods for m in names), f"--methods from {list(all_methods)}"
    headline = names[0]
    methods = {k: all_methods[k] for k in names}
    confs = {k: PicsConf(lam=LAM, maxiter=MAXITER, tol=TOL, toeplitz=True, precond=v) for k, v in methods.items()}
    conf = confs[headline]

    def make(c):
        p = Pics(traj_d, sens_d, ksp_dims=list(ksp.shape), conf=c, traj_dims=list(traj.shape),
                 sens_dims=list(sens.shape))
        if c.precond == 2:
            p.set_precnet(net)
        return p

    def step(c=conf):
        p = make(c)
        p.run(ksp_d, out=img_d)
        p.free()

    def solve_info(c):
        """iterations, residuals and device kernels of one step (untimed)"""
        p = make(c)
        p.run(ksp_d, out=img_d)
        it, rr, sc = p.stats()
        kn = p.kernels()
        tr = true_residual(dev, p, traj_d, sens_d, ksp_d, img_d, ksp.shape, traj.shape, sc)
        p.free()
        return it, rr, tr, kn

    for c in confs.values():
        for _ in range(max(3, args.warmup)):
            step(c)

    info = {k: solve_info(c) for k, c in confs.items()}
    iters, rres, tres, kernels_per_step = info[headline]

    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    with ClockSampler(local) as clk:
        ms = timed_steps(step, args.steps, flush, stream)
    ms_max = reduce_max(ms, dev)
    if world > 1:
        dist.barrier()

    # the other methods, same steps
    method_lines = {}
    for k, c in confs.items():
        mms = ms if k == headline else timed_steps(lambda: step(c), args.steps, flush, stream)
        it_k, rr_k, tr_k, _ = info[k]
        method_lines[k] = {"recons_per_s": args.steps / (mms / 1e3), "ms_per_recon": mms / args.steps,
                           "iterations": it_k, "recursive_rel_residual": rr_k, "true_rel_residual": tr_k}

    # dominant kernel: per-launch CUDA events over the same steps, run again
    # with the CG loop launched from the host (events cannot sit inside the
    # graph's while body) for exactly the iterations the solve took, so the
    # same kernels run on the same inputs
    conf_prof = PicsConf(lam=LAM, maxiter=iters, tol=0.0, toeplitz=True, precond=methods[headline])
    lib.bnufft_prof_start(DOMINANT.encode())
    timed_steps(lambda: step(conf_prof), args.steps, flush, stream)
    kms, kn = ctypes.c_double(), ctypes.c_long()
    lib.bnufft_prof_stop(ctypes.byref(kms), ctypes.byref(kn))

    # the same solve at a fixed 30 iterations (Toeplitz on and off)
    fixed = {}
    for toep in (() if args.lean else (True, False)):
        c = PicsConf(lam=LAM, maxiter=ITERS, toeplitz=toep)
        step(c)
        fms = timed_steps(lambda: step(c), max(3, args.steps // 4), flush, stream)
        fixed["toeplitz" if toep else "no_toeplitz"] = {"recons_per_s": max(3, args.steps // 4) / (fms / 1e3),
                                                        "ms_per_recon": fms / max(3, args.steps // 4)}

    # end to end through the host API: pinned host arrays in, host image out
    # (the library stages them through device buffers inside the call)
    def pinned(a):
        t = torch.empty(a.size, dtype=torch.complex64, pin_memory=True)
        v = t.numpy().reshape(a.shape, order="F")
        v[...] = a
        return t, v

    _keep = [pinned(traj), pinned(sens), pinned(ksp), pinned(np.zeros((N_IMG, N_IMG, 1), dtype=np.complex64))]
    traj_h, sens_h, ksp_h, img_h = (v for _, v in _keep)
    h2d = traj.nbytes + sens.nbytes + ksp.nbytes
    d2h = N_IMG * N_IMG * 8
    e2e_steps = max(3, args.steps // 2)

    def step_host():
        ph = Pics(traj_h, sens_h, ksp_dims=list(ksp.shape), conf=conf)
        ph.run(ksp_h, out=img_h)       # returns after the image is on the host
        ph.free()

    if args.lean:
        e2e_steps = 0
    else:
        step_host()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2e_t = 0.0
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        step_host()
        e2e_t += time.perf_counter() - t0
    e2e_s = reduce_max(e2e_t, dev)

    # roofline of the dominant kernel: Toeplitz column pass, per launch
    # reads + writes the [2X, Y, C] row-transformed buffer and reads the PSF
    G0, G1 = 2 * N_IMG, 2 * N_IMG
    alg_bytes = 2 * (G0 * N_IMG * COILS * 8) + G0 * G1 * 8
    k_avg_s = (kms.value / 1e3) / max(1, kn.value)
    peak, peak_src = peak_hbm()
    achieved = alg_bytes / k_avg_s / 1e9 if k_avg_s > 0 else None
    traffic = profiled_traffic(DOMINANT_PROFILE)
    # its FFT work: a forward and an inverse G1-point transform per column
    # (G0 columns x COILS), 5 n log2 n flop each
    fft_flop = 2 * G0 * COILS * 5 * G1 * np.log2(G1)
    fft_tflops = fft_flop / k_avg_s / 1e12 if k_avg_s > 0 else None

    nufft = nufft_throughput(dev) if (rank == 0 and not args.lean) else None
    vs_cufft = fft_vs_cufft(dev, traj, sens) if (rank == 0 and not args.lean) else None

    if rank == 0:
        value = aggregate_rate(world, args.steps, ms_max / 1e3)
        line = {"metric": METRIC, "value": value, "unit": "recons/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": workload_config(),
                "solver": {"method": {"cg": "plain CG (the reference's pics)",
                                      "fcg_circulant": "flexible CG with the reference's circulant PSF preconditioner",
                                      "fcg_learned": "flexible CG with the padded-circulant preconditioner and the learned correction (first iteration), then PCG",
                                      "fcg_padded": "PCG with the padded-circulant preconditioner"}[headline]
                                     + " (same normal equations and tolerance as the reference's plain-CG pics)",
                           "maxiter": MAXITER},
                "parallelism": f"replicas{world}",
                "l2": "flushed before every timed step (512 MB write); inside a step the ~60 MB "
                      "working set stays L2-resident across CG iterations",
                "inputs": inputs_record(traj, sens, ksp),
                "e2e": {"value": aggregate_rate(world, e2e_steps, e2e_s) if e2e_steps else None, "unit": "recons/s",
                        "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "gpu_launches": kernels_per_step * args.steps,
                "cg": {"method": headline, "iterations": iters, "recursive_rel_residual": rres,
                       "true_rel_residual": tres, "loop": "one CUDA graph with a while node per solve"},
                "methods": method_lines,
                "fixed_30_iters": fixed,
                "nufft": nufft,
                "toeplitz_normal_vs_cufft": vs_cufft,
                "roofline": {"bound": "hbm", "kernel": DOMINANT, "achieved": achieved, "peak": peak,
                             "peak_source": peak_src, "unit": "GB/s",
                             "frac": (achieved / peak) if achieved else None,
                             "traffic": traffic, "alg_bytes": alg_bytes,
                             "avg_launch_us": k_avg_s * 1e6, "launches": kn.value,
                             "fft_flop": fft_flop, "fp32_tflops": fft_tflops,
                             "fp32_peak_tflops": FP32_PEAK_TFLOPS,
                             "fp32_frac": (fft_tflops / FP32_PEAK_TFLOPS) if fft_tflops else None,
                             "fp32_peak_source": "nominal: 148 SMs x 128 lanes x 2 x 1.965 GHz",
                             "timing": "CUDA events per launch over the same steps, CG loop host-launched "
                                       "for the solve's iteration count"},
                "clocks": clk.summary()}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(traj, sens, ksp, method_lines["cg"]["iterations"])
        if world == 1 and not args.lean:
            # the other configs' workloads, timed in the same run: 3D
            # kooshball NUFFT + CG-SENSE, the batch of 512 uneven problems and
            # the ESPIRiT calibration
            torch.cuda.empty_cache()
            line["kooshball3d"] = run_nufft3d(dev, 3, 2)
            torch.cuda.empty_cache()
            line["kooshball3d"]["normal3d"] = run_normal3d(dev, 5, 3)
            torch.cuda.empty_cache()
            line["batch512"] = run_batch(dev, 2, 3, cpu_base=not args.no_cpu_baseline)
            torch.cuda.empty_cache()
            # ESPIRiT calibration of the maps (bart ecalib defaults), 256^2, 16 coils
            line["ecalib2d"] = run_ecalib(dev, 10, 3, coils=16, cpu_base=not args.no_cpu_baseline)
        print(json.dumps(line), flush=True)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
