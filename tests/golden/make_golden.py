"""Regenerate the golden fixtures from the reference's own CPU tools.

Runs the mrirecon/bart v1.0.00 tools built by ``oracle/refbuild/Makefile``
(``oracle/_ref/bin``: nufft, pics, traj, ecalib and the refnormal checker) on
seeded synthetic inputs and stores inputs and outputs as compressed .npz
files next to this script. Only needed when the fixtures change; the tests
read the .npz files and never run the reference.

    make -f oracle/refbuild/Makefile -j8
    python tests/golden/make_golden.py            # all fixtures
    python tests/golden/make_golden.py --uneven   # only the non-power-of-two sizes
    python tests/golden/make_golden.py --kb       # only the KB table and roll-off
    python tests/golden/make_golden.py --fullsize # only the C1 / C2 full-size cases
    python tests/golden/make_golden.py --gpu-gridding  # the reference's GPU-gridding test inputs
    python tests/golden/make_golden.py --kooshball     # 3D kooshball at 32^3, 2 coils
    python tests/golden/make_golden.py --basis         # subspace basis (nufft / pics -B)
    python tests/golden/make_golden.py --chain         # oversampling other than 2 (nufft -o)
    python tests/golden/make_golden.py --stream        # a k-space stream (copy --stream | tee -b)
    python tests/golden/make_golden.py --ecalib        # ESPIRiT calibration (ecalib)
"""

from __future__ import annotations

import os
import subprocess
import sys
import tempfile
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from bart_b200 import synth  # noqa: E402
from bart_b200.cfl import readcfl, writecfl  # noqa: E402

BIN = os.path.join(ROOT, "oracle", "_ref", "bin")


def run(*args, cwd, env=None):
    r = subprocess.run([os.path.join(BIN, args[0])] + list(args[1:]), cwd=cwd, capture_output=True, text=True,
                       env=env)
    if r.returncode != 0:
        raise RuntimeError(f"{args}: {r.stderr}")


def cplx(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def nufft_case(name, traj, img, periodic=False, normal=True, pattern=None):
    with tempfile.TemporaryDirectory() as d:
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        writecfl(os.path.join(d, "t"), traj)
        writecfl(os.path.join(d, "x"), img)
        P = ["-P"] if periodic else []
        if pattern is not None:
            writecfl(os.path.join(d, "w"), pattern)
            P += ["-p", "w"]
        run("nufft", *P, "t", "x", "k", cwd=d)
        fwd = readcfl(os.path.join(d, "k"))
        ksp = cplx(rng, fwd.shape)
        writecfl(os.path.join(d, "y"), ksp)
        dims = ":".join(str(s) for s in (list(img.shape) + [1, 1])[:3])
        run("nufft", *P, "-a", f"-x{dims}", "t", "y", "a", cwd=d)
        adj = readcfl(os.path.join(d, "a"))
        out = dict(traj=traj, img=img, fwd=fwd, ksp=ksp, adj=adj)
        if pattern is not None:
            out["pattern"] = pattern
        if normal:
            run("refnormal", *P, "t", "x", "n", "p", cwd=d)
            out["normal"] = readcfl(os.path.join(d, "n"))
            out["psf"] = readcfl(os.path.join(d, "p"))
            run("refnormal", *P, "--no-toeplitz", "t", "x", "ne", cwd=d)
            out["normal_explicit"] = readcfl(os.path.join(d, "ne"))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **{k: np.asarray(v) for k, v in out.items()})
    print(name, {k: np.shape(v) for k, v in out.items()})


def nudft_case(name, traj, img):
    """bart nufft -s (direct DFT), forward and adjoint."""
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "t"), traj)
        writecfl(os.path.join(d, "x"), img)
        run("nufft", "-s", "t", "x", "k", cwd=d)
        fwd = readcfl(os.path.join(d, "k"))
        ksp = cplx(rng, fwd.shape)
        writecfl(os.path.join(d, "y"), ksp)
        dims = ":".join(str(s) for s in (list(img.shape) + [1, 1])[:3])
        run("nufft", "-s", "-a", f"-x{dims}", "t", "y", "a", cwd=d)
        adj = readcfl(os.path.join(d, "a"))
    out = dict(traj=traj, img=img, fwd=fwd, ksp=ksp, adj=adj)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **{k: np.asarray(v) for k, v in out.items()})
    print(name, {k: np.shape(v) for k, v in out.items()})


def inverse_case(name, traj, ksp, dims):
    out = dict(traj=traj, ksp=ksp)
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "t"), traj)
        writecfl(os.path.join(d, "k"), ksp)
        x = ":".join(str(v) for v in dims)
        for key, args in [("inv_m5", ["-m5"]), ("inv_m5_l", ["-m5", "-l0.1"]), ("inv_m5_c", ["-m5", "-c"]),
                          ("inv_m5_c_l", ["-m5", "-c", "-l0.1"]), ("inv_m30_c", ["-m30", "-c"])]:
            run("nufft", "-i", f"-x{x}", *args, "t", "k", "o", cwd=d)
            out[key] = readcfl(os.path.join(d, "o"))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, {k: np.shape(v) for k, v in out.items()})


def sense_problem(N, C, spokes, seed, ndim=2):
    """Seeded CG-SENSE problem: trajectory, ellipse phantom, polynomial maps,
    k-space simulated by the oracle's SENSE forward model plus 40 dB noise.
    Deterministic: the full-size tests regenerate it from the seed."""
    from oracle.nufft_oracle import SenseOracle
    rng = np.random.default_rng(seed)
    traj = synth.radial_traj(N, spokes) if ndim == 2 else synth.kooshball_traj(N, spokes)
    truth = synth.ellipse_phantom(N, 20, rng, ndim=ndim)
    sens = synth.coil_maps(N, C, rng, ndim=ndim)
    A = SenseOracle(traj.real.reshape(3, -1, order="F"), sens)
    y = A.forward(truth.reshape(N, N, 1 if ndim == 2 else N, 1))
    y = synth.add_noise(y, 40.0, rng)
    ksp = y.reshape(1, traj.shape[1], traj.shape[2], C, order="F")
    return traj, truth, sens, ksp


def sha256(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes(order="F")).hexdigest()


def pics_case(name, N, C, spokes, seed, ndim=2, runs=None, store_inputs=True, spread=()):
    """Reference pics outputs on a seeded problem. store_inputs=False keeps
    only the seed and a checksum of the k-space (full-size cases); spread
    lists runs repeated with 1, 2, 4 and 8 OpenMP threads, whose largest
    difference to the stored run measures the reference's own run-to-run
    spread (its gridding adds with OpenMP atomics in thread order)."""
    traj, truth, sens, ksp = sense_problem(N, C, spokes, seed, ndim)
    out = dict(traj=traj, sens=sens, ksp=ksp, truth=truth) if store_inputs else \
        dict(seed=np.int64(seed), N=np.int64(N), C=np.int64(C), spokes=np.int64(spokes), ksp_sha256=sha256(ksp))
    runs = runs or [("x5_w1", ["-i5", "-w1"]), ("x30_w1", ["-i30", "-w1"]), ("x30", ["-i30"]),
                    ("x5_w1_notoep", ["-i5", "-w1", "--no-toeplitz"]), ("x30_rescale", ["-i30", "-S"])]
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "t"), traj)
        writecfl(os.path.join(d, "s"), sens)
        writecfl(os.path.join(d, "k"), ksp)
        for key, args in runs:
            run("pics", "-l2", "-r0.01", *args, "-t", "t", "k", "s", "o", cwd=d)
            out[key] = readcfl(os.path.join(d, "o"))
            if key in spread:
                sp = 0.0
                for th in ("1", "2", "4", "8"):
                    run("pics", "-l2", "-r0.01", *args, "-t", "t", "k", "s", "o1", cwd=d,
                        env=dict(os.environ, OMP_NUM_THREADS=th))
                    o1 = readcfl(os.path.join(d, "o1"))
                    sp = max(sp, np.linalg.norm((o1 - out[key]).ravel()) / np.linalg.norm(out[key].ravel()))
                out[key + "_spread"] = np.float64(sp)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, {k: (np.shape(v) if np.ndim(v) else v) for k, v in out.items()})


def gpu_gridding_case(name="pics2d_gpu_gridding_n128"):
    """The inputs of the reference's own GPU-gridding test
    (tests/gpu.mk:27-37, test-pics-gpu-noncart-gridding): radial trajectory
    256 x 64 scaled by 0.5, the analytic Shepp-Logan k-space on it, a
    128 x 128 map of ones; the reference's CPU pics -S -r0.001 (30
    iterations) is the result its GPU gridding must match to nrmse 0.007.
    Also stored: the spread of that output between 1 and all OpenMP threads."""
    with tempfile.TemporaryDirectory() as d:
        run("traj", "-r", "-x256", "-y64", "traj", cwd=d)
        run("scale", "0.5", "traj", "traj2", cwd=d)
        run("phantom", "-t", "traj2", "ksp", cwd=d)
        run("ones", "3", "128", "128", "1", "o", cwd=d)
        run("pics", "-S", "-r0.001", "-t", "traj2", "ksp", "o", "reco1", cwd=d)
        run("pics", "-S", "-r0.001", "-t", "traj2", "ksp", "o", "reco1t1", cwd=d,
            env=dict(os.environ, OMP_NUM_THREADS="1"))
        traj, ksp, reco = readcfl(os.path.join(d, "traj2")), readcfl(os.path.join(d, "ksp")), \
            readcfl(os.path.join(d, "reco1"))
        t1 = readcfl(os.path.join(d, "reco1t1"))
    spread = np.float64(np.linalg.norm((t1 - reco).ravel()) / np.linalg.norm(reco.ravel()))
    out = dict(traj=traj, ksp=ksp, reco=reco, spread=spread)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, {k: (np.shape(v) if np.ndim(v) else v) for k, v in out.items()})


def kooshball_case(name="nufft3d_n32_c2"):
    """3D golden-means kooshball at 32^3 (400 spokes x 64 samples), 2 coils:
    the reference's nufft forward, adjoint, and its Toeplitz normal with the
    PSF. Inputs regenerate from the seed (image) and the trajectory
    generator; only outputs and checksums are stored."""
    seed = 20261206
    rng = np.random.default_rng(seed)
    traj = synth.kooshball_traj(32, 400)
    img = cplx(rng, (32, 32, 32, 2))
    ksp = cplx(rng, (1, traj.shape[1], traj.shape[2], 2))
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "t"), traj)
        writecfl(os.path.join(d, "x"), img)
        writecfl(os.path.join(d, "y"), ksp)
        run("nufft", "t", "x", "k", cwd=d)
        run("nufft", "-a", "-x32:32:32", "t", "y", "a", cwd=d)
        run("refnormal", "t", "x", "n", "p", cwd=d)
        out = dict(seed=np.int64(seed), img_sha256=sha256(img), ksp_sha256=sha256(ksp),
                   fwd=readcfl(os.path.join(d, "k")), adj=readcfl(os.path.join(d, "a")),
                   normal=readcfl(os.path.join(d, "n")))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, {k: np.shape(v) for k, v in out.items()})


def fullsize_cases():
    """The configs' own sizes. C1: 256^2 image, 402 golden-angle spokes x 512
    samples, forward then adjoint of the forward's output. C2: 256^2, 16
    coils, 96 spokes x 512, pics -l2 -r0.01 at 30 iterations (automatic and
    unit scaling) and 5 iterations. Inputs regenerate from the seeds."""
    seed = 20261205
    rng = np.random.default_rng(seed)
    traj = synth.radial_traj(256, 402)
    img = cplx(rng, (256, 256))
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "t"), traj)
        writecfl(os.path.join(d, "x"), img)
        run("nufft", "t", "x", "k", cwd=d)
        fwd = readcfl(os.path.join(d, "k"))
        run("nufft", "-a", "-x256:256:1", "t", "k", "a", cwd=d)
        adj = readcfl(os.path.join(d, "a"))
    out = dict(seed=np.int64(seed), spokes=np.int64(402), img_sha256=sha256(img), fwd=fwd, adj=adj)
    np.savez_compressed(os.path.join(HERE, "nufft2d_c1_n256.npz"), **out)
    print("nufft2d_c1_n256", {k: np.shape(v) for k, v in out.items()})
    pics_case("pics2d_c2_n256_c16", 256, 16, 96, seed=1000, store_inputs=False,
              runs=[("x5_w1", ["-i5", "-w1"]), ("x30_w1", ["-i30", "-w1"]), ("x30", ["-i30"]),
                    ("x30_w1_notoep", ["-i30", "-w1", "--no-toeplitz"]), ("x30_notoep", ["-i30", "--no-toeplitz"]),
                    ("x300_w1", ["-i300", "-w1"]), ("x300", ["-i300"])],
              spread=("x30_w1", "x30", "x300_w1", "x300"))


ROLL_SIDES = (8, 12, 16, 40, 48, 64, 128, 256, 512)


def kb_case(name="kb_table"):
    """The reference's KB table, I0(beta) and per-axis roll-off (kbtable tool)."""
    r = subprocess.run([os.path.join(BIN, "kbtable"), "2", "6"] + [str(n) for n in ROLL_SIDES],
                       capture_output=True, text=True, check=True)
    kb, roll, out = {}, {}, {}
    for line in r.stdout.split("\n"):
        f = line.split()
        if not f:
            continue
        if f[0] == "beta":
            out["beta"] = np.float64(float.fromhex(f[1]))
        elif f[0] == "i0beta":
            out["i0beta"] = np.float64(float.fromhex(f[1]))
        elif f[0] == "kb":
            kb[int(f[1])] = float.fromhex(f[2])
        elif f[0] == "roll":
            roll.setdefault(int(f[1]), {})[int(f[2])] = float.fromhex(f[3])
    out["kb"] = np.array([kb[i] for i in range(len(kb))], dtype=np.float32)
    for n, v in roll.items():
        out[f"roll_{n}"] = np.array([v[i] for i in range(n)], dtype=np.float32)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, {k: np.shape(v) for k, v in out.items()})


def t24_traj():
    with tempfile.TemporaryDirectory() as d:
        run("traj", "-r", "-G", "-x24", "-o2", "-y10", "t", cwd=d)
        return readcfl(os.path.join(d, "t"))


def t16_traj():
    with tempfile.TemporaryDirectory() as d:
        run("traj", "-r", "-G", "-x16", "-o2", "-y8", "t", cwd=d)
        return readcfl(os.path.join(d, "t"))


def uneven_cases():
    """Image sides that are not powers of two (grids of 2N cells)."""
    rng = np.random.default_rng(20261204)
    with tempfile.TemporaryDirectory() as d:
        run("traj", "-r", "-G", "-x40", "-o2", "-y20", "t", cwd=d)
        t40 = readcfl(os.path.join(d, "t"))
    nufft_case("nufft2d_n40", t40, cplx(rng, (40, 40)))
    nufft_case("nufft2d_n40_periodic", t40, cplx(rng, (40, 40)), periodic=True)
    nufft_case("nufft3d_n12", synth.kooshball_traj(12, 64), cplx(rng, (12, 12, 12)))
    pics_case("pics2d_n48_c3", 48, 3, 20, seed=9)
    nudft_case("nudft2d_n24", t24_traj(), cplx(rng, (24, 24)))
    nudft_case("nudft2d_n16_coils2", t16_traj(), cplx(rng, (16, 16, 1, 2)))
    pics_case("pics3d_n16_c2", 16, 2, 120, seed=11, ndim=3,
              runs=[("x5_w1", ["-i5", "-w1"]), ("x5_w1_notoep", ["-i5", "-w1", "--no-toeplitz"])])


def basis_nufft_case(name, traj, img, basis, pattern=None):
    """nufft -B (forward, adjoint) and the Toeplitz / explicit normal with
    the basis: img [X, Y, 1, C, 1, 1, K], basis [1, 1, 1, 1, 1, T, K],
    traj [3, Mr, Ms(, 1, 1, T)], pattern [1, Mr, Ms, 1, 1, T]."""
    with tempfile.TemporaryDirectory() as d:
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        writecfl(os.path.join(d, "t"), traj)
        writecfl(os.path.join(d, "x"), img)
        writecfl(os.path.join(d, "b"), basis)
        P = ["-B", "b"]
        if pattern is not None:
            writecfl(os.path.join(d, "w"), pattern)
            P += ["-p", "w"]
        run("nufft", *P, "t", "x", "k", cwd=d)
        fwd = readcfl(os.path.join(d, "k"))
        ksp = cplx(rng, fwd.shape)
        writecfl(os.path.join(d, "y"), ksp)
        dims = ":".join(str(s) for s in (list(img.shape) + [1, 1])[:3])
        run("nufft", *P, "-a", f"-x{dims}", "t", "y", "a", cwd=d)
        adj = readcfl(os.path.join(d, "a"))
        run("refnormal", *P, "t", "x", "n", cwd=d)
        nrm = readcfl(os.path.join(d, "n"))
        run("refnormal", *P, "--no-toeplitz", "t", "x", "ne", cwd=d)
        nre = readcfl(os.path.join(d, "ne"))
    out = dict(traj=traj, img=img, basis=basis, fwd=fwd, ksp=ksp, adj=adj, normal=nrm, normal_explicit=nre)
    if pattern is not None:
        out["pattern"] = pattern
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **{k: np.asarray(v) for k, v in out.items()})
    print(name, {k: np.shape(v) for k, v in out.items()})


def basis_pics_case(name, traj, ksp, sens, basis, pattern, iters=10):
    """pics -B with a sampling pattern (tests/pics.mk test-pics-basis-noncart
    style): -l2 -r0.01 -i iters, automatic scaling, Toeplitz. Also stores the
    reference's own spread: its Toeplitz against its explicit normal
    (--no-toeplitz), the float32 sensitivity of these unconverged iterates."""
    with tempfile.TemporaryDirectory() as d:
        for n, a in (("t", traj), ("k", ksp), ("s", sens), ("b", basis), ("w", pattern)):
            writecfl(os.path.join(d, n), a)
        env = dict(os.environ, OMP_NUM_THREADS="1")
        run("pics", "-l2", "-r0.01", f"-i{iters}", "-B", "b", "-p", "w", "-t", "t", "k", "s", "o", cwd=d, env=env)
        out = readcfl(os.path.join(d, "o"))
        run("pics", "-l2", "-r0.01", f"-i{iters}", "-B", "b", "-p", "w", "--no-toeplitz", "-t", "t", "k", "s", "e",
            cwd=d, env=env)
        spread = float(np.linalg.norm(readcfl(os.path.join(d, "e")) - out) / np.linalg.norm(out))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), traj=traj, ksp=ksp, sens=sens, basis=basis,
                        pattern=pattern, out=out, iters=iters, spread=spread)
    print(name, out.shape, "reference spread", spread)


def chain_case(name, traj, img, oss, pattern=None):
    """nufft -o os (the reference's chained NUFFT) forward and adjoint for
    each oversampling factor in oss."""
    out = dict(traj=traj, img=img, oss=np.asarray(oss, dtype=np.float64))
    with tempfile.TemporaryDirectory() as d:
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        writecfl(os.path.join(d, "t"), traj)
        writecfl(os.path.join(d, "x"), img)
        P = []
        if pattern is not None:
            writecfl(os.path.join(d, "w"), pattern)
            P = ["-p", "w"]
            out["pattern"] = pattern
        dims = ":".join(str(s) for s in (list(img.shape) + [1, 1])[:3])
        for i, o in enumerate(oss):
            run("nufft", *P, "-o", str(o), "t", "x", "k", cwd=d)
            fwd = readcfl(os.path.join(d, "k"))
            if i == 0:
                out["ksp"] = cplx(rng, fwd.shape)
                writecfl(os.path.join(d, "y"), out["ksp"])
            run("nufft", *P, "-o", str(o), "-a", f"-x{dims}", "t", "y", "a", cwd=d)
            out[f"fwd_{i}"] = fwd
            out[f"adj_{i}"] = readcfl(os.path.join(d, "a"))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **{k: np.asarray(v) for k, v in out.items()})
    print(name, {k: np.shape(v) for k, v in out.items()})


def chain_cases():
    rng = np.random.default_rng(2468)
    with tempfile.TemporaryDirectory() as d:
        run("traj", "-r", "-G", "-x64", "-o2", "-y24", "t", cwd=d)
        t64 = readcfl(os.path.join(d, "t"))
    img = cplx(rng, (64, 64, 1, 2))
    chain_case("nufft2d_n64_chain", t64, img, [1.5, 1.25, 2.5])
    w = (0.2 + rng.random((1,) + t64.shape[1:3])).astype(np.complex64)
    chain_case("nufft2d_n64_chain_weights", t64, img[..., :1], [1.5], pattern=w)
    chain_case("nufft3d_n16_chain", synth.kooshball_traj(16, 64), cplx(rng, (16, 16, 16)), [1.5])


def stream_case(name="stream_ksp_c4_s3"):
    """Three k-space slices (dim 13) of the pics2d_n64_c4 problem, scaled
    differently, as the reference writes them into a pipe: `copy --stream
    8192 -- k - | tee -b` (tee -b: the data inline, a binary stream). Stores
    the array and the stream's bytes."""
    g = np.load(os.path.join(HERE, "pics2d_n64_c4.npz"))
    k = g["ksp"].reshape(list(g["ksp"].shape[:4]) + [1] * 9 + [1], order="F")
    ksp = np.concatenate([k * np.complex64(s) for s in (1.0, 0.5, 2.0)], axis=13).astype(np.complex64)
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "k"), ksp)
        r = subprocess.run(f"{os.path.join(BIN, 'copy')} --stream 8192 -- k - | {os.path.join(BIN, 'tee')} -b",
                           shell=True, cwd=d, capture_output=True)
        if r.returncode != 0:
            raise RuntimeError(r.stderr.decode())
        stream = r.stdout
    np.savez_compressed(os.path.join(HERE, name + ".npz"), ksp=ksp,
                        stream=np.frombuffer(stream, dtype=np.uint8))
    print(name, ksp.shape, len(stream), "stream bytes")


def basis_cases():
    rng = np.random.default_rng(555)
    T, K = 4, 3
    with tempfile.TemporaryDirectory() as d:
        run("traj", "-r", "-G", "-x32", "-o2", "-y48", "t", cwd=d)
        t48 = readcfl(os.path.join(d, "t"))            # [3, 64, 48]
    # frame t: spokes t, t + 4, ... (interleaved golden-angle frames)
    tf = np.stack([t48[:, :, f::T] for f in range(T)], axis=-1).reshape(3, 64, 12, 1, 1, T, order="F")
    basis = cplx(rng, (1, 1, 1, 1, 1, T, K)) / np.float32(2.0)
    img = cplx(rng, (32, 32, 1, 2, 1, 1, K))
    basis_nufft_case("nufft2d_n32_basis", tf, img, basis)
    # one trajectory shared by all frames, a sampling pattern per frame
    pat = np.zeros((1, 64, 12, 1, 1, T), dtype=np.complex64)
    for f in range(T):
        pat[0, :, f::T, 0, 0, f] = 1.0                 # frame f keeps spokes f, f + 4, ... of the shared 12
    basis_nufft_case("nufft2d_n32_basis_shared", t48[:, :, :12], img, basis, pattern=pat)
    # pics -B on a sampled phantom: an orthonormal basis (as a subspace
    # basis from an SVD is), 24 spokes per frame, coil maps from the SENSE
    # generator
    with tempfile.TemporaryDirectory() as d:
        run("traj", "-r", "-G", "-x32", "-o2", "-y96", "t", cwd=d)
        t96 = readcfl(os.path.join(d, "t"))
    tf = np.stack([t96[:, :, f::T] for f in range(T)], axis=-1).reshape(3, 64, 24, 1, 1, T, order="F")
    q, _ = np.linalg.qr(rng.standard_normal((T, K)) + 1j * rng.standard_normal((T, K)))
    basis = q.astype(np.complex64).reshape(1, 1, 1, 1, 1, T, K, order="F")
    N, C = 32, 4
    sens = synth.coil_maps(N, C, rng)
    truth = np.stack([synth.ellipse_phantom(N, 8, rng) for _ in range(K)], axis=-1).reshape(N, N, 1, 1, 1, 1, K)
    from oracle import nufft_oracle as orc
    ksp = np.zeros((1, 64, 24, C, 1, T), dtype=np.complex64)
    for f in range(T):
        A = orc.SenseOracle(tf[..., 0, 0, f].real.reshape(3, -1, order="F"), sens)
        xf = sum(basis[0, 0, 0, 0, 0, f, k] * truth[..., 0, 0, k].reshape(N, N, 1, 1) for k in range(K))
        ksp[:, :, :, :, 0, f] = A.forward(xf).reshape(1, 64, 24, C, order="F").astype(np.complex64)
    ksp = synth.add_noise(ksp, 40.0, rng)
    pat2 = np.ones((1, 64, 24, 1, 1, T), dtype=np.complex64)
    basis_pics_case("pics2d_n32_basis", tf, ksp, sens.astype(np.complex64), basis, pat2)


def ecalib_case(name, ksp, args):
    """The reference's ecalib (with -V: singular values) on Cartesian
    k-space; stores the inputs, the maps, the eigenvalue maps, the singular
    values, the number of kernels and the calibration region (its debug
    output)."""
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "k"), ksp)
        r = subprocess.run([os.path.join(BIN, "ecalib"), "-d4", "-V"] + args + ["k", "s", "e"], cwd=d,
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(r.stderr)
        sens, ev = readcfl(os.path.join(d, "s")), readcfl(os.path.join(d, "e"))
    svals = np.array([float(ln.split()[2]) for ln in r.stdout.splitlines() if ln.startswith("SVALS ")],
                     dtype=np.float32)
    nk = cd = None
    for ln in r.stderr.splitlines():
        if ln.startswith("Using "):
            nk = int(ln.split()[1].split("/")[0])
        if ln.startswith("Calibration region"):
            cd = [int(v) for v in ln.split("size: ")[1].split(",")[0].split("x")]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), ksp=ksp, sens=sens, emaps=ev, svals=svals,
                        nkernels=np.int64(nk), caldims=np.array(cd), args=np.array(args))
    print(name, ksp.shape, sens.shape, "kernels", nk, "caldims", cd)


def calone_case(name, ksp, args):
    """The reference's ecalib -1: the kernels' low-resolution covariance."""
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "k"), ksp)
        run("ecalib", "-1", *args, "k", "c", cwd=d)
        cov = readcfl(os.path.join(d, "c"))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), ksp=ksp, cov=cov, args=np.array(args))
    print(name, ksp.shape, cov.shape)


def ecalib_cases():
    """Cartesian k-space of ellipse phantoms and polynomial coil maps, 40 dB
    noise, a fully sampled centre and every other line outside it."""
    rng = np.random.default_rng(9001)
    N, C = 64, 8
    img = synth.ellipse_phantom(N, 12, rng)
    k = synth.cartesian_ksp(img, synth.coil_maps(N, C, rng), rng, 40.0, 24, 2)
    ecalib_case("ecalib2d_n64_c8", k, [])
    ecalib_case("ecalib2d_n64_c8_m3_soft", k, ["-m", "3", "-c", "0.1", "-S"])
    ecalib_case("ecalib2d_n64_c8_k5_r20_n30_P", k, ["-k", "5", "-r", "20", "-n", "30", "-P", "-c", "0.3"])
    ecalib_case("ecalib2d_n64_c8_I", k, ["-I", "-c", "0.5"])
    calone_case("calone2d_n64_c8", k, [])
    X, Y, C = 40, 48, 20
    img = synth.ellipse_phantom(48, 10, rng)[4:44, :, :]
    maps = synth.coil_maps(48, C, rng)[4:44]
    k = synth.cartesian_ksp(img, maps, rng, 40.0, 20, 3)
    ecalib_case("ecalib2d_40x48_c20", k, ["-r", "20", "-c", "0.5"])
    # odd image sides (odd-length centring of the sinc interpolation), six maps
    rng2 = np.random.default_rng(77)
    img = synth.ellipse_phantom(64, 10, rng2)[7:57, 9:54]
    k = synth.cartesian_ksp(img, synth.coil_maps(64, 8, rng2)[7:57, 9:54], rng2, 40.0, 20, 2)
    ecalib_case("ecalib2d_50x45_c8_m6", k, ["-r", "20", "-m", "6", "-c", "0.2"])
    N, C = 24, 4
    img = synth.ellipse_phantom(N, 6, rng, ndim=3)
    k = synth.cartesian_ksp(img, synth.coil_maps(N, C, rng, ndim=3), rng, 40.0, 12, 2)
    ecalib_case("ecalib3d_n24_c4", k, ["-r", "12", "-k", "4", "-c", "0.4"])


def main():
    if "--ecalib" in sys.argv:
        ecalib_cases()
        return
    if "--basis" in sys.argv:
        basis_cases()
        return
    if "--chain" in sys.argv:
        chain_cases()
        return
    if "--stream" in sys.argv:
        stream_case()
        return
    if "--uneven" in sys.argv:
        uneven_cases()
        return
    if "--kb" in sys.argv:
        kb_case()
        return
    if "--fullsize" in sys.argv:
        fullsize_cases()
        return
    if "--gpu-gridding" in sys.argv:
        gpu_gridding_case()
        return
    if "--kooshball" in sys.argv:
        kooshball_case()
        return
    rng = np.random.default_rng(20261203)
    with tempfile.TemporaryDirectory() as d:
        run("traj", "-r", "-G", "-x64", "-o2", "-y24", "t", cwd=d)
        t64 = readcfl(os.path.join(d, "t"))
        run("traj", "-r", "-G", "-x32", "-o2", "-y16", "t", cwd=d)
        t32 = readcfl(os.path.join(d, "t"))
    img64 = cplx(rng, (64, 64))
    nufft_case("nufft2d_n64", t64, img64)
    nufft_case("nufft2d_n64_periodic", t64, img64, periodic=True)
    nufft_case("nufft2d_n32_coils3", t32, cplx(rng, (32, 32, 1, 3)), normal=False)
    w64 = (0.2 + rng.random((1,) + t64.shape[1:3])).astype(np.complex64)   # real positive density weights
    nufft_case("nufft2d_n64_weights", t64, img64, pattern=w64)
    t3 = synth.kooshball_traj(16, 96)
    nufft_case("nufft3d_n16", t3, cplx(rng, (16, 16, 16)))
    pics_case("pics2d_n64_c4", 64, 4, 24, seed=7)
    g = np.load(os.path.join(HERE, "nufft2d_n32_coils3.npz"))
    inverse_case("inverse2d_n32_coils3", g["traj"], g["fwd"], (32, 32, 1))
    uneven_cases()
    kb_case()
    fullsize_cases()
    gpu_gridding_case()
    kooshball_case()
    ecalib_cases()


if __name__ == "__main__":
    main()
