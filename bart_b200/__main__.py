"""Command line mirror of ``bart nufft``, ``bart pics -t`` and ``bart ecalib`` with .cfl I/O.

  python -m bart_b200 nufft [-a|-i [-c] [-l lambda] [-m iter]] [-x X:Y:Z] [-P] [-r|-t]
                            [-p pattern] [-B basis] [-o os] traj input output
  python -m bart_b200 pics -l2 -r lambda [-i iter] -t traj [-w scale] [-S]
                           [--no-toeplitz] ksp sens output
  python -m bart_b200 -l flags pics ...   (or -p flags: the same here)
  python -m bart_b200 -l flags ecalib ... (one calibration per slice)
  python -m bart_b200 ecalib [-k k] [-r cal] [-m maps] [-t thr] [-c crop] [-S] [-P] [-I] [-1]
                             [-n numsv] [-p percent] [-V] kspace sens [emaps]

The k-space argument of pics may be "-": a stream of the reference's
(src/misc/stream.c, e.g. from `copy --stream flags -- ksp -`) on stdin.
With -l flags along the streamed dims every slice is reconstructed as soon
as it has arrived; without, the whole stream is read first.

pics also takes two options the reference does not have: --precond 1|3
(flexible CG with the reference's circulant preconditioner / PCG with the
padded-circulant one; default 0, the reference's plain CG) and --tol t
(stop at ||r|| <= t ||A^H y||; default 0, run -i iterations).

With -l / -p (src/bart.c:202-217) pics runs once per index of the flagged
dims (e.g. 8192 = slices, dim 13); all those problems run as one batched
graph launch and the images are joined along the flagged dims. Launched by
torchrun with several ranks (one per GPU), the problems are split over the
ranks by their cost and rank 0 gathers the images and writes the output.

Options follow src/nufft.c:75-101, src/pics.c:137-199 and src/ecalib.c:64-97;
options of the reference that are not built here are rejected with an error.
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

from .cfl import readcfl, writecfl
from .nufft import NufftConf, nufft_create2
from .pics import Pics, PicsConf


def _vec3(s: str):
    v = [int(x) for x in s.split(":")]
    if len(v) != 3:
        raise argparse.ArgumentTypeError("expected x:y:z")
    return v


def estimate_im_dims(traj: np.ndarray):
    """estimate_im_dims (src/noncart/traj.c): 2 * ceil(max |k|) per axis, 1 if all zero."""
    t = np.abs(np.real(traj.reshape(3, -1, order="F")))
    dims = []
    for ax in range(3):
        m = float(t[ax].max()) if t.shape[1] else 0.0
        dims.append(1 if m == 0.0 else int(2 * np.ceil(m)))
    return dims


def main_nufft(argv) -> int:
    ap = argparse.ArgumentParser(prog="nufft")
    ap.add_argument("-a", dest="adjoint", action="store_true")
    ap.add_argument("-i", dest="inverse", action="store_true")
    ap.add_argument("-x", dest="dims", type=_vec3)
    ap.add_argument("-t", dest="toeplitz", action="store_true")
    ap.add_argument("-r", dest="no_toeplitz", action="store_true")
    ap.add_argument("-P", dest="periodic", action="store_true")
    ap.add_argument("-g", dest="gpu", action="store_true")
    ap.add_argument("-c", dest="precond", action="store_true")
    ap.add_argument("-l", dest="lam", type=float, default=0.0)
    ap.add_argument("-m", dest="iters", type=int, default=50)
    ap.add_argument("-p", dest="pattern")
    ap.add_argument("-B", dest="basis", help="temporal (or other) basis [1,1,1,1,1,T,K]")
    ap.add_argument("-o", "--oversampling", dest="os", type=float, default=2.0,
                    help="oversampling (default 2; other values: the reference's chained NUFFT, no Toeplitz)")
    ap.add_argument("-s", dest="dft", action="store_true", help="direct non-uniform DFT")
    ap.add_argument("--lowmem", action="store_true", help="one coil's oversampled grid at a time")
    # the reference's other memory modes change what it holds, not its results;
    # the library precomputes no linear phases or fftmod tables, so they are accepted as they are
    ap.add_argument("--zero-mem", action="store_true", help="accepted (the reference's zero-overhead mode)")
    ap.add_argument("--no-precomp", action="store_true", help="accepted (no precomputed tables)")
    ap.add_argument("traj")
    ap.add_argument("input")
    ap.add_argument("output")
    a = ap.parse_args(argv)
    if a.adjoint and a.inverse:
        sys.stderr.write("Adjoint and inverse requested at the same time.\n")
        return 1
    traj = readcfl(a.traj)
    tdims = list(traj.shape)
    # the PSF is only built for the inverse (src/nufft.c:121-122); Toeplitz is on by default there
    conf = NufftConf(toeplitz=a.inverse and not a.no_toeplitz, periodic=a.periodic, lowmem=a.lowmem, os=a.os)
    inp = readcfl(a.input)
    pat = readcfl(a.pattern) if a.pattern else None
    bas = readcfl(a.basis) if a.basis else None
    bd = None if bas is None else (list(bas.shape) + [1] * 16)[:16]
    pd = None if pat is None else list(pat.shape)

    def create(kd, cd):
        return nufft_create2(kd, cd, tdims, traj, pd, pat, bd, bas, conf=conf)

    if bas is not None:     # src/nufft.c:169-176, 208-211, 284-288
        if a.dft or a.inverse:
            sys.stderr.write("-B: forward and adjoint only here\n")
            return 1
        if a.adjoint:
            kd = (list(inp.shape) + [1] * 16)[:16]
            cd = (a.dims or estimate_im_dims(traj)) + kd[3:]
            cd[5], cd[6] = 1, bd[6]
            op = create(kd, cd)
            writecfl(a.output, op.adjoint(inp).reshape(cd, order="F"))
        else:
            cd = (list(inp.shape) + [1] * 16)[:16]
            kd = [1, tdims[1], tdims[2]] + cd[3:]
            kd[5], kd[6] = bd[5], 1
            op = create(kd, cd)
            writecfl(a.output, op.forward(inp).reshape(kd, order="F"))
        op.free()
        return 0
    if a.dft:   # src/nufft.c:244, 297 (no basis, no pattern)
        from .nufft import Nudft
        if a.inverse or pat is not None:
            sys.stderr.write("-s: forward and adjoint only, without -p\n")
            return 1
        if a.adjoint:
            kd = list(inp.shape)
            cd = (a.dims or estimate_im_dims(traj)) + kd[3:]
            op = Nudft(kd, cd, tdims, traj)
            writecfl(a.output, op.adjoint(inp).reshape(cd, order="F"))
        else:
            cd = list(inp.shape)
            kd = [1, tdims[1], tdims[2]] + cd[3:]
            op = Nudft(kd, cd, tdims, traj)
            writecfl(a.output, op.forward(inp).reshape(kd, order="F"))
        op.free()
        return 0
    if a.inverse:
        kd = list(inp.shape)
        cd = (a.dims or estimate_im_dims(traj)) + kd[3:]
        op = nufft_create2(kd, cd, tdims, traj, None if pat is None else list(pat.shape), pat, conf=conf)
        writecfl(a.output, op.inverse(inp, lam=a.lam, maxiter=a.iters, precond=a.precond).reshape(cd, order="F"))
        op.free()
        return 0
    if a.adjoint:
        kd = list(inp.shape)
        cd = (a.dims or estimate_im_dims(traj)) + kd[3:]
        op = nufft_create2(kd, cd, tdims, traj, None if pat is None else list(pat.shape), pat, conf=conf)
        writecfl(a.output, op.adjoint(inp).reshape(cd, order="F"))
    else:
        cd = list(inp.shape)
        kd = [1, tdims[1], tdims[2]] + cd[3:]
        op = nufft_create2(kd, cd, tdims, traj, None if pat is None else list(pat.shape), pat, conf=conf)
        writecfl(a.output, op.forward(inp).reshape(kd, order="F"))
    op.free()
    return 0


def parse_pics(argv):
    """pics options and its three input arrays"""
    ap = argparse.ArgumentParser(prog="pics")
    ap.add_argument("-l", dest="reg", choices=["2"], help="only -l2 (CG) is built")
    ap.add_argument("-r", dest="lam", type=float, default=0.0)
    ap.add_argument("-i", dest="iters", type=int, default=30)
    ap.add_argument("-t", dest="traj", required=True)
    ap.add_argument("-w", dest="scaling", type=float, default=0.0)
    ap.add_argument("-S", dest="rescale", action="store_true")
    ap.add_argument("-g", dest="gpu", action="store_true")
    ap.add_argument("--no-toeplitz", dest="no_toeplitz", action="store_true")
    # not in the reference: the library's preconditioned solvers and a CG
    # tolerance (defaults keep the reference's plain CG for -i iterations)
    ap.add_argument("--precond", type=int, choices=[0, 1, 3], default=0,
                    help="0 plain CG, 1 flexible CG + circulant, 3 PCG + padded circulant")
    ap.add_argument("--tol", type=float, default=0.0, help="stop at ||r|| <= tol ||A^H y|| (0: run -i iterations)")
    ap.add_argument("ksp")
    ap.add_argument("sens")
    ap.add_argument("output")
    a = ap.parse_args(argv)
    if a.precond and a.no_toeplitz:
        ap.error("--precond needs the Toeplitz normal operator")
    a.traj_name = a.traj
    a.traj = readcfl(a.traj_name)
    if a.ksp == "-":	# a stream on stdin (src/misc/stream.c): read as it arrives
        from .stream import StreamReader
        a.ksp = StreamReader(sys.stdin.buffer)
    else:
        a.ksp = readcfl(a.ksp)
    a.sens = readcfl(a.sens)
    a.toeplitz = not a.no_toeplitz
    return a


def main_pics(argv, loop_flags: int = 0) -> int:
    a = parse_pics(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    from .stream import StreamReader
    if isinstance(a.ksp, StreamReader):
        if loop_flags and world == 1:	# each slice reconstructed as it arrives
            from .loop import stream_pics
            writecfl(a.output, stream_pics(loop_flags, a))
            return 0
        # without a loop: the whole stream is the k-space
        full = np.zeros(a.ksp.dims, dtype=np.complex64, order="F")
        for _, pos, block in a.ksp:
            sl = [slice(None)] * 16
            for d, p in zip(a.ksp.sdims, pos):
                sl[d] = slice(p, p + 1)
            full[tuple(sl)] = block
        a.ksp = full
    if loop_flags:
        from .loop import loop_pics
        if world == 1:
            writecfl(a.output, loop_pics(loop_flags, a))
            return 0
        # one rank per GPU (device = local rank mod GPU count, as the
        # reference's MPI ranks pick theirs, src/num/gpuops.c:169-187); the
        # ranks exchange only the finished images, on the host
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")) % torch.cuda.device_count())
        dist.init_process_group("gloo", timeout=timedelta(seconds=600))
        try:
            out = loop_pics(loop_flags, a)
            if rank == 0:
                writecfl(a.output, out)
            dist.barrier()
        finally:
            dist.destroy_process_group()
        return 0
    if rank != 0:	# one problem: rank 0 solves it, the others have nothing to do
        return 0
    conf = PicsConf(lam=a.lam, maxiter=a.iters, tol=a.tol, scaling=a.scaling, rescale=a.rescale, toeplitz=a.toeplitz,
                    precond=a.precond)
    p = Pics(a.traj, a.sens, ksp_dims=list(a.ksp.shape), conf=conf)
    img = p.run(a.ksp)
    p.free()
    sd = list(a.sens.shape) + [1] * 3
    writecfl(a.output, img.reshape(sd[:3], order="F"))
    return 0


def _vec3_or_one(s: str):
    """opt_vec3 (src/misc/opts.c:1075-1096): "x:y:z" or one value for all three."""
    v = s.split(":")
    if len(v) == 3:
        return [int(x) for x in v]
    return [int(v[0])] * 3


def main_ecalib(argv, loop_flags: int = 0) -> int:
    """bart ecalib (src/ecalib.c:46-262); with loop flags (bart -l / -p) one
    calibration per index of the flagged dims."""
    from .espirit import EcalibConf, ecalib
    ap = argparse.ArgumentParser(prog="ecalib")
    ap.add_argument("-t", dest="threshold", type=float, default=0.001)
    ap.add_argument("-c", dest="crop", type=float, default=0.8)
    ap.add_argument("-k", "-K", dest="kdims", type=_vec3_or_one, default=[6, 6, 6])
    ap.add_argument("-r", "-R", dest="calsize", type=_vec3_or_one, default=[24, 24, 24])
    ap.add_argument("-m", dest="maps", type=int, default=2)
    ap.add_argument("-S", dest="softcrop", action="store_true")
    ap.add_argument("-W", dest="weighting", action="store_true")
    ap.add_argument("-I", dest="intensity", action="store_true")
    ap.add_argument("-1", dest="one", action="store_true")
    ap.add_argument("-P", dest="norotphase", action="store_true")
    ap.add_argument("-N", dest="phase_normalize", action="store_true")
    ap.add_argument("-A", dest="nystroem", action="store_true")
    ap.add_argument("-O", dest="no_orthiter", action="store_true")
    ap.add_argument("-i", "--orthiter", dest="num_orthiter", type=int, default=30)
    ap.add_argument("-p", dest="percentsv", type=float, default=-1.0)
    ap.add_argument("-n", dest="numsv", type=int, default=-1)
    ap.add_argument("-a", dest="automate", action="store_true")
    ap.add_argument("-v", dest="var", type=float, default=-1.0)
    ap.add_argument("-V", dest="print_svals", action="store_true")
    ap.add_argument("-d", dest="debug", type=int, default=0)
    ap.add_argument("kspace")
    ap.add_argument("sens")
    ap.add_argument("emaps", nargs="?")
    a = ap.parse_args(argv)
    conf = EcalibConf(kdims=tuple(a.kdims), calsize=tuple(a.calsize), maps=a.maps, threshold=a.threshold,
                      numsv=a.numsv, percentsv=a.percentsv, crop=a.crop, softcrop=a.softcrop,
                      rotphase=not a.norotphase, num_orthiter=a.num_orthiter, intensity=a.intensity,
                      phase_normalize=a.phase_normalize, nystroem=a.nystroem, orthiter=not a.no_orthiter)
    if a.automate:				# src/ecalib.c:109-113
        conf.crop = -1.0
        conf.weighting = True
    if a.weighting:
        conf.weighting = True
    # under torchrun the slices are not split over the ranks: rank 0 alone
    # calibrates and writes the outputs, the others exit without work
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    ksp = readcfl(a.kspace)
    if loop_flags:
        if a.one:
            sys.stderr.write("ecalib: -1 inside a slice loop is not built\n")
            return 1
        from .loop import loop_ecalib
        sens, ev = loop_ecalib(loop_flags, ksp, conf, emaps=a.emaps is not None)
        writecfl(a.sens, sens)
        if a.emaps is not None:
            writecfl(a.emaps, ev)
        return 0
    if a.one:					# the first part alone (src/ecalib.c:171-190)
        from .espirit import calone
        cov, info = calone(ksp, conf)
        writecfl(a.sens, cov)
    else:
        sens, ev, info = ecalib(ksp, conf, emaps=a.emaps is not None)
        writecfl(a.sens, sens)
        if a.emaps is not None:
            writecfl(a.emaps, ev)
    if a.print_svals:
        for i, v in enumerate(info["svals"]):
            print(f"SVALS {i} {v:f}")
    return 0


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    flags = 0
    while argv and argv[0] in ("-l", "-p", "--loop", "--parallel-loop"):	# bart -l / -p flags
        if len(argv) < 2:
            sys.stderr.write(__doc__)
            return 2
        flags |= int(argv[1])
        argv = argv[2:]
    if not argv or argv[0] not in ("nufft", "pics", "ecalib") or (flags and argv[0] == "nufft"):
        sys.stderr.write(__doc__)
        return 2
    if "ecalib" == argv[0]:
        return main_ecalib(argv[1:], flags)
    if "pics" == argv[0]:
        return main_pics(argv[1:], flags)
    return main_nufft(argv[1:])


if __name__ == "__main__":
    sys.exit(main())
