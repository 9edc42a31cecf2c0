"""``bart -l flags`` / ``bart -p flags``: one tool run over the slices of its
files (src/bart.c:202-217, 568-600).

The reference runs the tool once per index of the flagged dimensions: every
input file is read at that index along each flagged dimension it has (a
file of size 1 there is used for every index), and the outputs are joined
along those dimensions. Here the per-index problems of ``pics`` are not run
one after another: each becomes its own SENSE model, and all of them run as
one batched graph launch (``bnufft_batch_create``: every problem's whole
solve an independent child graph), which the GPU overlaps. The results are
those of the loop of single runs up to float32 summation order.
"""

from __future__ import annotations

import itertools

import numpy as np

from .cfl import DIMS, dims16


def loop_dims(flags: int) -> list:
    """The dimensions selected by a BART loop bitmask."""
    if flags < 0 or flags >= (1 << DIMS):
        raise ValueError(f"loop flags {flags} outside the 16 dims")
    return [d for d in range(DIMS) if flags & (1 << d)]


def loop_sizes(shapes, dims) -> list:
    """Loop length per flagged dim: the files' sizes there must be 1 or one
    common value (as the reference's cfl loop requires)."""
    sizes = []
    for d in dims:
        vals = {dims16(s)[d] for s in shapes} - {1}
        if len(vals) > 1:
            raise ValueError(f"files disagree along looped dim {d}: sizes {sorted(vals)}")
        sizes.append(vals.pop() if vals else 1)
    return sizes


def loop_indices(sizes) -> list:
    """All index tuples, the first flagged dim fastest (the reference's
    default order)."""
    return [tuple(reversed(t)) for t in itertools.product(*[range(n) for n in reversed(sizes)])]


def slice_at(a: np.ndarray, dims, idx) -> np.ndarray:
    """``a`` at index idx along the flagged dims it has (size-1 dims are
    kept as they are), as an F-ordered array of the same rank."""
    a16 = a.reshape(dims16(a.shape), order="F")
    sl = [slice(None)] * DIMS
    for d, i in zip(dims, idx):
        if a16.shape[d] > 1:
            sl[d] = slice(i, i + 1)
    return np.asfortranarray(a16[tuple(sl)])


def place_at(out: np.ndarray, dims, idx, block: np.ndarray) -> None:
    """Write one index's result into the joined output."""
    sl = [slice(None)] * DIMS
    for d, i in zip(dims, idx):
        sl[d] = slice(i, i + 1)
    out[tuple(sl)] = block.reshape(out[tuple(sl)].shape, order="F")


def loop_pics(flags: int, a, dev=None) -> np.ndarray:
    """``bart -l flags pics ...``: every index of the flagged dims as one
    problem, all problems as one batched launch; returns the joined image
    (X, Y, Z and the flagged dims). ``a`` holds the parsed pics options and
    arrays (traj, ksp, sens). The looped dims must lie outside the ones the
    problem itself uses (0-3: readout / phase / partition, coils).

    Inside a process group of several ranks (one per GPU, as the reference's
    MPI slice loop, src/bart.c:361-409), every rank solves the share of the
    problems that the cost-model split gives it, with no exchange while it
    solves, and the images are gathered to rank 0, which returns the joined
    image; the other ranks return None."""
    import torch
    from .batch import BatchRecon
    from .dist import gather_to_root, partition, problem_cost, world_rank
    from .pics import Pics, PicsConf

    dims = loop_dims(flags)
    if any(d < 4 for d in dims):
        raise ValueError("pics: looped dims must be >= 4 (dims 0-3 are the image and coil axes)")
    shapes = [a.traj.shape, a.ksp.shape, a.sens.shape]
    sizes = loop_sizes(shapes, dims)
    idxs = loop_indices(sizes)
    img_dims = list(dims16(a.sens.shape)[:3])
    out_dims = img_dims + [1] * (DIMS - 3)
    for d, n in zip(dims, sizes):
        out_dims[d] = n
    out = np.zeros(out_dims, dtype=np.complex64, order="F")

    def problem(idx):
        traj = slice_at(a.traj, dims, idx).reshape(dims16(a.traj.shape)[:3], order="F")
        ksp = slice_at(a.ksp, dims, idx)
        ksp = ksp.reshape(dims16(ksp.shape)[:4], order="F")
        sens = slice_at(a.sens, dims, idx)
        sens = sens.reshape(dims16(sens.shape)[:4], order="F")
        return {"traj": traj, "sens": sens, "ksp": ksp}

    rank, world = world_rank()
    mine = list(range(len(idxs)))
    if world > 1:
        costs = [problem_cost(problem(i), a.iters, a.toeplitz) for i in idxs]
        mine = partition(costs, world)[rank]
    probs = [problem(idxs[k]) for k in mine]
    dev = dev or torch.device("cuda", torch.cuda.current_device())

    precond = getattr(a, "precond", 0)
    tol = getattr(a, "tol", 0.0)
    if not probs:
        imgs = []
    elif a.toeplitz and tol == 0.0:	# one graph launch for all problems (fixed iteration count)
        br = BatchRecon(probs, dev, lam=a.lam, maxiter=a.iters, scaling=a.scaling, rescale=a.rescale,
                        precond=precond).build()
        try:
            br.run()
            torch.cuda.synchronize(dev)
            imgs = [t.cpu().numpy() for t in br.img]
        finally:
            br.free()
    else:		# non-Toeplitz normal or a tolerance: one solve after another
        imgs = []
        for pr in probs:
            conf = PicsConf(lam=a.lam, maxiter=a.iters, tol=tol, scaling=a.scaling, rescale=a.rescale,
                            toeplitz=a.toeplitz, precond=precond)
            p = Pics(pr["traj"], pr["sens"], ksp_dims=list(pr["ksp"].shape), conf=conf)
            imgs.append(np.asarray(p.run(pr["ksp"])))
            p.free()

    got = dict(zip(mine, imgs))
    if world > 1:
        got = gather_to_root(got)
        if got is None:
            return None
    for k, idx in enumerate(idxs):
        place_at(out, dims, idx, got[k])
    return out


def stream_pics(flags: int, a) -> np.ndarray:
    """``bart -l flags pics ... - sens out`` with the k-space arriving as a
    stream (``a.ksp`` a bart_b200.stream.StreamReader) along the looped dims:
    each slice is reconstructed as soon as it has arrived (its own SENSE
    model and solve), and the images are joined along those dims."""
    from .pics import Pics, PicsConf

    r = a.ksp
    dims = loop_dims(flags)
    if any(d < 4 for d in dims):
        raise ValueError("pics: looped dims must be >= 4 (dims 0-3 are the image and coil axes)")
    if sorted(r.sdims) != dims:
        raise ValueError(f"the k-space stream runs along dims {r.sdims}, the loop along {dims}")
    sizes = loop_sizes([a.traj.shape, r.dims, a.sens.shape], dims)
    img_dims = list(dims16(a.sens.shape)[:3])
    out_dims = img_dims + [1] * (DIMS - 3)
    for d, n in zip(dims, sizes):
        out_dims[d] = n
    out = np.zeros(out_dims, dtype=np.complex64, order="F")
    conf = PicsConf(lam=a.lam, maxiter=a.iters, tol=getattr(a, "tol", 0.0), scaling=a.scaling, rescale=a.rescale,
                    toeplitz=a.toeplitz, precond=getattr(a, "precond", 0))
    for _, pos, block in r:
        idx = tuple(pos[r.sdims.index(d)] for d in dims)
        traj = slice_at(a.traj, dims, idx).reshape(dims16(a.traj.shape)[:3], order="F")
        sens = slice_at(a.sens, dims, idx)
        sens = sens.reshape(dims16(sens.shape)[:4], order="F")
        ksp = block.reshape(dims16(block.shape)[:4], order="F")
        p = Pics(traj, sens, ksp_dims=list(ksp.shape), conf=conf)
        try:
            place_at(out, dims, idx, np.asarray(p.run(ksp)))
        finally:
            p.free()
    return out


def loop_ecalib(flags: int, ksp: np.ndarray, conf, emaps: bool = True, workers: int = 4):
    """``bart -l flags ecalib ...``: one calibration per index of the
    flagged dims (which must lie outside the k-space's own dims 0-4), the
    maps and eigenvalue maps joined along them. Up to ``workers``
    calibrations run at once, each on a host thread with its own CUDA
    stream (a calibration is a few milliseconds of mostly latency-bound GPU
    work with three host synchronisations, so several overlap well); the
    results are those of one calibration after another. Returns (maps,
    emaps or None)."""
    import ctypes
    from concurrent.futures import ThreadPoolExecutor
    from .espirit import ecalib, output_dims

    dims = loop_dims(flags)
    if any(d < 5 for d in dims):
        raise ValueError("ecalib: looped dims must be >= 5 (dims 0-4 are the image, coil and maps axes)")
    sizes = loop_sizes([ksp.shape], dims)
    one = list(dims16(ksp.shape))
    for d in dims:
        one[d] = 1
    sd, ed = output_dims(one, conf)
    for d, n in zip(dims, sizes):
        sd[d] = n
        ed[d] = n
    sens = np.zeros(sd, dtype=np.complex64, order="F")
    ev = np.zeros(ed, dtype=np.complex64, order="F") if emaps else None
    import torch
    idxs = loop_indices(sizes)
    nw = max(1, min(int(workers), len(idxs)))
    streams = {}
    own_streams = nw > 1 and torch.cuda.is_available()

    def calibrate(idx):
        import threading
        stream = None
        if own_streams:
            t = threading.get_ident()
            if t not in streams:
                streams[t] = torch.cuda.Stream()
            stream = ctypes.c_void_p(streams[t].cuda_stream)
        k = slice_at(ksp, dims, idx)
        s, e, _ = ecalib(k.reshape(one, order="F"), conf, emaps=emaps, stream=stream)
        return idx, s, e

    if nw == 1:
        results = [calibrate(idx) for idx in idxs]
    else:
        with ThreadPoolExecutor(max_workers=nw) as pool:
            results = list(pool.map(calibrate, idxs))
    for idx, s, e in results:
        place_at(sens, dims, idx, s)
        if emaps:
            place_at(ev, dims, idx, e)
    return sens, ev
