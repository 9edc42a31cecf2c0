"""Learned preconditioner for flexible-CG CG-SENSE: network, training, evaluation.

The network (6 layers of 3x3 convolutions, 2 -> 32 -> ... -> 32 -> 2
channels, bf16 weights, float32 accumulation) runs and trains on the GPU
through libbnufft's own kernels (``bnufft_precnet_*``). Inside flexible CG
(``PicsConf(precond=2)``) the preconditioner is

    z = M_circ(r) + ||r|| net(r / ||r||)

where M_circ is the reference's circulant PSF preconditioner
(src/noncart/precond.c:48-164). With a zero last layer the network adds
nothing and the method is flexible CG with M_circ alone; if the residual
stops improving for 3 iterations the solve drops the learned term.

Training data come from the method itself: for each generated problem the
library's flexible CG (circulant preconditioner) is run for k = 0, 1, 2, ...
iterations and to convergence; with x* the converged solution, x_k the
iterate and r_k = b - (A^H A + lambda) x_k its true residual, the pair is

    input  = r_k / ||r_k||,   target = (x* - x_k - M_circ(r_k)) / ||r_k||

i.e. the network learns the part of the exact error A^-1 r_k that the
circulant preconditioner misses.

  python -m bart_b200.precnet train [--problems 2000] [--eval 256] [--out FILE]
  python -m bart_b200.precnet eval [--weights FILE] [--eval 256]
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np

from . import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "precnet_weights.npz")
CIN = [2, 32, 32, 32, 32, 32]
COUT = [32, 32, 32, 32, 32, 2]
LAM = 0.01
ITERS = (0, 1, 2, 4, 6, 9, 13)       # iterates whose residuals become training pairs


def layer_offsets():
    out, o = [], 0
    for ci, co in zip(CIN, COUT):
        w = co * 9 * ci
        out.append((o, o + w, o + w + co))
        o += w + co
    return out


def nparams() -> int:
    return layer_offsets()[-1][2]


def init_params(seed=0):
    """He-normal weights (fan-in 9 cin), zero biases, zero last layer (the
    untrained network adds nothing to the circulant preconditioner)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(nparams(), dtype=np.float32)
    for li, ((wo, bo, _), ci) in enumerate(zip(layer_offsets(), CIN)):
        if li < 5:
            p[wo:bo] = rng.standard_normal(bo - wo).astype(np.float32) * np.float32(np.sqrt(2.0 / (9 * ci)))
    return p


class PrecNet:
    """The network's parameters on the GPU (libbnufft handle)."""

    def __init__(self, params=None):
        lib = _lib.load()
        n = lib.bnufft_precnet_nparams()
        assert n == nparams()
        p = np.ascontiguousarray(init_params() if params is None else params, dtype=np.float32)
        assert p.size == n
        h = ctypes.c_void_p()
        _lib.check(lib.bnufft_precnet_create(ctypes.byref(h), ctypes.c_void_p(p.ctypes.data), None))
        self.handle = h

    @classmethod
    def load(cls, path=WEIGHTS):
        return cls(np.load(path)["params"])

    def params(self):
        p = np.empty(nparams(), dtype=np.float32)
        _lib.check(_lib.load().bnufft_precnet_get_params(self.handle, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                         None))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _lib.check(_lib.load().bnufft_precnet_set_params(self.handle, ctypes.c_void_p(p.ctypes.data), None))

    def save(self, path=WEIGHTS, **meta):
        np.savez(path, params=self.params(), meta=json.dumps(meta))

    def forward(self, x, X, Y, n=1):
        """net(x) for n complex images [X, Y] (torch CUDA tensor or numpy)."""
        from .nufft import _alloc_like, _ptr_in, _ptr_out, _stream_of
        P = X * Y * n
        out = _alloc_like(x, [X, Y, n])
        px, keep = _ptr_in(x, P)
        _lib.check(_lib.load().bnufft_precnet_forward(self.handle, _ptr_out(out, P), px, X, Y, n, _stream_of(x, out)))
        del keep
        return out

    def train_step(self, x, target, X, Y, n, lr, want_loss=True, grads=None):
        """One Adam step (lr > 0) on the batch; returns the loss (before the step)."""
        from .nufft import _ptr_in, _stream_of
        P = X * Y * n
        px, k1 = _ptr_in(x, P)
        pt, k2 = _ptr_in(target, P)
        loss = ctypes.c_double()
        gp = None if grads is None else ctypes.c_void_p(grads.ctypes.data)
        _lib.check(_lib.load().bnufft_precnet_train_step(self.handle, px, pt, X, Y, n, float(lr),
                                                         ctypes.byref(loss) if want_loss else None, gp,
                                                         _stream_of(x, target)))
        del k1, k2
        return loss.value if want_loss else None

    def free(self):
        if getattr(self, "handle", None) is not None:
            _lib.load().bnufft_precnet_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# training data from the method itself
# ---------------------------------------------------------------------------

def _model(prob, dev, precond, maxiter, tol):
    import torch
    from .pics import Pics, PicsConf

    def dt(a):
        return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).to(dev)

    traj, sens, ksp = prob["traj"], prob["sens"], prob["ksp"]
    p = Pics(dt(traj), dt(sens), ksp_dims=list(ksp.shape),
             conf=PicsConf(lam=LAM, maxiter=maxiter, tol=tol, precond=precond),
             traj_dims=list(traj.shape), sens_dims=list(sens.shape))
    return p, dt(ksp)


def training_pairs(prob, dev, iters=ITERS):
    """(inputs, targets): complex [len(iters), N*N] tensors on dev."""
    import torch
    N = prob["sens"].shape[0]
    p, ksp = _model(prob, dev, 1, 200, 1e-7)
    try:
        b = p.rhs(ksp)
        xs = p.run(ksp).clone()
        ins, tgs = [], []
        for k in iters:
            if k == 0:
                xk = torch.zeros_like(xs)
            else:
                q, _ = _model(prob, dev, 1, k, 0.0)
                try:
                    xk = q.run(ksp).clone()
                finally:
                    q.free()
            r = b - (p.normal(xk) + LAM * xk)
            nr = torch.linalg.vector_norm(r)
            mc = p.precond(r)
            ins.append(r / nr)
            tgs.append((xs - xk - mc) / nr)
        return torch.stack(ins), torch.stack(tgs)
    finally:
        p.free()


def make_dataset(nprob, seed, dev, N=256, coils=(8, 32), spokes=(48, 128), log=None):
    import torch
    from .problems import cgsense_problem
    rng = np.random.default_rng(seed)
    X, T = [], []
    t0 = time.time()
    for i in range(nprob):
        prob = cgsense_problem(rng, N=N, coils=coils, spokes=spokes)
        x, t = training_pairs(prob, dev)
        X.append(x)
        T.append(t)
        if log and (i + 1) % 100 == 0:
            log(f"data {i + 1}/{nprob} ({time.time() - t0:.1f} s)")
    return torch.cat(X), torch.cat(T)


# ---------------------------------------------------------------------------
# training and evaluation
# ---------------------------------------------------------------------------

def train(net, X, T, N, epochs=4, batch=8, lr=1e-3, seed=0, log=None):
    """Adam with cosine-decayed learning rate over shuffled batches."""
    import torch
    n = X.shape[0]
    steps = epochs * (n // batch)
    g = torch.Generator(device="cpu").manual_seed(seed)
    hist = []
    s = 0
    t0 = time.time()
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g)
        run = 0.0
        for j in range(n // batch):
            idx = perm[j * batch:(j + 1) * batch].to(X.device)
            xb = X.index_select(0, idx).contiguous().view(-1)
            tb = T.index_select(0, idx).contiguous().view(-1)
            lr_s = 0.5 * lr * (1 + np.cos(np.pi * s / max(1, steps)))
            want = (j % 50 == 0)
            loss = net.train_step(xb, tb, N, N, batch, lr_s, want_loss=want)
            if want:
                run = loss
                hist.append((s, loss))
            s += 1
        if log:
            log(f"epoch {ep + 1}/{epochs}: loss {run:.4g} ({time.time() - t0:.1f} s)")
    return hist


def dataset_loss(net, X, T, N, batch=8):
    tot, cnt = 0.0, 0
    for j in range(0, X.shape[0] - batch + 1, batch):
        tot += net.train_step(X[j:j + batch].contiguous().view(-1), T[j:j + batch].contiguous().view(-1),
                              N, N, batch, 0.0) * batch
        cnt += batch
    return tot / max(1, cnt)


def solve_stats(prob, dev, precond, net=None, tol=1e-4, maxiter=300, reps=3):
    """Iterations, ms per solve (model reused, CUDA events) and true residual."""
    import torch
    p, ksp = _model(prob, dev, precond, maxiter, tol)
    try:
        if net is not None:
            p.set_precnet(net)
        x = p.run(ksp)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            p.run(ksp, out=x)
        e1.record()
        torch.cuda.synchronize()
        it, _, _ = p.stats()
        b = p.rhs(ksp)
        r = b - (p.normal(x) + LAM * x)
        tr = float(torch.linalg.vector_norm(r) / torch.linalg.vector_norm(b))
        return {"iters": it, "ms": e0.elapsed_time(e1) / reps, "true_res": tr}
    finally:
        p.free()


def evaluate(net, nprob, seed, dev, N=256, coils=(8, 32), spokes=(48, 128), log=None):
    from .problems import cgsense_problem
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(nprob):
        prob = cgsense_problem(rng, N=N, coils=coils, spokes=spokes)
        row = {"coils": prob["coils"], "spokes": prob["spokes"],
               "cg": solve_stats(prob, dev, 0), "fcg_circ": solve_stats(prob, dev, 1),
               "fcg_learned": solve_stats(prob, dev, 2, net)}
        rows.append(row)
        if log and (i + 1) % 32 == 0:
            log(f"eval {i + 1}/{nprob}")
    return rows


def summarize(rows):
    out = {}
    for k in ("cg", "fcg_circ", "fcg_learned"):
        its = np.array([r[k]["iters"] for r in rows], dtype=float)
        ms = np.array([r[k]["ms"] for r in rows])
        tr = np.array([r[k]["true_res"] for r in rows])
        out[k] = {"iters_mean": float(its.mean()), "ms_mean": float(ms.mean()), "true_res_max": float(tr.max()),
                  "converged_frac": float(np.mean(tr <= 1.05e-4))}
    out["speedup_learned_vs_cg"] = out["cg"]["ms_mean"] / out["fcg_learned"]["ms_mean"]
    out["speedup_learned_vs_circ"] = out["fcg_circ"]["ms_mean"] / out["fcg_learned"]["ms_mean"]
    out["speedup_circ_vs_cg"] = out["cg"]["ms_mean"] / out["fcg_circ"]["ms_mean"]
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m bart_b200.precnet")
    ap.add_argument("cmd", choices=["train", "eval"])
    ap.add_argument("--problems", type=int, default=2000)
    ap.add_argument("--eval", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--weights", default=WEIGHTS)
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)

    import torch
    dev = torch.device("cuda", 0)

    def log(m):
        print(m, file=sys.stderr, flush=True)

    report = {}
    if a.cmd == "train":
        t0 = time.time()
        X, T = make_dataset(a.problems, 1, dev, log=log)
        report["data_s"] = time.time() - t0
        report["pairs"] = int(X.shape[0])
        net = PrecNet()
        Xh, Th = make_dataset(min(64, a.eval), 7, dev)
        report["heldout_loss_init"] = dataset_loss(net, Xh, Th, 256)
        t0 = time.time()
        hist = train(net, X, T, 256, epochs=a.epochs, batch=a.batch, lr=a.lr, log=log)
        torch.cuda.synchronize()
        report["train_s"] = time.time() - t0
        report["loss_history"] = hist
        report["heldout_loss_trained"] = dataset_loss(net, Xh, Th, 256)
        del X, T
        net.save(a.out, problems=a.problems, epochs=a.epochs, lr=a.lr, batch=a.batch)
    else:
        net = PrecNet.load(a.weights)
    rows = evaluate(net, a.eval, 2, dev, log=log)
    report["eval"] = summarize(rows)
    report["eval_problems"] = a.eval
    line = json.dumps(report)
    print(line, flush=True)
    if a.report:
        with open(a.report, "w") as f:
            json.dump({"report": report, "rows": rows}, f)


if __name__ == "__main__":
    main()
