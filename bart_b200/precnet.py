"""Learned preconditioner for flexible-CG CG-SENSE: network, training, evaluation.

The network (6 layers of 3x3 convolutions, 2 -> 32 -> ... -> 32 -> 2
channels, bf16 weights, float32 accumulation) runs and trains on the GPU
through libbnufft's own kernels (``bnufft_precnet_*``). Inside flexible CG
(``PicsConf(precond=2)``) the preconditioner is

    z = M(r) + ||M(r)|| net(M(r) / ||M(r)||)

where M is the padded-circulant preconditioner (the Toeplitz operator's own
circulant inverted on the zero-padded image, precond 3; the reference's
circulant PSF preconditioner, src/noncart/precond.c:48-164, is the weaker
Strang form of it). With a zero last layer the network adds nothing and the
method is flexible CG with M alone; the learned term is used in the first
``net_iters`` iterations (PicsConf.net_iters; 0 = all) and dropped for good
if the residual stops improving for 3 iterations.

Training data come from the method itself: for each generated problem the
library's flexible CG (padded-circulant preconditioner) is run for k = 0, 1,
2, ... iterations and to convergence (x*); each iterate x_k gives its true
residual r_k = b - (A^H A + lambda) x_k and exact error e_k = x* - x_k. The
loss is what one flexible-CG step along z = Mn + net(Mn), Mn = M(r)/||M(r)||,
leaves of the A-norm error after an exact line search,

    L = 1 - <z, r>^2 / (<z, A z> <e, r>),    A = A^H A + lambda,

scale-free in z like the solver; its gradient needs A z, applied with the
library's Toeplitz normal operator, and enters the network's own backward
kernels (bnufft_precnet_backward). Training is online: problems are drawn,
turned into a residual batch, and used for a few Adam steps.

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
ITERS = (0, 1, 2, 3, 5, 7, 10)      # iterates whose residuals become training pairs
BASE = 3                              # the preconditioner the network corrects (padded circulant)


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

    def backward(self, x, gout, X, Y, n, lr, grads=None):
        """Backward from a given d loss / d net(x), then an Adam step (lr > 0)."""
        from .nufft import _ptr_in, _stream_of
        P = X * Y * n
        px, k1 = _ptr_in(x, P)
        pg, k2 = _ptr_in(gout, P)
        gp = None if grads is None else ctypes.c_void_p(grads.ctypes.data)
        _lib.check(_lib.load().bnufft_precnet_backward(self.handle, px, pg, X, Y, n, float(lr), gp, _stream_of(x, gout)))
        del k1, k2

    def status(self):
        """0, or 1 if a tensor-core layer's bounded wait ran out (synchronises)."""
        st = ctypes.c_int(-1)
        _lib.check(_lib.load().bnufft_precnet_status(self.handle, ctypes.byref(st), None))
        return st.value

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

def _model(prob, dev, precond, maxiter, tol, net_iters=None):
    import torch
    from .pics import Pics, PicsConf

    def dt(a):
        return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).to(dev)

    traj, sens, ksp = prob["traj"], prob["sens"], prob["ksp"]
    p = Pics(dt(traj), dt(sens), ksp_dims=list(ksp.shape),
             conf=PicsConf(lam=LAM, maxiter=maxiter, tol=tol, precond=precond,
                           **({} if net_iters is None else {"net_iters": net_iters})),
             traj_dims=list(traj.shape), sens_dims=list(sens.shape))
    return p, dt(ksp)


def problem_samples(prob, dev, iters=ITERS):
    """The model (padded-circulant preconditioner) of one problem and, for
    its iterates k in iters, unit residuals R_k = r_k / ||r_k||, unit
    preconditioned steps Mn_k = M(r_k) / ||M(r_k)|| and E_k = <e_k, r_k> /
    ||r_k||^2 with e_k = x* - x_k = A^-1 r_k. The caller frees the model."""
    import torch
    p, ksp = _model(prob, dev, BASE, 200, 1e-7)
    b = p.rhs(ksp)
    xs = p.run(ksp).clone()
    R, Mn, E = [], [], []
    for k in iters:
        if k == 0:
            xk = torch.zeros_like(xs)
        else:
            p.set_iter(k, 0.0)
            xk = p.run(ksp).clone()
        r = b - (p.normal(xk) + LAM * xk)
        nr = torch.linalg.vector_norm(r)
        mc = p.precond(r)
        R.append(r / nr)
        Mn.append(mc / torch.linalg.vector_norm(mc))
        E.append(torch.sum(torch.conj(xs - xk) * r).real / nr ** 2)
    return p, torch.stack(R), torch.stack(Mn), torch.stack(E)


def anorm_loss(p, R, Mn, E, out):
    """Per sample, the fraction of the A-norm error that an exact line search
    along z = Mn + out leaves, L = 1 - <z, r>^2 / (<z, A z> <A^-1 r, r>)
    (A = A^H A + lambda; in [0, 1], scale-free in z like flexible CG), and
    d mean(L) / d out."""
    import torch
    K = R.shape[0]
    z = Mn + out.view(K, -1)
    Az = torch.stack([p.normal(z[k].contiguous()) + LAM * z[k] for k in range(K)])
    a = torch.sum(torch.conj(z) * R, dim=1).real
    q = torch.sum(torch.conj(z) * Az, dim=1).real
    L = 1 - a ** 2 / (q * E)
    g = -(2 * a / (q * E))[:, None] * (R - (a / q)[:, None] * Az)
    return L, (g / K).to(torch.complex64)


def train_online(net, nprob, seed, dev, N=256, coils=(8, 32), spokes=(48, 128), steps=3, lr=1e-3, log=None):
    """Adam on the A-norm line-search loss, problems generated on the fly;
    `steps` updates per problem on its residual batch; cosine-decayed rate."""
    import torch
    from .problems import cgsense_problem
    rng = np.random.default_rng(seed)
    total = nprob * steps
    hist = []
    s = 0
    t0 = time.time()
    for i in range(nprob):
        prob = cgsense_problem(rng, N=N, coils=coils, spokes=spokes)
        p, R, Mn, E = problem_samples(prob, dev)
        try:
            K = R.shape[0]
            x = Mn.contiguous().view(-1)
            for j in range(steps):
                out = net.forward(x, N, N, K)
                L, g = anorm_loss(p, R, Mn, E, out)
                if j == 0:
                    L0, _ = anorm_loss(p, R, Mn, E, torch.zeros_like(out))
                    hist.append((i, float(L0.mean()), float(L.mean())))
                lr_s = 0.5 * lr * (1 + np.cos(np.pi * s / max(1, total)))
                net.backward(x, g.contiguous().view(-1), N, N, K, lr_s)
                s += 1
        finally:
            p.free()
        if log and (i + 1) % 100 == 0:
            h = np.array(hist[-100:])
            log(f"problem {i + 1}/{nprob}: loss base {h[:, 1].mean():.4f} learned {h[:, 2].mean():.4f} "
                f"({time.time() - t0:.1f} s)")
    return hist


def heldout_loss(net, nprob, seed, dev, N=256):
    """Mean A-norm loss of the padded-circulant step and of the learned one."""
    import torch
    from .problems import cgsense_problem
    rng = np.random.default_rng(seed)
    lc, ll = [], []
    for _ in range(nprob):
        prob = cgsense_problem(rng, N=N)
        p, R, Mn, E = problem_samples(prob, dev)
        try:
            K = R.shape[0]
            out = net.forward(Mn.contiguous().view(-1), N, N, K)
            lc.append(anorm_loss(p, R, Mn, E, torch.zeros_like(out))[0].mean().item())
            ll.append(anorm_loss(p, R, Mn, E, out)[0].mean().item())
        finally:
            p.free()
    return float(np.mean(lc)), float(np.mean(ll))


def solve_stats(prob, dev, precond, net=None, tol=1e-4, maxiter=300, reps=3, net_iters=None):
    """Iterations, ms per solve (model reused, CUDA events) and true residual."""
    import torch
    p, ksp = _model(prob, dev, precond, maxiter, tol, net_iters)
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


def evaluate(net, nprob, seed, dev, N=256, coils=(8, 32), spokes=(48, 128), log=None, net_iters=(1,)):
    """Per problem: plain CG, FCG with the reference's circulant and with the
    padded-circulant preconditioner, and the learned method at each
    net_iters budget ("fcg_learned" = the first budget)."""
    from .problems import cgsense_problem
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(nprob):
        prob = cgsense_problem(rng, N=N, coils=coils, spokes=spokes)
        row = {"coils": prob["coils"], "spokes": prob["spokes"],
               "cg": solve_stats(prob, dev, 0), "fcg_circ": solve_stats(prob, dev, 1),
               "fcg_padded": solve_stats(prob, dev, 3)}
        for j, k in enumerate(net_iters):
            row["fcg_learned" if j == 0 else f"fcg_learned_k{k}"] = solve_stats(prob, dev, 2, net, net_iters=k)
        rows.append(row)
        if log and (i + 1) % 32 == 0:
            log(f"eval {i + 1}/{nprob}")
    return rows


def summarize(rows):
    out = {}
    for k in [k for k in rows[0] if k.startswith(("cg", "fcg"))]:
        its = np.array([r[k]["iters"] for r in rows], dtype=float)
        ms = np.array([r[k]["ms"] for r in rows])
        tr = np.array([r[k]["true_res"] for r in rows])
        out[k] = {"iters_mean": float(its.mean()), "ms_mean": float(ms.mean()), "true_res_max": float(tr.max()),
                  "converged_frac": float(np.mean(tr <= 1.05e-4))}
    out["speedup_learned_vs_cg"] = out["cg"]["ms_mean"] / out["fcg_learned"]["ms_mean"]
    out["speedup_learned_vs_circ"] = out["fcg_circ"]["ms_mean"] / out["fcg_learned"]["ms_mean"]
    out["speedup_learned_vs_padded"] = out["fcg_padded"]["ms_mean"] / out["fcg_learned"]["ms_mean"]
    out["speedup_circ_vs_cg"] = out["cg"]["ms_mean"] / out["fcg_circ"]["ms_mean"]
    return out


def time_forward(net, dev, N=256, reps=50):
    """Mean device time of one network forward on an N x N image with the
    tcgen05 layers and with the mma.sync layers (BNUFFT_NET_TC=0), CUDA
    events, after 3 warm-up passes; and whether the two outputs agree."""
    import torch
    x = torch.randn(N * N, dtype=torch.complex64, device=dev)
    res, outs = {}, {}
    old = os.environ.get("BNUFFT_NET_TC")
    try:
        for tc in ("1", "0"):
            os.environ["BNUFFT_NET_TC"] = tc
            for _ in range(3):
                net.forward(x, N, N, 1)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                net.forward(x, N, N, 1)
            e1.record()
            torch.cuda.synchronize()
            res["tcgen05_us" if tc == "1" else "mma_sync_us"] = e0.elapsed_time(e1) * 1e3 / max(1, reps)
            outs[tc] = net.forward(x, N, N, 1)
    finally:
        if old is None:
            os.environ.pop("BNUFFT_NET_TC", None)
        else:
            os.environ["BNUFFT_NET_TC"] = old
    res["max_abs_diff"] = float((outs["1"] - outs["0"]).abs().max())
    res["status"] = net.status()
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m bart_b200.precnet")
    ap.add_argument("cmd", choices=["train", "eval", "time"])
    ap.add_argument("--problems", type=int, default=2000)
    ap.add_argument("--eval", type=int, default=256)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--weights", default=WEIGHTS)
    ap.add_argument("--report", default=None)
    ap.add_argument("--reps", type=int, default=50, help="time: forward passes per layer kernel")
    ap.add_argument("--net-iters", default="1", help="comma list of learned-iteration budgets to evaluate")
    a = ap.parse_args(argv)

    import torch
    dev = torch.device("cuda", 0)

    def log(m):
        print(m, file=sys.stderr, flush=True)

    report = {}
    if a.cmd == "time":
        print(json.dumps(time_forward(PrecNet.load(a.weights), dev, reps=a.reps)), flush=True)
        return
    if a.cmd == "train":
        net = PrecNet()
        t0 = time.time()
        hist = train_online(net, a.problems, 1, dev, steps=a.steps, lr=a.lr, log=log)
        torch.cuda.synchronize()
        report["train_s"] = time.time() - t0
        report["loss_history"] = hist[::max(1, len(hist) // 50)]
        report["heldout_loss_circulant"], report["heldout_loss_learned"] = heldout_loss(net, 32, 7, dev)
        net.save(a.out, problems=a.problems, steps=a.steps, lr=a.lr)
    else:
        net = PrecNet.load(a.weights)
    rows = evaluate(net, a.eval, 2, dev, log=log, net_iters=tuple(int(v) for v in a.net_iters.split(",")))
    report["eval"] = summarize(rows)
    report["eval_problems"] = a.eval
    line = json.dumps(report)
    print(line, flush=True)
    if a.report:
        with open(a.report, "w") as f:
            json.dump({"report": report, "rows": rows}, f)


if __name__ == "__main__":
    main()
