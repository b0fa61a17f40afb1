"""Learned FSAI preconditioner: training and evaluation driver.

The network and every training step run on the GPU through the C ABI
(``mps_fsai_train_step``: tensor-core forward/backward kernels, probe loss,
Adam).  This module only chooses the systems and the probe vectors:

* each step draws one training system of the distribution the model is for
  (default: 512x512 log-normal diffusion, sigma 1.5, correlation length 16,
  training seeds 0..1999), built on the GPU;
* probes are Rademacher vectors plus Krylov residuals the solver itself
  generates: the residual of a short PCG run with the current factor, whose
  error lies in the slow, badly preconditioned modes;
* the loss is the probe estimate of ||I - G A G^T||_F^2 / n.

Trained weights live in ``weights/`` next to this file.
"""
from __future__ import annotations

import os
import time

import numpy as np
import torch

from . import workloads as W
from ._C import csr_tensor, fsai_model

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "fsai_lognormal512.npy")
SPEC_512 = dict(nx=512, ny=512, sigma=1.5, corr_len=16.0)


class LearnedFsai:
    """A network whose factor G is attached to csr_tensor objects for
    ``cgd(..., precond="fsai")`` and ``cg_mixed(..., precond="fsai")``."""

    def __init__(self, params: np.ndarray | None = None):
        self.model = fsai_model(None if params is None else torch.from_numpy(
            np.asarray(params, dtype=np.float32)))

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS) -> "LearnedFsai":
        return cls(np.load(path))

    def save(self, path: str = DEFAULT_WEIGHTS) -> None:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.save(path, self.model.params().numpy())

    def params(self) -> np.ndarray:
        return self.model.params().numpy()

    def attach(self, A: csr_tensor) -> None:
        A.attach_fsai(self.model)

    def train_system(self, A: csr_tensor, b: torch.Tensor, lr: float, seed: int,
                     n_probes: int = 4, residual_iters: int = 30) -> float:
        extra = None
        if residual_iters > 0:
            self.attach(A)
            x = torch.zeros_like(b)
            A.cgd(b, x, tol=1e-300, max_iter=residual_iters, precond="fsai")
            r = torch.empty_like(b)
            A.mv(x, r)
            r = b - r
            extra = (r / r.norm() * np.sqrt(r.numel())).contiguous()
        return A.fsai_train_step(self.model, n_probes=n_probes, extra=extra, lr=lr, seed=seed)

    def train(self, seeds, spec=SPEC_512, lr=2e-3, lr_final=2e-4, n_probes=4,
              residual_iters=30, log_every=100, log=print):
        seeds = list(seeds)
        t0 = time.time()
        losses = []
        e = torch.empty(0)
        for step, s in enumerate(seeds):
            frac = step / max(len(seeds) - 1, 1)
            rate = lr * (lr_final / lr) ** frac
            keys, vals, n = W.lognormal_diffusion_2d_torch(spec["nx"], spec["ny"], spec["sigma"],
                                                           spec["corr_len"], s)
            A = csr_tensor(keys, vals, e, e, e, n, n, fill_outputs=False)
            b = torch.from_numpy(W.rhs(n, s + 7)).cuda()
            losses.append(self.train_system(A, b, rate, s, n_probes, residual_iters))
            if log and (step + 1) % log_every == 0:
                log(f"step {step + 1}/{len(seeds)} loss {np.mean(losses[-log_every:]):.4f} "
                    f"lr {rate:.2e} {time.time() - t0:.1f}s")
        return losses


def _timed(fn):
    """fn() on the current stream, timed with CUDA events (device time)."""
    st = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    out = fn()
    b.record(st)
    torch.cuda.synchronize()
    return out, a.elapsed_time(b)


def evaluate(fsai: LearnedFsai | None, seeds, spec=SPEC_512, tol=1e-6, max_iter=40000,
             inner_tol=1e-4, timed=False):
    """Per held-out seed: iterations (and, with ``timed``, device time of a
    second solve on the same handle, after graph capture) to ``tol`` for the
    learned factor in mixed-precision PCG (FP64 true residual), Jacobi-PCG
    and plain CG in FP32 (their FP64 true residual reported beside)."""
    e = torch.empty(0)
    rows = []
    for s in seeds:
        keys, vals, n = W.lognormal_diffusion_2d_torch(spec["nx"], spec["ny"], spec["sigma"],
                                                       spec["corr_len"], s)
        A = csr_tensor(keys, vals, e, e, e, n, n, fill_outputs=False)
        b = torch.from_numpy(W.rhs(n, s + 7)).cuda()
        row = {"seed": s}
        if fsai is not None:
            b64 = b.double()

            def learned():
                fsai.attach(A)
                x = torch.zeros(n, dtype=torch.float64, device="cuda")
                return A.cg_mixed(b64, x, tol=tol, inner_tol=inner_tol, max_inner=max_iter,
                                  precond="fsai")
            info, ms = _timed(learned)
            if timed:
                info, ms = _timed(learned)
            row["fsai"] = {"iters": info["inner_iters"], "true_resid": info["rel_resid"],
                           "converged": bool(info["converged"])}
            if timed:
                row["fsai"]["ms"] = ms
        for name in ("jacobi", "none"):
            def solve():
                x = torch.zeros(n, device="cuda")
                return A.cgd(b, x, tol=tol, max_iter=max_iter, precond=name)
            info, ms = _timed(solve)
            if timed:
                info, ms = _timed(solve)
            row[name] = {"iters": info["iters"], "true_resid": info["true_resid"],
                         "converged": bool(info["converged"])}
            if timed:
                row[name]["ms"] = ms
        # Jacobi-PCG with the learned solve's precision scheme (FP64 x,
        # residual replacement): the like-for-like FP64-checked comparison
        b64j = b.double()

        def jacobi_mp():
            x = torch.zeros(n, dtype=torch.float64, device="cuda")
            return A.cg_mixed(b64j, x, tol=tol, inner_tol=inner_tol, max_inner=max_iter, precond="jacobi")
        info, ms = _timed(jacobi_mp)
        if timed:
            info, ms = _timed(jacobi_mp)
        row["jacobi_mp"] = {"iters": info["inner_iters"], "true_resid": info["rel_resid"],
                            "converged": bool(info["converged"])}
        if timed:
            row["jacobi_mp"]["ms"] = ms
        rows.append(row)
    return rows


def summarize(rows):
    """Mean / median / 95th percentile of iterations and times per method."""
    out = {"systems": len(rows)}
    for name in ("fsai", "jacobi", "none", "jacobi_mp"):
        if name not in rows[0]:
            continue
        it = np.array([r[name]["iters"] for r in rows], np.float64)
        d = {"iters_mean": float(it.mean()), "iters_median": float(np.median(it)),
             "iters_p95": float(np.percentile(it, 95)),
             "true_resid_max": float(max(r[name]["true_resid"] for r in rows)),
             "converged_fp64": int(sum(r[name]["converged"] for r in rows))}
        if "ms" in rows[0][name]:
            ms = np.array([r[name]["ms"] for r in rows], np.float64)
            d.update(ms_mean=float(ms.mean()), ms_median=float(np.median(ms)),
                     ms_p95=float(np.percentile(ms, 95)))
        out[name] = d
    if "fsai" in out:
        out["fsai_fewer_iters_than_jacobi"] = int(sum(r["fsai"]["iters"] < r["jacobi"]["iters"]
                                                     for r in rows))
        if "ms" in rows[0]["fsai"]:
            out["fsai_faster_than_jacobi_mp"] = int(sum(r["fsai"]["ms"] < r["jacobi_mp"]["ms"]
                                                        for r in rows))
    return out


def main():
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the learned FSAI network on the GPU and "
                                             "evaluate it on held-out systems")
    ap.add_argument("--systems", type=int, default=2000, help="training seeds 0..systems-1")
    ap.add_argument("--epochs", type=int, default=1)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--no-train", action="store_true", help="evaluate the weights in --out")
    ap.add_argument("--log", default=None, help="training record (JSON lines) written here")
    ap.add_argument("--eval", type=int, default=5, help="held-out systems evaluated")
    ap.add_argument("--eval-seed0", type=int, default=100_000)
    ap.add_argument("--timed", action="store_true", help="also time the evaluation solves")
    ap.add_argument("--report", default=None, help="evaluation rows + summary (JSON) written here")
    args = ap.parse_args()
    if args.no_train:
        f = LearnedFsai.load(args.out)
    else:
        f = LearnedFsai()
        seeds = [s for _ in range(args.epochs) for s in range(args.systems)]
        logf = open(args.log, "w") if args.log else None
        t0 = time.time()

        def log(msg):
            print(msg, flush=True)
        losses = f.train(seeds, lr=args.lr, log=log)
        f.save(args.out)
        if logf:
            logf.write(json.dumps({"command": "python -m mpsparse_b200.fsai " +
                                   f"--systems {args.systems} --epochs {args.epochs} --lr {args.lr}",
                                   "training_seeds": [0, args.systems - 1], "steps": len(seeds),
                                   "lr": [args.lr, 2e-4], "probes": 4, "residual_iters": 30,
                                   "seconds": time.time() - t0,
                                   "loss_first_100": float(np.mean(losses[:100])),
                                   "loss_last_100": float(np.mean(losses[-100:]))}) + "\n")
            for k in range(0, len(losses), 100):
                logf.write(json.dumps({"steps": [k + 1, min(k + 100, len(losses))],
                                       "loss_mean": float(np.mean(losses[k:k + 100]))}) + "\n")
            logf.close()
    rows = evaluate(f, range(args.eval_seed0, args.eval_seed0 + args.eval), timed=args.timed)
    summ = summarize(rows)
    print(json.dumps(summ))
    if args.report:
        with open(args.report, "w") as fh:
            json.dump({"summary": summ, "rows": rows}, fh)


if __name__ == "__main__":
    main()
