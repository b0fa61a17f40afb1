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


def evaluate(fsai: LearnedFsai | None, seeds, spec=SPEC_512, tol=1e-6, max_iter=40000):
    """PCG iterations to ``tol`` with the learned factor, Jacobi and none."""
    e = torch.empty(0)
    rows = []
    for s in seeds:
        keys, vals, n = W.lognormal_diffusion_2d_torch(spec["nx"], spec["ny"], spec["sigma"],
                                                       spec["corr_len"], s)
        A = csr_tensor(keys, vals, e, e, e, n, n, fill_outputs=False)
        b = torch.from_numpy(W.rhs(n, s + 7)).cuda()
        row = {"seed": s}
        for name in (["fsai"] if fsai is not None else []) + ["jacobi", "none"]:
            if name == "fsai":
                fsai.attach(A)
            x = torch.zeros(n, device="cuda")
            info = A.cgd(b, x, tol=tol, max_iter=max_iter, precond=name)
            row[name] = info["iters"]
        rows.append(row)
    return rows


def main():
    import argparse
    ap = argparse.ArgumentParser(description="train the learned FSAI network on the GPU")
    ap.add_argument("--systems", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=1)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--eval", type=int, default=5)
    args = ap.parse_args()
    f = LearnedFsai()
    seeds = [s for _ in range(args.epochs) for s in range(args.systems)]
    f.train(seeds, lr=args.lr)
    f.save(args.out)
    for r in evaluate(f, range(100_000, 100_000 + args.eval)):
        print(r)


if __name__ == "__main__":
    main()
