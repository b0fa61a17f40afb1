"""Learned FSAI on the GPU: features, tensor-core network forward/backward and
the probe-loss gradient against the CPU oracle; PCG with the factor.

Tolerances: features 1e-5 (FP32 logs/roots); network output and parameter
gradients 2e-2 relative in 2-norm (BF16 operands, FP32 tensor-core
accumulation against the oracle's FP64 with the same BF16 rounding points);
probe gradient 1e-4 relative (FP32 SpMVs against FP64)."""
import numpy as np
import pytest
import torch

from mpsparse_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _csr_tensor(mps, coo):
    e = torch.empty(0)
    return mps.spmv.csr_tensor(torch.from_numpy(coo.keys()), torch.from_numpy(coo.vals), e, e, e,
                               coo.n, coo.n)


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def _random_params(oracle, seed, scale=0.4):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(oracle.NPARAM) * scale).astype(np.float32)


@pytest.fixture(scope="module")
def small():
    return W.lognormal_diffusion_2d(40, 30, 1.5, 4.0, 3)


def test_features_match_oracle(mps, oracle, small):
    A = _csr_tensor(mps, small)
    X, rp, ci = (t.cpu().numpy() for t in A.fsai_features())
    Ao = oracle.Csr(*small.to_csr(), small.n)
    Xo, rpo, cio, _ = oracle.fsai_features(Ao)
    assert np.array_equal(rp, rpo) and np.array_equal(ci, cio)
    assert X.shape == Xo.shape and np.abs(X - Xo).max() <= 1e-5


def test_network_forward_matches_oracle(mps, oracle, small):
    A = _csr_tensor(mps, small)
    X = A.fsai_features()[0]
    p = _random_params(oracle, 0)
    m = mps._C.fsai_model(torch.from_numpy(p))
    out = m.forward(X).cpu().numpy()
    ref = oracle.mlp_forward(p, X.cpu().numpy())
    assert out.shape == ref.shape and _rel(out, ref) <= 2e-2
    # a row count that is not a multiple of the 128-row tile
    Xr = torch.randn(1000, 16, generator=torch.Generator().manual_seed(1))
    out = m.forward(Xr).cpu().numpy()
    assert _rel(out, oracle.mlp_forward(p, Xr.numpy())) <= 2e-2


def test_network_backward_matches_oracle(mps, oracle, small):
    A = _csr_tensor(mps, small)
    X = A.fsai_features()[0]
    p = _random_params(oracle, 1)
    m = mps._C.fsai_model(torch.from_numpy(p))
    dout = np.random.default_rng(2).standard_normal(X.shape[0]).astype(np.float32)
    g = m.backward(X, torch.from_numpy(dout)).cpu().numpy()
    ref = oracle.mlp_backward(p, X.cpu().numpy(), dout)
    bounds = np.cumsum([0, 16 * 64, 64, 64 * 64, 64, 64, 1])
    names = ["W1", "b1", "W2", "b2", "w3", "b3"]
    for name, a, b in zip(names, bounds[:-1], bounds[1:]):
        assert _rel(g[a:b], ref[a:b]) <= 2e-2, name


def test_probe_gradient_matches_oracle(mps, oracle, small):
    A = _csr_tensor(mps, small)
    m = mps._C.fsai_model(torch.from_numpy(_random_params(oracle, 3, 0.2)))
    A.attach_fsai(m)
    X, grp, gci = A.fsai_features()
    gv = A.fsai_g_values().cpu().numpy()
    Ao = oracle.Csr(*small.to_csr(), small.n)
    Go = oracle.Csr(grp.cpu().numpy(), gci.cpu().numpy(), gv, small.n)
    V = np.where(np.random.default_rng(4).random((3, small.n)) < 0.5, -1.0, 1.0).astype(np.float32)
    grad, loss = A.fsai_probe_grad(torch.from_numpy(V))
    lo, go = oracle.fsai_probe_loss_grad(Ao, Go, V)
    assert abs(loss - lo) <= 1e-4 * lo
    assert _rel(grad.cpu().numpy(), go) <= 1e-4
    # value map of the attached factor
    out = m.forward(X).cpu().numpy()
    _, _, row, _ = oracle.fsai_pattern(Ao)
    diag = np.zeros(small.n)
    rp, ci, cv = small.to_csr()
    for i in range(small.n):
        s = slice(rp[i], rp[i + 1])
        diag[i] = cv[s][ci[s] == i].sum()
    ref = oracle.fsai_value_map(out, row, gci.cpu().numpy(), diag)
    assert _rel(gv, ref) <= 1e-5


def test_fsai_pcg_and_training(mps, oracle):
    coo = W.lognormal_diffusion_2d(96, 96, 1.5, 8.0, 5)
    A = _csr_tensor(mps, coo)
    b = torch.from_numpy(W.rhs(coo.n, 6)).cuda()
    m = mps._C.fsai_model()
    A.attach_fsai(m)                     # untrained: close to Jacobi
    x = torch.zeros(coo.n, device="cuda")
    i_f = A.cgd(b, x, tol=1e-6, max_iter=20000, precond="fsai")
    i_j = A.cgd(b, torch.zeros(coo.n, device="cuda"), tol=1e-6, max_iter=20000, precond="jacobi")
    assert i_f["stop_rule_met"] and i_f["iters"] <= 1.2 * i_j["iters"]
    losses = [A.fsai_train_step(m, n_probes=4, lr=3e-3, seed=s) for s in range(40)]
    assert np.mean(losses[-5:]) < 0.8 * np.mean(losses[:5]), losses
    A.attach_fsai(m)
    x = torch.zeros(coo.n, device="cuda")
    i_t = A.cgd(b, x, tol=1e-6, max_iter=20000, precond="fsai")
    assert i_t["stop_rule_met"] and i_t["iters"] < i_j["iters"]
    Ao = oracle.Csr(*coo.to_csr(), coo.n)
    from tests.helpers import assert_solved_fp32
    assert_solved_fp32(oracle, Ao, b.cpu().numpy(), x.cpu().numpy(), 1e-6, i_t)


def test_stall_falls_back_to_jacobi(mps):
    coo = W.lognormal_diffusion_2d(64, 64, 1.5, 8.0, 7)
    A = _csr_tensor(mps, coo)
    n = coo.n
    # a deliberately poor (but SPD) factor: unit diagonal with large random
    # strictly-lower entries on tril(A)
    rp, ci, cv = coo.to_csr()
    keep = ci <= np.repeat(np.arange(n), np.diff(rp))
    rows = np.repeat(np.arange(n), np.diff(rp))[keep]
    gci = ci[keep]
    gv = np.where(gci == rows, 1.0, 5.0 * np.random.default_rng(0).standard_normal(keep.sum()))
    grp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int32)
    A.set_fsai(torch.from_numpy(grp), torch.from_numpy(gci.astype(np.int32)),
               torch.from_numpy(gv.astype(np.float32)))
    b = torch.from_numpy(W.rhs(n, 1)).cuda()
    x = torch.zeros(n, device="cuda")
    info = A.cgd(b, x, tol=1e-6, max_iter=20000, precond="fsai", stall_window=20)
    assert info["stalled"] and info["stop_rule_met"]


def test_bf16_entry_points_match(mps, oracle, small):
    """forward_bf16 / backward_bf16 (no allocation, no synchronisation) give
    what the FP32-input passes give (the same kernels after the same
    round-to-nearest BF16 conversion): the same bits forward; backward up to
    the order of the per-CTA float atomics that sum the weight gradients."""
    A = _csr_tensor(mps, small)
    X = A.fsai_features()[0]
    p = _random_params(oracle, 5)
    m = mps._C.fsai_model(torch.from_numpy(p))
    Xb = X.to(torch.bfloat16).contiguous()
    out = torch.empty(X.shape[0], device="cuda")
    m.forward_bf16(Xb, out)
    dout = torch.from_numpy(np.random.default_rng(6).standard_normal(X.shape[0]).astype(np.float32)).cuda()
    grad = torch.full((oracle.NPARAM,), float("nan"), device="cuda")
    m.backward_bf16(Xb, dout, grad)
    m.status()
    assert torch.equal(out, m.forward(X))
    g2 = m.backward(X, dout)
    assert torch.allclose(grad, g2, rtol=1e-5, atol=1e-6 * float(g2.abs().max()))


def test_committed_weights_beat_jacobi_on_held_out_512(mps):
    """The committed network (trained on seeds 0..1999) on a held-out 512^2
    log-normal diffusion system (sigma 1.5, correlation 16): FSAI-PCG needs
    clearly fewer iterations than Jacobi-PCG, and mixed-precision FSAI-PCG
    reaches an FP64 true residual of 1e-6."""
    from mpsparse_b200.fsai import LearnedFsai, evaluate
    row = evaluate(LearnedFsai.load(), [100_123])[0]
    assert row["fsai"]["converged"] and row["fsai"]["true_resid"] <= 1e-6
    assert row["fsai"]["iters"] < 0.75 * row["jacobi"]["iters"], row
    assert row["jacobi"]["iters"] < row["none"]["iters"]
