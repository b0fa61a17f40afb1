"""Reliable-update FSAI-PCG as one persistent cooperative kernel
(fsai_persistent.cu) against the graph form of the same solve and the FP64
oracle.

The two forms compute every row identically; only the FP64 sums of the
per-CTA partials group differently, so their iterates agree to rounding
early on and their iteration counts within a few percent at the end.
Tolerances: first iterates within 1e-6 relative of the graph form's;
final answers by the FP64 true residual (<= tol, checked by the oracle);
solutions of the two forms within 100 * tol of each other."""
import numpy as np
import pytest
import torch

from mpsparse_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _learned(mps, nx, ny, seed):
    from mpsparse_b200.fsai import LearnedFsai
    c = W.lognormal_diffusion_2d(nx, ny, 1.5, 8.0, seed)
    e = torch.empty(0)
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e, c.n, c.n)
    LearnedFsai.load().attach(A)
    A.set_fsai_apply("product")
    return c, A


def _solve(A, b, persistent, **kw):
    A.set_persistent(persistent)
    x = torch.zeros(b.numel(), dtype=torch.float64, device="cuda")
    info = A.cg_mixed(b, x, precond="fsai", **kw)
    return x, info


@pytest.mark.parametrize("shape", [(160, 120), (64, 64), (512, 512)])
def test_persistent_matches_graph_form(mps, oracle, shape):
    c, A = _learned(mps, *shape, 31)
    b = torch.from_numpy(W.rhs(c.n, 8).astype(np.float64)).cuda()
    xg, ig = _solve(A, b, False, tol=1e-9, inner_tol=1e-3, max_inner=40000)
    xp, ip = _solve(A, b, True, tol=1e-9, inner_tol=1e-3, max_inner=40000)
    assert ip["persistent"] and not ig["persistent"]
    assert ip["converged"] and ig["converged"]
    Ao = oracle.Csr(*c.to_csr(), c.n)
    bh = b.cpu().numpy()
    assert oracle.true_residual(Ao, bh, xp.cpu().numpy()) <= 1e-9 * 1.01
    assert abs(ip["inner_iters"] - ig["inner_iters"]) <= 0.05 * ig["inner_iters"] + 3, (ip, ig)
    rel = float((xp - xg).norm() / xg.norm())
    assert rel <= 1e-7, rel


def test_persistent_first_iterates(mps):
    """Capped at a few iterations (no replacement yet), the two forms return
    the same x to within FP32 rounding of the partial sums' grouping."""
    c, A = _learned(mps, 160, 120, 32)
    b = torch.from_numpy(W.rhs(c.n, 9).astype(np.float64)).cuda()
    for k in (1, 2, 5, 20):
        xg, ig = _solve(A, b, False, tol=1e-30, inner_tol=1e-30, max_inner=k, max_outer=1)
        xp, ip = _solve(A, b, True, tol=1e-30, inner_tol=1e-30, max_inner=k, max_outer=1)
        assert ip["persistent"] and ip["inner_iters"] == ig["inner_iters"] == k, (k, ip, ig)
        assert float((xp - xg).norm() / xg.norm()) <= 1e-6, k


def test_persistent_stall_fallback(mps):
    """A deliberately poor (but SPD) factor: the stall watch switches to
    Jacobi inside the persistent kernel as in the graph form, and the solve
    still reaches its FP64 target."""
    c = W.lognormal_diffusion_2d(64, 64, 1.5, 8.0, 7)
    e = torch.empty(0)
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e, c.n, c.n)
    n = c.n
    rp, ci, _ = c.to_csr()
    rows_all = np.repeat(np.arange(n), np.diff(rp))
    keep = ci <= rows_all
    rows, gci = rows_all[keep], ci[keep]
    gv = np.where(gci == rows, 1.0, 5.0 * np.random.default_rng(0).standard_normal(keep.sum()))
    grp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int32)
    A.set_fsai_apply("product")
    A.set_fsai(torch.from_numpy(grp), torch.from_numpy(gci.astype(np.int32)),
               torch.from_numpy(gv.astype(np.float32)))
    b = torch.from_numpy(W.rhs(n, 1).astype(np.float64)).cuda()
    A.set_persistent(True)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    info = A.cg_mixed(b, x, tol=1e-8, inner_tol=1e-3, max_inner=20000, precond="fsai")
    assert info["persistent"] and info["converged"] and info["rel_resid"] <= 1e-8


def test_persistent_stream_form_fsai(mps, oracle):
    """700^2 (3,311 rows per CTA): A's and M's rows no longer fit shared
    memory beside their vector window, nor alone, so the CTAs read them from
    L2 in every step (stream form) with the window staged as in the window
    form.  Without residual replacements the iterates agree with the graph
    form's to rounding of the FP64 partial sums through 2,000 iterations;
    the full solve reaches its FP64-checked target."""
    c, A = _learned(mps, 700, 700, 33)
    b = torch.from_numpy(W.rhs(c.n, 2).astype(np.float64)).cuda()
    xg, ig = _solve(A, b, False, tol=1e-30, inner_tol=1e-30, max_inner=2000, max_outer=1)
    xp, ip = _solve(A, b, True, tol=1e-30, inner_tol=1e-30, max_inner=2000, max_outer=1)
    assert ip["persistent_form"] == "stream" and ig["persistent_form"] is None
    assert ip["inner_iters"] == ig["inner_iters"] == 2000
    assert float((xp - xg).norm() / xg.norm()) <= 1e-12
    xp, ip = _solve(A, b, True, tol=1e-9, inner_tol=1e-3, max_inner=40000)
    assert ip["persistent_form"] == "stream" and ip["converged"]
    Ao = oracle.Csr(*c.to_csr(), c.n)
    assert oracle.true_residual(Ao, b.cpu().numpy(), xp.cpu().numpy()) <= 1e-9 * 1.01


def test_persistent_forms_bit_identical(mps):
    """512^2 fits one CTA per SM in all three forms (window, gather,
    stream).  They share the row partition, each row's arithmetic and the
    order of every sum, so learned-FSAI MP-PCG, plain CG and BiCGSTAB return
    bit-identical solutions and iteration counts in every form; an unknown
    form is rejected."""
    c, A = _learned(mps, 512, 512, 31)
    b = torch.from_numpy(W.rhs(c.n, 8).astype(np.float64)).cuda()
    forms = ("window", "gather", "stream")
    out = {}
    for form in forms:
        A.set_persistent(True, form=form)
        x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
        info = A.cg_mixed(b, x, tol=1e-9, inner_tol=1e-3, max_inner=40000, precond="fsai")
        assert info["persistent_form"] == form and info["converged"], (form, info)
        out[form] = (x, info["inner_iters"], info["outer_iters"])
    for form in forms[1:]:
        assert torch.equal(out[form][0], out["window"][0]), form
        assert out[form][1:] == out["window"][1:], (form, out[form][1:], out["window"][1:])
    # plain CG needs ~19,000 iterations on this system: 500 of each solver
    b32 = b.float()
    for solve, fs in (("cgd", forms), ("bicgstab", forms)):
        xs = {}
        for form in fs:
            A.set_persistent(True, form=form)
            x = torch.zeros(c.n, device="cuda")
            info = getattr(A, solve)(b32, x, tol=1e-300, max_iter=500)
            assert info["persistent_form"] == form and info["iters"] == 500, (solve, form, info)
            xs[form] = x
        for form in fs[1:]:
            assert torch.equal(xs[form], xs["window"]), (solve, form)
    with pytest.raises(ValueError):
        A.set_persistent(True, form="tiled")
    A.set_persistent(True)


@pytest.mark.parametrize("case", ["one_cta", "isolated_nodes"])
def test_persistent_forms_bit_identical_edge_cases(mps, case):
    """Forced forms on a one-CTA system (10x10 Laplacian: 100 rows, a grid of
    one CTA) and on a random graph with isolated nodes (5,000 rows, mean
    degree 1.5: rows of 1 to about 10 nonzeros, windows spanning the
    matrix): plain CG and BiCGSTAB over 30 iterations, and learned-FSAI
    MP-PCG to 1e-8, return bit-identical results in every form."""
    c = W.laplacian_2d(10) if case == "one_cta" else W.graph_laplacian(5000, 1.5, 4, shift=0.05)
    A = _cg_system(mps, c)
    b = torch.from_numpy(W.rhs(c.n, 2)).cuda()
    forms = ("window", "gather", "stream")
    for solve, fs in (("cgd", forms), ("bicgstab", forms)):
        xs = {}
        for form in fs:
            A.set_persistent(True, form=form)
            x = torch.zeros(c.n, device="cuda")
            info = getattr(A, solve)(b, x, tol=1e-300, max_iter=30)
            assert info["persistent_form"] == form, (solve, form, info)
            xs[form] = (x, info["iters"])
        for form in fs[1:]:
            assert torch.equal(xs[form][0], xs["window"][0]) and xs[form][1] == xs["window"][1], (solve, form)
    omega = 0.2 if case == "one_cta" else 0.05   # below 2 / lambda_max of each system
    xs = {}
    for form in forms:
        A.set_persistent(True, form=form)
        x = torch.zeros(c.n, device="cuda")
        info = A.richardson(b, x, omega=omega, iters=31)
        assert info["persistent_form"] == form and info["iters"] == 31, (form, info)
        xs[form] = x
    for form in forms[1:]:
        assert torch.equal(xs[form], xs["window"]), ("richardson", form)
    from mpsparse_b200.fsai import LearnedFsai
    LearnedFsai.load().attach(A)
    A.set_fsai_apply("product")
    b64 = b.double()
    out = {}
    for form in forms:
        A.set_persistent(True, form=form)
        x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
        info = A.cg_mixed(b64, x, tol=1e-8, inner_tol=1e-3, max_inner=20000, precond="fsai")
        assert info["persistent_form"] == form and info["converged"], (form, info)
        out[form] = (x, info["inner_iters"])
    for form in forms[1:]:
        assert torch.equal(out[form][0], out["window"][0]) and out[form][1] == out["window"][1], form
    A.set_persistent(True)


def test_rows_too_large_fall_back_to_graph_form(mps):
    """1600^2 (17,297 rows per CTA): not even the vector window and the own
    rows' vectors fit one CTA per SM, so the graph form runs."""
    c, A = _learned(mps, 1600, 1600, 33)
    b = torch.from_numpy(W.rhs(c.n, 2).astype(np.float64)).cuda()
    x, info = _solve(A, b, True, tol=1e-6, inner_tol=1e-4, max_inner=40000)
    assert not info["persistent"] and info["persistent_form"] is None and info["converged"]


def _cg_system(mps, c):
    e = torch.empty(0)
    return mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e, c.n, c.n)


@pytest.mark.parametrize("precond", ["none", "jacobi"])
def test_persistent_cg_matches_graph_form_and_oracle(mps, oracle, precond):
    """Plain CG / Jacobi-PCG (the drop-in cgd) as one persistent kernel:
    the first iterates agree with the graph form's and the FP64 oracle's
    (1e-5 relative, the cgd iterate bar), and converged solves need the same
    iterations within 2 and reach the same FP64 true residual bar."""
    from tests.helpers import assert_solved_fp32
    c = W.lognormal_diffusion_2d(96, 80, 1.0, 6.0, 12) if precond == "jacobi" else W.laplacian_2d(128)
    A = _cg_system(mps, c)
    Ao = oracle.Csr(*c.to_csr(), c.n)
    b = W.rhs(c.n, 5)
    bt = torch.from_numpy(b).cuda()
    for k in (1, 2, 5, 20):
        xs = []
        for persistent in (True, False):
            A.set_persistent(persistent)
            x = torch.zeros(c.n, device="cuda")
            info = A.cgd(bt, x, tol=1e-300, max_iter=k, precond=precond)
            assert info["iters"] == k and info["persistent"] == persistent
            xs.append(x.cpu().numpy().astype(np.float64))
        xo, _ = oracle.cg(Ao, b, tol=0.0, max_iter=k, precond=None if precond == "none" else "jacobi")
        for xk in xs:
            assert np.linalg.norm(xk - xo) / np.linalg.norm(xo) <= 1e-5, k
    infos = []
    for persistent in (True, False):
        A.set_persistent(persistent)
        x = torch.zeros(c.n, device="cuda")
        info = A.cgd(bt, x, tol=1e-6, max_iter=20000, precond=precond)
        assert info["stop_rule_met"] and info["persistent"] == persistent
        assert_solved_fp32(oracle, Ao, b, x.cpu().numpy(), 1e-6, info)
        infos.append(info)
    assert abs(infos[0]["iters"] - infos[1]["iters"]) <= 2, infos


def test_persistent_cg_edge_cases(mps):
    """b = 0 returns x = 0 at once; a non-finite b is rejected; the handle
    stays usable (the same rules as the graph form)."""
    c = W.laplacian_2d(64)
    A = _cg_system(mps, c)
    A.set_persistent(True)
    x = torch.ones(c.n, device="cuda")
    info = A.cgd(torch.zeros(c.n, device="cuda"), x)
    assert info["persistent"] and info["converged"] and info["iters"] == 0
    assert float(x.abs().max()) == 0.0
    bad = torch.ones(c.n, device="cuda")
    bad[3] = float("inf")
    with pytest.raises(RuntimeError, match="non-finite"):
        A.cgd(bad, x)
    info = A.cgd(torch.ones(c.n, device="cuda"), x, max_iter=3, tol=1e-300)
    assert info["iters"] == 3 and info["persistent"]


def test_persistent_cg_stream_form(mps, oracle):
    """1024^2 Laplacian (5.2 M nonzeros, 7,085 rows per CTA): A's rows do
    not fit shared memory, the vector windows do -- plain CG and Jacobi-PCG
    in the stream form agree with the graph form's first iterates (1e-5
    relative) and with the FP64 oracle's, and a converged solve needs the
    graph form's iterations within 1 % and meets the FP32 bar."""
    from tests.helpers import assert_solved_fp32
    c = W.laplacian_2d(1024)
    A = _cg_system(mps, c)
    Ao = oracle.Csr(*c.to_csr(), c.n)
    b = W.rhs(c.n, 1)
    bt = torch.from_numpy(b).cuda()
    for precond in ("none", "jacobi"):
        for k in (1, 5, 20):
            xs = []
            for persistent in (True, False):
                A.set_persistent(persistent)
                x = torch.zeros(c.n, device="cuda")
                info = A.cgd(bt, x, tol=1e-300, max_iter=k, precond=precond)
                assert info["iters"] == k
                assert info["persistent_form"] == ("stream" if persistent else None), info
                xs.append(x.cpu().numpy().astype(np.float64))
            assert np.linalg.norm(xs[0] - xs[1]) / np.linalg.norm(xs[1]) <= 1e-5, (precond, k)
            xo, _ = oracle.cg(Ao, b, tol=0.0, max_iter=k, precond=None if precond == "none" else "jacobi")
            for xk in xs:
                assert np.linalg.norm(xk - xo) / np.linalg.norm(xo) <= 1e-5, (precond, k)
    infos = []
    for persistent in (True, False):
        A.set_persistent(persistent)
        x = torch.zeros(c.n, device="cuda")
        info = A.cgd(bt, x, tol=1e-6, max_iter=40000)
        assert info["stop_rule_met"] and info["persistent"] == persistent
        assert_solved_fp32(oracle, Ao, b, x.cpu().numpy(), 1e-6, info)
        infos.append(info)
    assert abs(infos[0]["iters"] - infos[1]["iters"]) <= 0.01 * infos[1]["iters"] + 2, infos
    # reliable updates (cg_mixed) in the stream form reach the FP64 target
    A.set_persistent(True)
    x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
    info = A.cg_mixed(bt.double(), x, tol=1e-9, inner_tol=1e-3, max_inner=40000)
    assert info["persistent_form"] == "stream" and info["converged"], info
    assert oracle.true_residual(Ao, b.astype(np.float64), x.cpu().numpy()) <= 1e-9 * 1.01


def test_persistent_cg_falls_back_for_large_rows(mps):
    """1600^2 Laplacian (12.8 M nonzeros, 17,297 rows per CTA): not even the
    vector window fits one CTA per SM, so the graph form runs."""
    c = W.laplacian_2d(1600)
    A = _cg_system(mps, c)
    b = torch.from_numpy(W.rhs(c.n, 1)).cuda()
    x = torch.zeros(c.n, device="cuda")
    info = A.cgd(b, x, tol=1e-3, max_iter=200)
    assert not info["persistent"] and info["persistent_form"] is None and info["iters"] > 0


@pytest.mark.parametrize("precond", ["none", "jacobi"])
def test_persistent_reliable_cg_matches_graph_form(mps, oracle, precond):
    """cg_mixed without FSAI (FP32 recurrences, FP64 x, residual
    replacement) as one persistent kernel: the first iterates agree with
    the graph form's (1e-6 relative; only the grouping of the FP64 partial
    sums differs), and converged solves reach the FP64 target checked by
    the oracle, with iteration and replacement counts close to the graph
    form's."""
    c = W.lognormal_diffusion_2d(96, 80, 1.0, 6.0, 14) if precond == "jacobi" else W.laplacian_2d(128)
    A = _cg_system(mps, c)
    Ao = oracle.Csr(*c.to_csr(), c.n)
    b = torch.from_numpy(W.rhs(c.n, 6).astype(np.float64)).cuda()
    for k in (1, 2, 5, 20):
        xs = []
        for persistent in (True, False):
            A.set_persistent(persistent)
            x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
            info = A.cg_mixed(b, x, tol=1e-30, inner_tol=1e-30, max_inner=k, max_outer=1, precond=precond)
            assert info["persistent"] == persistent and info["inner_iters"] == k, (k, info)
            xs.append(x)
        assert float((xs[0] - xs[1]).norm() / xs[1].norm()) <= 1e-6, k
    infos, sols = [], []
    for persistent in (True, False):
        A.set_persistent(persistent)
        x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
        info = A.cg_mixed(b, x, tol=1e-9, inner_tol=1e-3, max_inner=40000, precond=precond)
        assert info["persistent"] == persistent and info["converged"], info
        assert oracle.true_residual(Ao, b.cpu().numpy(), x.cpu().numpy()) <= 1e-9 * 1.01
        infos.append(info)
        sols.append(x)
    ip, ig = infos
    assert abs(ip["inner_iters"] - ig["inner_iters"]) <= 0.05 * ig["inner_iters"] + 3, infos
    assert float((sols[0] - sols[1]).norm() / sols[1].norm()) <= 1e-7
    # b = 0: x = 0 at once, on the persistent form too
    A.set_persistent(True)
    x = torch.ones(c.n, dtype=torch.float64, device="cuda")
    info = A.cg_mixed(torch.zeros_like(b), x, precond=precond)
    assert info["persistent"] and info["converged"] and float(x.abs().max()) == 0.0


def test_persistent_gather_form_on_random_graph(mps, oracle):
    """A random graph Laplacian (60,000 rows, mean degree 6): every row block
    couples to columns all over the matrix, so the blocks' vector windows do
    not fit beside their rows and the persistent kernels gather the vector
    entries instead.  Plain CG and learned-FSAI mixed-precision PCG both
    agree with the graph form (first iterates) and reach their targets."""
    c = W.graph_laplacian(60000, 6.0, 3, shift=0.05)
    A = _cg_system(mps, c)
    Ao = oracle.Csr(*c.to_csr(), c.n)
    b = W.rhs(c.n, 7)
    bt = torch.from_numpy(b).cuda()
    for k in (1, 5, 20):
        xs = []
        for persistent in (True, False):
            A.set_persistent(persistent)
            x = torch.zeros(c.n, device="cuda")
            info = A.cgd(bt, x, tol=1e-300, max_iter=k)
            assert info["iters"] == k and info["persistent"] == persistent
            xs.append(x)
        assert float((xs[0] - xs[1]).norm() / xs[1].norm()) <= 1e-6, k
    A.set_persistent(True)
    x = torch.zeros(c.n, device="cuda")
    info = A.cgd(bt, x, tol=1e-6, max_iter=20000)
    assert info["persistent_form"] == "gather" and info["stop_rule_met"]
    # BiCGSTAB in the gather form: the graph form's first iterates, and a
    # converged solve; the window form does not fit here (graph form runs)
    for k in (1, 5, 20):
        xs = []
        for persistent in (True, False):
            A.set_persistent(persistent)
            x = torch.zeros(c.n, device="cuda")
            info = A.bicgstab(bt, x, tol=1e-300, max_iter=k)
            assert info["iters"] == k and info["persistent_form"] == ("gather" if persistent else None)
            xs.append(x)
        assert float((xs[0] - xs[1]).norm() / xs[1].norm()) <= 1e-5, k
    A.set_persistent(True)
    x = torch.zeros(c.n, device="cuda")
    info = A.bicgstab(bt, x, tol=1e-6, max_iter=20000)
    assert info["persistent_form"] == "gather" and info["stop_rule_met"]
    A.set_persistent(True, form="window")
    info = A.bicgstab(bt, x, tol=1e-6, max_iter=20000)
    assert not info["persistent"] and info["stop_rule_met"]
    A.set_persistent(True)
    from mpsparse_b200.fsai import LearnedFsai
    LearnedFsai.load().attach(A)
    A.set_fsai_apply("product")
    b64 = bt.double()
    sols = []
    for persistent in (True, False):
        A.set_persistent(persistent)
        x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
        info = A.cg_mixed(b64, x, tol=1e-8, inner_tol=1e-3, max_inner=40000, precond="fsai")
        assert info["converged"] and info["persistent"] == persistent, info
        assert oracle.true_residual(Ao, b, x.cpu().numpy()) <= 1e-8 * 1.01
        sols.append(x)
    assert float((sols[0] - sols[1]).norm() / sols[1].norm()) <= 1e-6


def test_persistent_560_window_form(mps, oracle):
    """560^2 fits one CTA per SM only in the window form (16-bit
    window-relative columns; 2,119 rows per CTA, more than two per thread).
    Without residual replacements the two forms' iterates agree to rounding
    of the FP64 partial sums through 2,000 iterations; the full solve reaches
    its FP64-checked target.  (Iteration counts of full solves are not
    compared here: on this system, at inner_tol 1e-3, last-bit differences
    of the grouped sums move a replacement by an iteration and the stall
    watch then branches differently -- measured 2,441 against 2,237, while
    at inner_tol 1e-2 and 1e-1 the counts agree within 5.)"""
    c, A = _learned(mps, 560, 560, 31)
    b = torch.from_numpy(W.rhs(c.n, 8).astype(np.float64)).cuda()
    xg, ig = _solve(A, b, False, tol=1e-30, inner_tol=1e-30, max_inner=2000, max_outer=1)
    xp, ip = _solve(A, b, True, tol=1e-30, inner_tol=1e-30, max_inner=2000, max_outer=1)
    assert ip["persistent_form"] == "window" and not ig["persistent"]
    assert ip["inner_iters"] == ig["inner_iters"] == 2000
    assert float((xp - xg).norm() / xg.norm()) <= 1e-12
    xp, ip = _solve(A, b, True, tol=1e-9, inner_tol=1e-3, max_inner=40000)
    assert ip["persistent"] and ip["converged"]
    Ao = oracle.Csr(*c.to_csr(), c.n)
    assert oracle.true_residual(Ao, b.cpu().numpy(), xp.cpu().numpy()) <= 1e-9 * 1.01


def _convection_diffusion(nx):
    """Nonsymmetric 5-point system: the 2D Laplacian with each east coupling
    halved (diagonally dominant, nonsingular)."""
    c = W.laplacian_2d(nx)
    vals = c.vals.copy()
    vals[c.cols == c.rows + 1] *= 0.5
    return W.Coo(c.rows, c.cols, vals.astype(np.float32), c.n)


@pytest.mark.parametrize("nx", [32, 128])
def test_persistent_bicgstab_matches_graph_form_and_oracle(mps, oracle, nx):
    """BiCGSTAB (the drop-in bicgstab) as one persistent kernel: the first
    iterates agree with the graph form's (1e-5 relative) and with the FP64
    oracle's (1e-5 relative up to 5 iterations, and up to 20 on the 32^2
    system; on 128^2 both FP32 forms drift from the FP64 recurrence by
    6e-5 after 20 iterations); converged solves need the same iterations
    within 2 and reach the FP64 true residual bar."""
    from tests.helpers import assert_solved_fp32
    c = _convection_diffusion(nx)
    A = _cg_system(mps, c)
    Ao = oracle.Csr(*c.to_csr(), c.n)
    b = W.rhs(c.n, 9)
    bt = torch.from_numpy(b).cuda()
    for k in (1, 2, 5, 20):
        xs = []
        for persistent in (True, False):
            A.set_persistent(persistent)
            x = torch.zeros(c.n, device="cuda")
            info = A.bicgstab(bt, x, tol=1e-300, max_iter=k)
            assert info["iters"] == k and info["persistent"] == persistent, (k, info)
            xs.append(x.cpu().numpy().astype(np.float64))
        assert np.linalg.norm(xs[0] - xs[1]) / np.linalg.norm(xs[1]) <= 1e-5, k
        if k <= 5 or nx == 32:
            xo, _ = oracle.bicgstab(Ao, b, tol=0.0, max_iter=k)
            for xk in xs:
                assert np.linalg.norm(xk - xo) / np.linalg.norm(xo) <= 1e-5, k
    infos = []
    for persistent in (True, False):
        A.set_persistent(persistent)
        x = torch.zeros(c.n, device="cuda")
        info = A.bicgstab(bt, x, tol=1e-6, max_iter=20000)
        assert info["stop_rule_met"] and info["persistent"] == persistent
        assert_solved_fp32(oracle, Ao, b, x.cpu().numpy(), 1e-6, info)
        infos.append(info)
    assert abs(infos[0]["iters"] - infos[1]["iters"]) <= 2, infos


def test_persistent_bicgstab_edge_cases(mps):
    """b = 0 returns x = 0 at once; a non-finite b is rejected; the handle
    stays usable; reference_compat keeps the graph form."""
    c = _convection_diffusion(64)
    A = _cg_system(mps, c)
    A.set_persistent(True)
    x = torch.ones(c.n, device="cuda")
    info = A.bicgstab(torch.zeros(c.n, device="cuda"), x)
    assert info["persistent"] and info["converged"] and info["iters"] == 0
    assert float(x.abs().max()) == 0.0
    bad = torch.ones(c.n, device="cuda")
    bad[5] = float("nan")
    with pytest.raises(RuntimeError, match="non-finite"):
        A.bicgstab(bad, x)
    info = A.bicgstab(torch.ones(c.n, device="cuda"), x, max_iter=4, tol=1e-300)
    assert info["iters"] == 4 and info["persistent"]
    info = A.bicgstab(torch.ones(c.n, device="cuda"), x, reference_compat=True)
    assert not info["persistent"]


def test_persistent_bicgstab_stream_form(mps, oracle):
    """BiCGSTAB on a 1024^2 nonsymmetric 5-point system in the stream form
    (rows from L2, the staged p and s windows in shared memory): the first
    iterates agree with the graph form's (1e-5 relative) and with the FP64
    oracle's up to 5 iterations; a converged solve needs the graph form's
    iterations within 2 % and meets the FP32 bar."""
    from tests.helpers import assert_solved_fp32
    c = _convection_diffusion(1024)
    A = _cg_system(mps, c)
    Ao = oracle.Csr(*c.to_csr(), c.n)
    b = W.rhs(c.n, 4)
    bt = torch.from_numpy(b).cuda()
    for k in (1, 5, 20):
        xs = []
        for persistent in (True, False):
            A.set_persistent(persistent)
            x = torch.zeros(c.n, device="cuda")
            info = A.bicgstab(bt, x, tol=1e-300, max_iter=k)
            assert info["iters"] == k
            assert info["persistent_form"] == ("stream" if persistent else None), info
            xs.append(x.cpu().numpy().astype(np.float64))
        assert np.linalg.norm(xs[0] - xs[1]) / np.linalg.norm(xs[1]) <= 1e-5, k
        if k <= 5:
            xo, _ = oracle.bicgstab(Ao, b, tol=0.0, max_iter=k)
            for xk in xs:
                assert np.linalg.norm(xk - xo) / np.linalg.norm(xo) <= 1e-5, k
    infos = []
    for persistent in (True, False):
        A.set_persistent(persistent)
        x = torch.zeros(c.n, device="cuda")
        info = A.bicgstab(bt, x, tol=1e-6, max_iter=40000)
        assert info["stop_rule_met"] and info["persistent"] == persistent
        assert_solved_fp32(oracle, Ao, b, x.cpu().numpy(), 1e-6, info)
        infos.append(info)
    assert abs(infos[0]["iters"] - infos[1]["iters"]) <= 0.02 * infos[1]["iters"] + 2, infos


def test_persistent_barrier_timeout_returns_error_and_handle_stays_usable(mps, oracle):
    """A bounded grid-barrier wait that runs out: the test hook makes CTA 3
    withhold its first arrival, so every CTA's first wait (bounded at
    20,000 polls, milliseconds) gives up and raises the abort word, and the
    kernel ends.  The call returns MPS_ERR_TIMEOUT; afterwards the same
    handle solves to the oracle's iterates, and the hook with no silent CTA
    is an ordinary 50-iteration solve."""
    import ctypes as C
    from tests import cabi
    L = cabi.lib()
    f = L.mps_test_persistent_barrier_timeout
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int32, C.c_void_p]
    f.restype = C.c_int
    c = W.laplacian_2d(128)
    keys = torch.from_numpy(c.keys()).cuda()
    vals = torch.from_numpy(c.vals).cuda()
    h = C.c_void_p()
    cabi.check(L.mps_csr_create_from_keys(cabi.ptr(keys), cabi.ptr(vals), c.nnz, c.n, c.n, C.byref(h), None))
    b = torch.from_numpy(W.rhs(c.n, 3)).cuda()
    x = torch.zeros(c.n, device="cuda")
    try:
        for _ in range(2):
            st = f(h, cabi.ptr(b), cabi.ptr(x), 20000, 3, None)
            assert st == 4, (st, L.mps_last_error_string())           # MPS_ERR_TIMEOUT
            msg = L.mps_last_error_string()
            assert b"watchdog" in msg or b"bounded device wait" in msg, msg
        torch.cuda.synchronize()
        assert f(h, cabi.ptr(b), cabi.ptr(x), 20000, -1, None) == 0
        o = cabi.SolveOpts()
        L.mps_solve_opts_default(C.byref(o))
        o.tol, o.max_iter = 1e-300, 20
        info = cabi.SolveInfo()
        x.zero_()
        cabi.check(L.mps_csr_cg(h, cabi.ptr(b), cabi.ptr(x), C.byref(o), C.byref(info), None))
        assert info.persistent and info.iters == 20
        Ao = oracle.Csr(*c.to_csr(), c.n)
        xo, _ = oracle.cg(Ao, b.cpu().numpy(), tol=0.0, max_iter=20)
        assert np.linalg.norm(x.cpu().numpy() - xo) / np.linalg.norm(xo) <= 1e-5
    finally:
        L.mps_csr_destroy(h)


def test_persistent_richardson_matches_graph_form_and_oracle(mps, oracle):
    """Richardson (the drop-in richardson, outside reference_compat) as one
    persistent kernel: x depends on no sum, so for a fixed iteration count
    (odd and even: the result buffer alternates) it is bit-identical to the
    graph form's, and within 1e-5 of the FP64 oracle's; with a tolerance
    both forms stop within one iteration of each other (the stop test's sum
    groups differently).  On a random graph the gather form runs."""
    c = W.laplacian_2d(128)
    A = _cg_system(mps, c)
    Ao = oracle.Csr(*c.to_csr(), c.n)
    b = W.rhs(c.n, 4)
    bt = torch.from_numpy(b).cuda()
    for iters in (1, 2, 301):
        xs = []
        for persistent in (True, False):
            A.set_persistent(persistent)
            x = torch.zeros(c.n, device="cuda")
            info = A.richardson(bt, x, omega=0.2, iters=iters)
            assert info["iters"] == iters
            assert info["persistent_form"] == ("window" if persistent else None), info
            xs.append(x)
        assert torch.equal(xs[0], xs[1]), iters
        xo, _ = oracle.richardson(Ao, b, compat=False, omega=0.2, iters=iters)
        assert np.linalg.norm(xs[0].cpu().numpy() - xo) / np.linalg.norm(xo) <= 1e-5, iters
    its = []
    for persistent in (True, False):
        A.set_persistent(persistent)
        x = torch.zeros(c.n, device="cuda")
        info = A.richardson(bt, x, omega=0.2, iters=20000, tol=0.3)
        assert info["converged"] and info["persistent"] == persistent, info
        its.append(info["iters"])
    assert abs(its[0] - its[1]) <= 1, its
    g = W.graph_laplacian(60000, 6.0, 3, shift=0.05)
    G = _cg_system(mps, g)
    bg = torch.from_numpy(W.rhs(g.n, 7)).cuda()
    xs = []
    for persistent in (True, False):
        G.set_persistent(persistent)
        x = torch.zeros(g.n, device="cuda")
        info = G.richardson(bg, x, omega=0.02, iters=50)
        assert info["persistent_form"] == ("gather" if persistent else None), info
        xs.append(x)
    assert torch.equal(xs[0], xs[1])
