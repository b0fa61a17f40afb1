"""BCSR (4x4 / 8x8) SpMV, GPU COO->BCSR and BCSR solvers against the oracle."""
import numpy as np
import pytest
import torch

from mpsparse_b200 import workloads as W
from tests.helpers import assert_solved_fp32

pytestmark = pytest.mark.gpu


def _bt(mps, bm, n=None):
    return mps.bcsr.bcsr_tensor(torch.empty(0), torch.from_numpy(bm.vals),
                                torch.from_numpy(bm.row_ptr), torch.from_numpy(bm.col_ind),
                                n or bm.n, n or bm.n, bm.block)


def test_golden_block16(mps, golden, oracle):
    g = golden("block16")
    bm = W.Bcsr(g["row_ptr"], g["col_ind"], g["vals"], 4, int(g["n"]))
    A = _bt(mps, bm)
    y = torch.zeros(bm.n)
    A.mv(torch.from_numpy(g["x"]), y)
    assert np.allclose(y.numpy(), g["y"], rtol=1e-5, atol=1e-4)
    for k in (1, 4, 8):
        x = torch.zeros(bm.n)
        A.bicgstab(torch.from_numpy(g["b"]), x, tol=1e-300, max_iter=k)
        ref = g["bicgstab_iterates"][k - 1]
        assert np.linalg.norm(x.numpy() - ref) <= 1e-5 * np.linalg.norm(ref)


@pytest.mark.parametrize("B,nbr", [(4, 3000), (8, 1500), (4, 65536)])
def test_spmv_vs_oracle(mps, oracle, B, nbr):
    bm = W.block_dominant(nbr, 8, seed=B, block=B)
    A = _bt(mps, bm)
    x = np.random.default_rng(0).standard_normal(bm.n).astype(np.float32)
    y = torch.zeros(bm.n, device="cuda")
    A.mv(torch.from_numpy(x).cuda(), y)
    Ao = oracle.Csr(bm.row_ptr, bm.col_ind, bm.vals, bm.n, B)
    ref = oracle.spmv(Ao, x)
    bound = oracle.spmv(oracle.Csr(bm.row_ptr, bm.col_ind, np.abs(bm.vals), bm.n, B), np.abs(x))
    assert np.all(np.abs(y.cpu().numpy() - ref) <= 1e-6 * bound)


@pytest.mark.parametrize("B", [4, 8])
def test_coo_to_bcsr_on_gpu(mps, B):
    bm = W.block_dominant(700, 5, seed=11, block=B)
    coo = bm.to_coo(drop_zeros=True).shuffled(3)
    A = mps.bcsr.bcsr_tensor(torch.from_numpy(coo.keys()), torch.from_numpy(coo.vals),
                             torch.empty(0, dtype=torch.int32), torch.empty(0, dtype=torch.int32),
                             bm.n, bm.n, B)
    rp, ci, v = (t.cpu().numpy() for t in A.bcsr())
    assert np.array_equal(rp, bm.row_ptr) and np.array_equal(ci, bm.col_ind)
    assert np.array_equal(v, bm.vals)


def test_unpadded_and_solvers(mps, oracle):
    bm = W.block_dominant(4096, 8, seed=1)
    n_logical = bm.n - 3                       # last block row padded
    coo = bm.to_coo(drop_zeros=True)
    keep = (coo.rows < n_logical) & (coo.cols < n_logical)
    sub = W.Coo(coo.rows[keep], coo.cols[keep], coo.vals[keep], n_logical)
    A = mps.bcsr.bcsr_tensor(torch.from_numpy(sub.keys()), torch.from_numpy(sub.vals),
                             torch.empty(0, dtype=torch.int32), torch.empty(0, dtype=torch.int32),
                             n_logical, n_logical, 4)
    assert A.padded_rows == bm.n
    b = W.rhs(n_logical, 3)
    x = torch.zeros(n_logical)
    info = A.bicgstab(torch.from_numpy(b), x, tol=1e-6)             # unpadded b accepted
    Ao = oracle.Csr(*sub.to_csr(), n_logical)
    assert info["stop_rule_met"]
    assert_solved_fp32(oracle, Ao, b, x.numpy(), 1e-6, info)
    # CG on an SPD block system (block diagonal 4x4 SPD blocks + coupling)
    spd = W.laplacian_2d(64)
    A2 = mps.bcsr.bcsr_tensor(torch.from_numpy(spd.keys()), torch.from_numpy(spd.vals),
                              torch.empty(0, dtype=torch.int32), torch.empty(0, dtype=torch.int32),
                              spd.n, spd.n, 4)
    b2 = W.rhs(spd.n, 4)
    x2 = torch.zeros(spd.n)
    info = A2.cgd(torch.from_numpy(b2), x2, tol=1e-6)
    A2o = oracle.Csr(*spd.to_csr(), spd.n)
    assert info["stop_rule_met"]
    assert_solved_fp32(oracle, A2o, b2, x2.numpy(), 1e-6, info)


def test_sparse_bsr_export(mps):
    """bcsr_tensor.sparse_bsr(): the padded BCSR as a torch.sparse_bsr_tensor
    (row-major B x B blocks) equal to the handle's arrays."""
    bm = W.block_dominant(300, 5, seed=4)
    c = bm.to_coo(drop_zeros=True).shuffled(5)
    ei = torch.empty(0, dtype=torch.int32)
    A = mps.bcsr.bcsr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), ei, ei, c.n, c.n, 4)
    S = A.sparse_bsr()
    assert S.layout == torch.sparse_bsr and tuple(S.shape) == (A.padded_rows, A.padded_rows)
    rp, ci, v = A.bcsr()
    assert torch.equal(S.crow_indices(), rp) and torch.equal(S.col_indices(), ci)
    assert torch.equal(S.values().reshape(-1), v)
    dense = torch.zeros(c.n, c.n, dtype=torch.float64)
    dense.index_put_((torch.from_numpy(c.rows), torch.from_numpy(c.cols)),
                     torch.from_numpy(c.vals).double(), accumulate=True)
    assert torch.equal(S.to_dense().cpu().double(), dense)
