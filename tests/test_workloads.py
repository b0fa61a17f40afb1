"""Synthetic systems have the sizes the measured configurations state."""
import numpy as np

from mpsparse_b200 import workloads as W


def test_laplacian_256_size():
    c = W.laplacian_256()
    assert c.n == 65536 and c.nnz == 326656


def test_block_dominant_shape():
    b = W.block_dominant(1024, 8, seed=0)
    assert b.col_ind.shape[0] == 1024 * 9 and b.vals.shape[0] == 1024 * 9 * 16
    for r in range(0, 1024, 97):
        cols = b.col_ind[b.row_ptr[r]:b.row_ptr[r + 1]]
        assert len(set(cols.tolist())) == 9 and r in cols
    A = b.to_coo(drop_zeros=False)
    import scipy.sparse as sp
    M = sp.csr_matrix((A.vals.astype(np.float64), (A.rows, A.cols)), shape=(b.n, b.n))
    d = M.diagonal()
    off = np.abs(M).sum(axis=1).A1 - np.abs(d)
    assert np.all(d > off)                      # strictly diagonally dominant


def test_diffusion_512_size_and_spd_pattern():
    c = W.diffusion_512sq(3)
    assert c.n == 512 * 512 and c.nnz == 5 * 512 * 512 - 4 * 512
    lower = (c.cols <= c.rows).sum()
    assert lower == 785408                      # nnz(tril(A)) = nnz(G)


def test_diffusion_3d_small():
    c = W.lognormal_diffusion_3d(16, 1.0, 8.0, 0)
    assert c.nnz == 7 * 16 ** 3 - 6 * 16 ** 2


def test_gaussian_field_stats():
    g = W.gaussian_field((256, 256), 1.5, 16.0, 0)
    assert abs(g.std() - 1.5) < 1e-9 and abs(g.mean()) < 1e-9


def test_graph_laplacian():
    c = W.graph_laplacian(5000, 8, 0)
    rp, ci, cv = c.to_csr()
    assert abs(c.nnz / c.n - 9.0) < 0.2         # mean degree 8 + diagonal
