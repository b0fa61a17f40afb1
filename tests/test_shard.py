"""Host logic of the multi-GPU path on CPU: nnz-balanced system shares and
the gather of per-system records over 2 gloo ranks."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from mpsparse_b200 import shard


def test_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    nnz = rng.integers(1000, 600000, 4096)
    parts = shard.partition_by_nnz(nnz, 8)
    allidx = np.sort(np.concatenate(parts))
    assert np.array_equal(allidx, np.arange(4096))
    loads = np.array([nnz[p].sum() for p in parts])
    assert loads.max() - loads.min() <= nnz.max()           # LPT bound
    assert shard.partition_by_nnz(nnz, 1)[0].shape[0] == 4096


def test_local_rows():
    row_off = np.array([0, 10, 15, 40, 41])
    loc = shard.local_rows(row_off, np.array([1, 3]))
    assert list(loc) == [0, 5, 6]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nnz = np.arange(1, 38) * 7 % 23 + 1
        parts = shard.partition_by_nnz(nnz, world)
        mine = parts[rank]
        vals = mine * 10.0 + 0.5                  # a per-system record
        merged = shard.gather_records(vals, mine, nnz.shape[0])
        t = shard.max_over_ranks(1.0 + rank)
        q.put((rank, merged.tolist(), t))
    finally:
        dist.destroy_process_group()


def test_gather_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, merged, t in out:
        assert np.allclose(merged, np.arange(37) * 10.0 + 0.5)
        assert t == 2.0


def _batch_worker(rank, world, port, q):
    """The batched leg's sharding path on CPU: each rank builds only its
    nnz-balanced share of a generated batch and the per-system records are
    gathered back into global system order."""
    import torch.distributed as dist
    from mpsparse_b200 import workloads as W
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n_sys, seed = 12, 5
        _, _, est = W.batch_plan(n_sys, seed, n_min=64, n_max=400)
        mine = shard.partition_by_nnz(est, world)[rank]
        keys, vals, off, kinds = W.batch_systems(n_sys, seed, n_min=64, n_max=400, device="cpu",
                                                 select=mine)
        rows = np.diff(off).astype(np.float64)
        nnz = np.array([((keys >> 32) >= off[k]).logical_and((keys >> 32) < off[k + 1]).sum().item()
                        for k in range(len(mine))], np.float64)
        merged_rows = shard.gather_records(rows, mine, n_sys)
        merged_nnz = shard.gather_records(nnz, mine, n_sys)
        q.put((rank, merged_rows.tolist(), merged_nnz.tolist(), kinds.tolist(), mine.tolist()))
    finally:
        dist.destroy_process_group()


def test_batched_shards_over_two_gloo_ranks():
    from mpsparse_b200 import workloads as W
    n_sys, seed = 12, 5
    keys, vals, off, kinds = W.batch_systems(n_sys, seed, n_min=64, n_max=400, device="cpu")
    rows = np.diff(off)
    rk = (keys >> 32).numpy()
    nnz = np.array([((rk >= off[k]) & (rk < off[k + 1])).sum() for k in range(n_sys)])
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shares = []
    for rank, mrows, mnnz, k_local, mine in out:
        assert np.array_equal(np.array(mrows), rows)          # same systems as the whole batch
        assert np.array_equal(np.array(mnnz), nnz)
        assert np.array_equal(np.array(k_local), kinds[mine])
        shares.append(mine)
    assert sorted(shares[0] + shares[1]) == list(range(n_sys))
