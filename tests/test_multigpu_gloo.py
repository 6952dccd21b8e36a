"""The multi-GPU sharding logic on world_size-2 gloo process groups (CPU).

Each rank takes its row shard of a power-law matrix with partition.rank_shard
(the call bench.py's ranks make for strong scaling), computes its y slice
with the oracle (the engine's kernels need a GPU), and the all-gathered slices
must equal the single-process product bit for bit; the shards' nonzeros are
balanced.  For batches, every matrix is assigned to exactly one rank and the
ranks' bytes are balanced.  No GPU: the host-side sharding exercised with real
process groups.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rows_worker(rank, world, port, q):
    import torch

    from matrix_format_performance_b200 import synth
    from matrix_format_performance_b200.partition import rank_shard
    from oracle import load_oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = synth.power_law(rows=60_000, seed=5).astype(np.float32)
        x = synth.vector(2, m.cols).astype(np.float32)
        s, lo, hi = rank_shard(m, rank, world)
        assert s.rows == hi - lo
        orc = load_oracle()
        y_local = orc.csr_spmv(s.rows, s.row_ptr, s.columns, s.data, x).astype(np.float32)
        sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(sizes, torch.tensor([s.rows]))
        n = max(int(v.item()) for v in sizes)
        buf = torch.zeros(n)
        buf[:s.rows] = torch.from_numpy(y_local)
        parts = [torch.zeros(n) for _ in range(world)]
        dist.all_gather(parts, buf)
        nnz = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(nnz, torch.tensor([s.nnz]))
        if rank == 0:
            y = np.concatenate([p[:int(sz.item())].numpy() for p, sz in zip(parts, sizes)])
            y_full = orc.csr_spmv(m.rows, m.row_ptr, m.columns, m.data, x).astype(np.float32)
            q.put((bool(np.array_equal(y.view(np.uint32), y_full.view(np.uint32))),
                   [int(v.item()) for v in nnz], int(m.nnz)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _batch_worker(rank, world, port, q):
    import torch

    from matrix_format_performance_b200.batch import uneven_set
    from matrix_format_performance_b200.partition import assign_matrices, matrix_bytes
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mats, _ = uneven_set(40, 1_000, 20_000)
        sizes = [matrix_bytes(m) for m in mats]
        mine = assign_matrices(sizes, world)[rank]
        flags = torch.zeros(len(mats), dtype=torch.int64)
        flags[mine] = 1
        dist.all_reduce(flags)
        load = torch.tensor([sum(sizes[i] for i in mine)], dtype=torch.int64)
        loads = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(loads, load)
        if rank == 0:
            q.put((flags.tolist(), [int(v.item()) for v in loads], max(sizes)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _guard(worker, rank, world, port, q):
    try:
        worker(rank, world, port, q)
    except BaseException as e:  # report instead of leaving the parent waiting
        q.put(("error", rank, repr(e)))
        raise


def _run(worker, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_guard, args=(worker, r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = q.get(timeout=180)
    assert not (isinstance(res, tuple) and res and res[0] == "error"), res
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


def test_row_partition_bounds():
    from matrix_format_performance_b200.partition import row_partition
    rp = np.array([0, 10, 10, 10, 50, 51, 52, 100], np.uint32)
    b = row_partition(rp, 3)
    assert b[0] == 0 and b[-1] == 7 and np.all(np.diff(b) >= 0)
    assert np.array_equal(row_partition(np.zeros(1, np.uint32), 4), np.zeros(5))


@pytest.mark.timeout(300)
def test_row_shards_gather_to_the_full_product():
    equal, nnz, total = _run(_rows_worker)
    assert equal
    assert sum(nnz) == total and max(nnz) <= 0.55 * total


@pytest.mark.timeout(300)
def test_batch_assignment_covers_and_balances():
    flags, loads, biggest = _run(_batch_worker)
    assert all(f == 1 for f in flags)
    assert max(loads) - min(loads) <= biggest
