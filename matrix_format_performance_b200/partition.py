"""Multi-GPU sharding of the SpMV path (one process per GPU).

SpMV with x replicated on every rank needs no exchange: rank r computes the
rows it owns and y is the concatenation of the ranks' slices.
- row_partition   contiguous row ranges balanced by nonzeros plus rows (a
                  prefix sum over row_ptr and a binary search per boundary)
- shard_csr       the CSR of one rank's rows (columns stay global)
- rank_shard      row_partition + shard_csr for one rank (what bench.py's
                  ranks run)
- assign_matrices whole matrices of a batch to ranks, balanced by bytes
                  (largest first onto the least-loaded rank)
An x distributed by rows would first need one all-gather of the x slices;
y never needs a reduction.
"""
from __future__ import annotations

import numpy as np

from .formats import csr_matrix_class


def row_partition(row_ptr: np.ndarray, world: int, row_weight: float = 1.0) -> np.ndarray:
    """world+1 row bounds; rank r owns rows [b[r], b[r+1]).  The cost of a row
    prefix is nnz + row_weight * rows, split into equal parts."""
    rp = np.asarray(row_ptr, np.int64)
    rows = rp.size - 1
    cost = rp + row_weight * np.arange(rows + 1)
    targets = cost[-1] * np.arange(1, world) / world
    inner = np.searchsorted(cost, targets, side="left")
    b = np.concatenate([[0], np.clip(inner, 0, rows), [rows]]).astype(np.int64)
    return np.maximum.accumulate(b)


def shard_csr(m: csr_matrix_class, lo: int, hi: int) -> csr_matrix_class:
    rp = m.row_ptr.astype(np.int64)
    e0, e1 = rp[lo], rp[hi]
    return csr_matrix_class.from_arrays(hi - lo, m.cols, (rp[lo:hi + 1] - e0).astype(np.uint32),
                                        m.columns[e0:e1], m.data[e0:e1], m.dtype)


def rank_shard(m: csr_matrix_class, rank: int, world: int) -> tuple[csr_matrix_class, int, int]:
    """The rows one rank runs in a strong-scaling SpMV of m (x replicated):
    (its CSR shard, first row, one past its last row).  bench.py's ranks and
    the multi-process tests both take their rows from here."""
    b = row_partition(m.row_ptr, world)
    lo, hi = int(b[rank]), int(b[rank + 1])
    return shard_csr(m, lo, hi), lo, hi


def matrix_bytes(m: csr_matrix_class) -> int:
    vs = np.dtype(m.dtype).itemsize
    return int(m.nnz * (vs + 4) + (m.rows + 1) * 4 + m.cols * vs + m.rows * vs)


def assign_matrices(sizes, world: int) -> list[list[int]]:
    """Indices of the matrices each rank runs: largest first onto the rank
    with the fewest bytes so far (ties to the lower rank)."""
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += sizes[i]
    return [sorted(v) for v in out]
