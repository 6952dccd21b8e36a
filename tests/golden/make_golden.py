"""Generates tests/golden/*.npz from the reference's own code.

    python tests/golden/make_golden.py

Needs oracle/_ref/libmfp_ref.so, which oracle/Makefile compiles from the
reference checkout (`make -C oracle ref`).  Each fixture holds a small COO
input (seeded numpy draws, written out in shuffled order like a Matrix Market
file) and, per value type, what the reference's converters and CPU loops
return for it:
  csr_*         csr_matrix_class           (matrix_converter.cpp:15-87)
  stats_*       get_rows_statistics        (:95-127)
  ell_*         ell_matrix_class (max)     (:139-174); arrays only up to
                SLOT_LIMIT padded slots, the width always
  coo_*         coo_matrix_class           (:211-240)
  hyb_*         hybrid_matrix_class 0.2    (:288-310)
  scoo_* / scoo_small_*   scoo_matrix_class with (148 SMs, 48 KiB) / (4, 1 KiB)
  rowblocks     fill_row_blocks, 64        (csr_adaptive_spmv.cu:180-240)
  y1_*, y1ro_*  cpu_csr_spmv_single_thread_naive(_with_reduce_order), x = 1
  yx_*, yxro_*  the same loops on values pre-multiplied by a seeded x
                (A * diag(x) with x = 1 is A * x, rounded per product in T)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import load_ref  # noqa: E402

OUT = Path(__file__).resolve().parent
SLOT_LIMIT = 100_000  # padded ELL arrays above this many slots keep only their width


class Coo:
    def __init__(self, rows, cols, r, c, v):
        self.rows, self.cols = rows, cols
        self.row_ids = np.ascontiguousarray(r, np.uint32)
        self.col_ids = np.ascontiguousarray(c, np.uint32)
        self.data = np.ascontiguousarray(v, np.float64)
        self.nnz = self.data.size


def shuffled(rows, cols, r, c, v, rng):
    p = rng.permutation(len(v))
    return Coo(rows, cols, np.asarray(r)[p], np.asarray(c)[p], np.asarray(v)[p])


def from_lengths(rows, cols, lengths, rng):
    r, c = [], []
    for i, n in enumerate(lengths):
        cc = rng.choice(cols, size=int(n), replace=False)
        r += [i] * int(n)
        c += list(cc)
    v = rng.uniform(-1, 1, size=len(r))
    return shuffled(rows, cols, r, c, v, rng)


def cases():
    rng = np.random.default_rng(20191115)
    out = {}
    n = 16
    r, c, v = [], [], []
    for i in range(n):
        for j in range(n):
            row = i * n + j
            for (di, dj, val) in ((-1, 0, -1.0), (0, -1, -1.0), (0, 0, 4.0), (0, 1, -1.0), (1, 0, -1.0)):
                ii, jj = i + di, j + dj
                if 0 <= ii < n and 0 <= jj < n:
                    r.append(row)
                    c.append(ii * n + jj)
                    v.append(val)
    out["laplacian_16"] = shuffled(n * n, n * n, r, c, v, rng)
    out["random_rect"] = from_lengths(300, 257, rng.integers(0, 13, size=300), rng)
    k = np.arange(1, 2001)
    p = k ** -2.0
    p /= p.sum()
    out["powerlaw_small"] = from_lengths(3000, 6000, rng.choice(k, size=3000, p=p), rng)
    out["edge_1x1"] = Coo(1, 1, [0], [0], [2.5])
    lens = np.zeros(50, np.int64)
    lens[[3, 17, 49]] = [4, 1, 9]
    out["edge_empty_rows"] = from_lengths(50, 64, lens, rng)
    lens = rng.integers(1, 6, size=40)
    lens[7] = 5000
    out["edge_long_row"] = from_lengths(40, 6000, lens, rng)
    # repeated (row, col) entries inside short rows
    rr = [0, 0, 0, 1, 1, 2, 2, 2, 2]
    cc = [5, 1, 5, 3, 3, 0, 7, 0, 7]
    vv = rng.uniform(-1, 1, size=len(rr))
    out["dups_short"] = Coo(3, 8, rr, cc, vv)
    return out


def main() -> None:
    ref = load_ref()
    if ref is None:
        raise SystemExit("oracle/_ref/libmfp_ref.so missing: run `make -C oracle ref` first")
    xrng = np.random.default_rng(7)
    for name, m in cases().items():
        arrays = {"rows": np.array([m.rows], np.uint32), "cols": np.array([m.cols], np.uint32),
                  "row_ids": m.row_ids, "col_ids": m.col_ids, "values": m.data,
                  "x": xrng.uniform(-1, 1, size=m.cols)}
        mn, mx, avg, sd = ref.rows_statistics(m)
        arrays["stats_u32"] = np.array([mn, mx, avg], np.uint32)
        arrays["stats_std"] = np.array([sd], np.float64)
        for dt, s in ((np.float32, "f32"), (np.float64, "f64")):
            rp, ci, d = ref.csr(m, dt)
            arrays[f"csr_row_ptr_{s}"], arrays[f"csr_columns_{s}"], arrays[f"csr_data_{s}"] = rp, ci, d
            w, ed, ec = ref.ell(m, dt)
            arrays[f"ell_width_{s}"] = np.array([w], np.uint32)
            if ed.size <= SLOT_LIMIT:
                arrays[f"ell_data_{s}"], arrays[f"ell_columns_{s}"] = ed, ec
            arrays[f"coo_data_{s}"], arrays[f"coo_cols_{s}"], arrays[f"coo_rows_{s}"] = ref.coo(m, dt)
            hw, hed, hec, hcd, hcc, hcr = ref.hybrid(m, dt, 0.2)
            arrays[f"hyb_width_{s}"] = np.array([hw], np.uint32)
            for k, a in zip(("ell_data", "ell_columns", "coo_data", "coo_cols", "coo_rows"), (hed, hec, hcd, hcc, hcr)):
                if not (k.startswith("ell") and a.size > SLOT_LIMIT):
                    arrays[f"hyb_{k}_{s}"] = a
            for tag, sm, smem in (("scoo", 148, 49152), ("scoo_small", 4, 1024)):
                prm, v, cx, rx, sp = ref.scoo(m, dt, sm, smem)
                arrays[f"{tag}_params_{s}"] = np.array(prm, np.uint32)
                arrays[f"{tag}_values_{s}"], arrays[f"{tag}_c_index_{s}"] = v, cx
                arrays[f"{tag}_r_index_{s}"], arrays[f"{tag}_slices_ptr_{s}"] = rx, sp
            arrays[f"y1_{s}"] = ref.spmv_ones(m, dt)
            arrays[f"y1ro_{s}"] = ref.spmv_ones(m, dt, reduce_order=True)
            # seeded x: pre-multiply the CSR values by x[col] in T, feed the reference with x = 1
            xt = arrays["x"].astype(dt)
            rows_of = np.repeat(np.arange(m.rows), np.diff(rp.astype(np.int64)))
            pre = (d * xt[ci]).astype(dt).astype(np.float64)
            mx_ = Coo(m.rows, m.cols, rows_of, ci, pre)
            arrays[f"yx_{s}"] = ref.spmv_ones(mx_, dt)
            arrays[f"yxro_{s}"] = ref.spmv_ones(mx_, dt, reduce_order=True)
            if s == "f32":
                arrays["rowblocks"] = ref.fill_row_blocks(m.rows, rp)
        np.savez_compressed(OUT / f"{name}.npz", **arrays)
        print(f"{name}: rows={m.rows} cols={m.cols} nnz={m.nnz}")


if __name__ == "__main__":
    main()
