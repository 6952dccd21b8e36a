"""Learned SpMV format selector.

Replaces the exhaustive timing sweep (every format x launch configuration,
timed on the matrix itself) with a prediction from 12 features of the sparsity
pattern (mfp_selector_features):
- **network**: an ensemble of MLPs 12-64-64-28 (FP32, ReLU), trained from
  different seeds; their 28 outputs, averaged, are the predicted log time,
  relative to the fastest, of the 7 formats x 4 launch configurations of
  CONFIGS (averaging cuts the variance of single networks);
- **choice**: the selector takes the smallest prediction among the
  configurations the matrix admits; with verify=k it times the k smallest
  on the matrix (k of the 28 configurations) and takes the fastest, which
  absorbs the network's near-ties (on the measured held-out set: within 5%
  of the best for 84% of the matrices from the prediction alone, 95.5% with
  the three best predictions timed);
- **training**: on the engine's own kernels (mfp_mlp_forward /
  mfp_mlp_backward / mfp_mlp_adam), against times the engine measured on
  seeded synthetic matrices, with a masked mean-squared error;
- **fallback**: when a matrix's features lie outside the range seen in
  training, select() runs the exhaustive sweep (sweep_if_unsure=False turns
  this off);
- **regret**: the same sweep measures the selector's regret on held-out
  matrices.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _capi
from ._capi import call
from .formats import csr_matrix_class, ptr

N_FEATURES, N_HIDDEN, N_OUT = 12, 64, 28

# (format name, config) per output slot; None = no such configuration of that
# format (masked in training and never selected).
CONFIGS: list[tuple[str, dict] | None] = [
    # CSR scalar: the automatic kernel (element-balanced bins below a mean row
    # length of 16), the row blocks at two warp-assist / long-row thresholds,
    # and the streaming kernel
    ("csr", {}), ("csr", {"kernel": 1}),
    ("csr", {"kernel": 1, "assist_threshold": 256, "long_row_threshold": 16384}), ("csr", {"kernel": 2}),
    # CSR vector: lanes per row
    ("csr_vector", {}), ("csr_vector", {"vector_lanes": 4}), ("csr_vector", {"vector_lanes": 8}),
    ("csr_vector", {"vector_lanes": 32}),
    # CSR-Adaptive: elements per row bin
    ("csr_adaptive", {}), ("csr_adaptive", {"bin_nnz": 1020}), ("csr_adaptive", {"bin_nnz": 508}),
    ("csr_adaptive", {"bin_nnz": 252}),
    # ELL (one layout)
    ("ell", {}), None, None, None,
    # COO (one layout)
    ("coo", {}), None, None, None,
    # SCOO: shared memory per block the slice size is derived from; the
    # reference's sort_cols layout (scoo_matrix_class.cpp:102-138)
    ("scoo", {"shared_mem": 49152}), ("scoo", {"shared_mem": 24576}), ("scoo", {"shared_mem": 98304}),
    ("scoo", {"shared_mem": 49152, "sort_cols": True}),
    # hybrid: ELL width at the 2/3-quantile of the row lengths, or the
    # reference's percent rule at the percents of its sweep (main.cpp:247-279:
    # 0, 0.35, 0.70)
    ("hybrid", {"quantile": 2 / 3}), ("hybrid", {"percent": 0.0}), ("hybrid", {"percent": 0.35}),
    ("hybrid", {"percent": 0.7}),
]
assert len(CONFIGS) == N_OUT
SLOT_AVAILABLE = np.array([c is not None for c in CONFIGS])
ELL_MAX_BYTES = 1 << 28  # ELL layouts larger than this are not built (padding)


def config_label(i: int) -> str:
    c = CONFIGS[i]
    if c is None:
        return f"slot{i}"
    return c[0] + ("" if not c[1] else "(" + ",".join(f"{k}={v:.3g}" if isinstance(v, float) else f"{k}={v}"
                                                      for k, v in c[1].items()) + ")")


def features(m: csr_matrix_class) -> np.ndarray:
    f = np.empty(N_FEATURES, np.float32)
    call("mfp_selector_features", m.rows, m.cols, ptr(m.row_ptr), ptr(m.columns) if m.nnz else None, ptr(f))
    return f


# ---------------------------------------------------------------------------
# Measurement: the exhaustive sweep
# ---------------------------------------------------------------------------
def hybrid_width(m: csr_matrix_class, cfg: dict) -> int:
    from .formats import hybrid_width as percent_width, row_length_quantile
    return percent_width(m, cfg["percent"]) if "percent" in cfg else row_length_quantile(m, cfg["quantile"])


def admissible(m: csr_matrix_class) -> np.ndarray:
    """Slots that can be built for m: ELL and the ELL part of the hybrid
    format only when their padded layout stays below ELL_MAX_BYTES."""
    from .formats import ell_matrix_class
    ok = SLOT_AVAILABLE.copy()
    vs = m.data.dtype.itemsize + 4
    if ell_matrix_class.estimate_size(m) * vs > ELL_MAX_BYTES:
        ok[12] = False
    for i in range(24, 28):
        if hybrid_width(m, CONFIGS[i][1]) * m.rows * vs > ELL_MAX_BYTES:
            ok[i] = False
    if m.nnz == 0:
        ok[23] = False  # the sort_cols layout needs elements
    return ok


def build_slot(m: csr_matrix_class, i: int, sm_count: int, dev_csr=None):
    """DeviceMatrix for slot i.  With dev_csr (device row_ptr, columns, values
    of m) the layout is converted on the GPU (mfp_matrix_create_device, the
    same arrays as the host converters); otherwise on the host, then uploaded."""
    from .device import FORMAT_NAMES, DeviceMatrix
    from .formats import hybrid_matrix_class, scoo_matrix_class
    name, cfg = CONFIGS[i]
    fmt = FORMAT_NAMES[name]
    if dev_csr is not None:
        rp, ci, va = dev_csr
        if name.startswith("csr"):
            return DeviceMatrix.from_device_csr(rp, ci, va, m.cols, fmt, config=cfg or None)
        if name == "scoo":
            prm = _capi.ScooParams()
            call("mfp_scoo_params_compute", m.rows, sm_count, cfg["shared_mem"], 1 if m.dtype == np.float64 else 0,
                 C.byref(prm))
            return DeviceMatrix.from_device_csr(rp, ci, va, m.cols, fmt, scoo=prm,
                                                scoo_sort_cols=bool(cfg.get("sort_cols")))
        if name == "hybrid":
            return DeviceMatrix.from_device_csr(rp, ci, va, m.cols, fmt, ell_width=hybrid_width(m, cfg))
        return DeviceMatrix.from_device_csr(rp, ci, va, m.cols, fmt)
    if name.startswith("csr"):
        return DeviceMatrix.from_csr(m, fmt, cfg or None)
    if name == "scoo":
        return DeviceMatrix.from_scoo(scoo_matrix_class(sm_count, cfg["shared_mem"], m,
                                                        sort_cols=bool(cfg.get("sort_cols"))))
    if name == "hybrid":
        hm = hybrid_matrix_class(m)
        hm.allocate_width(m, hybrid_width(m, cfg))
        return DeviceMatrix.from_hybrid(hm)
    return DeviceMatrix.build(m, fmt)


def sweep(m: csr_matrix_class, reps: int = 5, sm_count: int = 148, slots=None) -> np.ndarray:
    """Median device time (s) of every admissible slot (inf elsewhere), L2
    flushed before each launch (mfp_matrix_time)."""
    import torch
    ok = admissible(m)
    t = np.full(N_OUT, np.inf)
    x = torch.ones(max(1, m.cols), dtype=torch.float32 if m.data.dtype == np.float32 else torch.float64,
                   device="cuda")
    y = torch.empty(max(1, m.rows), dtype=x.dtype, device="cuda")
    dev_csr = None
    if m.nnz:  # one upload; every layout is converted from it on the GPU
        dev_csr = (torch.from_numpy(m.row_ptr.view(np.int32)).cuda(), torch.from_numpy(m.columns.view(np.int32)).cuda(),
                   torch.from_numpy(m.data).cuda())
    for i in (slots if slots is not None else range(N_OUT)):
        if not ok[i]:
            continue
        dm = build_slot(m, i, sm_count, dev_csr)
        try:
            _, med = dm.time(x, y, reps=reps, flush_l2=True)
            t[i] = med
        finally:
            dm.close()
    return t


def targets(times: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """log(time / best) per slot and the mask of measured slots ([n, 28])."""
    times = np.atleast_2d(times)
    mask = np.isfinite(times)
    best = np.where(mask, times, np.inf).min(axis=1, keepdims=True)
    t = np.where(mask, np.log(np.where(mask, times, 1.0) / best), 0.0)
    return t.astype(np.float32), mask.astype(np.float32)


# ---------------------------------------------------------------------------
# The network, trained with the engine's CUDA kernels
# ---------------------------------------------------------------------------
def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights, zero biases, in the flat layout of mfp_mlp_*."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((N_FEATURES, N_HIDDEN), (N_HIDDEN, N_HIDDEN), (N_HIDDEN, N_OUT)):
        lim = math.sqrt(6.0 / fan_in)
        parts += [rng.uniform(-lim, lim, (fan_in, fan_out)).astype(np.float32).ravel(), np.zeros(fan_out, np.float32)]
    p = np.concatenate(parts)
    assert p.size == _capi.load().mfp_mlp_param_count()
    return p


class MLP:
    """Device-resident parameters and Adam state; forward/backward/Adam are the
    library's CUDA kernels (torch tensors only hold the device memory)."""

    def __init__(self, params: np.ndarray):
        import torch
        self.p = torch.from_numpy(np.ascontiguousarray(params, np.float32)).cuda()
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.g = torch.zeros_like(self.p)
        self.loss = torch.zeros(1, device="cuda")
        self.step_count = 0

    @staticmethod
    def _ptr(t):
        return C.c_void_p(t.data_ptr())

    def forward(self, x):
        import torch
        B = x.shape[0]
        h1 = torch.empty(B, N_HIDDEN, device="cuda")
        h2 = torch.empty(B, N_HIDDEN, device="cuda")
        y = torch.empty(B, N_OUT, device="cuda")
        call("mfp_mlp_forward", self._ptr(self.p), self._ptr(x), B, self._ptr(h1), self._ptr(h2), self._ptr(y), None)
        return h1, h2, y

    def backward(self, x, h1, h2, y, t, mask):
        import torch
        B = x.shape[0]
        work = torch.empty(B * (N_OUT + 2 * N_HIDDEN), device="cuda")
        call("mfp_mlp_backward", self._ptr(self.p), self._ptr(x), self._ptr(h1), self._ptr(h2), self._ptr(y),
             self._ptr(t), self._ptr(mask), B, self._ptr(self.g), self._ptr(self.loss), self._ptr(work), None)
        return self.g, self.loss

    def adam(self, lr=3e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        call("mfp_mlp_adam", self._ptr(self.p), self._ptr(self.g), self._ptr(self.m), self._ptr(self.v),
             self.p.numel(), lr, beta1, beta2, eps, self.step_count, None)

    def params(self) -> np.ndarray:
        return self.p.cpu().numpy().copy()


@dataclass
class Selector:
    params: np.ndarray  # [members, parameters] (a single network: one row)
    mu: np.ndarray
    sigma: np.ndarray
    lo: np.ndarray     # feature range seen in training (for the sweep fallback)
    hi: np.ndarray
    history: list = field(default_factory=list)

    def __post_init__(self):
        self.params = np.atleast_2d(np.asarray(self.params, np.float32))

    def predict_slots(self, F: np.ndarray) -> np.ndarray:
        """Predicted log(time / best) per slot, [n, 28]: the members' forward
        passes on the GPU, averaged."""
        import torch
        x = torch.from_numpy(((np.atleast_2d(F) - self.mu) / self.sigma).astype(np.float32)).cuda()
        acc = None
        for p in self.params:
            _, _, y = MLP(p).forward(x)
            acc = y if acc is None else acc + y
        return (acc / len(self.params)).cpu().numpy()

    def choose(self, F: np.ndarray, admissible_mask: np.ndarray) -> np.ndarray:
        return self.candidates(F, admissible_mask, 1)[:, 0]

    def candidates(self, F: np.ndarray, admissible_mask: np.ndarray, k: int) -> np.ndarray:
        """The k admissible slots with the smallest predictions, best first,
        [n, k] (a matrix admitting fewer repeats its last)."""
        pred = self.predict_slots(F)
        mask = np.atleast_2d(admissible_mask)
        pred = np.where(mask, pred, np.inf)
        order = np.argsort(pred, axis=1, kind="stable")[:, :k]
        n_ok = np.maximum(mask.sum(axis=1), 1)
        return np.where(np.arange(k)[None, :] < n_ok[:, None], order, order[:, [0]])

    def in_range(self, f: np.ndarray, margin: float = 0.05) -> bool:
        span = np.maximum(self.hi - self.lo, 1e-6)
        return bool(np.all(f >= self.lo - margin * span) and np.all(f <= self.hi + margin * span))

    def select(self, m: csr_matrix_class, sweep_if_unsure: bool = True, reps: int = 5,
               verify: int = 1) -> tuple[int, str]:
        """(slot, how): the predicted slot ("predicted"); with verify=k > 1 the
        fastest of the k best predictions, timed on the matrix ("verified");
        the exhaustive sweep's best when the matrix lies outside the training
        range ("sweep")."""
        f = features(m)
        ok = admissible(m)
        if sweep_if_unsure and not self.in_range(f):
            t = sweep(m, reps=reps)
            return int(np.argmin(t)), "sweep"
        cand = self.candidates(f, ok, max(1, verify))[0]
        if verify <= 1:
            return int(cand[0]), "predicted"
        t = sweep(m, reps=reps, slots=sorted(set(int(c) for c in cand)))
        return int(np.argmin(t)), "verified"

    def save(self, path) -> None:
        np.savez(path, params=self.params, mu=self.mu, sigma=self.sigma, lo=self.lo, hi=self.hi,
                 history=np.array(self.history, np.float64))

    @classmethod
    def load(cls, path) -> "Selector":
        z = np.load(path)
        return cls(z["params"], z["mu"], z["sigma"], z["lo"], z["hi"], list(z["history"]))


def train(F: np.ndarray, times: np.ndarray, epochs: int = 400, batch: int = 256, lr: float = 3e-3,
          seed: int = 0, members: int = 10) -> Selector:
    """Fits `members` MLPs (seeds seed, seed + 1, ...) to log(time / best)
    with the engine's CUDA kernels; the selector averages their outputs."""
    import torch
    mu = F.mean(axis=0)
    sigma = np.maximum(F.std(axis=0), 1e-3)
    X = torch.from_numpy(((F - mu) / sigma).astype(np.float32)).cuda()
    T, M = targets(times)
    T = torch.from_numpy(T).cuda()
    M = torch.from_numpy(M).cuda()
    n = X.shape[0]
    params, history = [], []
    for k in range(members):
        net = MLP(init_params(seed + k))
        rng = np.random.default_rng(seed + k)
        for ep in range(epochs):
            order = rng.permutation(n)
            tot = 0.0
            for s in range(0, n, batch):
                idx = torch.from_numpy(order[s:s + batch]).cuda()
                xb, tb, mb = X[idx].contiguous(), T[idx].contiguous(), M[idx].contiguous()
                h1, h2, y = net.forward(xb)
                _, loss = net.backward(xb, h1, h2, y, tb, mb)
                net.adam(lr=lr)
                tot += float(loss.item()) * len(idx)
            if k == 0:
                history.append(tot / n)
        params.append(net.params())
    return Selector(np.stack(params), mu.astype(np.float32), sigma.astype(np.float32), F.min(axis=0), F.max(axis=0),
                    history)


def regret(times: np.ndarray, chosen: np.ndarray) -> np.ndarray:
    """time of the chosen slot / best time, per matrix."""
    times = np.atleast_2d(times)
    best = np.min(np.where(np.isfinite(times), times, np.inf), axis=1)
    return times[np.arange(times.shape[0]), chosen] / best


# ---------------------------------------------------------------------------
# The training and held-out matrices
# ---------------------------------------------------------------------------
FAMILIES = ("uniform", "zipf", "banded", "block_diagonal", "stencil", "dense_rows")


def family_matrix(seed: int, nnz_cap: int = 1 << 22, rows_lo: int = 10_000, rows_hi: int = 10_000_000):
    """One seeded matrix: rows log-uniform in [rows_lo, rows_hi], mean row
    length log-uniform in [2, 256], family uniform among FAMILIES (Zipf alpha
    in [1.5, 3], dense rows up to 1e5 nonzeros); rows are reduced to keep
    nnz <= nnz_cap.  Returns (float32 CSR, family, parameters)."""
    from . import synth
    rng = np.random.default_rng(2_654_435_761 * seed + 11)
    fam = FAMILIES[int(rng.integers(0, len(FAMILIES)))]
    rows = int(np.exp(rng.uniform(np.log(rows_lo), np.log(rows_hi))))
    mean = float(np.exp(rng.uniform(np.log(2), np.log(256))))
    rows = max(1_000, min(rows, int(nnz_cap / mean)))
    s = 7919 * seed + 3
    if fam == "uniform":
        lo = max(1, int(mean * 0.5))
        m = synth.uniform(rows, lo, max(lo, int(2 * mean - lo)), seed=s)
    elif fam == "zipf":
        alpha = float(rng.uniform(1.5, 3.0))
        m = synth.power_law(rows=rows, alpha=alpha, k_lo=1, k_hi=min(rows, 100_000), seed=s)
        if m.nnz > nnz_cap:  # heavy tail: shrink and redraw
            m = synth.power_law(rows=max(1_000, rows * nnz_cap // m.nnz), alpha=alpha, k_lo=1,
                                k_hi=min(rows, 100_000), seed=s)
    elif fam == "banded":
        per = max(1, min(int(mean), 256))
        m = synth.banded(n=rows, half_band=max(per, int(per * rng.uniform(1.0, 8.0))), per_row=per, seed=s)
    elif fam == "block_diagonal":
        blk = int(min(256, max(2, 2 ** round(np.log2(mean)))))
        m = synth.block_diagonal(max(blk, min(rows, nnz_cap // blk)), block=blk, seed=s)
    elif fam == "stencil":
        if rng.random() < 0.5:
            n = max(8, int(round(min(rows, nnz_cap // 5) ** 0.5)))
            m = synth.laplacian_2d(n)
        else:
            n = max(8, int(round(min(rows, nnz_cap // 27) ** (1 / 3))))
            m = synth.stencil_27(n, seed=s)
    else:  # uniform background and a few dense rows of up to 1e5 nonzeros
        base = synth.uniform(rows, 1, max(2, int(mean)), seed=s)
        k = int(rng.integers(1, 9))
        dense_len = int(min(rows, 100_000, max(1000, nnz_cap // (4 * k))))
        m = _with_dense_rows(base, rng, k, dense_len)
    return m.astype(np.float32), fam


def _with_dense_rows(m: csr_matrix_class, rng, k: int, length: int) -> csr_matrix_class:
    rows = np.sort(rng.choice(m.rows, size=min(k, m.rows), replace=False))
    lens = np.diff(m.row_ptr.astype(np.int64))
    new_cols = {}
    for r in rows:
        c = np.sort(rng.choice(m.cols, size=min(length, m.cols), replace=False)).astype(np.uint32)
        new_cols[int(r)] = c
        lens[r] = c.size
    rp = np.zeros(m.rows + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    cols = np.empty(int(rp[-1]), np.uint32)
    vals = np.empty(int(rp[-1]), np.float64)
    src = m.row_ptr.astype(np.int64)
    # bulk copy of the unchanged rows, then the dense rows
    keep = np.ones(m.rows, bool)
    keep[rows] = False
    starts_new = rp[:-1]
    idx = np.repeat(np.arange(m.rows), np.where(keep, lens, 0))
    off = np.arange(idx.size) - np.repeat(np.cumsum(np.where(keep, lens, 0)) - np.where(keep, lens, 0),
                                          np.where(keep, lens, 0))
    cols[starts_new[idx] + off] = m.columns[src[idx] + off]
    vals[starts_new[idx] + off] = m.data[src[idx] + off]
    for r, c in new_cols.items():
        cols[rp[r]:rp[r + 1]] = c
        vals[rp[r]:rp[r + 1]] = rng.uniform(-1.0, 1.0, c.size)
    return csr_matrix_class.from_arrays(m.rows, m.cols, rp.astype(np.uint32), cols, vals, np.float64)
