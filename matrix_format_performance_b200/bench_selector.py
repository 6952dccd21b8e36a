"""Learned format selector: data, training and regret (the selector configuration).

    python -m matrix_format_performance_b200.bench_selector [--train 2000] [--test 200] [--big 40]
        [--cap 4194304] [--big-cap 67108864] [--out DIR]
        [--dataset FILE]   (reuse a measured data set instead of sweeping)

1. Data: seeded matrices (selector.family_matrix: rows log-uniform in
   [1e4, 1e7], mean row length log-uniform in [2, 256], families uniform /
   Zipf alpha in [1.5, 3] / banded / block-diagonal / stencil / few dense
   rows up to 1e5 nonzeros; rows reduced to keep nonzeros under --cap).
   Each gets its 12 features and the exhaustive sweep (every admissible
   format x launch configuration, layouts converted on the GPU:
   mfp_matrix_time median of 5 launches, L2 flushed before each).  Training
   seeds 0..train-1, held-out seeds 1,000,000 + i, and a second held-out set
   at the configuration's full sizes (seeds 2,000,000 + i, nonzeros up to
   --big-cap) on which the selector is evaluated as is and with its sweep
   fallback for features outside the training range.
2. Training: an ensemble of MLPs 12-64-64-28 (--members, seeds 0, 1, ...)
   on the engine's CUDA kernels (Adam, masked MSE on log(time / best)); the
   selector averages the members' outputs.
3. Regret on the held-out matrices: time of the selected configuration /
   best time.  Reported beside it:
   - the method without the network: the single configuration that is best
     on average over the training matrices, and CSR scalar with its defaults;
   - the cost of the sweep the selector replaces.
Writes DIR/selector_dataset.npz and DIR/selector_weights.npz; prints one JSON
line.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import sys
import time
from pathlib import Path

import numpy as np


def measure_set(seeds, out_path: Path, tag: str, reps: int = 5, nnz_cap: int = 1 << 22):
    from . import selector as S
    from .device import device_info
    sm = device_info(0).sm_count
    F, T, fam, sweep_s = [], [], [], []
    pool = cf.ThreadPoolExecutor(max_workers=4)

    def prep(seed):
        m, f = S.family_matrix(seed, nnz_cap=nnz_cap)
        return m, f, S.features(m)
    futs = [pool.submit(prep, s) for s in seeds[:4]]
    t0 = time.time()
    for i, seed in enumerate(seeds):
        m, f, feat = futs[i].result()
        if i + 4 < len(seeds):
            futs.append(pool.submit(prep, seeds[i + 4]))
        futs[i] = None
        ts = time.time()
        times = S.sweep(m, reps=reps, sm_count=sm)
        sweep_s.append(time.time() - ts)
        F.append(feat)
        T.append(times)
        fam.append(f)
        if (i + 1) % 100 == 0 or i + 1 == len(seeds):
            np.savez(out_path, F=np.array(F, np.float32), T=np.array(T), fam=np.array(fam), seeds=np.array(seeds[:i + 1]),
                     sweep_s=np.array(sweep_s))
            print(f"[bench_selector] {tag}: {i + 1}/{len(seeds)} matrices in {time.time() - t0:.0f}s",
                  file=sys.stderr, flush=True)
    pool.shutdown()
    return np.array(F, np.float32), np.array(T), np.array(fam), np.array(sweep_s)


def verified_regret(sel, F, T, k: int) -> np.ndarray:
    """Regret of select(..., verify=k): the fastest of the k best predictions
    by the sweep's own times (the times select() measures, up to noise)."""
    from . import selector as S
    ok = np.isfinite(T)
    cand = sel.candidates(F, ok, k)
    tk = np.take_along_axis(np.where(ok, T, np.inf), cand, axis=1)
    return S.regret(T, cand[np.arange(len(T)), tk.argmin(axis=1)])


def full_size(sel, F, T, fam, sweep_s, fixed: int):
    """The selector on the full-size held-out matrices: as is, and with the
    sweep deciding for matrices outside the training range."""
    from . import selector as S
    if F is None or len(F) == 0:
        return None
    ok = np.isfinite(T)
    chosen = sel.choose(F, ok)
    r = S.regret(T, chosen)
    r3 = verified_regret(sel, F, T, 3)
    in_range = np.array([sel.in_range(f) for f in F])
    r_fb = np.where(in_range, r, 1.0)
    r3_fb = np.where(in_range, r3, 1.0)
    r_fixed = S.regret(T, np.where(ok[:, fixed], fixed, 0))
    return {"matrices": int(len(F)), "within_5pct": float(np.mean(r <= 1.05)),
            "mean_regret": float(np.mean(r)), "max_regret": float(np.max(r)),
            "with_sweep_fallback_within_5pct": float(np.mean(r_fb <= 1.05)),
            "verified_top3_within_5pct": float(np.mean(r3 <= 1.05)),
            "verified_top3_with_sweep_fallback_within_5pct": float(np.mean(r3_fb <= 1.05)),
            "fallback_matrices": int((~in_range).sum()),
            "best_fixed_within_5pct": float(np.mean(r_fixed <= 1.05)),
            "sweep_seconds_mean": float(np.mean(sweep_s)),
            "families": {f: float(np.mean(r[fam == f] <= 1.05)) for f in sorted(set(fam.tolist()))}}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--test", type=int, default=200)
    ap.add_argument("--big", type=int, default=40)
    ap.add_argument("--cap", type=int, default=1 << 22)
    ap.add_argument("--big-cap", type=int, default=1 << 26)
    ap.add_argument("--out", default="selector_out")
    ap.add_argument("--dataset", default=None)
    ap.add_argument("--epochs", type=int, default=400)
    ap.add_argument("--members", type=int, default=10)
    a = ap.parse_args()
    import torch

    from . import selector as S
    torch.cuda.set_device(0)
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    if a.dataset:
        z = np.load(a.dataset)
        Ftr, Ttr, fam_tr = z["F_train"], z["T_train"], z["fam_train"]
        Fte, Tte, fam_te = z["F_test"], z["T_test"], z["fam_test"]
        sweep_te = z["sweep_s_test"]
        Fbg, Tbg, fam_bg = (z["F_big"], z["T_big"], z["fam_big"]) if "F_big" in z.files else (None, None, None)
        sweep_bg = z["sweep_s_big"] if "F_big" in z.files else None
    else:
        Ftr, Ttr, fam_tr, _ = measure_set(list(range(a.train)), out / "_train_partial.npz", "train", nnz_cap=a.cap)
        Fte, Tte, fam_te, sweep_te = measure_set([1_000_000 + i for i in range(a.test)], out / "_test_partial.npz",
                                                 "held-out", nnz_cap=a.cap)
        Fbg, Tbg, fam_bg, sweep_bg = measure_set([2_000_000 + i for i in range(a.big)], out / "_big_partial.npz",
                                                 "held-out full size", nnz_cap=a.big_cap)
        np.savez_compressed(out / "selector_dataset.npz", F_train=Ftr, T_train=Ttr.astype(np.float32),
                            fam_train=fam_tr, F_test=Fte, T_test=Tte.astype(np.float32), fam_test=fam_te,
                            sweep_s_test=sweep_te, F_big=Fbg, T_big=Tbg.astype(np.float32), fam_big=fam_bg,
                            sweep_s_big=sweep_bg, nnz_cap=np.array([a.cap, a.big_cap]),
                            slots=np.array([S.config_label(i) for i in range(S.N_OUT)]))
    t0 = time.time()
    sel = S.train(Ftr, Ttr, epochs=a.epochs, members=a.members)
    train_s = time.time() - t0
    sel.save(out / "selector_weights.npz")

    ok_te = np.isfinite(Tte)
    t0 = time.time()
    chosen = sel.choose(Fte, ok_te)
    infer_s = time.time() - t0
    r = S.regret(Tte, chosen)
    in_range = np.array([sel.in_range(f) for f in Fte])
    r_fallback = np.where(in_range, r, 1.0)  # outside the training range the sweep decides
    # the method without the network
    tr_reg = np.where(np.isfinite(Ttr), Ttr / np.nanmin(np.where(np.isfinite(Ttr), Ttr, np.nan), axis=1,
                                                        keepdims=True), np.inf)
    fixed = int(np.argmin([np.mean(np.minimum(tr_reg[:, j], 10.0)) for j in range(S.N_OUT)]))
    r_fixed = S.regret(Tte, np.where(ok_te[:, fixed], fixed, 0))
    r_csr = S.regret(Tte, np.zeros(len(Tte), int))

    def summary(x):
        return {"within_5pct": float(np.mean(x <= 1.05)), "mean_regret": float(np.mean(x)),
                "p90_regret": float(np.quantile(x, 0.9)), "max_regret": float(np.max(x))}
    per_family = {f: summary(r[fam_te == f]) for f in sorted(set(fam_te.tolist()))}
    best_slots = np.bincount(np.argmin(np.where(ok_te, Tte, np.inf), axis=1), minlength=S.N_OUT)
    res = {"config": "learned_selector", "train_matrices": int(len(Ftr)), "held_out_matrices": int(len(Fte)),
           "network": f"ensemble of {a.members} MLPs 12-64-64-28 FP32 (outputs averaged), trained with "
                      "mfp_mlp_forward/backward/adam",
           "epochs": a.epochs, "train_seconds": train_s, "final_train_loss": float(sel.history[-1]),
           "selector": summary(r), "selector_with_sweep_fallback": {**summary(r_fallback),
                                                                   "fallback_matrices": int((~in_range).sum())},
           "selector_verified_top3": {**summary(verified_regret(sel, Fte, Tte, 3)),
                                      "how": "the 3 best predictions timed on the matrix, the fastest taken"},
           "without_network_best_fixed": {"slot": S.config_label(fixed), **summary(r_fixed)},
           "without_network_csr_default": summary(r_csr),
           "per_family": per_family,
           "best_slot_histogram_held_out": {S.config_label(i): int(c) for i, c in enumerate(best_slots) if c},
           "selection_cost_seconds": {"sweep_mean": float(np.mean(sweep_te)), "selector_batch_total": infer_s},
           "full_size_held_out": full_size(sel, Fbg, Tbg, fam_bg, sweep_bg, fixed),
           "target": "selected time within 5% of the exhaustive best on >= 90% of held-out matrices"}
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
