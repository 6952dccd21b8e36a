"""Format selector: features, the MLP's CUDA forward/backward/Adam kernels
against a NumPy CPU reference (itself checked by finite differences), and
training on a toy problem.

The NumPy functions below are the CPU oracle of the network: plain
restatements of a 12-64-64-28 ReLU MLP and its masked mean-squared error.
"""
import numpy as np
import pytest

from matrix_format_performance_b200 import selector as S
from matrix_format_performance_b200 import synth

L = [(12, 64), (64, 64), (64, 28)]


def unpack(p):
    out, o = [], 0
    for k, n in L:
        W = p[o:o + k * n].reshape(k, n)
        o += k * n
        b = p[o:o + n]
        o += n
        out.append((W, b))
    return out


def ref_forward(p, x):
    (W1, b1), (W2, b2), (W3, b3) = unpack(p.astype(np.float64))
    h1 = np.maximum(x @ W1 + b1, 0)
    h2 = np.maximum(h1 @ W2 + b2, 0)
    return h1, h2, h2 @ W3 + b3


def ref_loss(p, x, t, m):
    _, _, y = ref_forward(p, x)
    return float((m * (y - t) ** 2).sum() / m.sum())


def ref_grad(p, x, t, m):
    (W1, b1), (W2, b2), (W3, b3) = unpack(p.astype(np.float64))
    h1, h2, y = ref_forward(p, x)
    dy = 2 * m * (y - t) / m.sum()
    dW3, db3 = h2.T @ dy, dy.sum(0)
    dz2 = (dy @ W3.T) * (h2 > 0)
    dW2, db2 = h1.T @ dz2, dz2.sum(0)
    dz1 = (dz2 @ W2.T) * (h1 > 0)
    dW1, db1 = x.T @ dz1, dz1.sum(0)
    return np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])


def _problem(B=37, seed=0):
    rng = np.random.default_rng(seed)
    p = S.init_params(seed)
    p[p.size - 28:] = rng.normal(0, 0.1, 28)  # non-zero biases too
    x = rng.normal(0, 1, (B, 12))
    t = rng.normal(0, 1, (B, 28))
    m = (rng.random((B, 28)) < 0.7).astype(np.float64)
    return p, x, t, m


def test_reference_gradient_matches_finite_differences():
    p, x, t, m = _problem()
    g = ref_grad(p, x, t, m)
    rng = np.random.default_rng(1)
    p64 = p.astype(np.float64)
    for i in rng.choice(p.size, 40, replace=False):
        e = np.zeros_like(p64)
        e[i] = 1e-6
        fd = (ref_loss(p64 + e, x, t, m) - ref_loss(p64 - e, x, t, m)) / 2e-6
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(g[i])), i


def test_features_match_numpy():
    m = synth.power_law(rows=5000, seed=3)
    f = S.features(m)
    lens = np.diff(m.row_ptr.astype(np.int64))
    rows = np.repeat(np.arange(m.rows), lens)
    d = np.abs(m.columns.astype(np.int64) - rows)
    srt = np.sort(lens)
    gini = ((2 * np.arange(1, m.rows + 1) - m.rows - 1) * srt).sum() / (m.rows * lens.sum())
    want = [np.log10(m.rows), np.log10(m.cols), np.log10(m.nnz + 1), np.log2(1 + lens.mean()),
            np.log2(1 + lens.std()), np.log2(1 + lens.max()), gini, d.max() / max(m.rows, m.cols),
            (d <= 64).mean(), (d == 0).sum() / min(m.rows, m.cols), (lens == 0).mean(), lens[lens > 4096].sum() / m.nnz]
    assert np.allclose(f, np.array(want, np.float32), rtol=1e-5, atol=1e-6)


def test_generator_is_seeded_and_capped():
    a, fa = S.family_matrix(7, nnz_cap=1 << 18)
    b, fb = S.family_matrix(7, nnz_cap=1 << 18)
    assert fa == fb and np.array_equal(a.row_ptr, b.row_ptr) and np.array_equal(a.columns, b.columns)
    for s in range(30):
        m, fam = S.family_matrix(s, nnz_cap=1 << 18)
        assert m.nnz <= (1 << 18) * 1.6 + 100_000 and fam in S.FAMILIES
        assert np.all(np.diff(m.row_ptr.astype(np.int64)) >= 0) and m.row_ptr[-1] == m.nnz


def test_targets_and_regret():
    times = np.array([[2.0, 1.0, np.inf, 4.0], [1.0, 1.0, 3.0, np.inf]])
    t, mk = S.targets(times)
    assert np.allclose(t[0], [np.log(2), 0, 0, np.log(4)]) and np.array_equal(mk[0], [1, 1, 0, 1])
    assert np.allclose(S.regret(times, np.array([0, 2])), [2.0, 3.0])


@pytest.mark.gpu
def test_mlp_kernels_match_cpu_reference():
    import torch
    p, x, t, m = _problem(B=301, seed=4)
    net = S.MLP(p)
    xt = torch.from_numpy(x.astype(np.float32)).cuda()
    h1, h2, y = net.forward(xt)
    rh1, rh2, ry = ref_forward(p, x.astype(np.float32).astype(np.float64))
    assert np.allclose(y.cpu().numpy(), ry, rtol=1e-4, atol=1e-4)
    assert np.allclose(h2.cpu().numpy(), rh2, rtol=1e-4, atol=1e-4)
    tt = torch.from_numpy(t.astype(np.float32)).cuda()
    mt = torch.from_numpy(m.astype(np.float32)).cuda()
    g, loss = net.backward(xt, h1, h2, y, tt, mt)
    rg = ref_grad(p, x.astype(np.float32).astype(np.float64), t.astype(np.float32), m)
    assert abs(loss.item() - ref_loss(p, x.astype(np.float32).astype(np.float64), t.astype(np.float32), m)) < 1e-4
    gg = g.cpu().numpy()
    assert np.allclose(gg, rg, rtol=1e-3, atol=1e-5 * np.abs(rg).max())
    # deterministic: a second backward gives the same bits
    g2, _ = net.backward(xt, h1, h2, y, tt, mt)
    assert np.array_equal(gg.view(np.uint32), g2.cpu().numpy().view(np.uint32))
    # Adam on the GPU against the same update in NumPy
    p0 = net.params().astype(np.float64)
    net.adam(lr=1e-2)
    mm = 0.1 * gg
    vv = 0.001 * gg.astype(np.float64) ** 2
    want = p0 - 1e-2 * (mm / 0.1) / (np.sqrt(vv / 0.001) + 1e-8)
    assert np.allclose(net.params(), want, rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_training_fits_a_learnable_rule():
    """A synthetic 'best slot depends on two features' data set: the trained
    selector picks the best slot on held-out points far more often than any
    fixed slot does (at least 80%, and 30 points above the best fixed slot)."""
    rng = np.random.default_rng(0)
    F = rng.normal(0, 1, (1200, 12)).astype(np.float32)
    times = np.full((1200, 28), np.inf)
    for j in (0, 4, 8, 16, 24):
        times[:, j] = 1.0 + 0.3 * rng.random(1200)
    times[F[:, 0] > 0.5, 4] = 0.3
    times[F[:, 1] < -0.5, 16] = 0.2
    times[(F[:, 0] <= 0.5) & (F[:, 1] >= -0.5), 8] = 0.4
    sel = S.train(F[:1000], times[:1000], epochs=300, batch=128, lr=3e-3, members=2)
    assert sel.params.shape[0] == 2  # two members, outputs averaged
    assert sel.history[-1] < 0.25 * sel.history[0]
    ok = np.isfinite(times[1000:])
    chosen = sel.choose(F[1000:], ok)
    r = S.regret(times[1000:], chosen)
    fixed = min(np.mean(S.regret(times[1000:], np.full(200, j)) <= 1.05) for j in (0, 4, 8, 16, 24))
    # points next to the rule's sharp boundaries are the misses
    assert np.mean(r <= 1.05) >= 0.8 and np.mean(r <= 1.05) > fixed + 0.3


DATA = __import__("pathlib").Path(S.__file__).parent / "selector_data"


def _held_out():
    d = np.load(DATA / "selector_dataset.npz")
    w = S.Selector.load(DATA / "selector_weights.npz")
    return d, w


def ensemble_forward(w, F):
    """The committed ensemble with the NumPy network: members' outputs averaged."""
    x = (F - w.mu) / w.sigma
    return np.mean([ref_forward(p, x)[2] for p in w.params], axis=0)


def test_committed_selector_meets_target_on_cpu_reference():
    """The committed weights, evaluated with the NumPy network on the
    committed held-out measurements: timing the three best predictions
    (select(..., verify=3)) gives a configuration within 5% of the exhaustive
    best for >= 90% of the held-out matrices, the prediction alone for
    >= 80%; both far above the best fixed configuration."""
    d, w = _held_out()
    F, T = d["F_test"].astype(np.float64), d["T_test"].astype(np.float64)
    assert len(F) == 200 and len(d["F_train"]) == 2000
    y = np.where(np.isfinite(T), ensemble_forward(w, F), np.inf)
    chosen = y.argmin(axis=1)
    r = S.regret(T, chosen)
    assert np.mean(r <= 1.05) >= 0.8
    top3 = np.argsort(y, axis=1, kind="stable")[:, :3]
    t3 = np.take_along_axis(np.where(np.isfinite(T), T, np.inf), top3, axis=1)
    r3 = S.regret(T, top3[np.arange(len(T)), t3.argmin(axis=1)])
    assert np.mean(r3 <= 1.05) >= 0.9
    Ttr = d["T_train"].astype(np.float64)
    rel = np.where(np.isfinite(Ttr), Ttr / np.nanmin(np.where(np.isfinite(Ttr), Ttr, np.nan), axis=1, keepdims=True),
                   np.inf)
    fixed = int(np.argmin([np.mean(np.minimum(rel[:, j], 10.0)) for j in range(S.N_OUT)]))
    r_fixed = S.regret(T, np.where(np.isfinite(T[:, fixed]), fixed, 0))
    assert np.mean(r <= 1.05) > np.mean(r_fixed <= 1.05) + 0.3


@pytest.mark.gpu
def test_committed_selector_cuda_forward_agrees():
    """The CUDA forward kernels pick the same configurations as the NumPy
    network (up to exact ties) on the held-out features."""
    d, w = _held_out()
    F, T = d["F_test"], d["T_test"].astype(np.float64)
    ok = np.isfinite(T)
    g = w.choose(F, ok)
    y = ensemble_forward(w, F.astype(np.float64))
    c = np.where(ok, y, np.inf).argmin(axis=1)
    assert np.mean(g == c) >= 0.99
    assert np.mean(S.regret(T, g) <= 1.05) >= 0.8
    top3 = w.candidates(F, ok, 3)
    t3 = np.take_along_axis(np.where(ok, T, np.inf), top3, axis=1)
    assert np.mean(S.regret(T, top3[np.arange(len(T)), t3.argmin(axis=1)]) <= 1.05) >= 0.9


@pytest.mark.gpu
def test_select_end_to_end_and_sweep_fallback():
    """select() on a fresh matrix returns an admissible configuration; a matrix
    outside the training range goes to the exhaustive sweep."""
    d, w = _held_out()
    cap = int(d["nnz_cap"][0]) if "nnz_cap" in d.files else 1 << 21  # the training set's size cap
    m, _ = S.family_matrix(4_000_000, nnz_cap=cap)
    slot, how = w.select(m)
    assert how == "predicted" and S.admissible(m)[slot]
    tiny = synth.uniform(50, 1, 3, seed=1).astype(np.float32)  # 50 rows: below the training range
    slot, how = w.select(tiny, reps=2)
    assert how == "sweep" and S.admissible(tiny)[slot]
    # verify=3: the fastest of the three best predictions, timed
    f, ok = S.features(m), S.admissible(m)
    cand = w.candidates(f, ok, 3)[0]
    assert cand[0] == w.choose(f, ok)[0] and all(ok[c] for c in cand)
    slot, how = w.select(m, reps=2, verify=3)
    assert how == "verified" and slot in set(cand.tolist())
