"""Learned warm start on the host: the weight file format, the network's parameter layout, the
float64 oracle's reverse pass against finite differences, and the training code against the
oracle (the definitions the GPU kernels follow)."""

import re
from pathlib import Path

import numpy as np
import pytest

from oracle import warmstart_oracle as WO
from polysolve_b200 import synthetic
from polysolve_b200 import warmstart as W

ROOT = Path(__file__).resolve().parents[1]


def test_parameter_count_matches_header_and_oracle():
    hdr = (ROOT / "include" / "polysolve_mas.h").read_text()
    vals = {k: int(v) for k, v in re.findall(r"#define MAS_WS_(\w+) (\d+)", hdr)}
    assert vals == {"FEATURES": W.FEATURES, "HIDDEN": W.HIDDEN, "LAYERS": W.LAYERS, "PARAMS": W.PARAMS}
    assert WO.layout()[1] == W.PARAMS == 26051
    assert {k: v for k, v in W.layout().items()} == WO.layout()[0]


def test_weight_file_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    prm = rng.standard_normal(W.PARAMS).astype(np.float32)
    path = tmp_path / "w.psws"
    W.save(path, prm)
    assert np.array_equal(W.load(path), prm)
    raw = path.read_bytes()
    (tmp_path / "bad.psws").write_bytes(b"XXXXXXXX" + raw[8:])
    with pytest.raises(ValueError):
        W.load(tmp_path / "bad.psws")
    (tmp_path / "short.psws").write_bytes(raw[:-4])
    with pytest.raises(ValueError):
        W.load(tmp_path / "short.psws")


def test_shipped_weights_load():
    prm = W.default_weights()
    assert prm.shape == (W.PARAMS,) and np.all(np.isfinite(prm))


def _small_graph(V=40, seed=1):
    rng = np.random.default_rng(seed)
    src, dst = [], []
    for i in range(V):
        for j in rng.choice(V, size=4, replace=False):
            if j != i:
                src.append(j)
                dst.append(i)
    src, dst = np.array(src), np.array(dst)
    w = rng.uniform(0.1, 1.0, size=src.size)
    f = rng.standard_normal((V, W.FEATURES))
    return f, src, dst, w


def test_oracle_backward_matches_finite_differences():
    f, src, dst, w = _small_graph()
    rng = np.random.default_rng(2)
    prm = 0.3 * rng.standard_normal(W.PARAMS)
    g_out = rng.standard_normal((f.shape[0], 3))
    out, cache = WO.forward64(prm, f, src, dst, w)
    grad = WO.backward64(cache, g_out)
    lay, _ = WO.layout()
    idx = []
    for name, (o, s) in lay.items():
        idx += list(o + rng.choice(int(np.prod(s)), size=3, replace=False))
    eps = 1e-6
    for i in idx:
        p1, p2 = prm.copy(), prm.copy()
        p1[i] += eps
        p2[i] -= eps
        fd = (np.sum(WO.forward64(p1, f, src, dst, w)[0] * g_out) -
              np.sum(WO.forward64(p2, f, src, dst, w)[0] * g_out)) / (2 * eps)
        assert abs(fd - grad[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, grad[i])


def test_training_model_matches_oracle_forward():
    torch = pytest.importorskip("torch")
    from polysolve_b200 import warmstart_train as T

    f, src, dst, w = _small_graph(seed=3)
    prm = 0.3 * np.random.default_rng(4).standard_normal(W.PARAMS)
    model = T.build_model().double()
    model.load_flat(prm)
    out = model(torch.from_numpy(f), torch.from_numpy(src), torch.from_numpy(dst), torch.from_numpy(w))
    ref, _ = WO.forward64(prm, f, src, dst, w)
    assert np.allclose(out.detach().numpy(), ref, rtol=1e-12, atol=1e-12)


def test_training_features_match_oracle():
    from polysolve_b200 import warmstart_train as T

    s0, b = synthetic.workload_sequence60(3, seed=2, N=5)
    A = s0.scipy().tocsr()
    rng = np.random.default_rng(5)
    x1, x2 = rng.standard_normal(s0.n), rng.standard_normal(s0.n)
    src, dst, w, D = T.block_graph(A)
    x3 = rng.standard_normal(s0.n)
    xg = T.history_guess(A, b, [x1, x2, x3])
    f, sq, _, _ = T.features(A, b, x1, x2, D, xg)
    src_o, dst_o, w_o, D_o = WO.graph(A)
    order_t = np.lexsort((src, dst))
    order_o = np.lexsort((src_o, dst_o))
    assert np.array_equal(src[order_t], src_o[order_o]) and np.array_equal(dst[order_t], dst_o[order_o])
    assert np.allclose(w[order_t], w_o[order_o], rtol=1e-14)
    raw, sums = WO.features(A, b, x1, x2, D_o, xg)
    # the training's history guess follows the oracle's Galerkin rule (no c)
    y, _, _, _, _ = WO.galerkin(A, b, x1, x2, np.zeros_like(b), x3)
    xg_o = sum(yi * vi for yi, vi in zip(y, WO.galerkin_basis((x1, x2, x3), np.zeros_like(b))))
    assert np.linalg.norm(xg - xg_o) <= 1e-8 * np.linalg.norm(xg_o)
    fo = WO.normalise(raw, sums)
    assert np.allclose(f, fo, rtol=1e-10, atol=1e-12)
    assert abs(sq - WO.s_q(sums)) <= 1e-12 * sq
    # normalised q, v, p have unit rms
    for k in range(3):
        assert abs(np.sqrt(np.mean(fo[:, 3 * k:3 * k + 3] ** 2)) - 1.0) < 1e-12


def test_galerkin_oracle_is_never_worse_than_previous():
    s0, b = synthetic.workload_sequence60(0, seed=1, N=4)
    A = s0.scipy().tocsr()
    rng = np.random.default_rng(6)
    x1 = rng.standard_normal(s0.n)
    x2 = x1 + 0.1 * rng.standard_normal(s0.n)
    c = rng.standard_normal(s0.n)
    y, e, e1, fb, rank = WO.galerkin(A, b, x1, x2, c)
    assert e <= e1 and rank == 3 and not fb
    # a dependent correction (c = x1) is dropped
    y, e, e1, fb, rank = WO.galerkin(A, b, x1, x2, x1.copy())
    assert rank == 2 and e <= e1
