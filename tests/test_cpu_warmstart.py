"""Learned warm start on the host: the weight file format, the network's parameter layout, the
float64 oracle's reverse pass and training objective against finite differences, and the oracle's
emulation of the GPU training pass against the plain float64 one."""

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


def _spd(V, seed):
    import scipy.sparse as sp

    rng = np.random.default_rng(seed)
    M = sp.random(3 * V, 3 * V, density=0.05, random_state=rng)
    return (M @ M.T + 3 * V * sp.eye(3 * V)).tocsr()


def test_loss_gradient_matches_finite_differences():
    """The training objective 1 - rho through the float64 network: its reverse pass (backward64 of
    dL/dout) against central differences of the loss."""
    f, src, dst, w = _small_graph(V=30, seed=7)
    rng = np.random.default_rng(8)
    prm = 0.3 * rng.standard_normal(W.PARAMS)
    A = _spd(30, 9)
    e = rng.standard_normal(90)
    re = A @ e
    ere, s_q = float(e @ re), 0.7

    def loss_of(p):
        out, _ = WO.forward64(p, f, src, dst, w)
        return WO.loss_and_output_gradient(out, A, re, s_q, ere)[0]

    out, cache = WO.forward64(prm, f, src, dst, w)
    loss, rho, g_out = WO.loss_and_output_gradient(out, A, re, s_q, ere)
    assert 0.0 <= rho <= 1.0 + 1e-12 and abs(loss - (1 - rho)) < 1e-15
    grad = WO.backward64(cache, g_out)
    lay, _ = WO.layout()
    eps = 1e-6
    for name, (o, shape) in lay.items():
        for i in o + rng.choice(int(np.prod(shape)), size=2, replace=False):
            p1, p2 = prm.copy(), prm.copy()
            p1[i] += eps
            p2[i] -= eps
            fd = (loss_of(p1) - loss_of(p2)) / (2 * eps)
            assert abs(fd - grad[i]) <= 1e-5 * max(1.0, abs(fd)), (name, fd, grad[i])


def test_device_training_emulation_close_to_float64():
    """The emulation of the GPU training pass (bf16 at the tensor-core products) stays within BF16
    error of the plain float64 gradient, tensor by tensor."""
    from polysolve_b200 import warmstart_train as T

    f, src, dst, w = _small_graph(V=60, seed=10)
    rng = np.random.default_rng(11)
    prm = T.initial_params(2)  # the training's initial scale (BF16 error grows with random large weights)
    o = W.layout()["w_out"][0]
    prm[o:o + 3 * W.HIDDEN] *= 10.0
    A = _spd(60, 12)
    e = rng.standard_normal(180)
    re = A @ e
    ere, s_q = float(e @ re), 1.3
    loss_d, grad_d = WO.train_gradient_device(prm, f.astype(np.float32), src, dst, w, A, re, s_q, ere)
    out, cache = WO.forward64(prm.astype(np.float64), f.astype(np.float32).astype(np.float64), src, dst, w)
    loss, _, g_out = WO.loss_and_output_gradient(out, A, re, s_q, ere)
    grad = WO.backward64(cache, g_out)
    assert abs(loss_d - loss) <= 2e-2
    for name, (o, shape) in WO.layout()[0].items():
        a, b = grad_d[o:o + int(np.prod(shape))], grad[o:o + int(np.prod(shape))]
        assert np.linalg.norm(a - b) <= 6e-2 * np.linalg.norm(b), name


def test_initial_parameters_are_seeded_and_scaled():
    from polysolve_b200 import warmstart_train as T

    p1, p2 = T.initial_params(3), T.initial_params(3)
    assert np.array_equal(p1, p2) and p1.dtype == np.float32 and p1.size == W.PARAMS
    t = W.unpack(p1)
    assert np.abs(t["w_in"]).max() <= 1 / 4 and np.abs(t["w_0"]).max() <= 0.5 / np.sqrt(128)
    assert np.abs(t["w_out"]).max() <= 0.1 / 8


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
