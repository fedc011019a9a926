"""ORACLE — test infrastructure only (the checker, never the product path).

NumPy restatement of the learned warm start (``polysolve_b200/csrc/mas_warmstart.cu``). The
reference has no counterpart: it always starts PCG from x0 = 0 (MASSolver.cu:395-398), and its
caller re-solves every Newton step (Newton.cpp:173-214). The definitions restated here are the
solver's own (features, network, Galerkin combination):

* ``graph``:      neighbour weights w_ij = ||A_ij||_F / sum_{j' != i} ||A_ij'||_F over the
                  3x3 block pattern and the diagonal blocks;
* ``features``:   the 16 raw per-vertex features (from the residual of the history guess x_g)
                  and the five normalisation sums;
* ``forward_device``: the network as the GPU evaluates it (float32 input layer, bf16 hidden
                  states and layer weights with float32 accumulation, float32 output layer);
* ``forward64`` / ``backward64``: the same network in float64 with its reverse pass, checked
                  against finite differences (it is the reference for the training code);
* ``train_gradient_device``: the GPU training pass's loss and gradient with its rounding points
                  (bf16 where the GPU multiplies on tensor cores), for a tight check of its kernels;
* ``galerkin``:   the energy-minimising combination of {x1, x1 - x2, x2 - x3, x3 - x4, c} (missing
                  kept solutions give zero vectors, which are dropped) with the fallback to x1.

Only ``tests/`` import this.
"""

from __future__ import annotations

import math

import numpy as np

FEATURES, HIDDEN, LAYERS = 16, 64, 3


def layout():
    out, off = {}, 0
    for name, shape in [("w_in", (HIDDEN, FEATURES)), ("b_in", (HIDDEN,))] + \
            [(f"{k}_{lv}", s) for lv in range(LAYERS) for k, s in (("w", (HIDDEN, 2 * HIDDEN)), ("b", (HIDDEN,)))] + \
            [("w_out", (3, HIDDEN)), ("b_out", (3,))]:
        out[name] = (off, shape)
        off += int(np.prod(shape))
    return out, off


def unpack(params):
    lay, total = layout()
    params = np.asarray(params)
    assert params.size == total
    return {k: params[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in lay.items()}


def bf16(a):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def graph(A, bd=3):
    """(src, dst, w float64, D[V,3,3]) of a scipy matrix: edges j -> i for stored blocks i != j."""
    import scipy.sparse as sp

    coo = sp.coo_matrix(A)
    V = A.shape[0] // bd
    bi, bj = coo.row // bd, coo.col // bd
    key = bi.astype(np.int64) * V + bj
    uniq, inv = np.unique(key, return_inverse=True)
    fro2 = np.zeros(uniq.size)
    np.add.at(fro2, inv, coo.data ** 2)
    ri, cj = uniq // V, uniq % V
    off = ri != cj
    src, dst, nrm = cj[off], ri[off], np.sqrt(fro2[off])
    tot = np.zeros(V)
    np.add.at(tot, dst, nrm)
    w = np.where(tot[dst] > 0, nrm / np.where(tot[dst] > 0, tot[dst], 1.0), 0.0)
    D = np.zeros((V, bd, bd))
    diag = bi == bj
    np.add.at(D, (coo.row[diag] // bd, coo.row[diag] % bd, coo.col[diag] % bd), coo.data[diag])
    return src, dst, w, D


def features(A, b, x1, x2, D, xg=None):
    """(raw features float64 [V,16], sums[5]) with the residual r_g = b - A x_g of the history
    guess x_g (the solver's first Galerkin pass; default: the linear extrapolation 2 x1 - x2)."""
    V = D.shape[0]
    re = b - A @ ((2.0 * x1 - x2) if xg is None else xg)
    Dinv = np.linalg.inv(D)
    q = np.einsum("vij,vj->vi", Dinv, re.reshape(V, 3))
    v = (x1 - x2).reshape(V, 3)
    p = np.einsum("vij,vj->vi", Dinv, b.reshape(V, 3))
    tr = np.trace(D, axis1=1, axis2=2)
    t = tr / 3.0
    f = np.zeros((V, FEATURES))
    f[:, 0:3], f[:, 3:6], f[:, 6:9] = q, v, p
    f[:, 9], f[:, 10], f[:, 11] = D[:, 0, 0] / t, D[:, 1, 1] / t, D[:, 2, 2] / t
    f[:, 12], f[:, 13], f[:, 14] = D[:, 0, 1] / t, D[:, 0, 2] / t, D[:, 1, 2] / t
    f[:, 15] = np.log(tr)
    sums = np.array([np.sum(q * q), np.sum(v * v), np.sum(p * p), np.sum(np.log(tr)), float(V)])
    return f, sums


def normalise(f_raw, sums, dtype=np.float64):
    """Normalised features: q, v, p divided by their rms, log trace minus its mean."""
    cnt = sums[4]
    dofs = 3.0 * cnt
    scale = []
    for s in sums[:3]:
        r = math.sqrt(s / dofs)
        scale.append(1.0 / r if r > 0 else 0.0)
    f = np.array(f_raw, dtype=dtype)
    f[:, 0:3] *= dtype(scale[0])
    f[:, 3:6] *= dtype(scale[1])
    f[:, 6:9] *= dtype(scale[2])
    f[:, 15] -= dtype(sums[3] / cnt)
    return f


def s_q(sums):
    return math.sqrt(sums[0] / (3.0 * sums[4])) if sums[4] > 0 else 0.0


def forward_device(params, f_raw, sums, src, dst, w):
    """c (float64 [V,3]) as the GPU computes it (bf16 hidden states and layer weights)."""
    P = {k: np.asarray(v, dtype=np.float32) for k, v in unpack(params).items()}
    f = normalise(np.asarray(f_raw, dtype=np.float32), sums, dtype=np.float32)
    h = bf16(np.maximum(f @ P["w_in"].T + P["b_in"], 0.0))
    w32 = np.asarray(w, dtype=np.float32)
    for lv in range(LAYERS):
        m = np.zeros_like(h)
        np.add.at(m, dst, w32[:, None] * h[src])
        t = np.concatenate([h, bf16(m)], axis=1)
        acc = t @ bf16(P[f"w_{lv}"]).T
        h = bf16(h + np.maximum(acc + P[f"b_{lv}"], 0.0))
    out = h @ P["w_out"].T + P["b_out"]
    return s_q(sums) * out.astype(np.float64)


def forward64(params, f, src, dst, w):
    """The network in float64 on normalised features; returns (out [V,3], cache)."""
    P = {k: np.asarray(v, dtype=np.float64) for k, v in unpack(params).items()}
    cache = {"f": f, "src": src, "dst": dst, "w": w, "P": P}
    z0 = f @ P["w_in"].T + P["b_in"]
    h = np.maximum(z0, 0.0)
    cache["z0"] = z0
    hs, zs, ts = [h], [], []
    for lv in range(LAYERS):
        m = np.zeros_like(h)
        np.add.at(m, dst, w[:, None] * h[src])
        t = np.concatenate([h, m], axis=1)
        z = t @ P[f"w_{lv}"].T + P[f"b_{lv}"]
        h = h + np.maximum(z, 0.0)
        ts.append(t)
        zs.append(z)
        hs.append(h)
    cache.update(hs=hs, zs=zs, ts=ts)
    return h @ P["w_out"].T + P["b_out"], cache


def backward64(cache, g_out):
    """Gradient of sum(out * g_out) with respect to the flat parameter vector."""
    P, src, dst, w = cache["P"], cache["src"], cache["dst"], cache["w"]
    grads = {}
    h = cache["hs"][-1]
    grads["w_out"] = g_out.T @ h
    grads["b_out"] = g_out.sum(axis=0)
    gh = g_out @ P["w_out"]
    for lv in reversed(range(LAYERS)):
        z, t = cache["zs"][lv], cache["ts"][lv]
        gz = gh * (z > 0)
        grads[f"w_{lv}"] = gz.T @ t
        grads[f"b_{lv}"] = gz.sum(axis=0)
        gt = gz @ P[f"w_{lv}"]
        gh_prev = gh + gt[:, :HIDDEN]
        gm = gt[:, HIDDEN:]
        # m_i = sum_{(j -> i)} w h_j  =>  dh_j += w gm_i
        np.add.at(gh_prev, src, w[:, None] * gm[dst])
        gh = gh_prev
    gz0 = gh * (cache["z0"] > 0)
    grads["w_in"] = gz0.T @ cache["f"]
    grads["b_in"] = gz0.sum(axis=0)
    lay, total = layout()
    flat = np.zeros(total)
    for k, (o, s) in lay.items():
        flat[o:o + int(np.prod(s))] = grads[k].reshape(-1)
    return flat


def loss_and_output_gradient(out, A, re, s_q, ere):
    """(loss, rho, dL/dout) of the training objective 1 - rho, rho = (c . r_g)^2 / ((c . A c) (e . r_g)),
    c = s_q out (float64; the GPU's k_tr_spmv_loss and k_tr_out_bwd)."""
    c = s_q * np.asarray(out, dtype=np.float64).reshape(-1)
    Ac = A @ c
    a, q = float(c @ re), float(c @ Ac)
    if not (q > 0 and ere > 0):
        return 1.0, 0.0, np.zeros_like(np.asarray(out, dtype=np.float64))
    rho = a * a / (q * ere)
    g_c = -2.0 * a / (q * ere) * re + 2.0 * a * a / (q * q * ere) * Ac
    return 1.0 - rho, rho, (s_q * g_c).reshape(-1, 3)


def train_gradient_device(params, f, src, dst, w, A, re, s_q, ere):
    """(loss, flat gradient) of one training sample with the GPU training pass's rounding points
    (polysolve_b200/csrc/mas_ws_train.cu): the forward as ``forward_device`` (bf16 hidden states,
    messages and layer weights, float32 elsewhere) on normalised float32 features f; the reverse pass
    rounds gz = dL/dh' * [z > 0] and W_l to bf16 for the two tensor-core products, everything else
    float32 (sums here in float64). Messages m_i = sum_j w_ij h_j over edges j -> i."""
    P = {k: np.asarray(v, dtype=np.float32) for k, v in unpack(params).items()}
    f = np.asarray(f, dtype=np.float32)
    w32 = np.asarray(w, dtype=np.float32)
    z0 = f @ P["w_in"].T + P["b_in"]
    h = bf16(np.maximum(z0, 0.0))
    hs, ts, zs = [h], [], []
    for lv in range(LAYERS):
        m = np.zeros_like(h)
        np.add.at(m, dst, w32[:, None] * h[src])
        t = np.concatenate([h, bf16(m)], axis=1)
        z = t @ bf16(P[f"w_{lv}"]).T + P[f"b_{lv}"]
        h = bf16(h + np.maximum(z, 0.0))
        ts.append(t)
        zs.append(z)
        hs.append(h)
    out = (h @ P["w_out"].T + P["b_out"]).astype(np.float32)
    loss, _, g_out = loss_and_output_gradient(out, A, re, s_q, ere)
    g_out = g_out.astype(np.float32).astype(np.float64)
    grads = {"w_out": g_out.T @ hs[-1], "b_out": g_out.sum(axis=0)}
    gh = (g_out @ P["w_out"].astype(np.float64)).astype(np.float32).astype(np.float64)
    for lv in reversed(range(LAYERS)):
        gz = gh * (zs[lv] > 0)
        gzb = bf16(gz.astype(np.float32)).astype(np.float64)
        grads[f"w_{lv}"] = gzb.T @ ts[lv].astype(np.float64)
        grads[f"b_{lv}"] = gz.sum(axis=0)
        gt = gzb @ bf16(P[f"w_{lv}"]).astype(np.float64)
        gh_prev = gh + gt[:, :HIDDEN]
        np.add.at(gh_prev, src, w32[:, None].astype(np.float64) * gt[dst, HIDDEN:])
        gh = gh_prev.astype(np.float32).astype(np.float64)
    gz0 = gh * (z0 > 0)
    grads["w_in"] = gz0.T @ f.astype(np.float64)
    grads["b_in"] = gz0.sum(axis=0)
    lay, total = layout()
    flat = np.zeros(total)
    for k, (o, sh) in lay.items():
        flat[o:o + int(np.prod(sh))] = grads[k].reshape(-1)
    return loss, flat


def galerkin_basis(history, c):
    """The solver's basis: x1, the differences of consecutive kept solutions (x_{k-1} first; a
    missing one is zero), then c."""
    hist = list(history)
    V = [hist[0]]
    for i in range(1, 4):
        V.append(hist[i - 1] - hist[i] if i < len(hist) else np.zeros_like(hist[0]))
    V.append(c)
    return V


def galerkin(A, b, x1, x2, c, *older):
    """(coef[5], energy, energy of x1, fallback, rank) of the solver's combination rule over the
    basis of ``galerkin_basis((x1, x2, *older), c)``."""
    V = galerkin_basis((x1, x2) + tuple(older), c)
    AV = [A @ v for v in V]
    nb = len(V)
    G = np.array([[V[i] @ AV[j] for j in range(nb)] for i in range(nb)])
    G = 0.5 * (G + G.T)
    g = np.array([v @ b for v in V])
    keep = []
    for i in range(nb):
        if not (G[i, i] > 0 and np.isfinite(G[i, i])):
            continue
        S = keep
        d = G[i, i] - (G[i, S] @ np.linalg.solve(G[np.ix_(S, S)], G[S, i]) if S else 0.0)
        if d > 1e-10 * G[i, i] and np.isfinite(d):
            keep.append(i)
    y = np.zeros(nb)
    if keep:
        y[keep] = np.linalg.solve(G[np.ix_(keep, keep)], g[keep])
    e = 0.5 * y @ G @ y - y @ g
    e1 = 0.5 * G[0, 0] - g[0]
    ok = bool(keep) and np.isfinite(e) and e < e1
    if not ok:
        y0 = np.zeros(nb)
        y0[0] = 1.0
        return y0, e1, e1, True, len(keep)
    return y, e, e1, False, len(keep)
