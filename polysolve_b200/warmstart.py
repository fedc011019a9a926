"""Learned warm start: the message-passing network's definition and weight file format.

The solver's ``initial_guess: "learned"`` mode keeps the last four solutions of a sequence of
systems on the device and predicts the next starting guess from them, b and the diagonal blocks
(all on the GPU, ``csrc/mas_warmstart.cu``):

1. ``y_j = A x_{k-j}`` for the kept solutions (one SpMV each), the history guess ``x_g``: the
   Galerkin (energy-minimising) combination of x_{k-1} and the differences
   x_{k-1} - x_{k-2}, x_{k-2} - x_{k-3}, x_{k-3} - x_{k-4} (a polynomial extrapolation in the
   step index fitted in the energy norm; missing ones are dropped), and ``r_g = b - A x_g``
   (from the y_j, no SpMV);
2. per vertex i, with D_i the 3x3 diagonal block and t_i = trace(D_i) / 3, the 16 input features

   ====== =====================================  ==========================================
   index  raw value                               normalisation
   ====== =====================================  ==========================================
   0-2    q_i = D_i^-1 r_g,i                      / s_q = rms of q over all real DOFs
   3-5    v_i = x_{k-1,i} - x_{k-2,i}             / s_v = rms of v
   6-8    p_i = D_i^-1 b_i                        / s_p = rms of p
   9-11   D_i[0,0], D_i[1,1], D_i[2,2]            / t_i
   12-14  D_i[0,1], D_i[0,2], D_i[1,2]            / t_i
   15     log trace(D_i)                          - its mean over real vertices
   ====== =====================================  ==========================================

3. the network (hidden width H = 64, L = 3 message-passing layers over the vertex graph of A,
   neighbour weights w_ij = ||A_ij||_F / sum_{j' != i} ||A_ij'||_F):

   h   = relu(W_in f + b_in)                                  (16 -> 64)
   m_i = sum_j w_ij h_j;  h = h + relu(W_l [h ; m] + b_l)     (128 -> 64, three times)
   c_i = s_q (W_out h_i + b_out)                              (64 -> 3)

   On the GPU the hidden states and the layer weights W_l are BF16 (tensor-core products,
   FP32 accumulation); W_in, W_out and the biases stay FP32;
4. the starting guess is the Galerkin combination of the same basis plus c (the network is
   trained on the error of x_g, so c is the part the history cannot extrapolate); if its energy
   is not below that of x_{k-1} (or the system is degenerate), the guess falls back to x_{k-1}.
   PCG then runs to the tolerance as usual, so every accepted solve meets the same relative
   residual as a cold start.

Weight file (``.psws``): 8 bytes ``PSWSMPN1``, four little-endian int32 (features 16,
hidden 64, layers 3, parameter count), then the parameters as little-endian float32 in the
order W_in (64 x 16, row-major), b_in (64), for each layer W_l (64 x 128, row-major, columns
0-63 act on h and 64-127 on m) and b_l (64), W_out (3 x 64) and b_out (3).
"""

from __future__ import annotations

import os
from pathlib import Path

import numpy as np

FEATURES = 16
HIDDEN = 64
LAYERS = 3
HISTORY = 4            # kept solutions
BASIS = HISTORY + 1    # Galerkin basis: x1, x1 - x2, x2 - x3, x3 - x4, c
MAGIC = b"PSWSMPN1"


def param_count(features: int = FEATURES, hidden: int = HIDDEN, layers: int = LAYERS) -> int:
    return hidden * features + hidden + layers * (hidden * 2 * hidden + hidden) + 3 * hidden + 3


PARAMS = param_count()


def layout(features: int = FEATURES, hidden: int = HIDDEN, layers: int = LAYERS) -> dict[str, tuple[int, tuple]]:
    """name -> (offset, shape) of every tensor in the flat parameter vector."""
    out, off = {}, 0

    def put(name, shape):
        nonlocal off
        out[name] = (off, shape)
        off += int(np.prod(shape))

    put("w_in", (hidden, features))
    put("b_in", (hidden,))
    for lv in range(layers):
        put(f"w_{lv}", (hidden, 2 * hidden))
        put(f"b_{lv}", (hidden,))
    put("w_out", (3, hidden))
    put("b_out", (3,))
    assert off == param_count(features, hidden, layers)
    return out


def unpack(params: np.ndarray) -> dict[str, np.ndarray]:
    """Views of the flat parameter vector by tensor name."""
    params = np.asarray(params)
    if params.size != PARAMS:
        raise ValueError(f"expected {PARAMS} parameters, got {params.size}")
    return {k: params[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in layout().items()}


def save(path: str | os.PathLike, params: np.ndarray) -> None:
    params = np.ascontiguousarray(params, dtype="<f4")
    if params.size != PARAMS:
        raise ValueError(f"expected {PARAMS} parameters, got {params.size}")
    with open(path, "wb") as fh:
        fh.write(MAGIC)
        fh.write(np.array([FEATURES, HIDDEN, LAYERS, PARAMS], dtype="<i4").tobytes())
        fh.write(params.tobytes())


def load(path: str | os.PathLike) -> np.ndarray:
    """The float32 parameter vector of a ``.psws`` file (format checked)."""
    raw = Path(path).read_bytes()
    if len(raw) < 24 or raw[:8] != MAGIC:
        raise ValueError(f"{path}: not a warm-start weight file")
    dims = np.frombuffer(raw[8:24], dtype="<i4")
    if tuple(int(d) for d in dims) != (FEATURES, HIDDEN, LAYERS, PARAMS):
        raise ValueError(f"{path}: unsupported network shape {tuple(int(d) for d in dims)}")
    params = np.frombuffer(raw[24:], dtype="<f4")
    if params.size != PARAMS:
        raise ValueError(f"{path}: truncated ({params.size} of {PARAMS} parameters)")
    return params.astype(np.float32)


DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "data" / "warm_start_mpnn.psws"


def default_weights() -> np.ndarray:
    """The shipped network, trained by ``warmstart_train`` on seeded elasticity sequences."""
    return load(DEFAULT_WEIGHTS)


__all__ = ["FEATURES", "HIDDEN", "LAYERS", "HISTORY", "BASIS", "PARAMS", "layout", "unpack", "save", "load",
           "default_weights", "DEFAULT_WEIGHTS"]
