"""Training of the learned warm start (host side, PyTorch autograd as plumbing).

Data: seeded elasticity sequences built like the 60^3 sequence workload
(``synthetic.workload_sequence60``) on smaller grids; every step is solved to a relative
residual of 1e-12 on the host (a sparse LU of the first step's matrix preconditions CG for the
following steps, whose matrices differ by a few percent). A sample is step k of a sequence with
the two previous solutions: (A_k, b_k, x_{k-1}, x_{k-2}, x_k).

Objective: the network's correction c should point along the error of the history guess
x_g (the energy-minimising combination of the kept solutions x_{k-1} .. x_{k-4}, as the solver
computes it before the network), e = x_k - x_g, in the energy norm. With the optimal step along c
(the solver's final Galerkin combination does at least as well), the remaining squared energy
error is ||e||_A^2 (1 - rho) with rho = (c . r_g)^2 / ((c . A c) (e . r_g)), r_g = A e. The loss
is the mean of 1 - rho, which is invariant to the scale of c.

Run ``python -m polysolve_b200.warmstart_train --out polysolve_b200/data/warm_start_mpnn.psws``
to regenerate the shipped weights (seeded; data generation and training take tens of minutes
on 8 host cores).
"""

from __future__ import annotations

import argparse
import math
import multiprocessing as mp
import time

import numpy as np

from . import warmstart as W


# ----------------------------------------------------------------------------------------------
# Graph and features (the same definitions as the device kernels, in float64 on the host)
# ----------------------------------------------------------------------------------------------

def block_graph(A, bd: int = 3):
    """(src, dst, w, D): directed neighbour edges j -> i (i != j) of the block pattern with
    weights ||A_ij||_F / sum_{j' != i} ||A_ij'||_F, and the diagonal blocks D[V, 3, 3]."""
    import scipy.sparse as sp

    A = sp.csr_matrix(A)
    n = A.shape[0]
    V = n // bd
    coo = A.tocoo()
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
    diag = coo.row // bd == coo.col // bd
    np.add.at(D, (coo.row[diag] // bd, coo.row[diag] % bd, coo.col[diag] % bd), coo.data[diag])
    return src.astype(np.int64), dst.astype(np.int64), w, D


def history_guess(A, b, hist):
    """x_g: the energy-minimising combination of x1 and the differences of consecutive kept
    solutions (``hist`` newest first, 2 to 4 of them), with the solver's rule of dropping
    vectors whose Cholesky pivot falls below 1e-10 of their diagonal."""
    V = [hist[0]] + [hist[i - 1] - hist[i] for i in range(1, len(hist))]
    AV = [A @ v for v in V]
    G = np.array([[vi @ avj for avj in AV] for vi in V])
    g = np.array([v @ b for v in V])
    keep = []
    for i in range(len(V)):
        if not G[i, i] > 0:
            continue
        d = G[i, i] - (G[i, keep] @ np.linalg.solve(G[np.ix_(keep, keep)], G[keep, i]) if keep else 0.0)
        if d > 1e-10 * G[i, i]:
            keep.append(i)
    y = np.zeros(len(V))
    if keep:
        y[keep] = np.linalg.solve(G[np.ix_(keep, keep)], g[keep])
    return sum(yi * vi for yi, vi in zip(y, V))


def features(A, b, x1, x2, D, xg=None):
    """(f[V, 16] float64, s_q, r_g, x_g) of the definitions in ``polysolve_b200.warmstart``;
    x_g defaults to the linear extrapolation 2 x1 - x2."""
    V = D.shape[0]
    xe = 2.0 * x1 - x2 if xg is None else xg
    re = b - A @ xe
    Dinv = np.linalg.inv(D)
    q = np.einsum("vij,vj->vi", Dinv, re.reshape(V, 3))
    v = (x1 - x2).reshape(V, 3)
    p = np.einsum("vij,vj->vi", Dinv, b.reshape(V, 3))
    tr = np.trace(D, axis1=1, axis2=2)
    t = tr / 3.0

    def rms(a):
        return math.sqrt(float(np.sum(a * a)) / a.size)

    s_q, s_v, s_p = rms(q), rms(v), rms(p)
    f = np.zeros((V, W.FEATURES))
    f[:, 0:3] = q / s_q if s_q > 0 else 0.0
    f[:, 3:6] = v / s_v if s_v > 0 else 0.0
    f[:, 6:9] = p / s_p if s_p > 0 else 0.0
    f[:, 9] = D[:, 0, 0] / t
    f[:, 10] = D[:, 1, 1] / t
    f[:, 11] = D[:, 2, 2] / t
    f[:, 12] = D[:, 0, 1] / t
    f[:, 13] = D[:, 0, 2] / t
    f[:, 14] = D[:, 1, 2] / t
    lt = np.log(tr)
    f[:, 15] = lt - lt.mean()
    return f, s_q, re, xe


# ----------------------------------------------------------------------------------------------
# Data
# ----------------------------------------------------------------------------------------------

def solve_sequence_exact(N: int, seed: int, k0: int, steps: int):
    """(systems, rhs, solutions) of steps k0 .. k0+steps-1 of the seeded sequence on N^3."""
    import scipy.sparse.linalg as sla

    from . import synthetic

    systems, rhs, xs = [], [], []
    lu = None
    for k in range(k0, k0 + steps):
        s, b = synthetic.workload_sequence60(k, seed=seed, N=N)
        A = s.scipy().tocsr()
        if lu is None:
            lu = sla.splu(A.tocsc())
            x = lu.solve(b)
        else:
            M = sla.LinearOperator(A.shape, matvec=lu.solve)
            x0 = 2 * xs[-1] - xs[-2] if len(xs) >= 2 else xs[-1]
            x, info = sla.cg(A, b, x0=x0, M=M, rtol=1e-12, atol=0.0, maxiter=200)
            if info != 0:
                lu = sla.splu(A.tocsc())
                x = lu.solve(b)
        systems.append(A)
        rhs.append(b)
        xs.append(x)
    return systems, rhs, xs


def make_samples(job):
    """Samples of one sequence: everything the loss needs, float32 where it is bulk data."""
    N, seed, k0, steps = job
    systems, rhs, xs = solve_sequence_exact(N, seed, k0, steps)
    out = []
    for k in range(2, steps):
        A = systems[k]
        src, dst, w, D = block_graph(A)
        hist = [xs[k - j] for j in range(1, min(k, W.HISTORY) + 1)]
        xg = history_guess(A, rhs[k], hist)
        f, s_q, re, _ = features(A, rhs[k], xs[k - 1], xs[k - 2], D, xg)
        e = xs[k] - xg
        out.append({
            "N": N, "f": f.astype(np.float32), "src": src, "dst": dst, "w": w.astype(np.float32),
            "A_indptr": A.indptr.astype(np.int32), "A_indices": A.indices.astype(np.int32),
            "A_data": A.data.astype(np.float32), "re": re, "s_q": s_q, "ere": float(e @ re),
        })
    return out


def generate(jobs, processes: int = 8):
    """Samples of all jobs from a pool of single-threaded worker processes."""
    import os

    keys = ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")
    saved = {k: os.environ.get(k) for k in keys}
    os.environ.update({k: "1" for k in keys})  # inherited by the spawned workers
    try:
        ctx = mp.get_context("spawn")
        with ctx.Pool(processes) as pool:
            parts = pool.map(make_samples, sorted(jobs, key=lambda j: -j[0]), chunksize=1)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    return [s for p in parts for s in p]


def default_jobs(seed0: int = 1000, steps: int = 22):
    """About 2000 systems: sequences of 22 steps (20 samples each) on 12^3 to 28^3 grids."""
    rng = np.random.Generator(np.random.PCG64(seed0))
    jobs = []
    for N, count in ((12, 30), (16, 30), (20, 24), (24, 10), (28, 6)):
        for _ in range(count):
            jobs.append((N, int(rng.integers(0, 2 ** 31 - 1)), int(rng.integers(0, 200 - steps)), steps))
    return jobs


# ----------------------------------------------------------------------------------------------
# Model
# ----------------------------------------------------------------------------------------------

def build_model():
    import torch

    class MPNN(torch.nn.Module):
        def __init__(self):
            super().__init__()
            self.w_in = torch.nn.Linear(W.FEATURES, W.HIDDEN)
            self.layers = torch.nn.ModuleList([torch.nn.Linear(2 * W.HIDDEN, W.HIDDEN) for _ in range(W.LAYERS)])
            self.w_out = torch.nn.Linear(W.HIDDEN, 3)
            with torch.no_grad():
                for lin in self.layers:
                    lin.weight.mul_(0.5)
                self.w_out.weight.mul_(0.1)

        def forward(self, f, src, dst, w):
            h = torch.relu(self.w_in(f))
            for lin in self.layers:
                m = torch.zeros_like(h).index_add_(0, dst, w[:, None] * h[src])
                h = h + torch.relu(lin(torch.cat([h, m], dim=1)))
            return self.w_out(h)

        def flat(self) -> np.ndarray:
            parts = [self.w_in.weight, self.w_in.bias]
            for lin in self.layers:
                parts += [lin.weight, lin.bias]
            parts += [self.w_out.weight, self.w_out.bias]
            return np.concatenate([p.detach().cpu().numpy().reshape(-1) for p in parts]).astype(np.float32)

        def load_flat(self, params: np.ndarray) -> None:
            t = W.unpack(params)
            with torch.no_grad():
                self.w_in.weight.copy_(torch.from_numpy(np.array(t["w_in"])))
                self.w_in.bias.copy_(torch.from_numpy(np.array(t["b_in"])))
                for lv, lin in enumerate(self.layers):
                    lin.weight.copy_(torch.from_numpy(np.array(t[f"w_{lv}"])))
                    lin.bias.copy_(torch.from_numpy(np.array(t[f"b_{lv}"])))
                self.w_out.weight.copy_(torch.from_numpy(np.array(t["w_out"])))
                self.w_out.bias.copy_(torch.from_numpy(np.array(t["b_out"])))

    return MPNN()


def to_torch(sample):
    import torch

    n = sample["re"].size
    A = torch.sparse_csr_tensor(torch.from_numpy(sample["A_indptr"]), torch.from_numpy(sample["A_indices"]),
                                torch.from_numpy(sample["A_data"]), size=(n, n), check_invariants=False)
    return {"f": torch.from_numpy(sample["f"]), "src": torch.from_numpy(sample["src"]),
            "dst": torch.from_numpy(sample["dst"]), "w": torch.from_numpy(sample["w"]), "A": A,
            "re": torch.from_numpy(sample["re"]), "ere": sample["ere"], "s_q": sample["s_q"]}


def rho(model, t):
    """Squared energy-norm cosine between the correction and the extrapolation error."""
    import torch

    c = model(t["f"], t["src"], t["dst"], t["w"]).double().reshape(-1) * t["s_q"]
    Ac = torch.mv(t["A"], c.float()).double()
    return (c @ t["re"]) ** 2 / ((c @ Ac) * t["ere"])


def train(samples, epochs: int = 20, lr: float = 2e-3, seed: int = 0, val_fraction: float = 0.1, log=print):
    import torch

    torch.manual_seed(seed)
    rng = np.random.Generator(np.random.PCG64(seed))
    order = rng.permutation(len(samples))
    nval = max(1, int(len(samples) * val_fraction))
    val = [to_torch(samples[i]) for i in order[:nval]]
    tr = [samples[i] for i in order[nval:]]
    model = build_model()
    opt = torch.optim.Adam(model.parameters(), lr=lr)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, T_max=epochs * len(tr))
    vr = 0.0
    for ep in range(epochs):
        t0 = time.time()
        model.train()
        tot = 0.0
        for i in rng.permutation(len(tr)):
            opt.zero_grad()
            loss = 1.0 - rho(model, to_torch(tr[i]))
            loss.backward()
            opt.step()
            sched.step()
            tot += float(loss)
        model.eval()
        with torch.no_grad():
            vr = float(np.mean([float(rho(model, t)) for t in val]))
        log(f"epoch {ep}: train loss {tot / len(tr):.4f}  val rho {vr:.4f}  ({time.time() - t0:.1f}s)")
    return model, vr


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=str(W.DEFAULT_WEIGHTS))
    ap.add_argument("--epochs", type=int, default=15)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--processes", type=int, default=8)
    ap.add_argument("--sequences", type=int, default=0, help="limit the number of sequences (0: all)")
    args = ap.parse_args(argv)
    import torch

    torch.set_num_threads(args.processes)
    jobs = default_jobs()
    if args.sequences:
        jobs = jobs[:: max(1, len(jobs) // args.sequences)][: args.sequences]
    t0 = time.time()
    samples = generate(jobs, args.processes)
    print(f"{len(samples)} samples from {len(jobs)} sequences in {time.time() - t0:.0f}s", flush=True)
    model, vr = train(samples, epochs=args.epochs, lr=args.lr, log=lambda s: print(s, flush=True))
    W.save(args.out, model.flat())
    print(f"wrote {args.out} (validation rho {vr:.4f})", flush=True)


if __name__ == "__main__":
    main()
