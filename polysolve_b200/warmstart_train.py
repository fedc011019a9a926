"""Training of the learned warm start on the GPU, with this library's own kernels.

Data: seeded elasticity sequences built like the 60^3 sequence workload
(``synthetic.workload_sequence60``) on 12^3 to 28^3 grids, 100 sequences of 22 steps. Every step is
solved by the plain FP64 MAS-PCG on the GPU to a relative residual of 1e-9 (from the previous
step's solution); a sample is step k >= 2 with its kept solutions x_{k-1} .. x_{k-4} and the exact
solution x_k. The trainer (``WarmStartTrainer``, C ABI ``mas_ws_trainer_*``) runs the solver's own
prediction pipeline up to the features for each sample and keeps the sample in device memory.

Objective: the network's correction c should point along the error e = x_k - x_g of the history
guess x_g (the energy-minimising combination of the kept solutions, as the solver computes it before
the network) in the energy norm. With the optimal step along c (the solver's final Galerkin
combination does at least as well) the remaining squared energy error is ||e||_A^2 (1 - rho) with
rho = (c . r_g)^2 / ((c . A c) (e . r_g)), r_g = A e. The loss is 1 - rho (invariant to the scale of
c). Forward and reverse pass, the loss and Adam all run in the kernels of ``csrc/mas_ws_train.cu``
(BF16 tensor-core products with FP32 accumulation); one Adam step per sample, cosine-annealed
learning rate.

Run ``python -m polysolve_b200.warmstart_train --out polysolve_b200/data/warm_start_mpnn.psws`` on a
GPU to regenerate the shipped weights (seeded).
"""

from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import warmstart as W


def initial_params(seed: int = 0) -> np.ndarray:
    """Seeded initial parameters: every weight and bias U(-1/sqrt(fan_in), 1/sqrt(fan_in)), the
    message-passing layers' weights halved and the output layer's scaled by 0.1 (a small initial
    correction)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = np.zeros(W.PARAMS, dtype=np.float32)
    for name, (off, shape) in W.layout().items():
        fan_in = {"w_in": W.FEATURES, "b_in": W.FEATURES, "w_out": W.HIDDEN, "b_out": W.HIDDEN}.get(
            name, 2 * W.HIDDEN)
        bound = 1.0 / math.sqrt(fan_in)
        v = rng.uniform(-bound, bound, size=int(np.prod(shape)))
        if name.startswith("w_") and name[2:].isdigit():
            v *= 0.5
        if name == "w_out":
            v *= 0.1
        out[off:off + v.size] = v
    return out


def default_jobs(seed0: int = 1000, steps: int = 22):
    """About 2000 samples: sequences of 22 steps (20 samples each) on 12^3 to 28^3 grids."""
    rng = np.random.Generator(np.random.PCG64(seed0))
    jobs = []
    for N, count in ((12, 30), (16, 30), (20, 24), (24, 10), (28, 6)):
        for _ in range(count):
            jobs.append((N, int(rng.integers(0, 2 ** 31 - 1)), int(rng.integers(0, 200 - steps)), steps))
    return jobs


# The exact solutions: relative residual 1e-9 (the history guess's error e = x_k - x_g is some 1e-3
# of x_k, far above the solve's error). The systems are solved scaled by SOLVE_SCALE: PCG's absolute
# guard (alpha = 0 once |p.Ap| < 1e-20, MASSolver.cu:53) would otherwise stop it near 1e-9 on these
# unit-load systems. Scaling A and b changes neither x, the features (ratios and a centred log), the
# neighbour weights nor rho.
SOLVE_SCALE = 1e6
SOLVE_PARAMS = {"block_dim": 3, "relative_tolerance": 1e-9, "absolute_tolerance": 0.0, "max_iter": 5000,
                "precision": "fp64", "true_residual_period": 10, "check_period": 1, "initial_guess": "input"}


def collect(trainer, jobs, log=None) -> list[int]:
    """Solve every step of every job's sequence on the GPU and add the samples (steps >= 2) to the
    trainer. Returns the sample indices."""
    from . import Solver, synthetic

    idx = []
    for q, (N, seed, k0, steps) in enumerate(jobs):
        solver = Solver.create("MAS", "")
        solver.set_parameters({"MAS": dict(SOLVE_PARAMS)})
        xs = []
        for k in range(k0, k0 + steps):
            sk, bk = synthetic.workload_sequence60(k, seed=seed, N=N)
            if k == k0:
                solver.set_positions(sk.positions)
            solver.factorize(sk.scipy() * SOLVE_SCALE)
            bs = bk * SOLVE_SCALE
            x = xs[-1].copy() if xs else np.zeros(sk.n)
            solver.solve(bs, x)
            info = solver.get_info()
            if info["solver_status"] != "Reach relative tolerance":
                raise RuntimeError(f"sequence {q} step {k}: {info['solver_status']}")
            if len(xs) >= 2:
                hist = [xs[-j] for j in range(1, min(len(xs), W.HISTORY) + 1)]
                idx.append(trainer.add_sample(solver, bs, hist, x))
            xs.append(x)
        if log and (q + 1) % 10 == 0:
            log(f"collected {q + 1}/{len(jobs)} sequences, {len(idx)} samples")
    return idx


def train(trainer, samples, *, epochs: int = 15, lr: float = 2e-3, seed: int = 0, val_fraction: float = 0.1,
          log=print) -> dict:
    """Adam over the training samples (one step per sample, shuffled every epoch, cosine-annealed
    learning rate); rho of the held-out samples after every epoch."""
    rng = np.random.Generator(np.random.PCG64(seed))
    order = rng.permutation(np.asarray(samples))
    nval = max(1, int(len(order) * val_fraction))
    val, tr = order[:nval], order[nval:]
    total = epochs * len(tr)
    history = []
    step = 0
    t_train = 0.0
    rho0 = float(np.mean(trainer.evaluate(val)))
    for ep in range(epochs):
        perm = rng.permutation(tr)
        lrs = np.array([0.5 * lr * (1.0 + math.cos(math.pi * (step + i) / total)) for i in range(len(perm))],
                       dtype=np.float32)
        t0 = time.perf_counter()
        losses = trainer.train(perm, lrs)
        t_train += time.perf_counter() - t0
        step += len(perm)
        vr = float(np.mean(trainer.evaluate(val)))
        history.append({"epoch": ep, "train_loss": float(np.mean(losses)), "val_rho": vr})
        log(f"epoch {ep}: train loss {np.mean(losses):.4f}  val rho {vr:.4f}")
    return {"val_rho": history[-1]["val_rho"] if history else rho0, "val_rho_initial": rho0, "epochs": epochs,
            "train_samples": int(len(tr)), "val_samples": int(nval), "train_seconds": t_train,
            "history": history}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=str(W.DEFAULT_WEIGHTS))
    ap.add_argument("--epochs", type=int, default=15)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--sequences", type=int, default=0, help="limit the number of sequences (0: all)")
    ap.add_argument("--report", default="", help="write a JSON summary here")
    args = ap.parse_args(argv)
    from . import WarmStartTrainer

    jobs = default_jobs()
    if args.sequences:
        jobs = jobs[:: max(1, len(jobs) // args.sequences)][: args.sequences]
    trainer = WarmStartTrainer(initial_params(args.seed))
    t0 = time.perf_counter()
    samples = collect(trainer, jobs, log=lambda s: print(s, flush=True))
    t_collect = time.perf_counter() - t0
    print(f"{len(samples)} samples from {len(jobs)} sequences in {t_collect:.0f}s (GPU solves)", flush=True)
    rep = train(trainer, samples, epochs=args.epochs, lr=args.lr, seed=args.seed,
                log=lambda s: print(s, flush=True))
    W.save(args.out, trainer.params())
    rep.update(samples=len(samples), sequences=len(jobs), collect_seconds=t_collect)
    print(f"wrote {args.out} (validation rho {rep['val_rho']:.4f}, training {rep['train_seconds']:.1f}s)",
          flush=True)
    if args.report:
        with open(args.report, "w") as fh:
            json.dump(rep, fh, indent=1)


if __name__ == "__main__":
    main()
