"""Generates tests/golden/*.npz: small seeded systems with the CPU oracle's outputs.

The reference ships no golden vectors for MAS (its tests assert residual thresholds on data that
is not distributed), so these fixtures are the oracle's own answers on fixed inputs: the matrix,
the Morton partition, the coarse-space maps and counts, one preconditioner application and the
reference-mode PCG result. They pin the oracle (tests/test_cpu_oracle.py) and serve as known
answers for the GPU path (tests/test_gpu_golden.py).

Run from the repository root:  python tests/golden/make_golden.py
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from polysolve_b200 import synthetic  # noqa: E402

CASES = {
    "grid3": dict(N=3, kw=dict(seed=1)),
    "grid4_jitter": dict(N=4, kw=dict(young_sigma=1.0, jitter=0.2, seed=2)),
    "grid5_contact": dict(N=5, kw=dict(young_sigma=1.0, jitter=0.2, seed=3, contact_pairs=30)),
}


def make(name: str, N: int, kw: dict) -> dict:
    s = synthetic.elasticity(N, **kw)
    iso = O.isolated_blocks(s.outer, s.inner, s.n, 3)
    padded = O.morton_padded(s.positions, iso)
    perm, offsets = O.partition_from_padded(padded)
    orc = O.MasOracle(s.outer, s.inner, s.vals, s.n, 3, perm, offsets)
    r2p, cmap = orc.maps()
    r = np.random.Generator(np.random.PCG64(100)).standard_normal(orc.s.V * 3)
    z = orc.apply(r)
    b = synthetic.rhs(s.n, seed=101)
    x, info = orc.pcg(b, rel_tol=1e-8, abs_tol=0.0)
    return dict(n=s.n, outer=s.outer, inner=s.inner, vals=s.vals, positions=s.positions, padded=padded,
                perm=perm, offsets=offsets, r2p=r2p, cmap=cmap, cco_nums=orc.s.cco_nums,
                level_num=orc.s.level_num, mat_counts=orc.s.mat_counts, r=r, z=z, b=b, x=x,
                iters=info["solver_iter"], res=info["solver_error"])


def main() -> None:
    out = Path(__file__).resolve().parent
    for name, c in CASES.items():
        d = make(name, c["N"], c["kw"])
        np.savez_compressed(out / f"{name}.npz", **d)
        print(name, d["n"], "iters", d["iters"], "levels", d["level_num"], d["cco_nums"])


if __name__ == "__main__":
    main()
