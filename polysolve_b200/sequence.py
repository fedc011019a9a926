"""Warm starts for a sequence of related systems (a Newton loop or time stepping).

The reference's caller (`nonlinear::Newton`, Newton.cpp:173-214) re-factorizes a matrix with the
same pattern and new values at every step and solves from x0 = 0 (MASSolver.cu:395-398). With
``initial_guess: input`` the solver starts from a caller-supplied x0 instead; this module supplies
it from the previous solutions:

* ``previous``:    x0 = x_{k-1}
* ``extrapolate``: x0 = x_{k-1} + (x_{k-1} - x_{k-2})  (linear in the step index), falling back to
  ``previous`` for the second step and to zero for the first.

The relative tolerance stays relative to ||b_k||, so a good guess directly saves iterations.

``learned`` leaves the guess to the solver (``initial_guess: "learned"``, a network loaded with
``Solver.set_warm_start_model``): it keeps its last four solutions on the device and starts from
the energy-minimising combination of x_{k-1}, the differences of consecutive kept solutions and
the network's correction.
"""

from __future__ import annotations

import numpy as np

MODES = ("zero", "previous", "extrapolate", "learned")


class WarmStart:
    def __init__(self, mode: str = "extrapolate"):
        if mode not in MODES:
            raise ValueError(f"mode must be one of {MODES}")
        self.mode = mode
        self._hist: list[np.ndarray] = []

    def guess(self, n: int) -> np.ndarray | None:
        """x0 for the next step (None: start from zero)."""
        if self.mode in ("zero", "learned") or not self._hist:
            return None
        if self.mode == "previous" or len(self._hist) < 2:
            return self._hist[-1].copy()
        return 2.0 * self._hist[-1] - self._hist[-2]

    def record(self, x: np.ndarray) -> None:
        self._hist.append(np.array(x, dtype=np.float64, copy=True))
        del self._hist[:-2]

    def reset(self) -> None:
        self._hist.clear()


def solve_sequence(solver, systems, rhs, mode: str = "extrapolate", on_step=None, check: bool = True) -> list[dict]:
    """Factorize and solve each (A_k, b_k) with warm starts; returns per-step info (iterations,
    status, relative residual, x0 source). `solver` must have ``initial_guess: input`` for the
    previous / extrapolate modes and ``initial_guess: learned`` for the learned mode;
    the pattern of every A_k must be the same (values-only refactorization). With ``check`` the
    relative residual ||A x - b|| / ||b|| is recomputed on the host (scipy); otherwise it is the
    solver's own reported relative residual."""
    ws = WarmStart(mode)
    out = []
    for k, (A, b) in enumerate(zip(systems, rhs)):
        solver.factorize(A)
        x0 = ws.guess(A.shape[0])
        x = np.zeros(A.shape[0]) if x0 is None else np.ascontiguousarray(x0)
        solver.solve(b, x)
        ws.record(x)
        info = solver.get_info({})
        if check:
            rel = float(np.linalg.norm(A @ x - b) / np.linalg.norm(b))
        else:
            rel = float(info["relative_residual"])
        out.append({"step": k, "iterations": info["solver_iter"], "status": info["solver_status"], "rel": rel,
                    "x0_source": info.get("x0_source", "")})
        if on_step:
            on_step(k, x, info)
    return out


__all__ = ["WarmStart", "solve_sequence", "MODES"]
