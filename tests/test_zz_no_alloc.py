"""The SpMV + dot entry point that allocates nothing (mas_spmv_dot_noalloc).

It exists for callers that cannot allocate device memory when they call it -- inside a CUDA stream
capture, or in applications that reserve all device memory up front. Its reduction scratch is a
static device array shared by all calls. This file is collected last on purpose, so a run that stops
at the first failure has already run every other test.
"""

from __future__ import annotations

import numpy as np
import pytest

from polysolve_b200 import Solver, synthetic

pytestmark = pytest.mark.gpu


def test_spmv_dot_noalloc_matches_existing_entry_point():
    torch = pytest.importorskip("torch")
    system = synthetic.elasticity(7, young_sigma=1.0, jitter=0.2, seed=40)
    s = Solver.create("MAS", "")
    s.set_parameters({"MAS": {"block_dim": 3}})
    s.set_positions(system.positions)
    s.factorize(system.scipy())
    length = s.sizes()["nodes"] * 3
    stream = torch.cuda.current_stream()
    free_after_first = None
    # Two calls in a row, each checked against the existing SpMV entry point (mas_debug_spmv) and a
    # dot of its result, at the SpMV parity tolerance (1e-12 relative).
    for seed in (0, 1):
        x = np.random.default_rng(seed).standard_normal(length)
        y_ref = s.debug_spmv(x)
        dx = torch.tensor(x, device="cuda")
        dy = torch.full_like(dx, np.nan)
        dd = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        s.spmv_dot_noalloc(dx.data_ptr(), dy.data_ptr(), dd.data_ptr(), length, stream.cuda_stream)
        torch.cuda.synchronize()
        if free_after_first is None:
            free_after_first = torch.cuda.mem_get_info()[0]
        else:
            # nothing was allocated on the device by the second call
            assert torch.cuda.mem_get_info()[0] == free_after_first
        y = dy.cpu().numpy()
        assert np.linalg.norm(y - y_ref) <= 1e-12 * np.linalg.norm(y_ref)
        dot_ref = float(np.dot(x, y_ref))
        assert abs(float(dd.item()) - dot_ref) <= 1e-12 * np.linalg.norm(x) * np.linalg.norm(y_ref)


def test_spmv_dot_noalloc_rejects_bad_length():
    torch = pytest.importorskip("torch")
    from polysolve_b200 import MasError

    system = synthetic.elasticity(3, seed=41)
    s = Solver.create("MAS", "")
    s.set_parameters({"MAS": {"block_dim": 3}})
    s.factorize(system.scipy())
    length = s.sizes()["nodes"] * 3
    dx = torch.zeros(length, dtype=torch.float64, device="cuda")
    with pytest.raises(MasError) as e:
        s.spmv_dot_noalloc(dx.data_ptr(), dx.data_ptr(), dx.data_ptr(), length - 3)
    assert "len must be" in str(e.value)
