"""The SpMV + dot entry point that allocates nothing (mas_spmv_dot_noalloc).

It exists for callers that cannot allocate device memory when they call it -- inside a CUDA stream
capture, or in applications that reserve all device memory up front. Its reduction scratch is a
static device array shared by all calls. This file is collected last on purpose, so a run that stops
at the first failure has already run every other test.
"""

from __future__ import annotations

import numpy as np
import pytest

from polysolve_b200 import MasError, Solver, synthetic

pytestmark = pytest.mark.gpu


def _factorized(N, seed):
    system = synthetic.elasticity(N, young_sigma=1.0, jitter=0.2, seed=seed)
    s = Solver.create("MAS", "")
    s.set_parameters({"MAS": {"block_dim": 3}})
    s.set_positions(system.positions)
    s.factorize(system.scipy())
    return s, s.sizes()["nodes"] * 3


def _check(s, x, y, dot):
    """y and dot against the existing SpMV entry point (mas_debug_spmv) at the SpMV parity
    tolerance (1e-12 relative)."""
    y_ref = s.debug_spmv(x)
    assert np.linalg.norm(y - y_ref) <= 1e-12 * np.linalg.norm(y_ref)
    dot_ref = float(np.dot(x, y_ref))
    assert abs(dot - dot_ref) <= 1e-12 * np.linalg.norm(x) * np.linalg.norm(y_ref)


def test_spmv_dot_noalloc_matches_existing_entry_point():
    torch = pytest.importorskip("torch")
    # Another handle's call first loads the module and its static array on this device (lazy
    # module loading), so the free-memory readings below see only what the calls themselves do.
    warm, wlen = _factorized(3, 39)
    wx = torch.ones(wlen, dtype=torch.float64, device="cuda")
    wy, wd = torch.empty_like(wx), torch.empty(1, dtype=torch.float64, device="cuda")
    warm.spmv_dot_noalloc(wx.data_ptr(), wy.data_ptr(), wd.data_ptr(), wlen)
    torch.cuda.synchronize()

    s, length = _factorized(7, 40)
    stream = torch.cuda.current_stream()
    dx = torch.empty(length, dtype=torch.float64, device="cuda")
    dy = torch.empty_like(dx)
    dd = torch.empty(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    # Two calls in a row, each checked against the existing entry point.
    for seed in (0, 1):
        x = np.random.default_rng(seed).standard_normal(length)
        dx.copy_(torch.from_numpy(x))
        dy.fill_(np.nan)
        dd.fill_(np.nan)
        torch.cuda.synchronize()
        s.spmv_dot_noalloc(dx.data_ptr(), dy.data_ptr(), dd.data_ptr(), length, stream.cuda_stream)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free_before  # nothing was allocated on the device
        _check(s, x, dy.cpu().numpy(), float(dd.item()))


def test_spmv_dot_noalloc_inside_stream_capture():
    """The call can be captured into a CUDA graph (cudaMalloc would end the capture with an error)
    and each replay recomputes y and the dot from the current x, starting its ticket from zero."""
    torch = pytest.importorskip("torch")
    s, length = _factorized(6, 42)
    dx = torch.zeros(length, dtype=torch.float64, device="cuda")
    dy = torch.empty_like(dx)
    dd = torch.empty(1, dtype=torch.float64, device="cuda")
    s.spmv_dot_noalloc(dx.data_ptr(), dy.data_ptr(), dd.data_ptr(), length)  # uncaptured first call
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        s.spmv_dot_noalloc(dx.data_ptr(), dy.data_ptr(), dd.data_ptr(), length,
                           torch.cuda.current_stream().cuda_stream)
    for seed in (3, 4):
        x = np.random.default_rng(seed).standard_normal(length)
        dx.copy_(torch.from_numpy(x))
        dy.fill_(np.nan)
        dd.fill_(np.nan)
        g.replay()
        torch.cuda.synchronize()
        _check(s, x, dy.cpu().numpy(), float(dd.item()))
    del g


def test_spmv_dot_noalloc_rejects_bad_length_and_overlap():
    torch = pytest.importorskip("torch")
    s, length = _factorized(3, 41)
    dx = torch.zeros(2 * length + 8, dtype=torch.float64, device="cuda")
    with pytest.raises(MasError) as e:
        s.spmv_dot_noalloc(dx.data_ptr(), dx.data_ptr(), dx.data_ptr(), length - 3)
    assert "len must be" in str(e.value)
    x_ptr = dx.data_ptr()
    y_ptr = x_ptr + 8 * (length + 1)
    d_ptr = x_ptr + 8 * (2 * length + 4)
    # in place, partially overlapping vectors, the dot inside x or inside y
    for args in ((x_ptr, x_ptr, d_ptr), (x_ptr, x_ptr + 8 * 5, d_ptr), (x_ptr, y_ptr, x_ptr + 8 * 3),
                 (x_ptr, y_ptr, y_ptr + 8 * (length - 1))):
        with pytest.raises(MasError) as e:
            s.spmv_dot_noalloc(*args, length)
        assert "must not overlap" in str(e.value)
    # disjoint buffers inside one allocation are fine
    s.spmv_dot_noalloc(x_ptr, y_ptr, d_ptr, length)
    torch.cuda.synchronize()
