"""The allocation-free energy entry point, fz_energy_noalloc, against the handle-based fz_energy.

fz_energy_noalloc exists for callers that cannot allocate device memory -- their fields live in
a pool they manage themselves, or they run where a cudaMalloc (which may synchronise the device)
is not allowed. It takes the caller's device arrays and keeps its reduction scratch in a fixed
array inside the library. These tests call it through the C ABI: on two calls in a row (the
second one reusing the scratch the first left behind) it must give the energy fz_energy gives
for the same fields, and it must refuse sizes beyond its fixed scratch.
"""
import ctypes

import numpy as np
import pytest

from fases_b200 import _abi

# energies are accumulated in FP64 by both entry points; only the summation order differs
TOL = 1e-10


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = _abi.lib()
    dummy = ctypes.c_void_p(256)  # never dereferenced: the size check comes first
    rc = L.fz_energy_noalloc(dummy, dummy, dummy, dummy, _abi.FZ_NOALLOC_MAX_CELLS + 1, 1.2, 343.0, dummy, None)
    assert rc == _abi.FZ_EINVAL
    assert "exceed" in _abi.last_error()
    assert L.fz_energy_noalloc(None, dummy, dummy, dummy, 10, 1.2, 343.0, dummy, None) == _abi.FZ_EINVAL


@pytest.mark.gpu
def test_noalloc_energy_matches_fz_energy_on_two_calls():
    import torch

    from tests.helpers import run_gpu, small_room

    cfg = small_room(seed=21, steps=12)
    s = run_gpu(cfg, "fp32")
    L = _abi.lib()
    stream = torch.cuda.current_stream()
    results = []
    for call in range(2):
        if call == 1:
            s.run(7)  # different fields for the second call
        e_ref = s.energy()
        fields = [torch.tensor(a.astype(np.float32).ravel(), device="cuda") for a in s.fields()]
        out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        rc = L.fz_energy_noalloc(*(t.data_ptr() for t in fields), fields[0].numel(), cfg["rho"], cfg["c"],
                                 out.data_ptr(), stream.cuda_stream)
        assert rc == _abi.FZ_OK, _abi.last_error()
        torch.cuda.synchronize()
        e = out.item()
        assert e_ref > 0
        assert abs(e - e_ref) <= TOL * abs(e_ref), (call, e, e_ref)
        results.append(e)
    assert results[0] != results[1]
    s.close()


@pytest.mark.gpu
def test_noalloc_energy_ragged_many_blocks_and_empty():
    """Caller-owned arrays of a size that needs several blocks with a partial last one (and of
    size zero, where *out must become 0), against an FP64 torch sum of the same formula."""
    import torch

    L = _abi.lib()
    stream = torch.cuda.current_stream()
    rho, c = 1.2, 343.0
    g = torch.Generator(device="cuda").manual_seed(5)
    for n in (3 * 16384 + 5, 1, 0):
        # at least one element of storage each, so that the pointers are valid (never NULL) at n = 0
        store = [torch.randn(max(n, 1), generator=g, device="cuda", dtype=torch.float32) for _ in range(4)]
        fields = [t[:n] for t in store]
        out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        ptrs = [t.data_ptr() for t in store]
        assert all(ptrs)
        rc = L.fz_energy_noalloc(*ptrs, n, rho, c, out.data_ptr(), stream.cuda_stream)
        assert rc == _abi.FZ_OK, _abi.last_error()
        torch.cuda.synchronize()
        p, u, v, w = (t.double() for t in fields)
        want = 0.5 * float((p * p / (rho * c * c) + rho * (u * u + v * v + w * w)).sum())
        got = out.item()
        if n == 0:
            assert got == 0.0
        else:
            assert abs(got - want) <= 1e-12 * abs(want), (n, got, want)
