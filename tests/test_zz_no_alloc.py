"""The allocation-free FP64 electrogram contraction.

``phs_egm_contract_f64_noalloc`` serves callers that cannot allocate device
memory when they contract -- inside a global-mode stream capture, under another
allocator that owns the device memory, or in loops that cannot absorb
cudaFree's device-wide synchronisation.  Its split-K partial sums live in a
fixed array inside the library instead of a per-call allocation, so its result
must match the allocating entry point ``phs_egm_contract_f64`` on the same
inputs, call after call (the array keeps the previous call's contents).

This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from pyheartsim_b200 import _lib

# FP64 contraction; the two entry points may split K differently, so sums differ
# only by FP64 rounding of the split order
RTOL = 1e-12


def _contract(fn, T, n_v, n_e, V, Mt, out, stream):
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    return fn(T, n_v, n_e, p(V), n_v, p(Mt), p(out), ctypes.c_void_p(stream))


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_twice(cuda_device):
    import torch
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    # calls in a row, different sizes; the last fills the scratch exactly
    # (T * n_e = 2^21), which leaves room for one split-K slice only
    shapes = [(300, 20000, 64), (123, 7777, 40), (2048, 4096, 1024)]
    for call, (T, n_v, n_e) in enumerate(shapes):
        g = torch.Generator(device="cpu").manual_seed(100 + call)
        V = torch.randn(T, n_v, dtype=torch.float64, generator=g).to(cuda_device)
        Mt = torch.randn(n_e, n_v, dtype=torch.float64, generator=g).to(cuda_device)
        ref = torch.empty(T, n_e, dtype=torch.float64, device=cuda_device)
        got = torch.full((T, n_e), float("nan"), dtype=torch.float64, device=cuda_device)
        _lib.check(_contract(L.phs_egm_contract_f64, T, n_v, n_e, V, Mt, ref, stream), "phs_egm_contract_f64")
        _lib.check(_contract(L.phs_egm_contract_f64_noalloc, T, n_v, n_e, V, Mt, got, stream),
                   "phs_egm_contract_f64_noalloc")
        torch.cuda.synchronize()
        r, o = ref.cpu().numpy(), got.cpu().numpy()
        assert np.isfinite(o).all()
        np.testing.assert_allclose(o, r, rtol=RTOL, atol=RTOL * np.abs(r).max())


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = _lib.lib()
    cap = L.phs_egm_noalloc_capacity()
    assert cap == 1 << 21
    # rejected before any device work: T * n_e one past the capacity
    T, n_e = cap // 64 + 1, 64
    rc = L.phs_egm_contract_f64_noalloc(T, 16, n_e, ctypes.c_void_p(16), 16, ctypes.c_void_p(16),
                                        ctypes.c_void_p(16), None)
    assert rc == _lib.PHS_ERR_BAD_ARG
    assert b"exceeds the fixed scratch" in L.phs_last_error()
