"""The sort entry point that allocates nothing: tg_sort_pairs_noalloc.

Some callers of this library cannot allocate device memory -- a plugin host
that owns every GPU buffer and hands the library only its own, a real-time
loop where cudaMalloc's implicit device synchronisation is not acceptable, a
host without a caching allocator.  For them tg_sort_pairs_noalloc sorts with
its scratch kept in a static device array inside the library, so the caller
passes only keys, values and their ping-pong buffers.

The GPU test calls it through the C ABI and checks that it returns exactly
what tg_sort_pairs (caller-provided workspace) returns, on two calls in a row
-- the second at the size limit with all 64 key bits, the largest scratch the
static array must hold -- because every call reuses the same static scratch and
must start from a cleared state.  A second GPU test makes a bounded look-back
wait give up inside that static scratch (tg_sort_noalloc_lookback_selftest) and
checks that tg_sort_noalloc_status reports it, and that the next sort clears
it.  This file is named so that pytest collects it after every other test file.
"""
import ctypes

import numpy as np
import pytest
import torch

from textured_gaussians_b200 import _backend as B

MAX_PAIRS = 4194304  # TG_SORT_NOALLOC_MAX_PAIRS in include/tg2dgs.h


def _noalloc():
    fn = B.lib().tg_sort_pairs_noalloc
    fn.argtypes = [B.P, B.P, B.P, B.P, B.I64, B.I32, ctypes.POINTER(B.I32), B.P]
    fn.restype = ctypes.c_int
    return fn


def _keys(n, distinct, seed, end_bit):
    rng = np.random.default_rng(seed)
    if end_bit == 64:  # every bit sorted, negative int64 values included (the sort orders them as unsigned)
        return rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, size=n, dtype=np.int64)
    k = rng.integers(0, distinct, size=n, dtype=np.int64) * np.int64(0x9E3779B1) + rng.integers(0, 5, size=n)
    return (k & np.int64((1 << 60) - 1)) | (np.int64(1) << np.int64(61))  # bit 61 lies outside every sorted range


def _status():
    fn = B.lib().tg_sort_noalloc_status
    fn.argtypes = [B.P]
    fn.restype = ctypes.c_int
    return fn


def _workspace_sort(keys, vals, end_bit, stream):
    n = keys.numel()
    ka, va = torch.empty_like(keys), torch.empty_like(vals)
    wsb = B.lib().tg_sort_workspace_bytes(n, end_bit)
    ws = torch.empty((wsb,), dtype=torch.uint8, device=keys.device)
    in_alt = ctypes.c_int32(0)
    rc = B.lib().tg_sort_pairs(B.ptr(keys), B.ptr(vals), B.ptr(ka), B.ptr(va), n, end_bit, B.ptr(ws), wsb,
                               ctypes.byref(in_alt), stream)
    assert rc == 0, B.lib().tg_last_error()
    return (ka, va) if in_alt.value else (keys, vals)


@pytest.mark.gpu
def test_noalloc_sort_matches_workspace_sort_on_two_calls_in_a_row():
    fn = _noalloc()
    dev = torch.device("cuda:0")
    s = torch.cuda.Stream(dev)
    with torch.cuda.stream(s):
        for call, (n, end_bit, distinct) in enumerate([(1_000_003, 48, 1 << 20), (MAX_PAIRS, 64, 0)]):
            keys = torch.from_numpy(_keys(n, distinct, call, end_bit)).to(dev)
            vals = torch.arange(n, dtype=torch.int32, device=dev)
            ref_k, ref_v = _workspace_sort(keys.clone(), vals.clone(), end_bit, s.cuda_stream)
            k, v = keys.clone(), vals.clone()
            ka, va = torch.empty_like(k), torch.empty_like(v)
            in_alt = ctypes.c_int32(-1)
            rc = fn(B.ptr(k), B.ptr(v), B.ptr(ka), B.ptr(va), n, end_bit, ctypes.byref(in_alt), s.cuda_stream)
            assert rc == 0, B.lib().tg_last_error()
            got_k, got_v = (ka, va) if in_alt.value else (k, v)
            s.synchronize()
            assert torch.equal(got_k, ref_k), f"keys differ on call {call}"
            assert torch.equal(got_v, ref_v), f"values differ on call {call}"
            assert _status()(s.cuda_stream) == 0, B.lib().tg_last_error()


@pytest.mark.gpu
def test_noalloc_sort_reports_a_lookback_timeout_in_its_static_scratch():
    st = B.lib().tg_sort_noalloc_lookback_selftest
    st.argtypes = [B.P, B.P, B.P, B.P, B.P]
    st.restype = ctypes.c_int
    dev = torch.device("cuda:0")
    s = torch.cuda.Stream(dev)
    n = 8192
    with torch.cuda.stream(s):
        keys = torch.from_numpy(_keys(n, 1 << 12, 7, 48)).to(dev)
        vals = torch.arange(n, dtype=torch.int32, device=dev)
        ka, va = torch.empty_like(keys), torch.empty_like(vals)
        rc = st(B.ptr(keys), B.ptr(vals), B.ptr(ka), B.ptr(va), s.cuda_stream)
        assert rc == -5, (rc, B.lib().tg_last_error())  # TG_ERR_TIMEOUT: the wait gave up, the kernel returned
        assert _status()(s.cuda_stream) == -5
        assert b"gave up" in B.lib().tg_last_error()
        # the context is still usable and the next sort clears the flag
        fn = _noalloc()
        in_alt = ctypes.c_int32(-1)
        k, v = keys.clone(), vals.clone()
        rc = fn(B.ptr(k), B.ptr(v), B.ptr(ka), B.ptr(va), n, 48, ctypes.byref(in_alt), s.cuda_stream)
        assert rc == 0, B.lib().tg_last_error()
        assert _status()(s.cuda_stream) == 0
        got_k = ka if in_alt.value else k
        s.synchronize()
        ref = np.sort(keys.cpu().numpy().view(np.uint64), kind="stable").view(np.int64)
        assert np.array_equal(got_k.cpu().numpy(), ref)


def test_noalloc_sort_rejects_sizes_over_its_static_scratch():
    fn = _noalloc()
    in_alt = ctypes.c_int32(-1)
    rc = fn(None, None, None, None, MAX_PAIRS + 1, 48, ctypes.byref(in_alt), None)
    assert rc == -1 and in_alt.value == 0
    assert b"4194304" in B.lib().tg_last_error()
