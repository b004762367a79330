"""The allocation-free pair sort (cgs_sort_pairs_u32_noalloc) against the
context-based one (cgs_sort_pairs_u32).

It exists for callers that cannot let the library call cudaMalloc: an engine
that owns all device memory through its own allocator or budget, or a
real-time loop where an allocation could synchronise the device mid-frame. Its
scratch is a fixed array inside the library, shared by every call, so the test
sorts twice in a row with different data and sizes and checks each result
against the existing entry point exactly (an integer sort has no tolerance).
This file is collected last so a failure here never hides another test.
"""
import ctypes

import numpy as np
import pytest
import torch

from cindergs_b200 import _abi, radix_sort_u32_pairs

pytestmark = pytest.mark.gpu


def _pairs(n, seed, key_bits):
    rng = np.random.default_rng(seed)
    keys = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    if key_bits < 32:
        keys &= np.uint32((1 << key_bits) - 1) | np.uint32(0xF0000000)  # noise above key_bits
    vals = rng.permutation(n).astype(np.uint32)
    return keys, vals


def _dev(a):
    return torch.from_numpy(a.view(np.int32).copy()).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_context_sort_twice(gpu_state):
    lib = _abi.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call, (n, key_bits, digit_bits, seed) in enumerate(
            [(1_000_000, 32, 8, 1), (300_000, 24, 4, 2)]):
        keys, vals = _pairs(n, seed, key_bits)
        ref_k, ref_v = _dev(keys), _dev(vals)
        new_k, new_v = _dev(keys), _dev(vals)
        torch.cuda.synchronize()
        radix_sort_u32_pairs(gpu_state, ref_k.data_ptr(), ref_v.data_ptr(), n, key_bits,
                             digit_bits)
        rc = lib.cgs_sort_pairs_u32_noalloc(ctypes.c_void_p(new_k.data_ptr()),
                                            ctypes.c_void_p(new_v.data_ptr()), n, key_bits,
                                            digit_bits, stream)
        assert rc == _abi.CGS_OK, f"call {call}: status {rc}"
        torch.cuda.synchronize()
        np.testing.assert_array_equal(_host(new_k), _host(ref_k), err_msg=f"keys, call {call}")
        np.testing.assert_array_equal(_host(new_v), _host(ref_v), err_msg=f"values, call {call}")
        mask = np.uint32(0xFFFFFFFF if key_bits == 32 else (1 << key_bits) - 1)
        order = np.argsort(keys & mask, kind="stable")
        np.testing.assert_array_equal(_host(new_v), vals[order], err_msg=f"stable order {call}")


def test_noalloc_sort_rejects_sizes_beyond_its_scratch():
    lib = _abi.load()
    n = 1_048_577  # CGS_NOALLOC_SORT_MAX_PAIRS + 1: rejected on the host, no device work
    k = torch.zeros(n, dtype=torch.int32, device="cuda")
    v = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = lib.cgs_sort_pairs_u32_noalloc(ctypes.c_void_p(k.data_ptr()),
                                        ctypes.c_void_p(v.data_ptr()), n, 32, 8,
                                        ctypes.c_void_p(0))
    assert rc == _abi.CGS_E_CAPACITY
