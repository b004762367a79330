"""GPU scan and radix sort through the C ABI against exact CPU results
(the reference's cases, tests/gpu_parity_tests.rs:513-662, plus larger sizes)."""
import numpy as np
import pytest
import torch

from cindergs_b200 import exclusive_scan_u32, radix_sort_u32_pairs, radix_sort_u64_pairs

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def host(t, dtype=np.uint32):
    return t.cpu().numpy().view(dtype)


@pytest.mark.parametrize("n", [0, 1, 17, 512, 513, 4095, 4096, 4097, 100_000, 300_000, 5_000_000])
def test_scan(gpu_state, n):
    x = ((np.arange(n, dtype=np.uint64) * 37 + 11) % 7).astype(np.uint32)
    d_in = dev(x) if n else torch.zeros(1, dtype=torch.int32, device="cuda")
    d_out = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    total = exclusive_scan_u32(gpu_state, d_in.data_ptr(), d_out.data_ptr(), n)
    exp = np.zeros(n, np.uint64)
    if n:
        exp[1:] = np.cumsum(x[:-1], dtype=np.uint64)
    assert total == int(x.sum(dtype=np.uint64))
    np.testing.assert_array_equal(host(d_out)[:n], exp.astype(np.uint32))


@pytest.mark.parametrize("digit_bits", [8, 4])
@pytest.mark.parametrize("n", [0, 1, 317, 4096, 50_000, 3_000_000])
def test_radix_u32(gpu_state, n, digit_bits):
    i = np.arange(n, dtype=np.uint64)
    keys = (((i * 2654435761) >> 16) & 0x00FF0FFF).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    dk = dev(keys) if n else torch.zeros(1, dtype=torch.int32, device="cuda")
    dv = dev(vals) if n else torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    radix_sort_u32_pairs(gpu_state, dk.data_ptr(), dv.data_ptr(), n, 24, digit_bits)
    order = np.lexsort((vals, keys))
    np.testing.assert_array_equal(host(dk)[:n], keys[order])
    np.testing.assert_array_equal(host(dv)[:n], vals[order])


@pytest.mark.parametrize("key_bits", [1, 7, 13, 17, 31, 32])
def test_radix_u32_partial_bits_stable(gpu_state, key_bits):
    n = 200_000
    rng = np.random.default_rng(key_bits)
    keys = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    dk, dv = dev(keys), dev(vals)
    torch.cuda.synchronize()
    radix_sort_u32_pairs(gpu_state, dk.data_ptr(), dv.data_ptr(), n, key_bits, 8)
    mask = np.uint32(0xFFFFFFFF if key_bits == 32 else (1 << key_bits) - 1)
    order = np.argsort(keys & mask, kind="stable")
    np.testing.assert_array_equal(host(dv), vals[order])
    np.testing.assert_array_equal(host(dk), keys[order])


@pytest.mark.parametrize("n", [4096, 1_000_000])
def test_radix_u64_tile_depth(gpu_state, n):
    i = np.arange(n, dtype=np.uint64)
    tiles = ((i * 73 + 5) % 19).astype(np.uint32) if n == 4096 else \
        np.random.default_rng(0).integers(0, 129_600, n).astype(np.uint32)
    depths = (np.float32(0.5) + ((i * 19 + 3) % 100).astype(np.float32) * np.float32(0.1)
              ).astype(np.float32).view(np.uint32)
    ids = np.arange(n, dtype=np.uint32)
    dt, dd, di = dev(tiles), dev(depths), dev(ids)
    torch.cuda.synchronize()
    tile_bits = 5 if n == 4096 else 17
    radix_sort_u64_pairs(gpu_state, dt.data_ptr(), dd.data_ptr(), di.data_ptr(), n, tile_bits)
    order = np.lexsort((ids, depths, tiles))
    np.testing.assert_array_equal(host(dt), tiles[order])
    np.testing.assert_array_equal(host(dd), depths[order])
    np.testing.assert_array_equal(host(di), ids[order])
