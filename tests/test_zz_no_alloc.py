"""Allocation-free sumcheck entry point (whir_sumcheck_coeffs_noalloc).

Callers that cannot allocate device memory on this path (a host application
that hands out all device memory from its own pool, or a latency-critical loop
where allocation is not allowed) use this entry point: they pass their own
input and output buffers and the library keeps the per-block partial sums in a
fixed array of its own. This file is collected last so that a run stopping at
its first failure has already run every other test.

The test calls the entry point through the C ABI twice in a row, with
different inputs and sizes, and checks each result against the existing
whir_sumcheck_coeffs entry point exactly (the tests' tolerance for this exact
integer arithmetic is zero). It also checks that an out-of-range size is
rejected before any launch.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P = 0x7F000001


def _entry(pkg):
    fn = pkg.lib().whir_sumcheck_coeffs_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
    return fn


def _device_sync():
    import torch

    torch.cuda.synchronize()


def test_noalloc_matches_existing_entry_point_twice(pkg, gpu_ctx):
    fn = _entry(pkg)
    rng = np.random.default_rng(4242)
    for n in (18, 11):  # two calls in a row reuse the same scratch array
        f = rng.integers(0, P, 4 << n, dtype=np.uint64).astype(np.uint32)
        w = rng.integers(0, P, 4 << n, dtype=np.uint64).astype(np.uint32)
        d_f = pkg.DeviceArray.from_host(gpu_ctx, f)
        d_w = pkg.DeviceArray.from_host(gpu_ctx, w)
        d_out = pkg.DeviceArray(gpu_ctx, 8)
        _device_sync()
        rc = fn(d_f.ptr, d_w.ptr, n, d_out.ptr, None)
        assert rc == 0, pkg.lib().whir_last_error().decode()
        _device_sync()
        got = d_out.to_host()
        c0, c2 = pkg.sumcheck_coeffs(gpu_ctx, d_f, d_w, n)
        assert np.array_equal(got[:4], c0)
        assert np.array_equal(got[4:], c2)


@pytest.mark.parametrize("max_blocks", [1, 7, 100, 2048])
def test_capped_block_count_matches(pkg, gpu_ctx, max_blocks):
    """The allocation-free entry point caps its reduction at 2048 blocks, above
    the grid a B200 picks (8 CTAs per SM); the capped path, with caps below
    the natural grid, gives the same coefficients as the uncapped one."""
    rng = np.random.default_rng(900 + max_blocks)
    for n in (19, 9):
        f = rng.integers(0, P, 4 << n, dtype=np.uint64).astype(np.uint32)
        w = rng.integers(0, P, 4 << n, dtype=np.uint64).astype(np.uint32)
        d_f = pkg.DeviceArray.from_host(gpu_ctx, f)
        d_w = pkg.DeviceArray.from_host(gpu_ctx, w)
        want = pkg.sumcheck_coeffs(gpu_ctx, d_f, d_w, n)
        got = pkg.sumcheck_coeffs_shaped(gpu_ctx, d_f, d_w, n, max_blocks)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_noalloc_rejects_sizes_beyond_the_maximum(pkg, gpu_ctx):
    fn = _entry(pkg)
    d = pkg.DeviceArray(gpu_ctx, 64)
    assert fn(d.ptr, d.ptr, 31, d.ptr, None) == -1
    assert fn(d.ptr, d.ptr, 0, d.ptr, None) == -1
    assert fn(None, d.ptr, 4, d.ptr, None) == -1
