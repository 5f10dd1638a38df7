"""Kernel parity at the kernel micro-benchmarks' own sizes (the reference
workload's shapes): the commitment LDE of 16 columns of 2^20 -> 2^21, the
Poseidon2 Merkle tree over 2^21 leaves of 16 elements (P24 leaves, P16
nodes), the eq table of a 24-coordinate point (2^24 extension entries), the
extension evaluation and fold of 2^24 entries. Each compares every output word
with the oracle's; the smaller parity tests cover the other shapes."""
import numpy as np
import pytest

from oracle.oracle import P

pytestmark = pytest.mark.gpu


def rnd(rng, n):
    return rng.integers(0, P, n, dtype=np.uint64).astype(np.uint32)


def test_commit_lde_full_size(pkg, gpu_ctx, oracle):
    rng = np.random.default_rng(2024)
    x = rnd(rng, 1 << 24)
    want = oracle.dft_batch(x, 20, 4, 1, False)
    d_in = pkg.DeviceArray.from_host(gpu_ctx, x)
    d_out = pkg.DeviceArray(gpu_ctx, want.size)
    pkg.dft_batch(gpu_ctx, d_in, 20, 4, 1, False, d_out)
    assert np.array_equal(d_out.to_host(), want)


def test_merkle_2pow21_leaves(pkg, gpu_ctx, oracle):
    rng = np.random.default_rng(2121)
    log_h, words = 21, 16
    rows = rnd(rng, words << log_h)
    root_ref, dig_ref = oracle.merkle(rows, log_h, words, 0)
    d_rows = pkg.DeviceArray.from_host(gpu_ctx, rows)
    d_dig = pkg.DeviceArray(gpu_ctx, dig_ref.size)
    root = pkg.merkle_commit(gpu_ctx, d_rows, log_h, words, 0, d_dig)
    assert np.array_equal(root, root_ref)
    assert np.array_equal(d_dig.to_host(), dig_ref)


def test_eq_eval_fold_2pow24(pkg, gpu_ctx, oracle):
    rng = np.random.default_rng(2424)
    n = 24
    point = rnd(rng, 4 * n)
    scale = rnd(rng, 4)
    want = oracle.eq_table(point, tuple(int(v) for v in scale))
    d = pkg.DeviceArray(gpu_ctx, 4 << n)
    pkg.eq_table(gpu_ctx, point, scale, d)
    got = d.to_host()
    assert np.array_equal(got, want)
    # evaluation of the table's values as a multilinear polynomial at another point
    z = rnd(rng, 4 * n)
    assert np.array_equal(pkg.eval_ext(gpu_ctx, d, z), oracle.eval_ext(got, z))
    # one fold 2^24 -> 2^23
    r = rnd(rng, 4)
    want_fold = oracle.fold_ext(got, r)
    pkg.fold_ext(gpu_ctx, d, n, r)
    assert np.array_equal(d.to_host(4 << (n - 1)), want_fold)
