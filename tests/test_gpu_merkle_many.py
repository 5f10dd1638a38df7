"""Many independent Merkle trees committed together by the multi-instance
kernels (one leaf launch over all trees' leaves from a work queue, one launch
per level across the trees): every digest array and root equals the
single-tree commitment (which the other GPU tests tie to the oracle), for
uneven heights including one-leaf trees, both Poseidon2 leaf hashes and
base / extension row widths."""
import numpy as np
import pytest

from oracle.oracle import P

pytestmark = pytest.mark.gpu


def rnd(rng, n):
    return rng.integers(0, P, n, dtype=np.uint64).astype(np.uint32)


@pytest.mark.parametrize("row_words,leaf_hash,heights", [
    (16, 0, [0, 1, 2, 5, 9, 12, 13, 3]),
    (8, 1, [4, 0, 11, 7, 7, 1]),
    (64, 0, [6, 10, 2, 0]),
    (16, 0, [14]),
    (3, 1, [5, 2, 8]),
])
def test_many_trees_match_single_commits(pkg, gpu_ctx, oracle, row_words, leaf_hash, heights):
    rng = np.random.default_rng(sum(heights) + row_words)
    rows = [rnd(rng, row_words << h) for h in heights]
    d_rows = [pkg.DeviceArray.from_host(gpu_ctx, r) for r in rows]
    d_dig = [pkg.DeviceArray(gpu_ctx, (2 * (1 << h) - 1) * 8) for h in heights]
    roots = pkg.merkle_commit_many(gpu_ctx, d_rows, heights, row_words, leaf_hash, d_dig)
    for i, h in enumerate(heights):
        one = pkg.DeviceArray(gpu_ctx, (2 * (1 << h) - 1) * 8)
        root = pkg.merkle_commit(gpu_ctx, d_rows[i], h, row_words, leaf_hash, one)
        assert np.array_equal(roots[i], root), i
        assert np.array_equal(d_dig[i].to_host(), one.to_host()), i
    # one tree straight against the oracle
    i = int(np.argmax(heights))
    root_ref, dig_ref = oracle.merkle(rows[i], heights[i], row_words, leaf_hash)
    assert np.array_equal(roots[i], root_ref)


def test_many_trees_at_the_limit(pkg, gpu_ctx):
    """256 trees (the most one call takes) of 1 to 64 leaves."""
    rng = np.random.default_rng(256)
    heights = [int(h) for h in rng.integers(0, 7, 256)]
    rows = [pkg.DeviceArray.from_host(gpu_ctx, rnd(rng, 16 << h)) for h in heights]
    digs = [pkg.DeviceArray(gpu_ctx, (2 * (1 << h) - 1) * 8) for h in heights]
    roots = pkg.merkle_commit_many(gpu_ctx, rows, heights, 16, 0, digs)
    for i in (0, 17, 128, 255):
        one = pkg.DeviceArray(gpu_ctx, (2 * (1 << heights[i]) - 1) * 8)
        assert np.array_equal(roots[i], pkg.merkle_commit(gpu_ctx, rows[i], heights[i], 16, 0, one))


def test_many_trees_rejects_bad_arguments(pkg, gpu_ctx):
    rng = np.random.default_rng(3)
    rows = [pkg.DeviceArray.from_host(gpu_ctx, rnd(rng, 16 << 3))]
    digs = [pkg.DeviceArray(gpu_ctx, 15 * 8)]
    with pytest.raises(pkg.WhirError):
        pkg.merkle_commit_many(gpu_ctx, rows, [3], 16, 2, digs)  # Keccak trees are not batched
    with pytest.raises(pkg.WhirError):
        pkg.merkle_commit_many(gpu_ctx, rows, [31], 16, 0, digs)
    with pytest.raises(pkg.WhirError):
        pkg.merkle_commit_many(gpu_ctx, [], [], 16, 0, [])
