"""Kernel-level parity: every device kernel behind the C ABI against the
oracle on the same seeded inputs, bit for bit (all arithmetic is exact
integer mod p, so the tolerance is zero)."""
import ctypes as C

import numpy as np
import pytest

from oracle.oracle import Chal, P

pytestmark = pytest.mark.gpu


def rnd(rng, n):
    return rng.integers(0, P, n, dtype=np.uint64).astype(np.uint32)


def test_encode_decode_roundtrip(pkg, gpu_ctx):
    rng = np.random.default_rng(0)
    a = np.concatenate([rnd(rng, 1000), np.array([0, 1, P - 1, P - 2], dtype=np.uint32)])
    d = pkg.DeviceArray.from_host(gpu_ctx, a)
    assert np.array_equal(d.to_host(), a)
    # the device copy is Montgomery form
    raw = np.zeros(a.size, dtype=np.uint32)
    pkg._check(pkg.lib().whir_memcpy_d2h(gpu_ctx.handle, raw.ctypes.data, d.ptr, raw.size * 4))
    assert np.array_equal(raw, pkg.mont_encode(a))


DFT_SHAPES = [(0, 0, 0, 0), (0, 2, 3, 1), (3, 1, 1, 0), (5, 2, 3, 1), (10, 4, 1, 0), (12, 4, 1, 0), (13, 4, 1, 0),
              (11, 4, 2, 1), (12, 4, 2, 1), (4, 4, 11, 1), (16, 4, 2, 1), (14, 2, 3, 0), (18, 4, 1, 0), (8, 4, 8, 1),
              (15, 0, 2, 1), (20, 4, 1, 0)]


@pytest.mark.parametrize("log_chunk,log_w,log_blowup,ext", DFT_SHAPES)
def test_dft_batch(pkg, gpu_ctx, oracle, log_chunk, log_w, log_blowup, ext):
    rng = np.random.default_rng(log_chunk * 100 + log_w * 10 + log_blowup + 7 * ext)
    lanes = 4 if ext else 1
    x = rnd(rng, (1 << (log_chunk + log_w)) * lanes)
    want = oracle.dft_batch(x, log_chunk, log_w, log_blowup, bool(ext))
    d_in = pkg.DeviceArray.from_host(gpu_ctx, x)
    d_out = pkg.DeviceArray(gpu_ctx, want.size)
    pkg.dft_batch(gpu_ctx, d_in, log_chunk, log_w, log_blowup, bool(ext), d_out)
    assert np.array_equal(d_out.to_host(), want)


MERKLE_SHAPES = [(0, 16, 0), (1, 16, 0), (5, 16, 0), (9, 64, 0), (12, 16, 0), (8, 2, 0), (7, 1, 0), (10, 8, 1),
                 (6, 64, 1), (3, 5, 1), (14, 16, 0), (11, 64, 0)]


@pytest.mark.parametrize("log_h,row_words,leaf_hash", MERKLE_SHAPES)
def test_merkle_commit_and_open(pkg, gpu_ctx, oracle, log_h, row_words, leaf_hash):
    rng = np.random.default_rng(log_h * 1000 + row_words + leaf_hash)
    rows = rnd(rng, (1 << log_h) * row_words)
    root_ref, dig_ref = oracle.merkle(rows, log_h, row_words, leaf_hash)
    d_rows = pkg.DeviceArray.from_host(gpu_ctx, rows)
    d_dig = pkg.DeviceArray(gpu_ctx, dig_ref.size)
    root = pkg.merkle_commit(gpu_ctx, d_rows, log_h, row_words, leaf_hash, d_dig)
    assert np.array_equal(root, root_ref)
    assert np.array_equal(d_dig.to_host(), dig_ref)
    h = 1 << log_h
    for idx in sorted({0, h - 1, h // 2, int(rng.integers(0, h))}):
        row, path = pkg.merkle_open(gpu_ctx, d_rows, d_dig, log_h, row_words, idx)
        assert np.array_equal(row, rows[idx * row_words:(idx + 1) * row_words])
        off, n = 0, h
        for level in range(log_h):
            sib = (idx >> level) ^ 1
            assert np.array_equal(path[8 * level:8 * level + 8], dig_ref[(off + sib) * 8:(off + sib) * 8 + 8])
            off += n
            n //= 2


@pytest.mark.parametrize("n", [0, 1, 5, 11, 14, 17])
def test_eq_table(pkg, gpu_ctx, oracle, n):
    rng = np.random.default_rng(n + 11)
    z = rnd(rng, 4 * n)
    scale = rnd(rng, 4)
    want = oracle.eq_table(z, scale)
    d = pkg.DeviceArray(gpu_ctx, want.size)
    pkg.eq_table(gpu_ctx, z, scale, d)
    assert np.array_equal(d.to_host(), want)


@pytest.mark.parametrize("n", [0, 1, 2, 8, 9, 12, 13, 17, 20, 23])
def test_eval_base_and_ext(pkg, gpu_ctx, oracle, n):
    rng = np.random.default_rng(n + 21)
    f = rnd(rng, 1 << n)
    fe = rnd(rng, 4 << n)
    z = rnd(rng, 4 * n)
    assert np.array_equal(pkg.eval_base(gpu_ctx, pkg.DeviceArray.from_host(gpu_ctx, f), z), oracle.eval_base(f, z))
    assert np.array_equal(pkg.eval_ext(gpu_ctx, pkg.DeviceArray.from_host(gpu_ctx, fe), z), oracle.eval_ext(fe, z))


@pytest.mark.parametrize("n", [1, 2, 9, 16])
def test_folds(pkg, gpu_ctx, oracle, n):
    rng = np.random.default_rng(n + 31)
    r = rnd(rng, 4)
    fe = rnd(rng, 4 << n)
    d = pkg.DeviceArray.from_host(gpu_ctx, fe)
    pkg.fold_ext(gpu_ctx, d, n, r)
    assert np.array_equal(d.to_host(4 << (n - 1)), oracle.fold_ext(fe, r))
    fb = rnd(rng, 1 << n)
    db = pkg.DeviceArray.from_host(gpu_ctx, fb)
    out = pkg.DeviceArray(gpu_ctx, 4 << (n - 1))
    pkg.fold_base(gpu_ctx, db, n, r, out)
    assert np.array_equal(out.to_host(), oracle.fold_base(fb, r))
    for k in range(0, min(n, 6) + 1):
        rs = rnd(rng, 4 * k)
        out = pkg.DeviceArray(gpu_ctx, 4 << (n - k))
        pkg.fold_multi_base(gpu_ctx, db, n, rs, out)
        assert np.array_equal(out.to_host(), oracle.fold_multi_base(fb, rs)), k


@pytest.mark.parametrize("n", [1, 2, 7, 15, 19])
def test_sumcheck_coeffs(pkg, gpu_ctx, oracle, n):
    rng = np.random.default_rng(n + 41)
    f, w = rnd(rng, 4 << n), rnd(rng, 4 << n)
    c0, c2 = pkg.sumcheck_coeffs(gpu_ctx, pkg.DeviceArray.from_host(gpu_ctx, f), pkg.DeviceArray.from_host(gpu_ctx, w), n)
    r0, r2 = oracle.sumcheck_coeffs(f, w)
    assert np.array_equal(c0, r0) and np.array_equal(c2, r2)


@pytest.mark.parametrize("n,m", [(0, 1), (3, 2), (10, 3), (14, 1), (16, 5)])
def test_combine_eq(pkg, gpu_ctx, oracle, n, m):
    rng = np.random.default_rng(n * 10 + m)
    w = rnd(rng, 4 << n)
    pts = rnd(rng, 4 * n * m)
    g = rnd(rng, 4 * m)
    want = w.astype(np.uint64)
    for i in range(m):
        want = (want + oracle.eq_table(pts[4 * n * i:4 * n * (i + 1)], g[4 * i:4 * i + 4]).astype(np.uint64)) % P
    d = pkg.DeviceArray.from_host(gpu_ctx, w)
    pkg.combine_eq(gpu_ctx, d, n, pts, g)
    assert np.array_equal(d.to_host(), want.astype(np.uint32))


@pytest.mark.parametrize("n,m", [(0, 1), (1, 3), (5, 7), (8, 20), (12, 91), (16, 44)])
def test_combine_select(pkg, gpu_ctx, oracle, n, m):
    rng = np.random.default_rng(n * 100 + m)
    w = rnd(rng, 4 << n)
    vars_ = rnd(rng, m)
    vars_[0] = 0
    g = rnd(rng, 4 * m)
    d = pkg.DeviceArray.from_host(gpu_ctx, w)
    pkg.combine_select(gpu_ctx, d, n, vars_, g)
    assert np.array_equal(d.to_host(), oracle.combine_select(w, vars_, g))


# from 2^12 elements per segment the base-field dot streams through shared
# memory by bulk copies (one 4096-element chunk per stage)
@pytest.mark.parametrize("n,l", [(1, 1), (4, 4), (9, 3), (14, 4), (16, 4), (20, 6), (21, 3), (22, 8)])
def test_svo_partial_evals(pkg, gpu_ctx, oracle, n, l):
    rng = np.random.default_rng(n + 100 * l)
    f = rnd(rng, 1 << n)
    z = rnd(rng, 4 * n)
    parts, ev = pkg.svo_partial_evals(gpu_ctx, pkg.DeviceArray.from_host(gpu_ctx, f), n, l, z)
    assert np.array_equal(ev, oracle.eval_base(f, z))
    m = 1 << (n - l)
    for y in range(1 << l):
        assert np.array_equal(parts[4 * y:4 * y + 4], oracle.eval_base(f[y * m:(y + 1) * m], z[4 * l:]))


@pytest.mark.parametrize("window", [0, 3])
@pytest.mark.parametrize("bits", [1, 3, 8, 11, 12, 16])
def test_grind_smallest_witness(pkg, gpu_ctx, oracle, bits, window):
    """The smallest witness at every sponge position, with the latency window
    and with both lean windows (four-lane searches up to 11 bits, one-thread
    searches above)."""
    rng = np.random.default_rng(bits)
    ch = pkg.DuplexChallenger(gpu_ctx)
    oc = Chal()
    oracle.lib.or_chal_init(C.byref(oc))
    gpu_ctx.set_grind_window(window)
    try:
        for pending in range(8):  # the witness lands at position `pending` of the sponge
            vals = rnd(rng, 8 + pending)
            ch.observe_slice(vals)
            for v in vals:
                oracle.lib.or_chal_observe(C.byref(oc), C.byref(oracle.p16), int(v))
            w = ch.grind(bits)
            w_ref = oracle.lib.or_chal_grind(C.byref(oc), C.byref(oracle.p16), bits)
            assert w == w_ref
            assert list(ch.c.state) == list(oc.state)
    finally:
        gpu_ctx.set_grind_window(0)


def test_invalid_arguments_raise(pkg, gpu_ctx):
    d = pkg.DeviceArray(gpu_ctx, 64)
    with pytest.raises(pkg.WhirError):
        pkg.fold_multi_base(gpu_ctx, d, 8, np.zeros(28, np.uint32), d)  # k = 7 > 6
    with pytest.raises(pkg.WhirError):
        pkg.fold_ext(gpu_ctx, d, 0, np.zeros(4, np.uint32))
    with pytest.raises(pkg.WhirError):
        pkg.eval_base(gpu_ctx, d, np.full(4, P, np.uint32))  # non-canonical point
