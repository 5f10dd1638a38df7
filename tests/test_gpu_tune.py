"""Launch-shape tuner: every candidate shape the tuner may pick (DFT plans,
Merkle leaf/node batch widths, fold tiles) gives the oracle's values bit for
bit, and tuning on first use records a choice no slower than the default."""
import numpy as np
import pytest

from oracle.oracle import P

pytestmark = pytest.mark.gpu


def rnd(rng, n):
    return rng.integers(0, P, n, dtype=np.uint64).astype(np.uint32)


# one-pass shapes (chunk <= 2^12) and four-step shapes, base and extension;
# shapes with a pass of 2^8..2^12 points include register-pass plans
PLAN_SHAPES = [(6, 3, 2, 0), (10, 2, 1, 0), (12, 1, 1, 1), (9, 4, 3, 1), (14, 3, 1, 0), (13, 2, 2, 1),
               (16, 1, 1, 0), (18, 4, 1, 0), (20, 1, 4, 0), (14, 4, 2, 1), (12, 2, 5, 1), (8, 4, 8, 1)]


@pytest.mark.parametrize("log_chunk,log_w,log_blowup,ext", PLAN_SHAPES)
def test_every_dft_plan_matches_oracle(pkg, gpu_ctx, oracle, log_chunk, log_w, log_blowup, ext):
    rng = np.random.default_rng(1000 + log_chunk * 10 + log_w)
    lanes = 4 if ext else 1
    x = rnd(rng, (1 << (log_chunk + log_w)) * lanes)
    want = oracle.dft_batch(x, log_chunk, log_w, log_blowup, bool(ext))
    d_in = pkg.DeviceArray.from_host(gpu_ctx, x)
    d_out = pkg.DeviceArray(gpu_ctx, want.size)
    plans = pkg.dft_plans(log_chunk, log_w, log_blowup, bool(ext))
    assert len(plans) >= 2
    bad = []
    for plan in plans:
        pkg.dft_batch_plan(gpu_ctx, d_in, log_chunk, log_w, log_blowup, bool(ext), plan, d_out)
        if not np.array_equal(d_out.to_host(), want):
            bad.append(plan)
    assert not bad, bad


LEAF_SHAPES = [(128, 0), (128, 8), (128, 16), (256, 0), (256, 4), (256, 8), (256, 16), (512, 0), (512, 2), (512, 4),
               (512, 8)]
# variant bit 0: top kernel (cooperative subtrees / one CTA); bit 1: the two-level
# kernel's permutations one after the other; bit 2: the last two-level step with
# four-lane cooperative permutations
NODE_SHAPES = [(t, s, v) for v in (0, 1, 2, 3) for t, s in [(128, 0), (128, 8), (128, 16), (256, 0), (256, 8), (256, 16)]]
NODE_SHAPES += [(256, 0, 4), (128, 16, 4), (128, 0, 5), (256, 8, 5), (256, 16, 6), (128, 0, 7)]


# 2^17 and 2^13 leaves: leaf-digest kernel, two-level launches and either top
# kernel; 2^12: the smallest leaf-digest tree; 2^9: in-CTA leaf subtrees
@pytest.mark.parametrize("leaf_hash,row_words,log_h", [(0, 16, 17), (1, 8, 13), (0, 64, 12), (1, 16, 9)])
def test_every_merkle_shape_matches_oracle(pkg, gpu_ctx, oracle, leaf_hash, row_words, log_h):
    rng = np.random.default_rng(77 + leaf_hash + 10 * log_h)
    rows = rnd(rng, (1 << log_h) * row_words)
    root_ref, dig_ref = oracle.merkle(rows, log_h, row_words, leaf_hash)
    d_rows = pkg.DeviceArray.from_host(gpu_ctx, rows)
    d_dig = pkg.DeviceArray(gpu_ctx, dig_ref.size)
    shapes = [(t, s, 256, 16, 1) for t, s in LEAF_SHAPES] + [(256, 16, t, s, v) for t, s, v in NODE_SHAPES]
    for sh in shapes:
        root = pkg.merkle_commit_shaped(gpu_ctx, d_rows, log_h, row_words, leaf_hash, sh, d_dig)
        assert np.array_equal(root, root_ref), sh
        assert np.array_equal(d_dig.to_host(), dig_ref), sh


FOLD_SHAPES = [(128, 0), (128, 16), (256, 0), (256, 4), (256, 8), (256, 16), (512, 0), (512, 2), (512, 4), (512, 8)]


def test_every_fold_shape_matches_oracle(pkg, gpu_ctx, oracle):
    n = 15
    rng = np.random.default_rng(5)
    r = rnd(rng, 4)
    fe = rnd(rng, 4 << n)
    want = oracle.fold_ext(fe, r)
    for sh in FOLD_SHAPES:
        d = pkg.DeviceArray.from_host(gpu_ctx, fe)
        pkg.fold_ext_shaped(gpu_ctx, d, n, r, sh)
        assert np.array_equal(d.to_host(4 << (n - 1)), want), sh


def test_tuning_on_first_use(pkg, gpu_ctx, oracle):
    old = pkg.tune_mode()
    try:
        pkg.set_tune_mode(1)
        pkg.tune_clear()
        rng = np.random.default_rng(9)
        # DFT: one shape, tuned on the first call; the output is the oracle's
        log_chunk, log_w, log_blowup = 15, 2, 1
        x = rnd(rng, 1 << (log_chunk + log_w))
        want = oracle.dft_batch(x, log_chunk, log_w, log_blowup, False)
        d_in = pkg.DeviceArray.from_host(gpu_ctx, x)
        d_out = pkg.DeviceArray(gpu_ctx, want.size)
        pkg.dft_batch(gpu_ctx, d_in, log_chunk, log_w, log_blowup, False, d_out)
        assert np.array_equal(d_out.to_host(), want)
        # Merkle and fold
        log_h, rw = 16, 16
        rows = rnd(rng, (1 << log_h) * rw)
        root_ref, dig_ref = oracle.merkle(rows, log_h, rw, 0)
        d_rows = pkg.DeviceArray.from_host(gpu_ctx, rows)
        d_dig = pkg.DeviceArray(gpu_ctx, dig_ref.size)
        assert np.array_equal(pkg.merkle_commit(gpu_ctx, d_rows, log_h, rw, 0, d_dig), root_ref)
        n = 15
        r = rnd(rng, 4)
        fe = rnd(rng, 4 << n)
        d = pkg.DeviceArray.from_host(gpu_ctx, fe)
        pkg.fold_ext(gpu_ctx, d, n, r)
        assert np.array_equal(d.to_host(4 << (n - 1)), oracle.fold_ext(fe, r))
        entries = pkg.tune_entries()
        kinds = {e["kind"] for e in entries}
        assert {"dft", "merkle_leaves", "merkle_nodes", "fold"} <= kinds, entries
        for e in entries:
            assert e["candidates"] >= 2
            assert 0 < e["ms_best"] <= e["ms_default"] * 1.0001 + 1e-6, e
        dft = [e for e in entries if e["kind"] == "dft"][0]
        assert dft["key"] == [log_chunk, log_w, log_blowup, 1]
        # the chosen plan joins the fastest pass 1 and pass 2 of one split: each
        # pass is a candidate's, and the joined plan reproduces the oracle
        h2, t1, th1, t2, th2, reg1, reg2 = dft["choice"]
        cands = pkg.dft_plans(log_chunk, log_w, log_blowup, False)
        if h2 == 0:
            assert any(c[:3] == (0, t1, th1) for c in cands)
        else:
            assert any(c[:3] == (h2, t1, th1) and c[5] == reg1 for c in cands)
            assert any(c[0] == h2 and c[3:5] == (t2, th2) and c[6] == reg2 for c in cands)
        pkg.dft_batch_plan(gpu_ctx, d_in, log_chunk, log_w, log_blowup, False, dft["choice"], d_out)
        assert np.array_equal(d_out.to_host(), want)
        # cached: a second call adds nothing and still matches
        pkg.dft_batch(gpu_ctx, d_in, log_chunk, log_w, log_blowup, False, d_out)
        assert np.array_equal(d_out.to_host(), want)
        assert len(pkg.tune_entries()) == len(entries)
        # fixed shapes: nothing new is tuned
        pkg.set_tune_mode(0)
        pkg.tune_clear()
        pkg.dft_batch(gpu_ctx, d_in, log_chunk, log_w, log_blowup, False, d_out)
        assert np.array_equal(d_out.to_host(), want)
        assert pkg.tune_entries() == []
    finally:
        pkg.set_tune_mode(old)
