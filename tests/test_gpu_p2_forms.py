"""Both Poseidon2 external blocks on the GPU. The library's default is the
circulant (2, 3, 1, 1) of Plonky3's KoalaBear (`MDSMat4`), which the other GPU
suites use; here a context built with the paper's M4 (`HLMDSMat4`) is checked
against the oracle with the same block: Merkle trees through every kernel
path and launch shape, proof-of-work searches at every sponge position, and
whole proofs. Inputs drawn as the reference's benchmark draws them
(`SmallRng::seed_from_u64(0)`, benches/whir.rs:92-100) are proved with the
default block."""
import ctypes as C

import numpy as np
import pytest

from oracle.oracle import Chal, Oracle, P, make_params

pytestmark = pytest.mark.gpu


def rnd(rng, n):
    return rng.integers(0, P, n, dtype=np.uint64).astype(np.uint32)


@pytest.fixture(scope="module")
def hl_oracle():
    return Oracle(p2_seed=1, p2_mat=1)


@pytest.fixture(scope="module")
def hl_ctx(pkg):
    ctx = pkg.Context(0, *pkg.poseidon2_from_rng(1, pkg.P2_HL_MAT4))
    yield ctx
    ctx.close()


@pytest.mark.parametrize("log_h,row_words,leaf_hash", [(0, 16, 0), (5, 16, 0), (9, 64, 0), (10, 8, 1), (3, 5, 1),
                                                       (14, 16, 0), (16, 64, 0)])
def test_merkle_hl(pkg, hl_ctx, hl_oracle, log_h, row_words, leaf_hash):
    rng = np.random.default_rng(5 * log_h + row_words + leaf_hash)
    rows = rnd(rng, (1 << log_h) * row_words)
    root_ref, dig_ref = hl_oracle.merkle(rows, log_h, row_words, leaf_hash)
    d_rows = pkg.DeviceArray.from_host(hl_ctx, rows)
    d_dig = pkg.DeviceArray(hl_ctx, dig_ref.size)
    root = pkg.merkle_commit(hl_ctx, d_rows, log_h, row_words, leaf_hash, d_dig)
    assert np.array_equal(root, root_ref)
    assert np.array_equal(d_dig.to_host(), dig_ref)


@pytest.mark.parametrize("leaf_hash,row_words,log_h", [(0, 16, 17), (1, 8, 13)])
def test_merkle_hl_every_shape(pkg, hl_ctx, hl_oracle, leaf_hash, row_words, log_h):
    from test_gpu_tune import LEAF_SHAPES, NODE_SHAPES

    rng = np.random.default_rng(91 + log_h)
    rows = rnd(rng, (1 << log_h) * row_words)
    root_ref, dig_ref = hl_oracle.merkle(rows, log_h, row_words, leaf_hash)
    d_rows = pkg.DeviceArray.from_host(hl_ctx, rows)
    d_dig = pkg.DeviceArray(hl_ctx, dig_ref.size)
    shapes = [(t, s, 256, 16, 1) for t, s in LEAF_SHAPES] + [(256, 16, t, s, v) for t, s, v in NODE_SHAPES]
    for sh in shapes:
        root = pkg.merkle_commit_shaped(hl_ctx, d_rows, log_h, row_words, leaf_hash, sh, d_dig)
        assert np.array_equal(root, root_ref), sh
        assert np.array_equal(d_dig.to_host(), dig_ref), sh


@pytest.mark.parametrize("bits", [2, 9, 15])
def test_grind_hl_every_position(pkg, hl_ctx, hl_oracle, bits):
    rng = np.random.default_rng(300 + bits)
    ch = pkg.DuplexChallenger(hl_ctx)
    oc = Chal()
    hl_oracle.lib.or_chal_init(C.byref(oc))
    for pending in range(8):
        vals = rnd(rng, 8 + pending)
        ch.observe_slice(vals)
        for v in vals:
            hl_oracle.lib.or_chal_observe(C.byref(oc), C.byref(hl_oracle.p16), int(v))
        assert ch.grind(bits) == hl_oracle.lib.or_chal_grind(C.byref(oc), C.byref(hl_oracle.p16), bits)
        assert list(ch.c.state) == list(oc.state)


def _prove_both(pkg, ctx, orc, n, poly, pts, sec, pw, f, rate, rs, leaf, dig):
    params = pkg.ProtocolParameters(sec, pw, pkg.FoldingFactor.constant(f), pkg.SecurityAssumption.CapacityBound,
                                    rate, rs, "poseidon2_24" if leaf == 0 else "poseidon2_16", dig)
    proof, cp, evals = pkg.commit_and_prove(ctx, params, n, poly, pts)
    oprm = make_params(sec, pw, f, None, 2, rate, rs, leaf, dig)
    ref, ref_cp = orc.prove(oprm, n, poly, pts)
    assert proof.size == ref.size and np.array_equal(proof, ref) and np.array_equal(cp, ref_cp)
    rc, vcp = orc.verify(oprm, n, pts, evals, proof)
    assert rc == 0 and np.array_equal(vcp, cp)
    return proof


@pytest.mark.parametrize("n,f,rs,leaf,dig,npts", [(8, 2, 1, 1, 8, 1), (12, 3, 2, 0, 32, 2), (14, 4, 3, 1, 8, 0),
                                                  (18, 4, 3, 0, 32, 1), (20, 4, 1, 0, 32, 2)])
def test_e2e_hl(pkg, hl_ctx, hl_oracle, n, f, rs, leaf, dig, npts):
    rng = np.random.default_rng(7000 + n)
    poly = rnd(rng, 1 << n)
    pts = rnd(rng, 4 * n * npts) if npts else None
    _prove_both(pkg, hl_ctx, hl_oracle, n, poly, pts, 64 if n < 16 else 100, 10 if n < 16 else 16, f, 1, rs, leaf,
                dig)


def test_blocks_give_different_roots(pkg, gpu_ctx, hl_ctx):
    rows = np.arange(16 << 12, dtype=np.uint32) % P
    roots = []
    for ctx in (gpu_ctx, hl_ctx):
        d_rows = pkg.DeviceArray.from_host(ctx, rows)
        d_dig = pkg.DeviceArray(ctx, ((2 << 12) - 1) * 8)
        roots.append(pkg.merkle_commit(ctx, d_rows, 12, 16, 0, d_dig))
    assert not np.array_equal(roots[0], roots[1])


@pytest.mark.parametrize("n", [16, 20])
def test_e2e_benchmark_inputs(pkg, gpu_ctx, oracle, n):
    """The polynomial and constraint point as the reference's benchmark draws
    them: 2^n elements, then n extension coordinates, from one
    SmallRng::seed_from_u64(0); k = 4, rate 1/2, 100-bit CapacityBound,
    pow_bits 16, rs reduction 3, Poseidon2-24 leaves, DIGEST_ELEMS 32."""
    draw = pkg.rng_koalabear(0, (1 << n) + 4 * n)
    assert np.array_equal(draw, oracle.rng_fields(0, (1 << n) + 4 * n))
    poly, pts = draw[: 1 << n], draw[1 << n:]
    _prove_both(pkg, gpu_ctx, oracle, n, poly, pts, 100, 16, 4, 1, 3, 0, 32)
