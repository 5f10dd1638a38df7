"""The Keccak configuration of the reference (src/whir/mod.rs:236-383,
test_whir_keccak_end_to_end) on the GPU: the Keccak MMCS kernels against the
oracle's tree (digests, root and openings word for word), and whole proofs on
the SerializingChallenger32 transcript equal to the oracle's, with the
oracle's verifier accepting them. Includes the reference test's own
configuration (n = 10, k = 4, 32-bit security, CapacityBound, no grinding,
two points, DIGEST_ELEMS 4) and variants with grinding on the Keccak
challenger (the GPU search must return the smallest witness, as the oracle's)."""
import numpy as np
import pytest

from oracle.oracle import P, make_params

pytestmark = pytest.mark.gpu


def rnd(rng, n):
    return rng.integers(0, P, n, dtype=np.uint64).astype(np.uint32)


@pytest.mark.parametrize("log_h,row_words", [(0, 16), (1, 16), (5, 16), (10, 16), (11, 64), (12, 4), (9, 7),
                                              (6, 35), (14, 16)])
def test_keccak_merkle_commit_and_open(pkg, gpu_ctx, oracle, log_h, row_words):
    rng = np.random.default_rng(log_h * 100 + row_words)
    rows = rnd(rng, (1 << log_h) * row_words)
    root_ref, dig_ref = oracle.merkle(rows, log_h, row_words, 2)
    d_rows = pkg.DeviceArray.from_host(gpu_ctx, rows)
    d_dig = pkg.DeviceArray(gpu_ctx, dig_ref.size)
    root = pkg.merkle_commit(gpu_ctx, d_rows, log_h, row_words, 2, d_dig)
    assert np.array_equal(root, root_ref)
    assert np.array_equal(d_dig.raw(), dig_ref)
    h = 1 << log_h
    for idx in sorted({0, h - 1, h // 2, int(rng.integers(0, h))}):
        row, path = pkg.merkle_open(gpu_ctx, d_rows, d_dig, log_h, row_words, idx, leaf_hash=2)
        assert np.array_equal(row, rows[idx * row_words:(idx + 1) * row_words])
        off, n = 0, h
        for level in range(log_h):
            sib = (idx >> level) ^ 1
            assert np.array_equal(path[8 * level:8 * level + 8], dig_ref[(off + sib) * 8:(off + sib) * 8 + 8])
            off += n
            n //= 2


def run_keccak(pkg, ctx, oracle, n, sec, pw, k, snd, rate, rs, npts, seed):
    rng = np.random.default_rng(seed)
    poly = rnd(rng, 1 << n)
    pts = rnd(rng, 4 * n * npts)
    params = pkg.ProtocolParameters(sec, pw, pkg.FoldingFactor.constant(k), pkg.SecurityAssumption(snd), rate, rs,
                                    "keccak", 4)
    proof, cp, evals = pkg.commit_and_prove(ctx, params, n, poly, pts if npts else None)
    oprm = make_params(sec, pw, k, None, snd, rate, rs, 2, 4)
    ref, ref_cp = oracle.prove(oprm, n, poly, pts if npts else None)
    assert proof.size == ref.size
    if not np.array_equal(proof, ref):
        first = int(np.nonzero(proof != ref)[0][0])
        raise AssertionError(f"proof differs at word {first} of {proof.size}")
    assert np.array_equal(cp, ref_cp)
    rc, vcp = oracle.verify(oprm, n, pts if npts else None, evals if npts else None, proof)
    assert rc == 0 and np.array_equal(vcp, cp)
    return proof


def test_keccak_reference_configuration(pkg, gpu_ctx, oracle):
    """make_whir_things_keccak(10, Constant(4), 2, CapacityBound, 0, 1, ..)."""
    run_keccak(pkg, gpu_ctx, oracle, 10, 32, 0, 4, 2, 1, 1, 2, 11)


@pytest.mark.parametrize("n,pw,k,snd,rate,rs,npts", [(12, 8, 4, 2, 1, 1, 1), (14, 12, 4, 0, 1, 2, 2),
                                                     (16, 10, 3, 1, 2, 1, 1), (18, 14, 4, 2, 1, 3, 1)])
def test_keccak_proofs_with_grinding(pkg, gpu_ctx, oracle, n, pw, k, snd, rate, rs, npts):
    run_keccak(pkg, gpu_ctx, oracle, n, 64, pw, k, snd, rate, rs, npts, 500 + n)


def test_keccak_grinding_throughput_window(pkg, gpu_ctx, oracle):
    """Keccak-challenger searches with both lean candidate windows: the same
    proof as the oracle's."""
    gpu_ctx.set_grind_window(3)
    try:
        run_keccak(pkg, gpu_ctx, oracle, 14, 64, 12, 4, 0, 1, 2, 2, 514)
    finally:
        gpu_ctx.set_grind_window(0)


@pytest.mark.parametrize("n,k,rs,npts", [(2, 1, 1, 1), (4, 2, 1, 0), (6, 3, 2, 2), (8, 4, 3, 1), (9, 2, 1, 3)])
def test_keccak_small_shapes(pkg, gpu_ctx, oracle, n, k, rs, npts):
    """Small sizes and folding factors (one-CTA trees, no four-step DFT)."""
    run_keccak(pkg, gpu_ctx, oracle, n, 32, 4, k, 2, 1, rs, npts, 900 + 10 * n + k)


def test_keccak_split_api_refused(pkg, gpu_ctx):
    """The split commit / prove API carries the duplex challenger's state; the
    Keccak configuration is refused there with an error, not proved wrongly."""
    params = pkg.ProtocolParameters(32, 0, pkg.FoldingFactor.constant(4), pkg.SecurityAssumption.CapacityBound, 1, 1,
                                    "keccak", 4)
    st = pkg.InitialStatement(rnd(np.random.default_rng(1), 1 << 10), 10)
    writer = pkg.CommitmentWriter(pkg.WhirConfig(10, params))
    with pytest.raises(pkg.WhirError):
        writer.commit(gpu_ctx, pkg.DuplexChallenger(gpu_ctx), st)


def test_keccak_in_batch_and_with_device_transcript_switch(pkg, gpu_ctx, oracle):
    """Keccak jobs through the worker pool mixed with Poseidon2 jobs give the
    same proofs as one at a time; the device-transcript switch, which covers
    the duplex challenger only, leaves a Keccak proof unchanged."""
    rng = np.random.default_rng(31)
    jobs = []
    for i, (n, leaf) in enumerate([(12, "keccak"), (13, "poseidon2_24"), (14, "keccak"), (12, "poseidon2_16")]):
        params = pkg.ProtocolParameters(64, 10, pkg.FoldingFactor.constant(4), pkg.SecurityAssumption.CapacityBound,
                                        1, 1, leaf, 4 if leaf == "keccak" else 8)
        jobs.append((params, n, rnd(rng, 1 << n), rnd(rng, 4 * n)))
    alone = [pkg.commit_and_prove(gpu_ctx, p, n, poly, pt)[0] for p, n, poly, pt in jobs]
    with pkg.Batch(gpu_ctx.device, workers=3) as b:
        reqs = [pkg.ProofRequest(p, n, poly, pt) for p, n, poly, pt in jobs]
        b.run(reqs)
    for r, a in zip(reqs, alone):
        assert np.array_equal(r.proof, a)
    gpu_ctx.set_device_transcript(True)
    try:
        p, n, poly, pt = jobs[2]
        again = pkg.commit_and_prove(gpu_ctx, p, n, poly, pt)[0]
    finally:
        gpu_ctx.set_device_transcript(False)
    assert np.array_equal(again, alone[2])
