"""End-to-end parity of the GPU prover: for the same seeded polynomial,
constraints and parameters the proof words and the post-proof transcript
checkpoint equal the oracle's exactly, and the oracle's verifier accepts."""
import numpy as np
import pytest

from oracle.oracle import P, make_params

pytestmark = pytest.mark.gpu


def rnd(rng, n):
    return rng.integers(0, P, n, dtype=np.uint64).astype(np.uint32)


def run_both(pkg, ctx, oracle, n, sec, pw, f0, f, snd, rate, rs, leaf, dig, npts, seed):
    rng = np.random.default_rng(seed)
    poly = rnd(rng, 1 << n)
    pts = rnd(rng, 4 * n * npts)
    params = pkg.ProtocolParameters(sec, pw, pkg.FoldingFactor(f0, f), pkg.SecurityAssumption(snd), rate, rs,
                                    "poseidon2_24" if leaf == 0 else "poseidon2_16", dig)
    proof, cp, evals = pkg.commit_and_prove(ctx, params, n, poly, pts if npts else None)
    oprm = make_params(sec, pw, f, f0, snd, rate, rs, leaf, dig)
    ref, ref_cp = oracle.prove(oprm, n, poly, pts if npts else None)
    assert proof.size == ref.size
    if not np.array_equal(proof, ref):
        first = int(np.nonzero(proof != ref)[0][0])
        raise AssertionError(f"proof differs at word {first} of {proof.size}")
    assert np.array_equal(cp, ref_cp)
    rc, vcp = oracle.verify(oprm, n, pts if npts else None, evals if npts else None, proof)
    assert rc == 0 and np.array_equal(vcp, cp)
    return proof


def grid():
    cases = []
    for rs in (1, 2, 3):
        for f0, f in [(1, 1), (2, 2), (3, 3), (4, 4), (2, 1), (3, 1), (3, 2), (5, 2)]:
            if f0 < rs:
                continue
            for n in range(f0, 3 * f0 + 1):
                cases.append((rs, f0, f, n))
    return cases


@pytest.mark.parametrize("rs,f0,f,n", grid())
def test_e2e_grid(pkg, gpu_ctx, oracle, rs, f0, f, n):
    """The parameter grid of the reference's test_whir_end_to_end1
    (src/whir/mod.rs:177-232), with a rotating subset of (points, soundness, pow)."""
    for j in range(3):
        npts = (n + j) % 3
        snd = (n + f0 + j) % 3
        pw = (0, 5, 10)[(f + j) % 3]
        run_both(pkg, gpu_ctx, oracle, n, 32, pw, f0, f, snd, 1, rs, 1, 8, npts, 1000 * rs + 100 * f0 + 10 * f + n + j)


@pytest.mark.parametrize("leaf,dig", [(0, 32), (1, 8), (0, 8)])
def test_e2e_hash_and_separator_choices(pkg, gpu_ctx, oracle, leaf, dig):
    run_both(pkg, gpu_ctx, oracle, 14, 64, 8, 4, 4, 2, 1, 2, leaf, dig, 2, 77 + leaf + dig)


def test_e2e_cli_default_shape_n18(pkg, gpu_ctx, oracle):
    """n = 18, k = 4, rate 1/2, 90-bit CapacityBound, pow_bits 16, rs reduction
    3, one constraint: the CLI's security level, rate, pow_bits and rs
    reduction defaults (src/bin/main.rs:41-67; its defaults for the variable
    count and folding factor are 25 and 5), at a size the oracle proves in
    about a second."""
    run_both(pkg, gpu_ctx, oracle, 18, 90, 16, 4, 4, 2, 1, 3, 0, 32, 1, 18)


def test_e2e_n20_rs1_four_constraints(pkg, gpu_ctx, oracle):
    run_both(pkg, gpu_ctx, oracle, 20, 100, 16, 4, 4, 2, 1, 1, 0, 32, 4, 20)


def test_split_commit_then_prove_matches(pkg, gpu_ctx):
    """CommitmentWriter::commit then Prover::prove (two calls, device-resident
    polynomial) gives the same proof as the one-call path."""
    rng = np.random.default_rng(5)
    n = 16
    poly = rnd(rng, 1 << n)
    pt = rnd(rng, 4 * n)
    params = pkg.ProtocolParameters(80, 10, pkg.FoldingFactor.constant(4), pkg.SecurityAssumption.CapacityBound, 1, 2)
    one, cp1, _ = pkg.commit_and_prove(gpu_ctx, params, n, poly, pt)
    cfg = pkg.WhirConfig(n, params)
    ch = pkg.DuplexChallenger(gpu_ctx)
    pkg.DomainSeparator(cfg).observe_domain_separator(ch)
    dpoly = pkg.DeviceArray.from_host(gpu_ctx, poly)
    st = pkg.InitialStatement(dpoly, n)
    st.evaluate(pt)
    wit = pkg.CommitmentWriter(cfg).commit(gpu_ctx, ch, st)
    two = pkg.Prover(cfg).prove(gpu_ctx, ch, wit)
    wit.free()
    assert np.array_equal(one, two)
    assert np.array_equal(ch.sample_algebra_element(), cp1)


@pytest.mark.parametrize("n,k,rate", [(20, 4, 1), (18, 3, 2), (18, 5, 1)])
def test_pipelined_upload_matches_device_resident(pkg, gpu_ctx, n, k, rate):
    """A host polynomial goes up in eight chunk groups, each group's DFT first
    pass queued behind its copy once the DFT plan of the shape is known; the
    proof equals the one from a device-resident polynomial, and the launch
    count shows the pipelined path ran (eight encodings and eight first-pass
    launches in place of one encoding and one first pass)."""
    rng = np.random.default_rng(n * 10 + k)
    poly = rnd(rng, 1 << n)
    pt = rnd(rng, 4 * n)
    params = pkg.ProtocolParameters(90, 12, pkg.FoldingFactor.constant(k), pkg.SecurityAssumption.CapacityBound,
                                    rate, 1)
    dpoly = pkg.DeviceArray.from_host(gpu_ctx, poly)
    ref, ref_cp, ref_ev = pkg.commit_and_prove(gpu_ctx, params, n, dpoly, pt)  # tunes the shapes
    l0 = pkg.kernel_launches()
    again = pkg.commit_and_prove(gpu_ctx, params, n, dpoly, pt)
    dev_launches = pkg.kernel_launches() - l0
    for _ in range(2):
        l0 = pkg.kernel_launches()
        proof, cp, ev = pkg.commit_and_prove(gpu_ctx, params, n, poly, pt)
        host_launches = pkg.kernel_launches() - l0
        assert np.array_equal(proof, ref) and np.array_equal(cp, ref_cp) and np.array_equal(ev, ref_ev)
        assert host_launches == dev_launches + 15, (host_launches, dev_launches)
    assert np.array_equal(again[0], ref)


def test_e2e_headline_n24(pkg, gpu_ctx, oracle):
    """The reference's benchmark configuration (benches/whir.rs:34-120): n = 24,
    k = 4, rate 1/2, 100-bit CapacityBound, pow_bits 16, rs reduction 3, one
    constraint, Poseidon2-24 leaves, DIGEST_ELEMS 32, with the polynomial and
    point drawn as the benchmark draws them (SmallRng::seed_from_u64(0))."""
    n = 24
    draw = pkg.rng_koalabear(0, (1 << n) + 4 * n)
    poly, pts = draw[: 1 << n], draw[1 << n:]
    params = pkg.ProtocolParameters(100, 16, pkg.FoldingFactor.constant(4), pkg.SecurityAssumption.CapacityBound, 1, 3,
                                    "poseidon2_24", 32)
    proof, cp, evals = pkg.commit_and_prove(gpu_ctx, params, n, poly, pts)
    oprm = make_params(100, 16, 4, None, 2, 1, 3, 0, 32)
    ref, ref_cp = oracle.prove(oprm, n, poly, pts)
    assert np.array_equal(proof, ref) and np.array_equal(cp, ref_cp)
    rc, vcp = oracle.verify(oprm, n, pts, evals, proof)
    assert rc == 0 and np.array_equal(vcp, cp)


def test_e2e_n26_four_constraints_word_identical(pkg, gpu_ctx, oracle):
    """n = 26 with four constraints (the larger full-prove configuration),
    rs reduction 3: proof words and checkpoint equal the oracle's."""
    run_both(pkg, gpu_ctx, oracle, 26, 100, 16, 4, 4, 2, 1, 3, 0, 32, 4, 2626)


def test_e2e_n26_verified(pkg, gpu_ctx, oracle):
    """n = 26 (the larger size of the full-prove configuration), rs reduction 1,
    four constraints: the GPU proof is accepted by the oracle's verifier with an
    agreeing transcript checkpoint (proving n = 26 on the CPU oracle as well
    would take about a minute; n <= 24 is compared word for word above)."""
    rng = np.random.default_rng(26)
    n = 26
    poly = rnd(rng, 1 << n)
    pts = rnd(rng, 4 * n * 4)
    params = pkg.ProtocolParameters(100, 16, pkg.FoldingFactor.constant(4), pkg.SecurityAssumption.CapacityBound, 1, 1,
                                    "poseidon2_24", 32)
    proof, cp, evals = pkg.commit_and_prove(gpu_ctx, params, n, poly, pts)
    oprm = make_params(100, 16, 4, None, 2, 1, 1, 0, 32)
    rc, vcp = oracle.verify(oprm, n, pts, evals, proof)
    assert rc == 0 and np.array_equal(vcp, cp)
    for i in range(4):
        assert np.array_equal(evals[4 * i:4 * i + 4], oracle.eval_base(poly, pts[4 * n * i:4 * n * (i + 1)]))


@pytest.mark.parametrize("n,f,rs,pw", [(12, 3, 1, 10), (18, 4, 3, 16), (20, 4, 1, 16)])
def test_device_transcript_matches_host_round_trips(pkg, gpu_ctx, oracle, n, f, rs, pw):
    """Sumcheck stages with the transcript on the device and with one host
    round trip per step (the default) give the same proof, equal to the
    oracle's."""
    rng = np.random.default_rng(4400 + n)
    poly = rnd(rng, 1 << n)
    pts = rnd(rng, 4 * n)
    params = pkg.ProtocolParameters(100, pw, pkg.FoldingFactor.constant(f), pkg.SecurityAssumption.CapacityBound, 1,
                                    rs, "poseidon2_24", 32)
    out = []
    for device in (False, True):
        gpu_ctx.set_device_transcript(device)
        try:
            out.append(pkg.commit_and_prove(gpu_ctx, params, n, poly, pts))
        finally:
            gpu_ctx.set_device_transcript(False)
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    ref, ref_cp = oracle.prove(make_params(100, pw, f, None, 2, 1, rs, 0, 32), n, poly, pts)
    assert np.array_equal(out[1][0], ref) and np.array_equal(out[1][1], ref_cp)
