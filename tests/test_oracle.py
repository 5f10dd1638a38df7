"""The oracle (CPU restatement) against the reference's own known-answer
tests and relations.

The reference pins no golden roots, transcripts or proofs (its tests check
prover/verifier agreement and algebraic identities on small inputs), so these
tests pin exactly what it pins:
  * WhirConfig parameter schedules (src/whir/parameters.rs:81-234), checked
    against schedules derived independently from the same formulas;
  * compute_number_of_rounds (src/parameters/mod.rs:217-290 test cases);
  * multilinear evaluation KATs (src/poly/evals.rs:911-1200);
  * extrapolate_012 KATs (src/sumcheck/lagrange.rs:236-256);
  * end-to-end prover -> verifier acceptance and transcript checkpoint
    agreement over the grid of src/whir/mod.rs:177-232, and rejection of a
    tampered proof.
"""
import numpy as np
import pytest

from oracle.oracle import P, make_params

INV = lambda a: pow(int(a), P - 2, P)


def ef(*c):
    v = list(c) + [0] * (4 - len(c))
    return np.array([x % P for x in v], dtype=np.uint32)


def pt(*coords):
    return np.concatenate([ef(c) for c in coords])


# (n, k, rate, security, rs_reduction) -> (commit_ood, start_fold_pow, rounds[(log_domain, queries, pow,
# folding_pow, ood)], final_queries, final_pow, final_sumcheck_rounds)
SCHEDULES = {
    (24, 4, 1, 100, 1): (2, 7, [(25, 91, 15, 12, 2), (24, 22, 15, 17, 2), (23, 13, 17, 22, 2), (22, 9, 18, 27, 2)],
                         7, 9, 4),
    (24, 4, 1, 100, 3): (2, 7, [(25, 91, 15, 6, 2), (22, 44, 15, 11, 2), (21, 18, 13, 16, 2), (20, 11, 15, 21, 2)],
                         8, 12, 4),
    (26, 4, 1, 100, 1): (2, 9, [(27, 91, 17, 14, 2), (26, 22, 17, 19, 2), (25, 13, 19, 24, 2), (24, 9, 20, 29, 2)],
                         7, 9, 6),
    (18, 4, 1, 90, 1): (2, 0, [(19, 80, 15, 0, 2), (18, 19, 15, 1, 2)], 11, 13, 6),
}


@pytest.mark.parametrize("key", sorted(SCHEDULES))
def test_whir_config_schedule(oracle, key):
    n, k, r, sec, rs = key
    cfg = oracle.config(make_params(sec, 16, k, starting_log_inv_rate=r, rs_reduction=rs), n)
    ood, sfp, rounds, fq, fp, fin = SCHEDULES[key]
    got = [(cfg.rounds[i].domain_size.bit_length() - 1, cfg.rounds[i].num_queries, cfg.rounds[i].pow_bits,
            cfg.rounds[i].folding_pow_bits, cfg.rounds[i].ood_samples) for i in range(cfg.n_rounds)]
    assert (cfg.commitment_ood_samples, cfg.starting_folding_pow_bits) == (ood, sfp)
    assert got == rounds
    assert (cfg.final_queries, cfg.final_pow_bits, cfg.final_sumcheck_rounds) == (fq, fp, fin)
    assert cfg.final_folding_pow_bits == 0  # max(0, 100 - 123)


def test_compute_number_of_rounds(oracle):
    # src/parameters/mod.rs:217-290 with MAX_NUM_VARIABLES_TO_SEND_COEFFS = 6
    M = 6
    for n, expect in [(M - 1, (0, M - 3 - 1)), (M, (0, M - 3)), (M + 1, (0, M - 3 + 1)), (M + 3, (0, M)),
                      (M + 3 + 1, (1, M - 3 + 1)), (M + 6 + 1, (2, M - 3 + 1))]:
        cfg = oracle.config(make_params(32, 0, 3, soundness="UniqueDecoding"), n)
        assert (cfg.n_rounds, cfg.final_sumcheck_rounds) == expect
    for n, expect in [(M - 1, (0, M - 4 - 1)), (M, (0, M - 4)), (M + 1, (0, M - 4 + 1)), (M + 4, (0, M)),
                      (M + 4 + 1, (1, M - 3 + 1)), (M + 4 + 3 + 1, (2, M - 3 + 1))]:
        cfg = oracle.config(make_params(32, 0, 3, folding_factor_0=4, soundness="UniqueDecoding"), n)
        assert (cfg.n_rounds, cfg.final_sumcheck_rounds) == expect


def test_eval_multilinear_kats(oracle):
    # evals.rs:911-921: 1-d at x = 1/2
    a, b = 5, 10
    x = INV(2)
    assert (oracle.eval_base(np.array([a, b], np.uint32), pt(x)) == ef(a + (b - a) * x)).all()
    # evals.rs:1070-1110: f = 5 + 6 x2 + 7 x1 + 8 x1 x2 at (x1, x2) = (2, 1)
    e0, e1, e2, e3 = 5, 6, 7, 8
    evals = np.array([e0, e0 + e1, e0 + e2, e0 + e1 + e2 + e3], np.uint32)
    assert (oracle.eval_base(evals, pt(2, 1)) == ef(e0 + e1 * 1 + e2 * 2 + e3 * 2 * 1)).all()
    # evals.rs:1112-1190: 3 variables at (2, 3, 4)
    c = [1, 2, 3, 4, 5, 6, 7, 8]
    ev = [c[0], c[0] + c[1], c[0] + c[2], c[0] + c[1] + c[2] + c[3], c[0] + c[4], c[0] + c[1] + c[4] + c[5],
          c[0] + c[2] + c[4] + c[6], sum(c)]
    x0, x1, x2 = 2, 3, 4
    want = (c[0] + c[1] * x2 + c[2] * x1 + c[3] * x1 * x2 + c[4] * x0 + c[5] * x0 * x2 + c[6] * x0 * x1
            + c[7] * x0 * x1 * x2)
    assert (oracle.eval_base(np.array(ev, np.uint32), pt(x0, x1, x2)) == ef(want)).all()
    # the same polynomial lifted to the extension (evals.rs test_eval_extension_3_variables)
    evx = np.concatenate([ef(v) for v in ev])
    assert (oracle.eval_ext(evx, pt(x0, x1, x2)) == ef(want)).all()
    # evals.rs:924-945: 2-d interpolation formula at (1/2, 1/2)
    a, b, c2, d = 1, 2, 3, 4
    h = INV(2)
    want = ((1 - h) * (1 - h) * a + (1 - h) * h * b + h * (1 - h) * c2 + h * h * d) % P
    assert (oracle.eval_base(np.array([a, b, c2, d], np.uint32), pt(h, h)) == ef(want)).all()


def test_extrapolate_kats(oracle):
    # lagrange.rs:236-256
    e0, e1, e2 = ef(7), ef(13), ef(23)
    for r, want in [(0, e0), (1, e1), (2, e2)]:
        assert (oracle.extrapolate_012(e0, e1, e2, ef(r)) == want).all()
    assert (oracle.extrapolate_012(ef(1), ef(2), ef(5), ef(3)) == ef(10)).all()
    assert (oracle.extrapolate_012(ef(1), ef(2), ef(5), ef(4)) == ef(17)).all()


def test_eq_table_and_fold_identities(oracle):
    rng = np.random.default_rng(5)
    n = 6
    f = rng.integers(0, P, (1 << n) * 4, dtype=np.uint64).astype(np.uint32)
    z = rng.integers(0, P, n * 4, dtype=np.uint64).astype(np.uint32)
    eq = oracle.eq_table(z)
    # sum_x eq(z, x) f(x) == f(z)
    acc = np.zeros(4, dtype=object)
    from itertools import product  # noqa: F401

    def efmul(a, b):
        t = [0] * 7
        for i in range(4):
            for j in range(4):
                t[i + j] += int(a[i]) * int(b[j])
        return [(t[k] + 3 * (t[k + 4] if k + 4 < 7 else 0)) % P for k in range(4)]

    for x in range(1 << n):
        m = efmul(eq[4 * x:4 * x + 4], f[4 * x:4 * x + 4])
        acc = [(acc[i] + m[i]) % P for i in range(4)]
    assert [int(v) for v in oracle.eval_ext(f, z)] == acc
    # folding by z0 then evaluating at z[1:] equals evaluating at z
    g = oracle.fold_ext(f, z[:4])
    assert (oracle.eval_ext(g, z[4:]) == oracle.eval_ext(f, z)).all()


def _grid():
    cases = []
    for rs_red in (1, 2, 3):
        for f0, f in [(1, 1), (2, 2), (3, 3), (4, 4), (2, 1), (3, 1), (3, 2), (5, 2)]:
            if f0 < rs_red:
                continue
            for n in range(f0, 3 * f0 + 1):
                cases.append((rs_red, f0, f, n))
    return cases


@pytest.mark.parametrize("rs_red,f0,f,n", _grid())
def test_prove_verify_grid(oracle, rs_red, f0, f, n):
    """src/whir/mod.rs:177-232 (BabyBear there, KoalaBear here): every proof
    verifies and the post-proof challenger sample agrees. A rotating subset of
    (points, soundness, pow) keeps the CPU suite short."""
    rng = np.random.default_rng(1000 * rs_red + 100 * f0 + 10 * f + n)
    for j in range(3):
        npts = (n + j) % 3
        snd = (n + f0 + j) % 3
        pw = (0, 5, 10)[(f + j) % 3]
        prm = make_params(32, pw, f, f0, snd, 1, rs_red, 1, 8)
        poly = rng.integers(0, P, 1 << n, dtype=np.uint64).astype(np.uint32)
        pts = rng.integers(0, P, max(npts, 1) * n * 4, dtype=np.uint64).astype(np.uint32)[: npts * n * 4]
        evs = np.concatenate([oracle.eval_base(poly, pts[i * n * 4:(i + 1) * n * 4]) for i in range(npts)]) \
            if npts else None
        proof, cp = oracle.prove(prm, n, poly, pts if npts else None)
        rc, cp2 = oracle.verify(prm, n, pts if npts else None, evs, proof)
        assert rc == 0
        assert (cp == cp2).all()


def test_tampered_proof_rejected(oracle):
    rng = np.random.default_rng(7)
    n = 10
    prm = make_params(32, 5, 2, soundness="CapacityBound", rs_reduction=1, leaf_hash=1, ds_digest_elems=8)
    poly = rng.integers(0, P, 1 << n, dtype=np.uint64).astype(np.uint32)
    pts = rng.integers(0, P, n * 4, dtype=np.uint64).astype(np.uint32)
    evs = oracle.eval_base(poly, pts)
    proof, _ = oracle.prove(prm, n, poly, pts)
    assert oracle.verify(prm, n, pts, evs, proof)[0] == 0
    # a wrong claimed evaluation is rejected
    bad = evs.copy()
    bad[0] = (int(bad[0]) + 1) % P
    assert oracle.verify(prm, n, pts, bad, proof)[0] != 0
    # flipping any of a spread of proof words is rejected
    for pos in np.linspace(2, len(proof) - 1, 40).astype(int):
        t = proof.copy()
        t[pos] = (int(t[pos]) + 1) % P
        assert oracle.verify(prm, n, pts, evs, t)[0] != 0, pos
