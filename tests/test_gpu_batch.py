"""Batching and serving: jobs proved concurrently by the worker pool give
exactly the proofs and transcript checkpoints of one-at-a-time proving (which
the other GPU tests tie to the oracle), whatever the mix, the admission budget
or the arrival order."""
import time

import numpy as np
import pytest

from oracle.oracle import P, make_params

pytestmark = pytest.mark.gpu


def make_jobs(pkg, count, seed, n_lo=10, n_hi=16):
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(count):
        n = int(rng.integers(n_lo, n_hi + 1))
        k = int(rng.choice([3, 4]))
        r = int(rng.choice([1, 2]))
        params = pkg.ProtocolParameters(64, 8, pkg.FoldingFactor.constant(k), pkg.SecurityAssumption.CapacityBound, r,
                                        min(3, k), "poseidon2_24", 32)
        poly = rng.integers(0, P, 1 << n, dtype=np.uint64).astype(np.uint32)
        pts = rng.integers(0, P, 4 * n * int(rng.integers(0, 3)), dtype=np.uint64).astype(np.uint32)
        jobs.append((params, n, poly, pts))
    return jobs


def check_against_single(pkg, ctx, jobs, reqs):
    for (params, n, poly, pts), req in zip(jobs, reqs):
        assert req.job.status == 0
        proof, cp, _ = pkg.commit_and_prove(ctx, params, n, poly, pts if pts.size else None)
        assert np.array_equal(req.proof, proof)
        assert np.array_equal(req.checkpoint, cp)


def test_batch_matches_one_at_a_time(pkg, gpu_ctx, oracle):
    jobs = make_jobs(pkg, 32, 1, 10, 19)  # mixed sizes: concurrent DFTs of different shapes
    reqs = [pkg.ProofRequest(p, n, poly, pts if pts.size else None) for p, n, poly, pts in jobs]
    with pkg.Batch(0, workers=8) as b:
        b.run(reqs)
    check_against_single(pkg, gpu_ctx, jobs, reqs)
    # and one of them against the oracle directly
    params, n, poly, pts = jobs[0]
    ref, ref_cp = oracle.prove(make_params(64, 8, params.folding_factor.rest, None, 2, params.starting_log_inv_rate,
                                           params.rs_domain_initial_reduction_factor, 0, 32),
                               n, poly, pts if pts.size else None)
    assert np.array_equal(reqs[0].proof, ref) and np.array_equal(reqs[0].checkpoint, ref_cp)


def test_admission_budget_limits_concurrency(pkg, gpu_ctx):
    jobs = make_jobs(pkg, 8, 2, 14, 16)
    reqs = [pkg.ProofRequest(p, n, poly, pts if pts.size else None) for p, n, poly, pts in jobs]
    biggest = max(pkg.job_footprint(p, n) for p, n, _, _ in jobs)
    with pkg.Batch(0, workers=4, hbm_budget_bytes=biggest) as b:  # at most one job fits at a time
        b.run(reqs)
    # with a budget of one job, runs never overlap
    spans = sorted((r.job.t_start_ms, r.job.t_done_ms) for r in reqs)
    for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
        assert s1 >= e0 - 1e-6
    check_against_single(pkg, gpu_ctx, jobs, reqs)


def test_serving_requests_arriving_in_the_mix(pkg, gpu_ctx):
    """Requests submitted while others are on the GPU: each result is the
    same as proving it alone."""
    jobs = make_jobs(pkg, 12, 3, 12, 17)
    reqs = [pkg.ProofRequest(p, n, poly, pts if pts.size else None) for p, n, poly, pts in jobs]
    rng = np.random.default_rng(9)
    with pkg.Batch(0, workers=4) as b:
        for r in reqs:
            b.submit(r)
            time.sleep(float(rng.exponential(0.002)))
        for r in reqs:
            b.wait(r)
    check_against_single(pkg, gpu_ctx, jobs, reqs)
