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


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_lean_grind_windows_in_batch(pkg, gpu_ctx, mode):
    """Workers with lean grinding windows (fewer candidates in flight) give the
    same proofs as one-at-a-time proving with the latency window."""
    jobs = make_jobs(pkg, 12, 5 + mode, 10, 17)
    reqs = [pkg.ProofRequest(p, n, poly, pts if pts.size else None) for p, n, poly, pts in jobs]
    with pkg.Batch(0, workers=4) as b:
        b.set_grind_window(mode)
        b.run(reqs)
    check_against_single(pkg, gpu_ctx, jobs, reqs)
    with pytest.raises(pkg.WhirError):
        gpu_ctx.set_grind_window(4)


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


def test_device_memory_stays_within_budget(pkg, gpu_ctx):
    """A tight HBM budget with mixed sizes: the device memory in use
    (cudaMemGetInfo, sampled every half millisecond while the pool runs) never
    exceeds the budget by more than 64 MiB, jobs still run concurrently, and
    every proof equals the one-at-a-time result."""
    import threading

    import torch

    jobs = make_jobs(pkg, 24, 5, 14, 19)
    workers = 6
    # the first proof of a shape tunes its launch shapes on scratch arrays
    # outside the job's footprint: tune every shape first, as a server warms up
    seen = set()
    for p, n, poly, pts in jobs:
        key = (p.folding_factor.rest, p.starting_log_inv_rate, p.rs_domain_initial_reduction_factor, n)
        if key not in seen:
            seen.add(key)
            pkg.commit_and_prove(gpu_ctx, p, n, poly, pts if pts.size else None)
    with pkg.Batch(0, workers=1) as probe:
        per_ctx = probe.memory()[0]
    # a job is charged its footprint plus one 32 MiB pool chunk: room for two
    # of the largest
    biggest = max(pkg.job_footprint(p, n) for p, n, _, _ in jobs) + (32 << 20)
    budget = workers * per_ctx + int(2.5 * biggest)
    torch.cuda.synchronize()
    base = torch.cuda.mem_get_info()
    base_used = base[1] - base[0]
    peak = [0]
    stop = threading.Event()

    def sample():
        while not stop.is_set():
            free, total = torch.cuda.mem_get_info()
            peak[0] = max(peak[0], total - free - base_used)
            time.sleep(0.0005)

    reqs = [pkg.ProofRequest(p, n, poly, pts if pts.size else None) for p, n, poly, pts in jobs]
    th = threading.Thread(target=sample)
    th.start()
    try:
        with pkg.Batch(0, workers=workers, hbm_budget_bytes=budget) as b:
            b.run(reqs)
            fixed, _ = b.memory()
    finally:
        stop.set()
        th.join()
    assert fixed == workers * per_ctx
    assert peak[0] <= budget + (64 << 20), (peak[0], budget)
    spans = sorted((r.job.t_start_ms, r.job.t_done_ms) for r in reqs)
    overlapped = any(s1 < e0 for (s0, e0), (s1, e1) in zip(spans, spans[1:]))
    assert overlapped, "the budget leaves room for two jobs, yet none ran concurrently"
    check_against_single(pkg, gpu_ctx, jobs, reqs)


def test_small_jobs_pass_a_large_waiting_one(pkg, gpu_ctx):
    """First-fit admission: with a large job waiting for memory, a small job
    queued behind it starts before it."""
    big = make_jobs(pkg, 2, 11, 21, 21)
    small = make_jobs(pkg, 1, 12, 12, 12)
    jobs = [big[0], big[1], small[0]]
    for p, n, poly, pts in (big[0], small[0]):  # tune both shapes first
        pkg.commit_and_prove(gpu_ctx, p, n, poly, pts if pts.size else None)
    with pkg.Batch(0, workers=1) as probe:
        per_ctx = probe.memory()[0]
    # charges: footprint plus one 32 MiB pool chunk
    fp_big = max(pkg.job_footprint(p, n) for p, n, _, _ in big) + (32 << 20)
    fp_small = pkg.job_footprint(small[0][0], small[0][1]) + (32 << 20)
    budget = 3 * per_ctx + fp_big + fp_small + fp_small // 2  # one big job at a time, a small one beside it
    reqs = [pkg.ProofRequest(p, n, poly, pts if pts.size else None) for p, n, poly, pts in jobs]
    with pkg.Batch(0, workers=3, hbm_budget_bytes=budget) as b:
        b.run(reqs)
    assert reqs[2].job.t_start_ms < reqs[1].job.t_start_ms
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
