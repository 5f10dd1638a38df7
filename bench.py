#!/usr/bin/env python
"""WHIR commit + prove at 2^24 variables on B200.

Workload (the reference's own benchmark, benches/whir.rs:34-120 "prove"):
KoalaBear / quartic extension, num_variables = 24, folding factor 4, rate 1/2,
100-bit CapacityBound, pow_bits 16, rs_domain_initial_reduction_factor 3, one
evaluation constraint, Poseidon2-24 leaf hashing, Poseidon2-16 compression and
duplex challenger, DIGEST_ELEMS 32. Inputs are drawn as the reference's
benchmark draws them: SmallRng::seed_from_u64(0) yields the 2^24-element
polynomial, then the constraint point; the Poseidon2 permutations are
new_from_rng_128 on SmallRng::seed_from_u64(1) with Plonky3's KoalaBear
external block.

One step = one full commit + prove of one polynomial on each GPU (replicas:
one independent proof per rank, no collective on the data path). Rank 0 prints
one JSON line; `value` is milliseconds per proof for the whole job (the max
over ranks of the timed region divided by the proofs all ranks produced).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Batching (64 independent proofs, num_variables log-uniform in [16, 22],
folding factor in {3, 4}, rate 1/2 or 1/4) and serving (Poisson arrivals,
num_variables uniform in [16, 24], 120 GB HBM budget) against the plain
one-proof-at-a-time path:

  python bench.py --batch [--workers W]
  python bench.py --serve [--rates 10,50,100,200,500] [--workers W]

Kernel-level microbenchmarks (the kernel configuration of the benchmark
suite: eq expansion / evaluation / fold over 2^24 extension elements, the
2^24 -> 2^25 LDE, a Poseidon2 Merkle tree over 2^21 leaves of 16 elements, and
proof-of-work grinding), each timed alone with CUDA events on the context's
stream and printed as one JSON line per kernel:

  python bench.py --micro all|eq|eval|fold|dft|merkle|grind [--steps K]

The default run (N = 1) also reports, in its one JSON line: `extra` (n = 24
with four constraints, n = 26 with one and four), `micro` (the kernel
micro-benchmarks above, 5 timed runs each), `batched`, `served` (the rate
sweep), `cpu_baseline`, the per-stage `rooflines` and `autotune`.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_VARS = 24
CONFIG = dict(workload="whir_commit_prove", num_variables=N_VARS, folding_factor=4, starting_log_inv_rate=1,
              security_level=100, soundness="CapacityBound", pow_bits=16, rs_domain_initial_reduction_factor=3,
              constraints=1, leaf_hash="poseidon2_24", compress="poseidon2_16", challenger="duplex_poseidon2_16",
              ds_digest_elems=32, l2="flushed between timed steps (256 MiB write)")
METRIC = "WHIR prove ms @2^24 vars"
UNIT = "ms/proof"
P = 0x7F000001


def reduce_over_ranks(local_ms: float, dist, device=None) -> float:
    """Max of a per-rank device time over all ranks (the slowest rank bounds a
    weak-scaling step); without a process group it is the local value."""
    if dist is None:
        return float(local_ms)
    import torch

    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(max_total_ms: float, steps: int, world: int) -> tuple[float, float]:
    """(ms per step, whole-job ms per proof): every rank proves one polynomial
    per step, so a step yields `world` proofs."""
    step_ms = max_total_ms / steps
    return step_ms, step_ms / world


def inputs(draw, rank: int, n: int):
    """The benchmark's inputs as benches/whir.rs:92-100 draws them: 2^n base
    elements, then n extension coordinates, from SmallRng::seed_from_u64(0)
    (rank r of a replica run uses seed r). `draw(seed, count)` is the
    product's whir_rng_koalabear or, on the CPU legs, the oracle's restatement
    of the same generator."""
    v = draw(rank, (1 << n) + 4 * n)
    return v[: 1 << n], v[1 << n:]


def inputs_m(draw, rank: int, n: int, m: int):
    """inputs() with m constraint points drawn after the polynomial, one after
    the other (the loop of src/bin/main.rs:131-133)."""
    v = draw(rank, (1 << n) + 4 * n * m)
    return v[: 1 << n], v[1 << n:]


def measure_config(pkg, ctx, stream, flush, n: int, m: int, steps: int, warmup: int) -> dict:
    """Device-resident commit + prove of the benchmark's workload at n
    variables with m constraints: ms per proof over `steps` timed proofs (CUDA
    events on the context's stream, L2 flushed before each), after `warmup`."""
    import torch

    params = pkg.ProtocolParameters(100, 16, pkg.FoldingFactor.constant(4), pkg.SecurityAssumption.CapacityBound, 1, 3,
                                    "poseidon2_24", 32)
    poly, pts = inputs_m(pkg.rng_koalabear, 0, n, m)
    d_poly = pkg.DeviceArray.from_host(ctx, poly)
    for _ in range(max(warmup, 1)):
        pkg.commit_and_prove(ctx, params, n, d_poly, pts)
    total = 0.0
    for _ in range(steps):
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        pkg.commit_and_prove(ctx, params, n, d_poly, pts)
        e.record(stream)
        e.synchronize()
        total += s.elapsed_time(e)
    del d_poly
    return {"num_variables": n, "constraints": m, "value": round(total / steps, 4), "unit": UNIT, "steps": steps,
            "warmup": max(warmup, 1), "rs_domain_initial_reduction_factor": 3, "inputs": "SmallRng(0) draw"}


def oracle_params():
    from oracle.oracle import make_params

    return make_params(100, 16, 4, None, 2, 1, 3, 0, 32)


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.proc = None
        # raw samples beside the run's other outputs when BENCH_OUT_DIR names a
        # folder, else in the temporary directory; the JSON line summarises them
        out_dir = os.environ.get("BENCH_OUT_DIR") or tempfile.gettempdir()
        self.path = pathlib.Path(out_dir) / f"clocks_rank{index}.csv"
        try:
            self.path.parent.mkdir(exist_ok=True)
            q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # wait (up to 2 s) until the sampler has produced its first line
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < 2.0:
            try:
                if self.path.stat().st_size > 0:
                    break
            except OSError:
                pass
            time.sleep(0.02)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for name, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# Warp instructions one warp issues for 32 permutations (one per thread) in
# each Poseidon2 stage, from ncu's smsp__inst_executed.sum divided by the
# permutations of the captured launches, measured once on this build (Poseidon2
# with Plonky3's KoalaBear external block): the grind from an 18-bit search,
# leaves and tree levels from the n = 24 proof's launches (the tree stage mixes
# one-thread and four-lane permutations). The DFT stage's instructions per
# algorithmic byte come from the same proof's DFT launches. The issue ceiling
# is 4 warp instructions per clock per SM at the SM clock sampled during the
# timed run.
WARP_INST_PER_32_PERMS = {"grind": 4810, "merkle_leaves": 8270, "merkle_upper": 5540}
DFT_WARP_INST_PER_BYTE = 0.7064


def stage_rooflines(stages, work, steps, sm_mhz):
    """One roofline entry per measured kernel stage. Poseidon2 stages (grinding,
    leaf hashing, tree compression) are bound by instruction issue: achieved
    = permutations per second (the stage's counted permutations over its live
    CUDA-event time) times warp instructions per permutation, against SMs x 4
    x the sampled SM clock. The DFT is bound by HBM: achieved = algorithmic
    bytes (chunks read once, LDE written once) over its live time, against the
    measured copy bandwidth; its instruction issue is reported beside it (the
    passes run below the HBM limit because they are issue-bound)."""
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    import torch

    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    issue_peak = sms * 4 * sm_mhz * 1e6 / 1e9  # G warp-instructions / s
    names = {"grind": "k_grind (Poseidon2-16 proof-of-work search)",
             "merkle_leaves": "k_leaf_digests (Poseidon2-24 leaf sponge)",
             "merkle_upper": "k_merkle_two_levels / tree tops (Poseidon2-16 compression)",
             "dft": "k_dft_cols_reg + k_dft_rows_reg / k_dft_coset (LDE)"}
    out = []
    for st, label in names.items():
        ms, launches = stages[st]
        units = work.get(st, 0)
        if ms <= 0 or units <= 0:
            continue
        sec = ms * 1e-3
        e = {"kernel": label, "stage": st, "ms_per_proof": round(ms / steps, 4),
             "launches_per_proof": round(launches / steps, 2)}
        if st == "dft":
            gbs = units / sec / 1e9
            e.update({"bound": "hbm", "achieved": round(gbs, 1), "peak": hbm, "unit": "GB/s",
                      "frac": round(gbs / hbm, 4), "traffic": None,
                      "algorithmic_bytes_per_proof": units // steps,
                      "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650 GB/s"})
            ach = units * DFT_WARP_INST_PER_BYTE / sec / 1e9
            e["issue"] = {"achieved": round(ach, 2), "peak": round(issue_peak, 2), "unit": "G warp-instructions/s",
                          "frac": round(ach / issue_peak, 4), "warp_instructions_per_algorithmic_byte":
                          DFT_WARP_INST_PER_BYTE}
        else:
            rate = units / sec
            e.update({"permutations_per_proof": units // steps, "permutations_per_s": round(rate)})
            ipp = WARP_INST_PER_32_PERMS.get(st)
            if ipp:
                ach = rate / 32.0 * ipp / 1e9
                e.update({"bound": "issue", "achieved": round(ach, 2), "peak": round(issue_peak, 2),
                          "unit": "G warp-instructions/s", "frac": round(ach / issue_peak, 4), "traffic": None,
                          "warp_instructions_per_32_permutations": ipp,
                          "peak_source": f"{sms} SMs x 4 issue slots x {sm_mhz:.0f} MHz sampled"})
            else:
                e.update({"bound": "issue", "achieved": None, "peak": round(issue_peak, 2),
                          "unit": "G warp-instructions/s", "frac": None, "traffic": None})
        out.append(e)
    return out


def run_reference(args) -> None:
    """The reference's CPU prover cannot be built here (Rust, no cargo); the
    CPU arm runs the oracle port of the same algorithm on all host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.oracle import Oracle

    o = Oracle()
    prm = oracle_params()
    poly, point = inputs(o.rng_fields, 0, N_VARS)
    cores = os.cpu_count() or 1
    # a CPU proof takes seconds: one warm-up proof, then at most as many timed
    # proofs as fit in about two and a half minutes (at least one), so the
    # whole arm ends within a few minutes whatever --steps asks
    for _ in range(min(max(args.warmup, 0), 1)):
        o.prove(prm, N_VARS, poly, point)
    times = []
    budget_s, start = 150.0, time.perf_counter()
    for _ in range(max(args.steps, 1)):
        t0 = time.perf_counter()
        o.prove(prm, N_VARS, poly, point)
        times.append((time.perf_counter() - t0) * 1e3)
        if time.perf_counter() - start + times[-1] / 1e3 > budget_s:
            break
    ms = float(np.mean(times))
    line = {"metric": METRIC, "value": ms, "unit": UNIT, "n_gpus": args.gpus, "steps": len(times),
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32 (KoalaBear mod p)",
            "data": "synthetic: the reference benchmark's SmallRng(0) polynomial and point",
            "config": dict(CONFIG, parallelism="cpu"), "impl": "reference",
            "cpu_baseline": {"value": ms, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{len(times)} full n=24 commit+prove runs of the oracle port (OpenMP)"},
            "e2e": {"value": ms, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_sample() -> dict:
    from oracle.oracle import Oracle

    o = Oracle()
    poly, point = inputs(o.rng_fields, 0, N_VARS)
    t0 = time.perf_counter()
    o.prove(oracle_params(), N_VARS, poly, point)
    ms = (time.perf_counter() - t0) * 1e3
    return {"value": ms, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
            "sample": "one full n=24 commit+prove of the oracle port on all host cores (OpenMP)"}


def run_micro(args) -> None:
    kinds = ["eq", "eval", "fold", "dft", "merkle", "grind"] if args.micro == "all" else [args.micro]
    micro_lines(kinds, args.steps, args.warmup, echo=True)


def micro_lines(kinds, steps: int, warmup: int, echo: bool = False) -> list:
    """The kernel micro-benchmarks (eq table, evaluations and fold of 2^24
    extension entries, the commitment LDE, the 2^21-leaf Merkle tree, an
    18-bit proof-of-work search), each timed alone with CUDA events; one dict
    per measurement (printed as a JSON line each with `echo`)."""
    import torch

    import __graft_entry__

    pkg = __graft_entry__.load_package()
    torch.cuda.set_device(0)
    ctx = pkg.Context(0)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    rng = np.random.default_rng(7)
    reps = max(steps, 1)
    lines = []

    def timed(fn):
        for _ in range(max(warmup, 1)):  # the launch-shape tuner runs here, on first use
            fn()
        total = 0.0
        # the timed launches only, for a profiler run with --profile-from-start off
        torch.cuda.profiler.start()
        for _ in range(reps):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            e.synchronize()
            total += s.elapsed_time(e)
        torch.cuda.profiler.stop()
        return total / reps

    def emit(name, ms, alg_bytes=None, units=None, unit_name=None, extra=None):
        line = {"micro": name, "ms": round(ms, 5)}
        if alg_bytes is not None:
            gbs = alg_bytes / (ms * 1e-3) / 1e9
            line.update({"algorithmic_bytes": alg_bytes, "GB/s": round(gbs, 1), "hbm_frac": round(gbs / hbm, 4)})
        if units is not None:
            line[unit_name] = round(units / (ms * 1e-3), 1)
        line.update(extra or {})
        lines.append(line)
        if echo:
            print(json.dumps(line), flush=True)

    n = 24
    N = 1 << n
    if any(k in kinds for k in ("eq", "eval", "fold")):
        f = pkg.DeviceArray(ctx, 4 * N)
        point = rng.integers(0, P, 4 * n, dtype=np.uint64).astype(np.uint32)
        scale = np.array([1, 0, 0, 0], dtype=np.uint32)
        pkg.eq_table(ctx, point, scale, f)  # also initialises f with data
    if "eq" in kinds:
        emit("eq_table 2^24 ext", timed(lambda: pkg.eq_table(ctx, point, scale, f)), alg_bytes=16 * N)
    if "eval" in kinds:
        fb = pkg.DeviceArray.from_host(ctx, rng.integers(0, P, N, dtype=np.uint64).astype(np.uint32))
        emit("eval_base 2^24 base", timed(lambda: pkg.eval_base(ctx, fb, point)), alg_bytes=4 * N)
        emit("eval_ext 2^24 ext", timed(lambda: pkg.eval_ext(ctx, f, point)), alg_bytes=16 * N)
    if "fold" in kinds:
        r = rng.integers(0, P, 4, dtype=np.uint64).astype(np.uint32)
        # in-place compress of the first variable: reads 2^24, writes 2^23 elements
        emit("fold_ext 2^24 -> 2^23 ext", timed(lambda: pkg.fold_ext(ctx, f, n, r)), alg_bytes=16 * N + 8 * N)
    if "dft" in kinds:
        x = pkg.DeviceArray.from_host(ctx, rng.integers(0, P, N, dtype=np.uint64).astype(np.uint32))
        out = pkg.DeviceArray(ctx, 2 * N)
        # KoalaBear's two-adicity is 24, so a single 2^25-point subgroup DFT does not exist; the rate-1/2
        # LDE of 2^24 values is measured in the shape the prover runs it: 16 columns of 2^20 -> 2^21.
        emit("dft 16 x 2^20 -> 16 x 2^21 (commit LDE)", timed(lambda: pkg.dft_batch(ctx, x, n - 4, 4, 1, False, out)),
             alg_bytes=4 * N + 8 * N)
        # the same transform at one fixed plan (split 2^10 x 2^11, register passes, 8 columns per CTA)
        # with pass 2 reading its tile directly and with the tile staged by a TMA tensor copy
        for label, reg2 in (("register pass 2", 1), ("TMA-staged register pass 2", 2)):
            plan = (11, 3, 256, 3, 256, 1, reg2)
            emit(f"dft commit LDE, plan {list(plan)} ({label})",
                 timed(lambda: pkg.dft_batch_plan(ctx, x, n - 4, 4, 1, False, plan, out)), alg_bytes=4 * N + 8 * N)
    if "merkle" in kinds:
        log_h, words = 21, 16
        rows = pkg.DeviceArray.from_host(ctx, rng.integers(0, P, words << log_h, dtype=np.uint64).astype(np.uint32))
        dig = pkg.DeviceArray(ctx, (2 * (1 << log_h) - 1) * 8)
        ms = timed(lambda: pkg.merkle_commit(ctx, rows, log_h, words, 0, dig))
        emit("merkle 2^21 leaves x 16 (P24 leaves, P16 nodes)", ms, alg_bytes=4 * words << log_h,
             units=2 * (1 << log_h) - 1, unit_name="permutations/s")
        # the Keccak MMCS of the reference's Keccak configuration on the same rows
        ms = timed(lambda: pkg.merkle_commit(ctx, rows, log_h, words, 2, dig))
        emit("merkle 2^21 leaves x 16 (Keccak MMCS)", ms, alg_bytes=4 * words << log_h,
             units=2 * (1 << log_h) - 1, unit_name="keccak_f/s")
        # 64 independent trees of 2^10 .. 2^16 leaves x 16 (a batch's commitments): one call per tree
        # (each returning its root) against one multi-instance call for all of them
        hs = [int(h) for h in np.random.default_rng(64).integers(10, 17, 64)]
        trows = [pkg.DeviceArray.from_host(ctx, rng.integers(0, P, words << h, dtype=np.uint64).astype(np.uint32))
                 for h in hs]
        tdig = [pkg.DeviceArray(ctx, (2 * (1 << h) - 1) * 8) for h in hs]
        perms = sum(2 * (1 << h) - 1 for h in hs)
        one = timed(lambda: [pkg.merkle_commit(ctx, r, h, words, 0, d) for r, h, d in zip(trows, hs, tdig)])
        many = timed(lambda: pkg.merkle_commit_many(ctx, trows, hs, words, 0, tdig))
        emit("merkle 64 trees of 2^10..2^16 leaves x 16, one call per tree", one, units=perms,
             unit_name="permutations/s")
        emit("merkle 64 trees of 2^10..2^16 leaves x 16, multi-instance kernels", many, units=perms,
             unit_name="permutations/s", extra={"speedup_vs_one_call_per_tree": round(one / many, 3)})
    if "grind" in kinds:
        bits = 18
        ch = pkg.DuplexChallenger(ctx)
        seq = iter(range(1 << 30))

        evaluated = []

        def grind():
            ch.observe(next(seq))
            ch.grind(bits)
            evaluated.append(ctx.stage_work(reset=True)["grind"])

        ctx.set_profiling(True)  # counts the candidates each search evaluated
        ms = timed(grind)
        ctx.set_profiling(False)
        ctx.stage_times(reset=True)
        timed_evals = evaluated[-reps:]
        emit(f"grind {bits} bits", ms, units=float(np.mean(timed_evals)), unit_name="permutations/s",
             extra={"candidates_evaluated_per_call": [int(v) for v in evaluated],
                    "note": "one Poseidon2-16 permutation per evaluated candidate; expected 2^bits per search"})
        # a small search (the four-lane form, latency-bound: one permutation's latency per pass)
        bits = 10
        evaluated.clear()
        ctx.set_profiling(True)
        ms = timed(grind)
        ctx.set_profiling(False)
        ctx.stage_times(reset=True)
        emit(f"grind {bits} bits (four-lane form)", ms,
             extra={"candidates_evaluated_per_call": [int(v) for v in evaluated[-reps:]]})
    ctx.close()
    return lines


def batch_jobs(pkg, count: int, seed: int):
    """The batching workload: num_variables log-uniform in [16, 22], folding
    factor 3 or 4, starting rate 1/2 or 1/4, 100-bit CapacityBound, pow 16,
    rs reduction 3, one constraint each."""
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(count):
        n = int(round(float(np.exp(rng.uniform(np.log(16), np.log(22))))))
        k = int(rng.choice([3, 4]))
        r = int(rng.choice([1, 2]))
        params = pkg.ProtocolParameters(100, 16, pkg.FoldingFactor.constant(k), pkg.SecurityAssumption.CapacityBound,
                                        r, 3, "poseidon2_24", 32)
        poly = rng.integers(0, P, 1 << n, dtype=np.uint64).astype(np.uint32)
        point = rng.integers(0, P, 4 * n, dtype=np.uint64).astype(np.uint32)
        jobs.append((params, n, poly, point))
    return jobs


def warm_shapes(pkg, ctx, jobs) -> None:
    """One proof per distinct (parameters, size) on one context before any
    timing, so that the launch-shape tuner has already chosen every shape the
    timed runs use and neither arm pays for tuning."""
    seen = set()
    for params, n, poly, point in jobs:
        key = (params.folding_factor.first, params.folding_factor.rest, params.starting_log_inv_rate,
               params.rs_domain_initial_reduction_factor, n)
        if key in seen:
            continue
        seen.add(key)
        pkg.commit_and_prove(ctx, params, n, poly, point)


def run_batch(pkg, ctx, jobs, workers: int) -> dict:
    import time as _t

    warm_shapes(pkg, ctx, jobs)
    t0 = _t.perf_counter()
    plain = [pkg.commit_and_prove(ctx, params, n, poly, point)[0] for params, n, poly, point in jobs]
    t_plain = _t.perf_counter() - t0
    with pkg.Batch(ctx.device, workers=workers) as b:
        # every worker context proves each distinct shape once before timing,
        # and the largest job once (a context's memory pool grows to the
        # largest footprint it has served, and growing it mid-run stalls)
        b.run([pkg.ProofRequest(p, n, poly, pt) for p, n, poly, pt in jobs])
        b.run([pkg.ProofRequest(*largest_job(pkg, jobs)) for _ in range(workers)])
        runs = []
        for _ in range(3):
            reqs = [pkg.ProofRequest(p, n, poly, pt) for p, n, poly, pt in jobs]
            t0 = _t.perf_counter()
            b.run(reqs)
            runs.append(_t.perf_counter() - t0)
    t_batch = sorted(runs)[1]
    same = all(np.array_equal(r.proof, q) for r, q in zip(reqs, plain))
    return {"instances": len(jobs), "workers": workers, "plain_proofs_per_s": round(len(jobs) / t_plain, 2),
            "batched_proofs_per_s": round(len(jobs) / t_batch, 2), "speedup": round(t_plain / t_batch, 3),
            "batched_runs_proofs_per_s": [round(len(jobs) / t, 1) for t in runs],
            "identical_to_plain": bool(same), "timing": "host wall clock around all proofs, median of 3 runs"}


def largest_job(pkg, jobs):
    """The job of the largest device footprint in a list of (params, n, poly, point)."""
    return max(jobs, key=lambda j: pkg.job_footprint(j[0], j[1]))


_SERVE_POLYS: dict = {}


def serve_requests(pkg, count: int, seed: int):
    """Requests with num_variables uniform in [16, 24] (k = 4, rate 1/2), each
    with its own evaluation point; one seeded polynomial per size is shared."""
    rng = np.random.default_rng(seed)
    params = pkg.ProtocolParameters(100, 16, pkg.FoldingFactor.constant(4), pkg.SecurityAssumption.CapacityBound,
                                    1, 3, "poseidon2_24", 32)
    reqs = []
    for _ in range(count):
        n = int(rng.integers(16, 25))
        if n not in _SERVE_POLYS:
            _SERVE_POLYS[n] = np.random.default_rng(100 + n).integers(0, P, 1 << n, dtype=np.uint64).astype(np.uint32)
        point = rng.integers(0, P, 4 * n, dtype=np.uint64).astype(np.uint32)
        reqs.append((params, n, _SERVE_POLYS[n], point))
    return reqs


def run_serve(pkg, ctx, device: int, rate: float, workers: int, count: int, seed: int) -> dict:
    """Poisson arrivals at `rate` req/s into the pool (served) and into a single
    worker (the plain sequential path), same requests and arrival times."""
    import time as _t

    items = serve_requests(pkg, count, seed)
    warm_shapes(pkg, ctx, items)
    gaps = np.random.default_rng(seed + 1).exponential(1.0 / rate, count)
    out = {}
    for label, w in (("served", workers), ("plain", 1)):
        with pkg.Batch(device, workers=w, hbm_budget_bytes=120 << 30) as b:
            # warm up: every worker proves the largest request once, so no
            # context grows its memory pool while serving
            b.run([pkg.ProofRequest(p, n, poly, pt) for p, n, poly, pt in items[: max(w, 2)]])
            b.run([pkg.ProofRequest(*largest_job(pkg, items)) for _ in range(w)])
            reqs = [pkg.ProofRequest(p, n, poly, pt) for p, n, poly, pt in items]
            t0 = _t.perf_counter()
            due = 0.0
            for r, g in zip(reqs, gaps):
                due += g
                wait = due - (_t.perf_counter() - t0)
                if wait > 0:
                    _t.sleep(wait)
                b.submit(r)
            b.wait_all()
            elapsed = max(r.job.t_done_ms for r in reqs) - min(r.job.t_submit_ms for r in reqs)
        lat = np.array([r.latency_ms for r in reqs])
        out[label] = {"throughput_per_s": round(count / (elapsed / 1e3), 2), "p50_ms": round(float(np.percentile(lat, 50)), 3),
                      "p99_ms": round(float(np.percentile(lat, 99)), 3), "workers": w}
        out[label + "_proofs"] = [r.proof for r in reqs]
    same = all(np.array_equal(a, b) for a, b in zip(out.pop("served_proofs"), out.pop("plain_proofs")))
    return {"rate_per_s": rate, "requests": count, **out, "identical_in_mix_and_alone": bool(same),
            "throughput_ratio": round(out["served"]["throughput_per_s"] / out["plain"]["throughput_per_s"], 3)}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--micro", default=None, choices=["all", "eq", "eval", "fold", "dft", "merkle", "grind"])
    ap.add_argument("--batch", action="store_true")
    ap.add_argument("--serve", action="store_true")
    ap.add_argument("--workers", type=int, default=16)
    ap.add_argument("--rates", default="10,50,100,200,500")
    ap.add_argument("--no-batch", action="store_true", help="skip the batch/serve summary in the default run")
    ap.add_argument("--n", type=int, default=N_VARS, help="num_variables of the headline workload")
    ap.add_argument("--constraints", type=int, default=1, help="evaluation constraints of the headline workload")
    ap.add_argument("--no-extra", action="store_true", help="skip the n=26 / four-constraint lines")
    ap.add_argument("--device-transcript", action="store_true",
                    help="run the sumcheck stages' transcript steps on the device (Context.set_device_transcript)")
    args = ap.parse_args()
    if args.micro:
        run_micro(args)
        return
    if args.batch or args.serve:
        import torch

        import __graft_entry__

        pkg = __graft_entry__.load_package()
        torch.cuda.set_device(0)
        ctx = pkg.Context(0)
        if args.batch:
            print(json.dumps({"mode": "batch", **run_batch(pkg, ctx, batch_jobs(pkg, 64, 4), args.workers)}), flush=True)
        if args.serve:
            for rate in [float(x) for x in args.rates.split(",")]:
                count = int(min(400, max(40, rate * 1.0)))
                print(json.dumps({"mode": "serve", **run_serve(pkg, ctx, 0, rate, args.workers, count, 5)}), flush=True)
        ctx.close()
        return
    if args.impl == "reference":
        run_reference(args)
        return

    import torch

    import __graft_entry__

    pkg = __graft_entry__.load_package()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    ctx = pkg.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.set_device_transcript(args.device_transcript)
    params = pkg.ProtocolParameters(100, 16, pkg.FoldingFactor.constant(4), pkg.SecurityAssumption.CapacityBound, 1, 3,
                                    "poseidon2_24", 32)
    n_vars = args.n
    poly, point = inputs_m(pkg.rng_koalabear, rank, n_vars, args.constraints)
    d_poly = pkg.DeviceArray.from_host(ctx, poly)  # resident in HBM, Montgomery form
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def step(poly_arg):
        return pkg.commit_and_prove(ctx, params, n_vars, poly_arg, point)

    for _ in range(max(args.warmup, 3)):
        step(d_poly)
    ref_proof = step(d_poly)[0]
    tuned = pkg.tune_entries()
    autotune = {"mode": pkg.tune_mode(), "shapes": len(tuned),
                "default_ms_sum": round(sum(e["ms_default"] for e in tuned), 4),
                "tuned_ms_sum": round(sum(e["ms_best"] for e in tuned), 4),
                "choices": [f'{e["kind"]}{e["key"]}->{e["choice"]} {e["ms_default"]:.4f}->{e["ms_best"]:.4f} ms'
                            for e in tuned]}

    # ---- device-resident timing (value) ----
    clocks = Clocks(local)
    barrier()
    l0 = pkg.kernel_launches()
    total_ms = 0.0
    torch.cuda.profiler.start()  # the timed steps only, for a profiler run with --profile-from-start off
    for _ in range(args.steps):
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        proof = step(d_poly)[0]
        e.record(stream)
        e.synchronize()
        total_ms += s.elapsed_time(e)
        assert np.array_equal(proof, ref_proof)
    torch.cuda.profiler.stop()
    barrier()
    launches = pkg.kernel_launches() - l0
    clk = clocks.stop()
    step_ms, value = job_value(reduce_over_ranks(total_ms, dist, "cuda"), args.steps, world)

    # ---- end to end through the public API with host buffers ----
    host_poly = torch.from_numpy(poly).pin_memory()
    host_np = host_poly.numpy()
    for _ in range(max(args.warmup, 1)):  # untimed: the pool takes the uploaded polynomial's size once
        step(host_np)
    barrier()
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        proof = step(host_np)[0]
        e.record(stream)
        e.synchronize()
        e2e_ms += s.elapsed_time(e)
    barrier()
    e2e_value = job_value(reduce_over_ranks(e2e_ms, dist, "cuda"), args.steps, world)[1]
    h2d = poly.nbytes + point.nbytes
    d2h = int(proof.size) * 4

    # ---- per-stage device times and work, timed live with CUDA events on the
    # context's stream over a second pass of the same steps ----
    ctx.set_profiling(True)
    ctx.stage_times(reset=True)
    ctx.stage_work(reset=True)
    for _ in range(args.steps):
        flush.zero_()
        step(d_poly)
    stages = ctx.stage_times(reset=True)
    work = ctx.stage_work(reset=True)
    ctx.set_profiling(False)
    stages_ms = {k: round(v[0] / args.steps, 4) for k, v in stages.items()}
    rooflines = stage_rooflines(stages, work, args.steps, clk.get("sm_mhz") or 1965.0)
    primary = max(rooflines, key=lambda r: r["ms_per_proof"])

    extra = None
    if rank == 0 and world == 1 and not args.no_extra:
        # the other sizes of the full-prove configuration: n = 24 and 26, one
        # and four constraints
        extra = [measure_config(pkg, ctx, stream, flush, n, m, 5, 2)
                 for n, m in ((24, 1), (24, 4), (26, 1), (26, 4)) if (n, m) != (n_vars, args.constraints)]
    batch = serve = None
    if rank == 0 and world == 1 and not args.no_batch:
        batch = run_batch(pkg, ctx, batch_jobs(pkg, 64, 4), args.workers)
        serve = []
        for rate in [float(x) for x in args.rates.split(",")]:
            count = int(min(400, max(40, rate * 1.0)))
            serve.append(run_serve(pkg, ctx, local, rate, args.workers, count, 5))
    micro = None
    if rank == 0 and world == 1 and not args.no_extra:
        # the kernel micro-benchmarks at their reference sizes (5 timed runs each)
        micro = micro_lines(["eq", "eval", "fold", "dft", "merkle", "grind"], 5, 2)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample()
    if rank == 0:
        metric = METRIC if n_vars == N_VARS else METRIC.replace("2^24", f"2^{n_vars}")
        line = {"metric": metric, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": round(step_ms, 4), "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "u32 (KoalaBear mod p, exact)",
                "data": "synthetic: the reference benchmark's SmallRng(0) polynomial and point",
                "config": dict(CONFIG, num_variables=n_vars, constraints=args.constraints,
                               parallelism=f"replicas x{world} (one proof per GPU per step)",
                               transcript="device" if args.device_transcript else "host"),
                "proofs_per_s": round(1e3 / value, 3), "proof_words": int(ref_proof.size),
                "e2e": {"value": round(e2e_value, 4), "unit": UNIT, "h2d_bytes_per_step": h2d * world,
                        "d2h_bytes_per_step": d2h * world},
                "gpu_launches": int(launches), "roofline": primary, "rooflines": rooflines,
                "stages_ms_per_proof": stages_ms,
                "autotune": autotune,
                "cpu_baseline": cpu, "clocks": clk,
                "extra": extra, "micro": micro, "batched": batch, "served": serve}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
