"""C-ABI boundary checks that need no GPU: the library loads, exports every
symbol declared in include/whir_b200.h, and its host-side logic (Poseidon2
data and permutation, WhirConfig derivation, domain separator, duplex
challenger) agrees with the oracle word for word."""
import re

import numpy as np
import pytest

from conftest import ROOT
from oracle.oracle import Chal, P, make_params


def header_functions():
    text = (ROOT / "include" / "whir_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(whir_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol(pkg):
    lib = pkg.lib()
    names = header_functions()
    assert len(names) >= 35
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_host_only_context_rejects_device_work(pkg, host_ctx):
    arr_ptr = None
    with pytest.raises(pkg.WhirError) as e:
        pkg.lib()
        pkg._check(pkg.lib().whir_monty_encode(host_ctx.handle, arr_ptr, 0))
    assert e.value.code == -6


def test_default_poseidon2_matches_oracle(pkg, oracle):
    p16, p24 = pkg.default_poseidon2()
    for a, b in ((p16, oracle.p16), (p24, oracle.p24)):
        assert (a.width, a.rounds_f, a.rounds_p) == (b.width, b.rounds_f, b.rounds_p)
        assert list(a.ext_rc) == list(b.ext_rc)
        assert list(a.int_rc) == list(b.int_rc)
        assert list(a.diag) == list(b.diag)


@pytest.mark.parametrize("width", [16, 24])
def test_internal_matrix_conditions(oracle, width):
    """The fixed internal matrix 1*1^T + diag(mu) meets the Poseidon2 paper's
    conditions (eprint 2023/323, sec. 5.3): invertible, and the characteristic
    polynomial of every power M^k, k = 1 .. 2t, irreducible (no invariant
    subspace trails)."""
    sympy = pytest.importorskip("sympy")
    d = [int(v) for v in (oracle.p16 if width == 16 else oracle.p24).diag[:width]]
    assert all(d) and (1 + sum(pow(v, P - 2, P) for v in d)) % P != 0
    m = sympy.Matrix(width, width, lambda i, j: (1 + (d[i] if i == j else 0)) % P)
    x = sympy.symbols("x")
    mk = m
    for k in range(1, 2 * width + 1):
        if k > 1:
            mk = (mk * m).applyfunc(lambda v: v % P)
        assert sympy.Poly(mk.charpoly(x).as_expr(), x, modulus=P).is_irreducible, k


def test_custom_internal_diagonal_rejected(pkg):
    """The internal diagonal is fixed, as in p3-koala-bear; a parameter set
    carrying another one is refused at context creation."""
    p16, p24 = pkg.default_poseidon2()
    p24.diag[5] = (p24.diag[5] + 1) % P
    with pytest.raises(pkg.WhirError) as e:
        pkg.Context(-1, p16, p24)
    assert e.value.code == -1 and "diagonal" in str(e.value)


@pytest.mark.parametrize("width", [16, 24])
def test_permutation_matches_oracle(host_ctx, oracle, width):
    rng = np.random.default_rng(width)
    for _ in range(20):
        s = rng.integers(0, P, width, dtype=np.uint64).astype(np.uint32)
        assert np.array_equal(host_ctx.permute(s), oracle.permute(s))
    # edge values
    for v in (0, 1, P - 1):
        s = np.full(width, v, dtype=np.uint32)
        assert np.array_equal(host_ctx.permute(s), oracle.permute(s))


def _cfg_tuple(c):
    rounds = [(r.pow_bits, r.folding_pow_bits, r.num_queries, r.ood_samples, r.num_variables, r.folding_factor,
               r.domain_size, r.folded_domain_gen) for r in list(c.rounds)[: c.n_rounds]]
    return (c.num_variables, c.commitment_ood_samples, c.starting_folding_pow_bits, c.n_rounds, rounds,
            c.final_queries, c.final_pow_bits, c.final_sumcheck_rounds, c.final_folding_pow_bits)


CONFIG_GRID = [(n, sec, pw, f0, f, snd, r, rs) for n in (1, 4, 7, 10, 16, 18, 20, 24, 26)
               for sec in (32, 90, 100, 128) for pw in (0, 16, 20) for (f0, f) in ((1, 1), (2, 2), (3, 2), (4, 4), (5, 2))
               for snd in (0, 1, 2) for r in (1, 2) for rs in (1, 2, 3)
               if f0 <= n and f <= n and rs <= f0 and n + r - f0 <= 24]


def test_config_matches_oracle(pkg, oracle):
    checked = 0
    for (n, sec, pw, f0, f, snd, r, rs) in CONFIG_GRID:
        params = pkg.ProtocolParameters(sec, pw, pkg.FoldingFactor(f0, f), pkg.SecurityAssumption(snd), r, rs)
        mine = pkg.WhirConfig(n, params)
        ref = oracle.config(make_params(sec, pw, f, f0, snd, r, rs), n)
        assert _cfg_tuple(mine._c) == _cfg_tuple(ref), (n, sec, pw, f0, f, snd, r, rs)
        for dig in (8, 32):
            assert np.array_equal(pkg.DomainSeparator(mine, dig).pattern, oracle.domain_separator(ref, dig))
        checked += 1
    assert checked > 1000


def test_config_rejects_invalid(pkg):
    with pytest.raises(pkg.WhirError):
        pkg.WhirConfig(3, pkg.ProtocolParameters(folding_factor=pkg.FoldingFactor.constant(5)))
    with pytest.raises(pkg.WhirError):
        pkg.WhirConfig(10, pkg.ProtocolParameters(folding_factor=pkg.FoldingFactor.constant(2),
                                                  rs_domain_initial_reduction_factor=3))
    with pytest.raises(pkg.WhirError):
        pkg.WhirConfig(10, pkg.ProtocolParameters(folding_factor=pkg.FoldingFactor.constant(0)))


def test_challenger_matches_oracle(pkg, host_ctx, oracle):
    import ctypes as C

    rng = np.random.default_rng(3)
    ch = pkg.DuplexChallenger(host_ctx)
    oc = Chal()
    oracle.lib.or_chal_init(C.byref(oc))
    for step in range(300):
        op = rng.integers(0, 4)
        if op == 0:
            vals = rng.integers(0, P, rng.integers(1, 20), dtype=np.uint64).astype(np.uint32)
            ch.observe_slice(vals)
            for v in vals:
                oracle.lib.or_chal_observe(C.byref(oc), C.byref(oracle.p16), int(v))
        elif op == 1:
            assert ch.sample() == oracle.lib.or_chal_sample(C.byref(oc), C.byref(oracle.p16))
        elif op == 2:
            bits = int(rng.integers(0, 31))
            assert ch.sample_bits(bits) == oracle.lib.or_chal_sample_bits(C.byref(oc), C.byref(oracle.p16), bits)
        else:
            bits = int(rng.integers(1, 4))
            w = int(rng.integers(0, 64))
            a = ch.check_witness(bits, w)
            b = bool(oracle.lib.or_chal_check_witness(C.byref(oc), C.byref(oracle.p16), bits, w))
            assert a == b
    assert list(ch.c.state) == list(oc.state)


def test_job_footprint_grows_with_size(pkg):
    params = pkg.ProtocolParameters(100, 16, pkg.FoldingFactor.constant(4), pkg.SecurityAssumption.CapacityBound, 1, 3)
    sizes = [pkg.job_footprint(params, n) for n in range(12, 27)]
    assert all(a < b for a, b in zip(sizes, sizes[1:]))
    # n = 24: polynomial 64 + commit codeword 128 + commit digests 128 + f, w 32 MiB, plus the round-1
    # peak: round-0 tree (64 + 16) + round-1 codeword 32 + digests 8 + DFT scratch 32 = 152 MiB
    assert sizes[24 - 12] == (64 + 128 + 128 + 32 + 152) * 2**20
    assert pkg.job_footprint(params, 24, True) == sizes[24 - 12] - 64 * 2**20


@pytest.mark.parametrize("log_chunk,log_w,log_blowup,ext", [(20, 4, 1, 0), (16, 4, 3, 1), (8, 4, 3, 1), (0, 0, 0, 0),
                                                           (12, 0, 12, 0), (4, 12, 1, 1), (24, 0, 0, 0)])
def test_dft_candidate_plans_are_in_bounds(pkg, log_chunk, log_w, log_blowup, ext):
    """Every plan the tuner may time keeps each pass <= 2^12 points, its tiles
    within 128 KiB of shared memory and its tile counts within the shape."""
    plans = pkg.dft_plans(log_chunk, log_w, log_blowup, bool(ext))
    assert plans, "the default plan is always a candidate"
    lanes = 4 if ext else 1
    log_h = log_chunk + log_blowup
    def reg_ok(m, lt, threads):
        # register pass: 2^m points as E x G (E >= G) with G threads per vector and 2^lt
        # vectors per CTA, holding 2^lt * E * (G + 1) words of shared memory (plus padding)
        lg = m // 2
        le = m - lg
        return 8 <= m <= 12 and threads == 1 << (lg + lt) and (4 << lt) * (1 << le) * ((1 << lg) + 1) <= 128 * 1024

    for h2, t1, th1, t2, th2, reg1, reg2 in plans:
        if h2 == 0:
            assert not reg1 and not reg2 and th1 in (128, 256, 512)
            assert log_chunk <= 12 and 0 <= t1 <= log_w
            assert (4 * lanes << t1 << log_chunk) <= 128 * 1024
        else:
            h1 = log_h - h2
            ls = 2 if ext else 0  # register passes count tiles in words
            assert 1 <= h2 <= min(12, log_chunk) and 0 <= h1 <= 12
            if reg1:
                assert 2 <= t1 <= 4 and t1 <= h2 + ls and reg_ok(h1, t1, th1)
            else:
                assert 0 <= t1 <= h2 and th1 in (128, 256, 512) and (4 * lanes << t1 << h1) <= 128 * 1024
            if reg2:
                assert ls <= t2 <= 4 and t2 <= log_w + ls and reg_ok(h2, t2, th2)
            else:
                assert 0 <= t2 <= log_w and th2 in (128, 256, 512) and (4 * lanes << t2 << h2) <= 128 * 1024


def test_tune_mode_switch(pkg):
    assert pkg.tune_mode() == 1
    with pytest.raises(pkg.WhirError):
        pkg.set_tune_mode(2)
    pkg.set_tune_mode(0)
    assert pkg.tune_mode() == 0
    pkg.set_tune_mode(1)
    pkg.tune_clear()
    assert pkg.tune_entries() == []
