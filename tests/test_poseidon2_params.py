"""Poseidon2 set-up of the reference (src/bin/main.rs:100-102,
benches/whir.rs:66-68): `Poseidon2KoalaBear<16>::new_from_rng_128` then
`<24>::new_from_rng_128` on one `SmallRng::seed_from_u64(1)`, and the
RNG-drawn benchmark inputs (benches/whir.rs:92-100). No GPU needed.

Pins, from the outside in:
  - the oracle's xoshiro256++ against the outputs of the algorithm's reference
    implementation from state (1, 2, 3, 4), and its seed expansion against
    SplitMix64's outputs for seed 0 (published known answers);
  - a plain-Python restatement of the sampler (next_u32 = high half of
    next_u64; v = next_u32 >> 1, rejected if v >= p; v is the Montgomery word)
    and of p3-poseidon2's constant order (initial external rows, terminal
    external rows, internal constants) against the oracle and the product;
  - the product's host permutations against the oracle's, for both external
    blocks (the circulant (2, 3, 1, 1) of Plonky3's KoalaBear, and the paper's
    M4).
How rand wires SmallRng::seed_from_u64 to the generator and how Plonky3 maps
a sample to a field element are documented behaviour restated here; no
reference output pins them (the reference cannot run in this environment)."""
import ctypes as C

import numpy as np
import pytest

from oracle.oracle import Oracle, P

M64 = (1 << 64) - 1


def _rotl(x, k):
    return ((x << k) | (x >> (64 - k))) & M64


class PySmallRng:
    """xoshiro256++ seeded by SplitMix64 (plain-Python restatement)."""

    def __init__(self, seed):
        self.s = []
        for _ in range(4):
            seed = (seed + 0x9E3779B97F4A7C15) & M64
            z = seed
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
            self.s.append(z ^ (z >> 31))

    def next_u64(self):
        s = self.s
        r = (_rotl((s[0] + s[3]) & M64, 23) + s[0]) & M64
        t = (s[1] << 17) & M64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = _rotl(s[3], 45)
        return r

    def field(self):
        r_inv = pow(1 << 32, P - 2, P)
        while True:
            v = (self.next_u64() >> 32) >> 1
            if v < P:
                return v * r_inv % P


def py_constants(seed):
    g = PySmallRng(seed)
    out = []
    for width, rp in ((16, 20), (24, 23)):
        ext = [g.field() for _ in range(8 * width)]
        internal = [g.field() for _ in range(rp)]
        out.append((ext, internal))
    return out


def test_xoshiro256pp_reference_outputs(oracle):
    # outputs of the xoshiro256++ reference implementation from state (1, 2, 3, 4)
    want = [41943041, 58720359, 3588806011781223, 3591011842654386, 9228616714210784205, 9973669472204895162,
            14011001112246962877, 12406186145184390807, 15849039046786891736, 10450023813501588000]
    st = (C.c_uint64 * 4)(1, 2, 3, 4)
    out = (C.c_uint64 * 10)()
    oracle.lib.or_rng_u64_from_state(st, out, 10)
    assert list(out) == want


def test_splitmix64_seed_expansion(oracle):
    # SplitMix64's first four outputs for seed 0
    st = (C.c_uint64 * 4)()
    oracle.lib.or_rng_seed_state(C.c_uint64(0), st)
    assert list(st) == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F, 0xF88BB8A8724C81EC]


@pytest.mark.parametrize("seed", [0, 1, 7, 2**63 + 5])
def test_field_sampler_matches(pkg, oracle, seed):
    g = PySmallRng(seed)
    want = np.array([g.field() for _ in range(3000)], dtype=np.uint32)
    assert np.array_equal(oracle.rng_fields(seed, 3000), want)
    assert np.array_equal(pkg.rng_koalabear(seed, 3000), want)


@pytest.mark.parametrize("seed", [1, 0, 42])
@pytest.mark.parametrize("mat", [0, 1])
def test_constants_follow_new_from_rng_order(pkg, seed, mat):
    (e16, i16), (e24, i24) = py_constants(seed)
    p16, p24 = pkg.poseidon2_from_rng(seed, mat)
    o = Oracle(p2_seed=seed, p2_mat=mat)
    for prm, oprm, ext, internal, width, rp in ((p16, o.p16, e16, i16, 16, 20), (p24, o.p24, e24, i24, 24, 23)):
        assert (prm.width, prm.rounds_f, prm.rounds_p, prm.external_matrix) == (width, 8, rp, mat)
        assert list(prm.ext_rc[: 8 * width]) == ext and list(prm.int_rc[:rp]) == internal
        assert (oprm.width, oprm.rounds_f, oprm.rounds_p, oprm.mat) == (width, 8, rp, mat)
        assert list(oprm.ext_rc) == list(prm.ext_rc) and list(oprm.int_rc) == list(prm.int_rc)
        assert list(oprm.diag) == list(prm.diag)


def test_default_is_seed_one_with_plonky3_block(pkg):
    d16, d24 = pkg.default_poseidon2()
    s16, s24 = pkg.poseidon2_from_rng(1, pkg.P2_MDS_MAT4)
    assert bytes(d16) == bytes(s16) and bytes(d24) == bytes(s24)
    assert d16.external_matrix == 0 and d24.external_matrix == 0


@pytest.mark.parametrize("mat", [0, 1])
@pytest.mark.parametrize("width", [16, 24])
def test_host_permutation_both_blocks(pkg, mat, width):
    p16, p24 = pkg.poseidon2_from_rng(1, mat)
    o = Oracle(p2_seed=1, p2_mat=mat)
    rng = np.random.default_rng(100 + width + mat)
    with pkg.Context(-1, p16, p24) as ctx:
        for t in range(30):
            s = rng.integers(0, P, width, dtype=np.uint64).astype(np.uint32)
            if t < 3:
                s[:] = (0, 1, P - 1)[t]
            assert np.array_equal(ctx.permute(s), o.permute(s))


def test_blocks_give_different_permutations(pkg):
    a = pkg.poseidon2_from_rng(1, 0)
    b = pkg.poseidon2_from_rng(1, 1)
    s = np.arange(16, dtype=np.uint32)
    with pkg.Context(-1, *a) as ca, pkg.Context(-1, *b) as cb:
        assert not np.array_equal(ca.permute(s), cb.permute(s))


def test_mixed_or_unknown_blocks_rejected(pkg):
    m16, _ = pkg.poseidon2_from_rng(1, 0)
    _, h24 = pkg.poseidon2_from_rng(1, 1)
    with pytest.raises(pkg.WhirError) as e:
        pkg.Context(-1, m16, h24)
    assert e.value.code == -1 and "external matrix" in str(e.value)
    p16, p24 = pkg.poseidon2_from_rng(1, 0)
    p16.external_matrix = p24.external_matrix = 2
    with pytest.raises(pkg.WhirError):
        pkg.Context(-1, p16, p24)
    with pytest.raises(pkg.WhirError):
        pkg.poseidon2_from_rng(1, 2)
