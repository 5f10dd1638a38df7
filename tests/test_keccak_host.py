"""The library's host Keccak-256 (the Keccak challenger's hash, whir_keccak256)
against the oracle's and the published known answers; a host-only entry point,
so it runs without a GPU."""
import numpy as np

KATS = {
    b"": "c5d2460186f7233c927e7db2dcc703c0e500b653ca82273b7bfad8045d85a470",
    b"abc": "4e03657aea45a94fc7d47ba826c8d667c0d1e6e33a64a036ec44f58fa12d6c45",
}


def test_host_keccak256_known_answers(pkg):
    for msg, want in KATS.items():
        assert pkg.keccak256(msg).hex() == want


def test_host_keccak256_matches_oracle(pkg, oracle):
    rng = np.random.default_rng(9)
    for n in list(range(0, 300, 7)) + [135, 136, 137, 271, 272, 273, 1000]:
        msg = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert pkg.keccak256(msg) == oracle.keccak256(msg), n
