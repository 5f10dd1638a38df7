"""Proof wire format (whir_proof_to_bincode / whir_proof_from_bincode): the
library's flat proof stream and the bytes bincode::serialize gives for the
reference's WhirProof (src/whir/proof.rs:11-141, src/bin/main.rs:221). The
oracle's proofs are encoded by the library and by a separate Python encoder
written here from the same layout rules, compared byte for byte, and decoded
back to the same words. The Plonky3 serde forms (field elements as their
Montgomery u32, digests and extension elements as fixed arrays, Merkle proofs
as Vec<[F; 8]>) are assumed, not checked against the reference. No GPU."""
import struct

import numpy as np
import pytest

from oracle.oracle import P, make_params

R = (1 << 32) % P


def py_encode(words):
    """bincode 1.3 default options: little-endian fixed-width integers, u64
    sequence lengths, one-byte Option tags, structs as their fields in order,
    fixed arrays without a length, internally tagged QueryOpening."""
    w = [int(x) for x in words]
    pos = [2]
    out = bytearray()

    def nxt():
        v = w[pos[0]]
        pos[0] += 1
        return v

    def fields(k):
        for _ in range(k):
            out.extend(struct.pack("<I", nxt() * R % P))

    def seq(k):
        out.extend(struct.pack("<Q", k))

    def sumcheck():
        n = nxt()
        seq(n)
        fields(8 * n)
        m = nxt()
        seq(m)
        fields(m)

    def queries():
        nq = nxt()
        seq(nq)
        for _ in range(nq):
            kind = nxt()
            tag = b"extension" if kind else b"base"
            seq(len(tag))
            out.extend(tag)
            nv = nxt()
            seq(nv)
            fields(nv * (4 if kind else 1))
            path = nxt()
            seq(path)
            fields(8 * path)

    assert w[0] == 0x50524857 and w[1] == 1
    out.append(1)
    fields(8)
    n = nxt()
    seq(n)
    fields(4 * n)
    sumcheck()
    nr = nxt()
    seq(nr)
    for _ in range(nr):
        out.append(1)
        fields(8)
        n = nxt()
        seq(n)
        fields(4 * n)
        fields(1)
        queries()
        sumcheck()
    nf = nxt()
    out.append(1)
    seq(nf)
    fields(4 * nf)
    fields(1)
    queries()
    has = nxt()
    out.append(has)
    if has:
        sumcheck()
    assert pos[0] == len(w)
    return bytes(out)


CASES = [(8, 2, 2, 1, 1, 8, 1, 10), (10, 3, 3, 2, 0, 32, 2, 0), (12, 4, 4, 1, 0, 32, 1, 5), (9, 5, 2, 1, 1, 8, 0, 0),
         (14, 4, 4, 3, 0, 32, 1, 8)]


@pytest.mark.parametrize("n,f0,f,rs,leaf,dig,npts,pw", CASES)
def test_bincode_round_trip(pkg, oracle, n, f0, f, rs, leaf, dig, npts, pw):
    rng = np.random.default_rng(n * 31 + f)
    poly = rng.integers(0, P, 1 << n, dtype=np.uint64).astype(np.uint32)
    pts = rng.integers(0, P, 4 * n * npts, dtype=np.uint64).astype(np.uint32) if npts else None
    proof, _ = oracle.prove(make_params(32, pw, f, f0, 2, 1, rs, leaf, dig), n, poly, pts)
    data = pkg.proof_to_bincode(proof)
    assert data == py_encode(proof)
    assert data[0] == 1 and struct.unpack("<8I", data[1:33]) == tuple(int(v) * R % P for v in proof[2:10])
    assert np.array_equal(pkg.proof_from_bincode(data), proof)


def test_bincode_rejects_malformed(pkg, oracle):
    rng = np.random.default_rng(1)
    poly = rng.integers(0, P, 1 << 10, dtype=np.uint64).astype(np.uint32)
    proof, _ = oracle.prove(make_params(32, 0, 2, None, 2, 1, 1, 0, 8), 10, poly, None)
    data = pkg.proof_to_bincode(proof)
    for bad in (data[:-1], data + b"\x00", b"\x00" + data[1:], data[:1] + b"\xff\xff\xff\x7f" + data[5:]):
        with pytest.raises(pkg.WhirError):
            pkg.proof_from_bincode(bad)
    with pytest.raises(pkg.WhirError):
        pkg.proof_to_bincode(proof[:-1])
    tag = data.find(b"base")
    if tag >= 0:
        with pytest.raises(pkg.WhirError):
            pkg.proof_from_bincode(data[:tag] + b"bass" + data[tag + 4:])
