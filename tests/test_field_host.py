"""The product's field header (whir-p3_b200/csrc/kb.cuh) compiled for the host
and checked exactly against Python integer arithmetic: Montgomery products,
the wide reduction used for sums of four products, and the quartic extension
product (X^4 = 3). No GPU needed."""
import random
import subprocess

import pytest

from conftest import ROOT

P = 0x7F000001
R_INV = pow(1 << 32, P - 2, P)


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    exe = tmp_path_factory.mktemp("kb") / "kb_host_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "whir-p3_b200" / "csrc"),
                    str(ROOT / "tests" / "kb_host_check.cpp"), "-o", str(exe)], check=True)
    return exe


def run(exe, lines):
    out = subprocess.run([str(exe)], input="\n".join(lines) + "\n", capture_output=True, text=True, check=True)
    return out.stdout.split("\n")


def efmul(a, b):
    t = [0] * 7
    for i in range(4):
        for j in range(4):
            t[i + j] += a[i] * b[j]
    return [(t[k] + 3 * (t[k + 4] if k + 4 < 7 else 0)) % P for k in range(4)]


def test_mul(harness):
    rnd = random.Random(1)
    edge = [0, 1, 2, P - 1, P - 2, (P - 1) // 2, 1 << 24, (1 << 31) - (1 << 24)]
    pairs = [(a, b) for a in edge for b in edge] + [(rnd.randrange(P), rnd.randrange(P)) for _ in range(3000)]
    got = run(harness, [f"mul {a} {b}" for a, b in pairs])
    for (a, b), g in zip(pairs, got):
        assert int(g) == a * b % P


def test_reduce_wide_full_range(harness):
    rnd = random.Random(2)
    limit = 2 * P * (1 << 32)
    ts = [0, 1, limit - 1, 4 * (P - 1) ** 2, P << 32, (P << 32) + 12345, ((2 * P - 1) << 32) + (1 << 32) - 1]
    ts += [rnd.randrange(limit) for _ in range(3000)]
    ts += [rnd.randrange(P << 32, limit) for _ in range(3000)]  # the range where the sign must come from the borrow
    got = run(harness, [f"red {t}" for t in ts])
    for t, g in zip(ts, got):
        assert int(g) == t * R_INV % P, t


def test_extension_mul(harness):
    rnd = random.Random(3)
    cases = [([P - 1] * 4, [P - 1] * 4), ([0] * 4, [1, 2, 3, 4]), ([1, 0, 0, 0], [5, 6, 7, 8])]
    cases += [([rnd.randrange(P) for _ in range(4)], [rnd.randrange(P) for _ in range(4)]) for _ in range(2000)]
    got = run(harness, ["ef " + " ".join(map(str, a + b)) for a, b in cases])
    for (a, b), g in zip(cases, got):
        assert list(map(int, g.split())) == efmul(a, b)


def test_shoup_constant_product_any_32bit_input(harness):
    """mul_shoup(a, w, shoup_const(w)) = a * w mod p, fully reduced, for every
    32-bit a (Montgomery states never exceed p, but the bound holds to 2^32)."""
    rnd = random.Random(4)
    ws = [0, 1, 2, P - 1, P - 2, (P - 1) // 2, 1 << 24] + [rnd.randrange(P) for _ in range(40)]
    aa = [0, 1, P - 1, P, P + 1, 2 * P - 1, 2 * P, (1 << 32) - 1, (1 << 31)] + [rnd.randrange(1 << 32) for _ in range(60)]
    pairs = [(a, w) for a in aa for w in ws]
    got = run(harness, [f"shoup {a} {w}" for a, w in pairs])
    for (a, w), g in zip(pairs, got):
        assert int(g) == a * w % P, (a, w)
