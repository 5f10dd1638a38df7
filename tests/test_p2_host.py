"""The device Poseidon2 header (whir-p3_b200/csrc/poseidon2.cuh) compiled for
the host: the specialised forms the kernels run (the grinding check of output
word 7 with its folded initial layer, for every witness position; the sponge's
zero-capacity and digest-only permutations; each internal-diagonal product; the
64-bit internal sum) agree exactly with the plain permutation and with direct
modular arithmetic. The host and device builds share these templates and
differ only in how the S-box forms its products. No GPU needed."""
import subprocess

from conftest import ROOT


def test_specialised_poseidon2_forms_match_plain(tmp_path):
    exe = tmp_path / "p2_host_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "whir-p3_b200" / "csrc"),
                    str(ROOT / "tests" / "p2_host_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    words = out.stdout.split()
    assert words[0] == "ok" and int(words[1]) > 5000, out.stdout


def test_device_sbox_method_on_unreduced_inputs():
    """The device S-box (poseidon2.cuh `cube`) forms t = v^2 - q p with
    q = round(v * fl(v / p)) (an FMA with 1.5 * 2^52), t in (-p, p) kept
    signed, then r = t * v - q' p with q' = round(t * fl(v / p)) and one
    correction of r, all products modulo 2^32. Its inputs are round-constant
    sums that skip their reduction (below 2p), so it must hold for every
    v < 2^32. Emulated here in IEEE double with an exactly rounded FMA."""
    import random
    import struct
    from fractions import Fraction

    p = 2**31 - 2**24 + 1
    inv_p, magic = 1.0 / p, 6755399441055744.0

    def low_word(ad, bp):
        q = float(Fraction(ad) * Fraction(bp) + Fraction(magic))
        return struct.unpack("<Q", struct.pack("<d", q))[0] & 0xFFFFFFFF

    def cube(v):
        vd = float(v)
        vp = vd * inv_p
        t = (v * v - low_word(vd, vp) * p) & 0xFFFFFFFF
        ts = t - (1 << 32) if t >= 1 << 31 else t
        assert -p < ts < p
        r = (t * v - low_word(float(ts), vp) * p) & 0xFFFFFFFF
        return min(r, (r + p) & 0xFFFFFFFF)

    rng = random.Random(3)
    vals = [0, 1, p - 1, p, p + 1, 2 * p - 2, 2**31 - 1, 2**31, 2**32 - 2, 2**32 - 1]
    vals += [rng.randrange(2 * p) for _ in range(6000)] + [rng.randrange(2**32) for _ in range(6000)]
    for v in vals:
        assert cube(v) == pow(v, 3, p), v
