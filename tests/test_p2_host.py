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
