"""Oracle loader (test infrastructure only).

ctypes bindings for oracle/_build/liboracle.so, the CPU restatement of the
WHIR prover hot path. Only tests/, __graft_entry__.smoke() and the CPU-baseline
leg of bench.py import this module, and only as the checker or the timed CPU
baseline; the product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
P = 0x7F000001


def build(force: bool = False) -> pathlib.Path:
    if force or not LIB_PATH.exists():
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


class P2Params(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("rounds_f", C.c_uint32),
        ("rounds_p", C.c_uint32),
        ("mat", C.c_uint32),
        ("ext_rc", C.c_uint32 * (8 * 24)),
        ("int_rc", C.c_uint32 * 32),
        ("diag", C.c_uint32 * 24),
    ]


class Params(C.Structure):
    _fields_ = [
        ("security_level", C.c_int32),
        ("pow_bits", C.c_int32),
        ("folding_factor_0", C.c_int32),
        ("folding_factor", C.c_int32),
        ("soundness", C.c_int32),
        ("starting_log_inv_rate", C.c_int32),
        ("rs_reduction", C.c_int32),
        ("leaf_hash", C.c_int32),
        ("ds_digest_elems", C.c_int32),
    ]


class RoundCfg(C.Structure):
    _fields_ = [
        ("pow_bits", C.c_int32),
        ("folding_pow_bits", C.c_int32),
        ("num_queries", C.c_int32),
        ("ood_samples", C.c_int32),
        ("num_variables", C.c_int32),
        ("folding_factor", C.c_int32),
        ("domain_size", C.c_uint64),
        ("folded_domain_gen", C.c_uint32),
    ]


class Config(C.Structure):
    _fields_ = [
        ("num_variables", C.c_int32),
        ("security_level", C.c_int32),
        ("max_pow_bits", C.c_int32),
        ("commitment_ood_samples", C.c_int32),
        ("starting_log_inv_rate", C.c_int32),
        ("starting_folding_pow_bits", C.c_int32),
        ("folding_factor_0", C.c_int32),
        ("folding_factor", C.c_int32),
        ("rs_reduction", C.c_int32),
        ("soundness", C.c_int32),
        ("n_rounds", C.c_int32),
        ("rounds", RoundCfg * 32),
        ("final_queries", C.c_int32),
        ("final_pow_bits", C.c_int32),
        ("final_sumcheck_rounds", C.c_int32),
        ("final_folding_pow_bits", C.c_int32),
    ]


class Chal(C.Structure):
    _fields_ = [
        ("state", C.c_uint32 * 16),
        ("inp", C.c_uint32 * 8),
        ("in_len", C.c_int32),
        ("out", C.c_uint32 * 8),
        ("out_len", C.c_int32),
    ]


SOUNDNESS = {"UniqueDecoding": 0, "JohnsonBound": 1, "CapacityBound": 2}

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


class Oracle:
    def __init__(self, path: os.PathLike | None = None, p2_seed: int = 1, p2_mat: int = 0):
        """p2_seed, p2_mat: the Poseidon2 permutations, new_from_rng_128 on
        SmallRng::seed_from_u64(p2_seed) with external block p2_mat (0: the
        circulant (2, 3, 1, 1) of Plonky3's KoalaBear; 1: the paper's M4)."""
        self.lib = C.CDLL(str(path or build()))
        L = self.lib
        L.or_p2_default.argtypes = [C.POINTER(P2Params), C.POINTER(P2Params)]
        L.or_p2_from_rng.argtypes = [C.c_uint64, C.c_uint32, C.POINTER(P2Params), C.POINTER(P2Params)]
        L.or_p2_select.argtypes = [C.POINTER(P2Params), C.POINTER(P2Params)]
        L.or_rng_fields.argtypes = [C.c_uint64, _u32p, C.c_size_t]
        L.or_rng_seed_state.argtypes = [C.c_uint64, C.POINTER(C.c_uint64)]
        L.or_rng_u64_from_state.argtypes = [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_size_t]
        L.or_p2_permute.argtypes = [C.POINTER(P2Params), _u32p]
        L.or_config_new.argtypes = [C.POINTER(Params), C.c_int, C.POINTER(Config)]
        L.or_config_new.restype = C.c_int
        L.or_chal_init.argtypes = [C.POINTER(Chal)]
        L.or_chal_observe.argtypes = [C.POINTER(Chal), C.POINTER(P2Params), C.c_uint32]
        L.or_chal_sample.argtypes = [C.POINTER(Chal), C.POINTER(P2Params)]
        L.or_chal_sample.restype = C.c_uint32
        L.or_chal_sample_bits.argtypes = [C.POINTER(Chal), C.POINTER(P2Params), C.c_int]
        L.or_chal_sample_bits.restype = C.c_uint64
        L.or_chal_grind.argtypes = [C.POINTER(Chal), C.POINTER(P2Params), C.c_int]
        L.or_chal_grind.restype = C.c_uint32
        L.or_chal_check_witness.argtypes = [C.POINTER(Chal), C.POINTER(P2Params), C.c_int, C.c_uint32]
        L.or_chal_check_witness.restype = C.c_int
        L.or_domain_separator.argtypes = [C.POINTER(Config), C.c_int, C.c_void_p, C.c_int]
        L.or_domain_separator.restype = C.c_int
        L.or_dft_batch.argtypes = [_u32p, C.c_int, C.c_int, C.c_int, C.c_int, _u32p]
        L.or_merkle_build.argtypes = [C.POINTER(P2Params), C.POINTER(P2Params), C.c_int, _u32p, C.c_int,
                                      C.c_int, _u32p, _u32p]
        L.or_eq_table.argtypes = [_u32p, C.c_int, _u32p, _u32p]
        L.or_eval_base.argtypes = [_u32p, C.c_int, _u32p, _u32p]
        L.or_eval_ext.argtypes = [_u32p, C.c_int, _u32p, _u32p]
        L.or_fold_ext.argtypes = [_u32p, C.c_int, _u32p]
        L.or_fold_base.argtypes = [_u32p, C.c_int, _u32p, _u32p]
        L.or_fold_multi_base.argtypes = [_u32p, C.c_int, _u32p, C.c_int, _u32p]
        L.or_sumcheck_coeffs.argtypes = [_u32p, _u32p, C.c_int, _u32p, _u32p]
        L.or_extrapolate_012.argtypes = [_u32p, _u32p, _u32p, _u32p, _u32p]
        L.or_combine_select.argtypes = [_u32p, C.c_int, _u32p, C.c_int, _u32p]
        L.or_whir_prove.argtypes = [C.POINTER(Params), C.c_int, _u32p, C.c_void_p, C.c_int,
                                    C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_size_t), _u32p]
        L.or_whir_prove.restype = C.c_int
        L.or_whir_verify.argtypes = [C.POINTER(Params), C.c_int, C.c_void_p, C.c_void_p, C.c_int, _u32p,
                                     C.c_size_t, _u32p]
        L.or_whir_verify.restype = C.c_int
        L.or_free.argtypes = [C.c_void_p]
        L.or_keccak256.argtypes = [C.c_char_p, C.c_size_t, C.c_void_p]
        L.or_keccak_f1600.argtypes = [C.c_void_p]
        self.p16 = P2Params()
        self.p24 = P2Params()
        L.or_p2_from_rng(p2_seed, p2_mat, C.byref(self.p16), C.byref(self.p24))

    # ---- primitives -------------------------------------------------------
    def keccak256(self, data: bytes) -> bytes:
        """Keccak-256 (original Keccak padding, as p3-keccak's Keccak256Hash)."""
        out = (C.c_uint8 * 32)()
        self.lib.or_keccak256(data, len(data), out)
        return bytes(out)

    def keccak_f1600(self, lanes: np.ndarray) -> np.ndarray:
        """Keccak-f[1600] on 25 64-bit lanes (lane x + 5y)."""
        st = np.ascontiguousarray(lanes, dtype=np.uint64).copy()
        self.lib.or_keccak_f1600(st.ctypes.data)
        return st

    def rng_fields(self, seed: int, count: int) -> np.ndarray:
        """rng.random::<KoalaBear>() drawn `count` times from SmallRng::seed_from_u64(seed)."""
        out = np.empty(count, dtype=np.uint32)
        self.lib.or_rng_fields(seed, out, count)
        return out

    def permute(self, state: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(state, dtype=np.uint32).copy()
        self.lib.or_p2_permute(C.byref(self.p16 if len(s) == 16 else self.p24), s)
        return s

    def config(self, params: Params, n: int) -> Config:
        c = Config()
        rc = self.lib.or_config_new(C.byref(params), n, C.byref(c))
        if rc:
            raise ValueError(f"or_config_new failed: {rc}")
        return c

    def domain_separator(self, cfg: Config, digest_elems: int) -> np.ndarray:
        n = self.lib.or_domain_separator(C.byref(cfg), digest_elems, None, 0)
        out = np.zeros(n, dtype=np.uint32)
        self.lib.or_domain_separator(C.byref(cfg), digest_elems, out.ctypes.data, n)
        return out

    def dft_batch(self, chunks: np.ndarray, log_chunk: int, log_width: int, log_blowup: int, ext: bool):
        lanes = 4 if ext else 1
        out = np.zeros((1 << (log_chunk + log_blowup)) * (1 << log_width) * lanes, dtype=np.uint32)
        self.lib.or_dft_batch(np.ascontiguousarray(chunks, dtype=np.uint32), log_chunk, log_width, log_blowup,
                              int(ext), out)
        return out

    def merkle(self, rows: np.ndarray, log_h: int, row_words: int, leaf_hash: int = 0):
        h = 1 << log_h
        dig = np.zeros((2 * h - 1) * 8, dtype=np.uint32)
        root = np.zeros(8, dtype=np.uint32)
        self.lib.or_merkle_build(C.byref(self.p16), C.byref(self.p24), leaf_hash,
                                 np.ascontiguousarray(rows, dtype=np.uint32), log_h, row_words, dig, root)
        return root, dig

    def eq_table(self, point: np.ndarray, scale=(1, 0, 0, 0)) -> np.ndarray:
        n = len(point) // 4
        out = np.zeros((1 << n) * 4, dtype=np.uint32)
        self.lib.or_eq_table(np.ascontiguousarray(point, dtype=np.uint32), n,
                             np.array(scale, dtype=np.uint32), out)
        return out

    def eval_base(self, evals, point) -> np.ndarray:
        out = np.zeros(4, dtype=np.uint32)
        n = len(point) // 4
        self.lib.or_eval_base(np.ascontiguousarray(evals, dtype=np.uint32), n,
                              np.ascontiguousarray(point, dtype=np.uint32), out)
        return out

    def eval_ext(self, evals, point) -> np.ndarray:
        out = np.zeros(4, dtype=np.uint32)
        n = len(point) // 4
        self.lib.or_eval_ext(np.ascontiguousarray(evals, dtype=np.uint32), n,
                             np.ascontiguousarray(point, dtype=np.uint32), out)
        return out

    def fold_ext(self, evals, r) -> np.ndarray:
        e = np.ascontiguousarray(evals, dtype=np.uint32).copy()
        n = (len(e) // 4).bit_length() - 1
        self.lib.or_fold_ext(e, n, np.array(r, dtype=np.uint32))
        return e[: len(e) // 2]

    def fold_base(self, evals, r) -> np.ndarray:
        e = np.ascontiguousarray(evals, dtype=np.uint32)
        n = len(e).bit_length() - 1
        out = np.zeros(len(e) // 2 * 4, dtype=np.uint32)
        self.lib.or_fold_base(e, n, np.array(r, dtype=np.uint32), out)
        return out

    def fold_multi_base(self, evals, rs) -> np.ndarray:
        e = np.ascontiguousarray(evals, dtype=np.uint32)
        n = len(e).bit_length() - 1
        k = len(rs) // 4
        out = np.zeros((1 << (n - k)) * 4, dtype=np.uint32)
        self.lib.or_fold_multi_base(e, n, np.ascontiguousarray(rs, dtype=np.uint32), k, out)
        return out

    def sumcheck_coeffs(self, f, w):
        n = (len(f) // 4).bit_length() - 1
        c0 = np.zeros(4, dtype=np.uint32)
        c2 = np.zeros(4, dtype=np.uint32)
        self.lib.or_sumcheck_coeffs(np.ascontiguousarray(f, dtype=np.uint32),
                                    np.ascontiguousarray(w, dtype=np.uint32), n, c0, c2)
        return c0, c2

    def extrapolate_012(self, e0, e1, e2, r) -> np.ndarray:
        out = np.zeros(4, dtype=np.uint32)
        a = [np.ascontiguousarray(v, dtype=np.uint32) for v in (e0, e1, e2, r)]
        self.lib.or_extrapolate_012(*a, out)
        return out

    def combine_select(self, weights, vars_, gamma_pows) -> np.ndarray:
        w = np.ascontiguousarray(weights, dtype=np.uint32).copy()
        n = (len(w) // 4).bit_length() - 1
        self.lib.or_combine_select(w, n, np.ascontiguousarray(vars_, dtype=np.uint32), len(vars_),
                                   np.ascontiguousarray(gamma_pows, dtype=np.uint32))
        return w

    # ---- end to end -------------------------------------------------------
    def prove(self, params: Params, n: int, poly: np.ndarray, points: np.ndarray | None):
        poly = np.ascontiguousarray(poly, dtype=np.uint32)
        npts = 0 if points is None else len(points) // (4 * n)
        pts = None if points is None or npts == 0 else np.ascontiguousarray(points, dtype=np.uint32)
        out = C.POINTER(C.c_uint32)()
        words = C.c_size_t()
        cp = np.zeros(4, dtype=np.uint32)
        self.lib.or_p2_select(C.byref(self.p16), C.byref(self.p24))
        rc = self.lib.or_whir_prove(C.byref(params), n, poly, None if pts is None else pts.ctypes.data, npts,
                                    C.byref(out), C.byref(words), cp)
        if rc:
            raise ValueError(f"or_whir_prove failed: {rc}")
        proof = np.ctypeslib.as_array(out, shape=(words.value,)).copy()
        self.lib.or_free(out)
        return proof, cp

    def verify(self, params: Params, n: int, points, evals, proof) -> tuple[int, np.ndarray]:
        npts = 0 if points is None else len(points) // (4 * n)
        pts = None if npts == 0 else np.ascontiguousarray(points, dtype=np.uint32)
        evs = None if npts == 0 else np.ascontiguousarray(evals, dtype=np.uint32)
        cp = np.zeros(4, dtype=np.uint32)
        proof = np.ascontiguousarray(proof, dtype=np.uint32)
        self.lib.or_p2_select(C.byref(self.p16), C.byref(self.p24))
        rc = self.lib.or_whir_verify(C.byref(params), n, None if pts is None else pts.ctypes.data,
                                     None if evs is None else evs.ctypes.data, npts, proof, len(proof), cp)
        return rc, cp


def make_params(security_level=100, pow_bits=16, folding_factor=4, folding_factor_0=None,
                soundness="CapacityBound", starting_log_inv_rate=1, rs_reduction=1, leaf_hash=0,
                ds_digest_elems=32) -> Params:
    return Params(security_level, pow_bits,
                  folding_factor if folding_factor_0 is None else folding_factor_0, folding_factor,
                  SOUNDNESS[soundness] if isinstance(soundness, str) else soundness,
                  starting_log_inv_rate, rs_reduction, leaf_hash, ds_digest_elems)
