"""whir_p3_b200 — Python face of the B200 WHIR prover hot path.

Mirrors the reference crate's interface for the prover path (tcoratger/whir-p3):
ProtocolParameters / FoldingFactor / SecurityAssumption
(src/parameters/mod.rs, src/parameters/errors.rs), WhirConfig
(src/whir/parameters.rs), DomainSeparator (src/fiat_shamir/domain_separator.rs),
the DuplexChallenger / GrindingChallenger calls (p3-challenger),
InitialStatement (src/whir/constraints/statement/initial.rs), CommitmentWriter
(src/whir/committer/writer.rs) and Prover (src/whir/prover/mod.rs), plus the
Plonky3 DFT / MMCS and multilinear kernels. Every call goes through the C ABI
of lib/libwhir_b200.so (include/whir_b200.h); there is no Python or CPU
fallback for device work, and importing fails loudly if the library is absent.

Host-side values are canonical uint32 numpy arrays; extension elements are 4
consecutive words.
"""
from __future__ import annotations

import ctypes as C
import enum
import pathlib
from dataclasses import dataclass, field

import numpy as np

_PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = _PKG / "lib" / "libwhir_b200.so"
P = 0x7F000001

WHIR_OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of memory", -4: "proof-of-work not found",
          -5: "buffer too small", -6: "no CUDA device"}


class WhirError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


# external 4x4 block of the Poseidon2 external layer
P2_MDS_MAT4 = 0  # circ(2, 3, 1, 1): Plonky3's Monty-31 MDSMat4, the KoalaBear permutation
P2_HL_MAT4 = 1   # the Poseidon2 paper's M4 (Plonky3's HLMDSMat4)


class Poseidon2Params(C.Structure):
    _fields_ = [("width", C.c_uint32), ("rounds_f", C.c_uint32), ("rounds_p", C.c_uint32),
                ("external_matrix", C.c_uint32), ("ext_rc", C.c_uint32 * (8 * 24)), ("int_rc", C.c_uint32 * 32), ("diag", C.c_uint32 * 24)]


class _Params(C.Structure):
    _fields_ = [("security_level", C.c_int32), ("pow_bits", C.c_int32), ("folding_factor_0", C.c_int32),
                ("folding_factor", C.c_int32), ("soundness", C.c_int32), ("starting_log_inv_rate", C.c_int32),
                ("rs_reduction", C.c_int32), ("leaf_hash", C.c_int32), ("ds_digest_elems", C.c_int32)]


class _Round(C.Structure):
    _fields_ = [("pow_bits", C.c_int32), ("folding_pow_bits", C.c_int32), ("num_queries", C.c_int32),
                ("ood_samples", C.c_int32), ("num_variables", C.c_int32), ("folding_factor", C.c_int32),
                ("domain_size", C.c_uint64), ("folded_domain_gen", C.c_uint32)]


class _Config(C.Structure):
    _fields_ = [("num_variables", C.c_int32), ("security_level", C.c_int32), ("max_pow_bits", C.c_int32),
                ("commitment_ood_samples", C.c_int32), ("starting_log_inv_rate", C.c_int32),
                ("starting_folding_pow_bits", C.c_int32), ("folding_factor_0", C.c_int32),
                ("folding_factor", C.c_int32), ("rs_reduction", C.c_int32), ("soundness", C.c_int32),
                ("n_rounds", C.c_int32), ("rounds", _Round * 32), ("final_queries", C.c_int32),
                ("final_pow_bits", C.c_int32), ("final_sumcheck_rounds", C.c_int32),
                ("final_folding_pow_bits", C.c_int32)]


class _Chal(C.Structure):
    _fields_ = [("state", C.c_uint32 * 16), ("input", C.c_uint32 * 8), ("input_len", C.c_int32),
                ("output", C.c_uint32 * 8), ("output_len", C.c_int32)]


class Job(C.Structure):
    _fields_ = [("params", _Params), ("n", C.c_int32), ("poly", C.c_void_p), ("poly_on_device", C.c_int32),
                ("points", C.c_void_p), ("num_points", C.c_int32), ("evals_out", C.c_void_p),
                ("proof_out", C.c_void_p), ("proof_cap", C.c_size_t), ("proof_words", C.c_size_t),
                ("checkpoint", C.c_uint32 * 4), ("status", C.c_int32), ("done", C.c_int32),
                ("footprint_bytes", C.c_uint64), ("t_submit_ms", C.c_double), ("t_start_ms", C.c_double),
                ("t_done_ms", C.c_double), ("error", C.c_char * 160)]


_u32 = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_vp = C.c_void_p
_i32 = C.c_int32

# name -> (restype, argtypes)
_SIGS = {
    "whir_last_error": (C.c_char_p, []),
    "whir_kernel_launches": (C.c_uint64, []),
    "whir_poseidon2_default_params": (C.c_int, [C.POINTER(Poseidon2Params), C.POINTER(Poseidon2Params)]),
    "whir_poseidon2_params_from_rng": (C.c_int, [C.c_uint64, C.c_uint32, C.POINTER(Poseidon2Params),
                                                 C.POINTER(Poseidon2Params)]),
    "whir_rng_koalabear": (C.c_int, [C.c_uint64, _vp, C.c_size_t]),
    "whir_proof_to_bincode": (C.c_int, [_vp, C.c_size_t, _vp, C.c_size_t, C.POINTER(C.c_size_t)]),
    "whir_proof_from_bincode": (C.c_int, [_vp, C.c_size_t, _vp, C.c_size_t, C.POINTER(C.c_size_t)]),
    "whir_ctx_create": (C.c_int, [_i32, C.POINTER(Poseidon2Params), C.POINTER(Poseidon2Params), C.POINTER(_vp)]),
    "whir_ctx_destroy": (C.c_int, [_vp]),
    "whir_ctx_set_stream": (C.c_int, [_vp, _vp]),
    "whir_ctx_synchronize": (C.c_int, [_vp]),
    "whir_poseidon2_permute": (C.c_int, [_vp, _u32, _i32]),
    "whir_ctx_set_profiling": (C.c_int, [_vp, _i32]),
    "whir_ctx_stage_times": (C.c_int, [_vp, _vp, _vp, _i32, _i32]),
    "whir_ctx_stage_work": (C.c_int, [_vp, _vp, _i32, _i32]),
    "whir_ctx_set_device_transcript": (C.c_int, [_vp, _i32]),
    "whir_config_new": (C.c_int, [C.POINTER(_Params), _i32, C.POINTER(_Config)]),
    "whir_domain_separator": (C.c_int, [C.POINTER(_Config), _i32, _vp, _i32]),
    "whir_challenger_init": (None, [C.POINTER(_Chal)]),
    "whir_challenger_observe": (C.c_int, [_vp, C.POINTER(_Chal), _u32, C.c_size_t]),
    "whir_challenger_sample": (C.c_int, [_vp, C.POINTER(_Chal), _u32, C.c_size_t]),
    "whir_challenger_sample_bits": (C.c_int, [_vp, C.POINTER(_Chal), _i32, C.POINTER(C.c_uint64)]),
    "whir_challenger_grind": (C.c_int, [_vp, C.POINTER(_Chal), _i32, C.POINTER(C.c_uint32)]),
    "whir_challenger_check_witness": (C.c_int, [_vp, C.POINTER(_Chal), _i32, C.c_uint32]),
    "whir_device_alloc": (C.c_int, [_vp, C.c_size_t, C.POINTER(_vp)]),
    "whir_device_free": (C.c_int, [_vp, _vp]),
    "whir_memcpy_h2d": (C.c_int, [_vp, _vp, _vp, C.c_size_t]),
    "whir_memcpy_d2h": (C.c_int, [_vp, _vp, _vp, C.c_size_t]),
    "whir_monty_encode": (C.c_int, [_vp, _vp, C.c_size_t]),
    "whir_monty_decode": (C.c_int, [_vp, _vp, C.c_size_t]),
    "whir_dft_batch": (C.c_int, [_vp, _vp, _i32, _i32, _i32, _i32, _vp]),
    "whir_merkle_commit": (C.c_int, [_vp, _vp, _i32, _i32, _i32, _vp, _u32]),
    "whir_merkle_commit_many": (C.c_int, [_vp, _i32, _vp, _vp, _i32, _i32, _vp, _vp]),
    "whir_merkle_open": (C.c_int, [_vp, _vp, _vp, _i32, _i32, C.c_uint64, _u32, _u32]),
    "whir_merkle_open_ex": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _i32, C.c_uint64, _u32, _u32]),
    "whir_keccak256": (C.c_int, [C.c_char_p, C.c_size_t, _vp]),
    "whir_eq_table": (C.c_int, [_vp, _vp, _i32, _u32, _vp]),
    "whir_eval_base": (C.c_int, [_vp, _vp, _i32, _vp, _u32]),
    "whir_eval_ext": (C.c_int, [_vp, _vp, _i32, _vp, _u32]),
    "whir_fold_ext": (C.c_int, [_vp, _vp, _i32, _u32]),
    "whir_fold_base": (C.c_int, [_vp, _vp, _i32, _u32, _vp]),
    "whir_fold_multi_base": (C.c_int, [_vp, _vp, _i32, _vp, _i32, _vp]),
    "whir_sumcheck_coeffs": (C.c_int, [_vp, _vp, _vp, _i32, _u32, _u32]),
    "whir_combine_eq": (C.c_int, [_vp, _vp, _i32, _vp, _i32, _vp]),
    "whir_combine_select": (C.c_int, [_vp, _vp, _i32, _vp, _i32, _vp]),
    "whir_svo_partial_evals": (C.c_int, [_vp, _vp, _i32, _i32, _vp, _u32, _u32]),
    "whir_commit": (C.c_int, [_vp, C.POINTER(_Params), _i32, _vp, _i32, _vp, _i32, _vp, C.POINTER(_Chal),
                              C.POINTER(_vp)]),
    "whir_prove": (C.c_int, [_vp, _vp, C.POINTER(_Chal), _vp, C.c_size_t, C.POINTER(C.c_size_t)]),
    "whir_witness_free": (C.c_int, [_vp]),
    "whir_commit_and_prove": (C.c_int, [_vp, C.POINTER(_Params), _i32, _vp, _i32, _vp, _i32, _vp, _vp, C.c_size_t,
                                        C.POINTER(C.c_size_t), _vp]),
    "whir_job_footprint": (C.c_int, [C.POINTER(_Params), _i32, _i32, C.POINTER(C.c_uint64)]),
    "whir_batch_create": (C.c_int, [_i32, _i32, C.POINTER(Poseidon2Params), C.POINTER(Poseidon2Params), C.c_uint64,
                                    C.POINTER(_vp)]),
    "whir_batch_destroy": (C.c_int, [_vp]),
    "whir_batch_memory": (C.c_int, [_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "whir_batch_set_device_transcript": (C.c_int, [_vp, _i32]),
    "whir_batch_set_wait_spin": (C.c_int, [_vp, _i32]),
    "whir_ctx_set_wait_spin": (C.c_int, [_vp, _i32]),
    "whir_ctx_set_grind_window": (C.c_int, [_vp, _i32]),
    "whir_batch_set_grind_window": (C.c_int, [_vp, _i32]),
    "whir_batch_submit": (C.c_int, [_vp, C.POINTER(Job)]),
    "whir_batch_wait": (C.c_int, [_vp, C.POINTER(Job), _i32]),
    "whir_batch_wait_all": (C.c_int, [_vp]),
    "whir_batch_run": (C.c_int, [_vp, C.POINTER(Job), _i32]),
    "whir_tune_set_mode": (C.c_int, [_i32]),
    "whir_tune_get_mode": (C.c_int, []),
    "whir_tune_entries": (C.c_int, [_vp, _i32]),
    "whir_tune_clear": (C.c_int, []),
    "whir_dft_plans": (C.c_int, [_i32, _i32, _i32, _i32, _vp, _i32]),
    "whir_dft_batch_plan": (C.c_int, [_vp, _vp, _i32, _i32, _i32, _i32, _vp, _vp]),
    "whir_merkle_commit_shaped": (C.c_int, [_vp, _vp, _i32, _i32, _i32, _vp, _vp, _u32]),
    "whir_fold_ext_shaped": (C.c_int, [_vp, _vp, _i32, _u32, _vp]),
    "whir_sumcheck_coeffs_shaped": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _u32, _u32]),
}

_lib = None


def lib() -> C.CDLL:
    """Load libwhir_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with whir-p3_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(code: int) -> int:
    if code < 0:
        raise WhirError(code, lib().whir_last_error().decode())
    return code


def _arr(a, n_words=None) -> np.ndarray:
    out = np.ascontiguousarray(np.asarray(a, dtype=np.uint32).reshape(-1))
    if n_words is not None and out.size != n_words:
        raise ValueError(f"expected {n_words} words, got {out.size}")
    return out


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def kernel_launches() -> int:
    return int(lib().whir_kernel_launches())


# ---------------------------------------------------------------------------
# Parameters (src/parameters/mod.rs, src/parameters/errors.rs, src/whir/parameters.rs)
# ---------------------------------------------------------------------------

class SecurityAssumption(enum.IntEnum):
    UniqueDecoding = 0
    JohnsonBound = 1
    CapacityBound = 2


@dataclass(frozen=True)
class FoldingFactor:
    first: int
    rest: int

    @staticmethod
    def constant(k: int) -> "FoldingFactor":
        return FoldingFactor(k, k)

    @staticmethod
    def constant_from_second_round(first: int, rest: int) -> "FoldingFactor":
        return FoldingFactor(first, rest)

    def at_round(self, r: int) -> int:
        return self.first if r == 0 else self.rest


# hash families (whir_b200.h WHIR_LEAF_*): "keccak" is the Keccak MMCS with the
# SerializingChallenger32 of src/whir/mod.rs:236-383 (commit_and_prove only)
LEAF_HASH = {"poseidon2_24": 0, "poseidon2_16": 1, "keccak": 2}


@dataclass
class ProtocolParameters:
    security_level: int = 100
    pow_bits: int = 16
    folding_factor: FoldingFactor = field(default_factory=lambda: FoldingFactor.constant(4))
    soundness_type: SecurityAssumption = SecurityAssumption.CapacityBound
    starting_log_inv_rate: int = 1
    rs_domain_initial_reduction_factor: int = 1
    leaf_hash: str = "poseidon2_24"   # PaddingFreeSponge<P24,24,16,8>; "poseidon2_16" = <P16,16,8,8>; "keccak"
    ds_digest_elems: int = 32          # DIGEST_ELEMS given to DomainSeparator::commit_statement

    def _c(self) -> _Params:
        return _Params(self.security_level, self.pow_bits, self.folding_factor.first, self.folding_factor.rest,
                       int(self.soundness_type), self.starting_log_inv_rate,
                       self.rs_domain_initial_reduction_factor, LEAF_HASH[self.leaf_hash], self.ds_digest_elems)


@dataclass
class RoundConfig:
    pow_bits: int
    folding_pow_bits: int
    num_queries: int
    ood_samples: int
    num_variables: int
    folding_factor: int
    domain_size: int
    folded_domain_gen: int


class WhirConfig:
    """WhirConfig::new (src/whir/parameters.rs:81-234)."""

    def __init__(self, num_variables: int, params: ProtocolParameters):
        self.params = params
        self._c = _Config()
        _check(lib().whir_config_new(C.byref(params._c()), num_variables, C.byref(self._c)))
        c = self._c
        for name, _ in _Config._fields_:
            if name != "rounds":
                setattr(self, name, getattr(c, name))
        self.round_parameters = [RoundConfig(r.pow_bits, r.folding_pow_bits, r.num_queries, r.ood_samples,
                                             r.num_variables, r.folding_factor, r.domain_size, r.folded_domain_gen)
                                 for r in list(c.rounds)[: c.n_rounds]]

    def n_rounds(self) -> int:
        return self._c.n_rounds

    def max_fft_size(self) -> int:
        return self.num_variables + self.starting_log_inv_rate - self.folding_factor_0

    def check_pow_bits(self) -> bool:
        m = self.max_pow_bits
        if self.starting_folding_pow_bits > m or self.final_pow_bits > m or self.final_folding_pow_bits > m:
            return False
        return all(r.pow_bits <= m and r.folding_pow_bits <= m for r in self.round_parameters)

    def proof_words_bound(self) -> int:
        """Upper bound on the encoded proof length in words."""
        n = self.num_variables
        k0 = self.folding_factor_0
        words = 64 + 4 * self.commitment_ood_samples + self._sc_words(k0)
        log_h = n + self.starting_log_inv_rate - k0
        row = 1 << k0
        for r in self.round_parameters:
            words += 16 + 4 * r.ood_samples + r.num_queries * (3 + row + 8 * log_h)
            nxt = self.folding_factor
            new_dom = r.domain_size >> (self.rs_reduction if r is self.round_parameters[0] else 1)
            log_h = new_dom.bit_length() - 1 - nxt
            row = 4 << nxt
            words += self._sc_words(nxt)
        words += 8 + 4 * (1 << self.final_sumcheck_rounds) + self.final_queries * (3 + row + 8 * log_h)
        words += self._sc_words(self.final_sumcheck_rounds)
        return words

    @staticmethod
    def _sc_words(rounds: int) -> int:
        return 2 + 9 * rounds


class DomainSeparator:
    """DomainSeparator::commit_statement + add_whir_proof (domain_separator.rs:95-213)."""

    def __init__(self, config: WhirConfig, digest_elems: int | None = None):
        d = config.params.ds_digest_elems if digest_elems is None else digest_elems
        n = _check(lib().whir_domain_separator(C.byref(config._c), d, None, 0))
        self.pattern = np.zeros(n, dtype=np.uint32)
        lib().whir_domain_separator(C.byref(config._c), d, self.pattern.ctypes.data, n)

    def observe_domain_separator(self, challenger: "DuplexChallenger") -> None:
        challenger.observe_slice(self.pattern)


# ---------------------------------------------------------------------------
# Context and device buffers
# ---------------------------------------------------------------------------

def default_poseidon2() -> tuple[Poseidon2Params, Poseidon2Params]:
    a, b = Poseidon2Params(), Poseidon2Params()
    _check(lib().whir_poseidon2_default_params(C.byref(a), C.byref(b)))
    return a, b


def poseidon2_from_rng(seed: int, external_matrix: int = P2_MDS_MAT4) -> tuple[Poseidon2Params, Poseidon2Params]:
    """Poseidon2KoalaBear<16>::new_from_rng_128 then <24>::new_from_rng_128 on
    one SmallRng::seed_from_u64(seed) stream (src/bin/main.rs:100-102)."""
    a, b = Poseidon2Params(), Poseidon2Params()
    _check(lib().whir_poseidon2_params_from_rng(seed, external_matrix, C.byref(a), C.byref(b)))
    return a, b


def proof_to_bincode(proof: np.ndarray) -> bytes:
    """The flat proof stream as the bytes bincode::serialize gives for the
    reference's WhirProof (src/whir/proof.rs:11-141)."""
    w = np.ascontiguousarray(proof, dtype=np.uint32)
    n = C.c_size_t(0)
    rc = lib().whir_proof_to_bincode(w.ctypes.data, w.size, None, 0, C.byref(n))
    if rc not in (0, -5):
        _check(rc)
    out = np.empty(n.value, dtype=np.uint8)
    _check(lib().whir_proof_to_bincode(w.ctypes.data, w.size, out.ctypes.data, out.size, C.byref(n)))
    return out.tobytes()


def proof_from_bincode(data: bytes) -> np.ndarray:
    """bincode bytes of a WhirProof back to the flat proof stream."""
    b = np.frombuffer(data, dtype=np.uint8)
    n = C.c_size_t(0)
    rc = lib().whir_proof_from_bincode(b.ctypes.data, b.size, None, 0, C.byref(n))
    if rc not in (0, -5):
        _check(rc)
    out = np.empty(n.value, dtype=np.uint32)
    _check(lib().whir_proof_from_bincode(b.ctypes.data, b.size, out.ctypes.data, out.size, C.byref(n)))
    return out


def rng_koalabear(seed: int, count: int) -> np.ndarray:
    """The first `count` KoalaBear elements (canonical uint32) that
    `rng.random::<F>()` draws from SmallRng::seed_from_u64(seed)
    (benches/whir.rs:92-100 draws the polynomial, then the point, this way)."""
    out = np.empty(count, dtype=np.uint32)
    _check(lib().whir_rng_koalabear(seed, out.ctypes.data, count))
    return out


class Context:
    """One device (or host-only with device=-1) and one CUDA stream."""

    def __init__(self, device: int = 0, p16: Poseidon2Params | None = None, p24: Poseidon2Params | None = None):
        h = _vp()
        _check(lib().whir_ctx_create(device, None if p16 is None else C.byref(p16),
                                     None if p24 is None else C.byref(p24), C.byref(h)))
        self.handle = h
        self.device = device

    def close(self) -> None:
        if self.handle:
            lib().whir_ctx_destroy(self.handle)
            self.handle = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self) -> None:
        _check(lib().whir_ctx_synchronize(self.handle))

    def set_stream(self, stream_ptr: int) -> None:
        _check(lib().whir_ctx_set_stream(self.handle, stream_ptr))

    STAGES = ["dft", "merkle_leaves", "merkle_upper", "grind", "sumcheck", "eval", "weights", "open"]

    def set_profiling(self, enable: bool) -> None:
        _check(lib().whir_ctx_set_profiling(self.handle, int(enable)))

    def stage_times(self, reset: bool = True) -> dict:
        ms = np.zeros(8, dtype=np.float64)
        cnt = np.zeros(8, dtype=np.uint64)
        _check(lib().whir_ctx_stage_times(self.handle, ms.ctypes.data, cnt.ctypes.data, 8, int(reset)))
        return {name: (float(m), int(c)) for name, m, c in zip(self.STAGES, ms, cnt)}

    def set_wait_spin(self, microseconds: int) -> None:
        """How long a wait for a small device result spins before yielding."""
        _check(lib().whir_ctx_set_wait_spin(self.handle, int(microseconds)))

    GRIND_LATENCY, GRIND_LEAN_SMALL, GRIND_LEAN_LARGE = 0, 1, 2

    def set_grind_window(self, mode: int) -> None:
        """Candidates in flight of proof-of-work searches: GRIND_LATENCY (0, each search as
        fast as possible on an idle GPU), or the bits GRIND_LEAN_SMALL (searches of up to 11
        bits with 2x the expected candidates in flight instead of 8x) and GRIND_LEAN_LARGE
        (larger searches with one CTA per SM). The witness is the same in every mode."""
        _check(lib().whir_ctx_set_grind_window(self.handle, int(mode)))

    def set_device_transcript(self, enable: bool) -> None:
        """Sumcheck stages with their transcript steps on the device, or with
        one host round trip per step (default); the proofs are the same."""
        _check(lib().whir_ctx_set_device_transcript(self.handle, int(enable)))

    def stage_work(self, reset: bool = True) -> dict:
        """Work per stage while profiling was on: DFT algorithmic bytes, Merkle
        leaf permutations, Merkle compressions, grinding candidates (one
        Poseidon2-16 permutation each)."""
        w = np.zeros(8, dtype=np.uint64)
        _check(lib().whir_ctx_stage_work(self.handle, w.ctypes.data, 8, int(reset)))
        return {name: int(v) for name, v in zip(self.STAGES, w)}

    def permute(self, state) -> np.ndarray:
        s = _arr(state).copy()
        _check(lib().whir_poseidon2_permute(self.handle, s, s.size))
        return s


class DeviceArray:
    """Device buffer of field words in Montgomery form (owned by the context)."""

    def __init__(self, ctx: Context, words: int):
        self.ctx = ctx
        self.words = int(words)
        p = _vp()
        _check(lib().whir_device_alloc(ctx.handle, max(self.words, 1) * 4, C.byref(p)))
        self.ptr = p.value

    @staticmethod
    def from_host(ctx: Context, values) -> "DeviceArray":
        a = _arr(values)
        d = DeviceArray(ctx, a.size)
        _check(lib().whir_memcpy_h2d(ctx.handle, d.ptr, a.ctypes.data, a.size * 4))
        _check(lib().whir_monty_encode(ctx.handle, d.ptr, a.size))
        return d

    def to_host(self, words: int | None = None) -> np.ndarray:
        return mont_decode(self.raw(words))

    def raw(self, words: int | None = None) -> np.ndarray:
        """The words as stored (Keccak digests are raw bytes, not field words)."""
        w = self.words if words is None else words
        out = np.zeros(w, dtype=np.uint32)
        _check(lib().whir_memcpy_d2h(self.ctx.handle, out.ctypes.data, self.ptr, w * 4))
        return out

    def free(self) -> None:
        if self.ptr:
            lib().whir_device_free(self.ctx.handle, self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


_R_INV = pow(1 << 32, P - 2, P)


def mont_decode(a: np.ndarray) -> np.ndarray:
    return ((a.astype(np.uint64) * _R_INV) % P).astype(np.uint32)


def mont_encode(a: np.ndarray) -> np.ndarray:
    return ((np.asarray(a, dtype=np.uint64) << 32) % P).astype(np.uint32)


# ---------------------------------------------------------------------------
# Challenger (DuplexChallenger<F, Poseidon2-16, 16, 8> + GrindingChallenger)
# ---------------------------------------------------------------------------

class DuplexChallenger:
    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.c = _Chal()
        lib().whir_challenger_init(C.byref(self.c))

    def clone(self) -> "DuplexChallenger":
        o = DuplexChallenger(self.ctx)
        C.memmove(C.byref(o.c), C.byref(self.c), C.sizeof(_Chal))
        return o

    def observe(self, v: int) -> None:
        self.observe_slice([v])

    def observe_slice(self, vals) -> None:
        a = _arr(vals)
        _check(lib().whir_challenger_observe(self.ctx.handle, C.byref(self.c), a, a.size))

    def observe_algebra_element(self, e) -> None:
        self.observe_slice(_arr(e, 4))

    def sample(self) -> int:
        out = np.zeros(1, dtype=np.uint32)
        _check(lib().whir_challenger_sample(self.ctx.handle, C.byref(self.c), out, 1))
        return int(out[0])

    def sample_algebra_element(self) -> np.ndarray:
        out = np.zeros(4, dtype=np.uint32)
        _check(lib().whir_challenger_sample(self.ctx.handle, C.byref(self.c), out, 4))
        return out

    def sample_bits(self, bits: int) -> int:
        v = C.c_uint64()
        _check(lib().whir_challenger_sample_bits(self.ctx.handle, C.byref(self.c), bits, C.byref(v)))
        return int(v.value)

    def grind(self, bits: int) -> int:
        w = C.c_uint32()
        _check(lib().whir_challenger_grind(self.ctx.handle, C.byref(self.c), bits, C.byref(w)))
        return int(w.value)

    def check_witness(self, bits: int, witness: int) -> bool:
        return bool(_check(lib().whir_challenger_check_witness(self.ctx.handle, C.byref(self.c), bits, witness)))


# ---------------------------------------------------------------------------
# Plonky3 trait kernels and multilinear kernels on device arrays
# ---------------------------------------------------------------------------

def dft_batch(ctx: Context, chunks: DeviceArray, log_chunk: int, log_width: int, log_blowup: int, ext: bool,
              out: DeviceArray) -> DeviceArray:
    _check(lib().whir_dft_batch(ctx.handle, chunks.ptr, log_chunk, log_width, log_blowup, int(ext), out.ptr))
    return out


def merkle_commit(ctx: Context, rows: DeviceArray, log_height: int, row_words: int, leaf_hash: int,
                  digests: DeviceArray) -> np.ndarray:
    root = np.zeros(8, dtype=np.uint32)
    _check(lib().whir_merkle_commit(ctx.handle, rows.ptr, log_height, row_words, leaf_hash, digests.ptr, root))
    return root


def merkle_commit_many(ctx: Context, rows: list, log_heights, row_words: int, leaf_hash: int,
                       digests: list) -> np.ndarray:
    """Independent trees (DeviceArrays of rows and digests, one per tree) committed together by the
    multi-instance kernels; returns the roots, one row of 8 canonical words per tree."""
    n = len(rows)
    if n != len(digests) or n != len(log_heights):
        raise ValueError("rows, log_heights and digests must have one entry per tree")
    rp = np.array([r.ptr for r in rows], dtype=np.uint64)
    dp = np.array([d.ptr for d in digests], dtype=np.uint64)
    lh = np.ascontiguousarray(log_heights, dtype=np.int32)
    roots = np.zeros((n, 8), dtype=np.uint32)
    _check(lib().whir_merkle_commit_many(ctx.handle, n, rp.ctypes.data, lh.ctypes.data, row_words, leaf_hash,
                                         dp.ctypes.data, roots.ctypes.data))
    return roots


# ---------------------------------------------------------------------------
# launch-shape tuning
# ---------------------------------------------------------------------------

TUNE_KINDS = {1: "dft", 2: "merkle_leaves", 3: "merkle_nodes", 4: "fold"}


class TuneEntry(C.Structure):
    _fields_ = [("kind", C.c_int32), ("device", C.c_int32), ("key", C.c_int32 * 4), ("choice", C.c_int32 * 7),
                ("candidates", C.c_int32), ("ms_default", C.c_float), ("ms_best", C.c_float)]


def set_tune_mode(mode: int) -> None:
    """1: time every candidate launch shape on first use of a shape (default); 0: fixed default shapes."""
    _check(lib().whir_tune_set_mode(int(mode)))


def tune_mode() -> int:
    return int(lib().whir_tune_get_mode())


def tune_clear() -> None:
    _check(lib().whir_tune_clear())


def tune_entries() -> list[dict]:
    """The cached launch-shape choices as dicts (kind, device, key, choice, candidates, ms_default, ms_best)."""
    n = _check(lib().whir_tune_entries(None, 0))
    arr = (TuneEntry * max(n, 1))()
    n = min(n, _check(lib().whir_tune_entries(C.cast(arr, _vp), n)))
    return [{"kind": TUNE_KINDS.get(e.kind, str(e.kind)), "device": e.device, "key": list(e.key),
             "choice": list(e.choice), "candidates": e.candidates, "ms_default": e.ms_default,
             "ms_best": e.ms_best} for e in arr[:n]]


def dft_plans(log_chunk: int, log_width: int, log_blowup: int, ext: bool) -> list[tuple[int, ...]]:
    """Candidate DFT plans (log_h2, log_t1, threads1, log_t2, threads2, reg1, reg2) the tuner times for a shape."""
    n = _check(lib().whir_dft_plans(log_chunk, log_width, log_blowup, int(ext), None, 0))
    buf = np.zeros(max(n, 1) * 7, dtype=np.int32)
    _check(lib().whir_dft_plans(log_chunk, log_width, log_blowup, int(ext), buf.ctypes.data, n))
    return [tuple(int(v) for v in buf[7 * i: 7 * i + 7]) for i in range(n)]


def dft_batch_plan(ctx: Context, chunks: DeviceArray, log_chunk: int, log_width: int, log_blowup: int, ext: bool,
                   plan, out: DeviceArray) -> DeviceArray:
    p = np.ascontiguousarray(plan, dtype=np.int32)
    _check(lib().whir_dft_batch_plan(ctx.handle, chunks.ptr, log_chunk, log_width, log_blowup, int(ext),
                                     p.ctypes.data, out.ptr))
    return out


def merkle_commit_shaped(ctx: Context, rows: DeviceArray, log_height: int, row_words: int, leaf_hash: int,
                         shape, digests: DeviceArray) -> np.ndarray:
    """merkle_commit with shape = (leaf threads, leaf CTAs/SM, node threads, node CTAs/SM, node variant:
    bit 0 one-CTA top kernel, bit 1 sequential two-level kernel, bit 2 cooperative last two-level step)."""
    sh = np.ascontiguousarray(shape, dtype=np.int32)
    root = np.zeros(8, dtype=np.uint32)
    _check(lib().whir_merkle_commit_shaped(ctx.handle, rows.ptr, log_height, row_words, leaf_hash, sh.ctypes.data,
                                           digests.ptr, root))
    return root


def fold_ext_shaped(ctx: Context, evals: DeviceArray, n: int, r, shape) -> None:
    sh = np.ascontiguousarray(shape, dtype=np.int32)
    _check(lib().whir_fold_ext_shaped(ctx.handle, evals.ptr, n, _arr(r, 4), sh.ctypes.data))


def merkle_open(ctx: Context, rows: DeviceArray, digests: DeviceArray, log_height: int, row_words: int,
                index: int, leaf_hash: int = 0) -> tuple[np.ndarray, np.ndarray]:
    row = np.zeros(row_words, dtype=np.uint32)
    path = np.zeros(max(log_height, 1) * 8, dtype=np.uint32)
    _check(lib().whir_merkle_open_ex(ctx.handle, rows.ptr, digests.ptr, log_height, row_words, leaf_hash, index,
                                     row, path))
    return row, path[: log_height * 8]


def keccak256(data: bytes) -> bytes:
    """Keccak256Hash (p3-keccak): Keccak-256 with the original padding, on the host."""
    out = (C.c_uint8 * 32)()
    _check(lib().whir_keccak256(data, len(data), out))
    return bytes(out)


def eq_table(ctx: Context, point, scale, out: DeviceArray) -> DeviceArray:
    p = _arr(point)
    _check(lib().whir_eq_table(ctx.handle, _ptr(p), p.size // 4, _arr(scale, 4), out.ptr))
    return out


def eval_base(ctx: Context, evals: DeviceArray, point) -> np.ndarray:
    p = _arr(point)
    out = np.zeros(4, dtype=np.uint32)
    _check(lib().whir_eval_base(ctx.handle, evals.ptr, p.size // 4, _ptr(p), out))
    return out


def eval_ext(ctx: Context, evals: DeviceArray, point) -> np.ndarray:
    p = _arr(point)
    out = np.zeros(4, dtype=np.uint32)
    _check(lib().whir_eval_ext(ctx.handle, evals.ptr, p.size // 4, _ptr(p), out))
    return out


def fold_ext(ctx: Context, evals: DeviceArray, n: int, r) -> None:
    _check(lib().whir_fold_ext(ctx.handle, evals.ptr, n, _arr(r, 4)))


def fold_base(ctx: Context, evals: DeviceArray, n: int, r, out: DeviceArray) -> None:
    _check(lib().whir_fold_base(ctx.handle, evals.ptr, n, _arr(r, 4), out.ptr))


def fold_multi_base(ctx: Context, evals: DeviceArray, n: int, rs, out: DeviceArray) -> None:
    r = _arr(rs)
    _check(lib().whir_fold_multi_base(ctx.handle, evals.ptr, n, _ptr(r), r.size // 4, out.ptr))


def sumcheck_coeffs(ctx: Context, f: DeviceArray, w: DeviceArray, n: int) -> tuple[np.ndarray, np.ndarray]:
    c0 = np.zeros(4, dtype=np.uint32)
    c2 = np.zeros(4, dtype=np.uint32)
    _check(lib().whir_sumcheck_coeffs(ctx.handle, f.ptr, w.ptr, n, c0, c2))
    return c0, c2


def sumcheck_coeffs_shaped(ctx: Context, f: DeviceArray, w: DeviceArray, n: int,
                           max_blocks: int) -> tuple[np.ndarray, np.ndarray]:
    """sumcheck_coeffs with the reduction's block count capped at max_blocks."""
    c0 = np.zeros(4, dtype=np.uint32)
    c2 = np.zeros(4, dtype=np.uint32)
    _check(lib().whir_sumcheck_coeffs_shaped(ctx.handle, f.ptr, w.ptr, n, max_blocks, c0, c2))
    return c0, c2


def combine_eq(ctx: Context, w: DeviceArray, n: int, points, gamma_pows) -> None:
    p, g = _arr(points), _arr(gamma_pows)
    _check(lib().whir_combine_eq(ctx.handle, w.ptr, n, _ptr(p), g.size // 4, _ptr(g)))


def combine_select(ctx: Context, w: DeviceArray, n: int, vars_, gamma_pows) -> None:
    v, g = _arr(vars_), _arr(gamma_pows)
    _check(lib().whir_combine_select(ctx.handle, w.ptr, n, _ptr(v), v.size, _ptr(g)))


def svo_partial_evals(ctx: Context, poly: DeviceArray, n: int, l: int, point) -> tuple[np.ndarray, np.ndarray]:
    out = np.zeros(4 << l, dtype=np.uint32)
    ev = np.zeros(4, dtype=np.uint32)
    _check(lib().whir_svo_partial_evals(ctx.handle, poly.ptr, n, l, _ptr(_arr(point)), out, ev))
    return out, ev


# ---------------------------------------------------------------------------
# Protocol entry points
# ---------------------------------------------------------------------------

class InitialStatement:
    """InitialStatement (src/whir/constraints/statement/initial.rs): the
    polynomial (2^n canonical values on the host, or a DeviceArray in
    Montgomery form) plus its evaluation constraints."""

    def __init__(self, poly, num_variables: int):
        self.poly = poly
        self.n = num_variables
        self.points: list[np.ndarray] = []

    def evaluate(self, point) -> None:
        p = _arr(point, 4 * self.n)
        self.points.append(p)


class Witness:
    def __init__(self, handle, evals: np.ndarray):
        self.handle = handle
        self.evals = evals

    def free(self) -> None:
        if self.handle:
            lib().whir_witness_free(self.handle)
            self.handle = _vp()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class CommitmentWriter:
    """CommitmentWriter::commit (src/whir/committer/writer.rs:56-109)."""

    def __init__(self, config: WhirConfig):
        self.config = config

    def commit(self, ctx: Context, challenger: DuplexChallenger, statement: InitialStatement) -> Witness:
        pts = np.concatenate(statement.points) if statement.points else None
        evals = np.zeros(4 * len(statement.points), dtype=np.uint32)
        on_dev = isinstance(statement.poly, DeviceArray)
        if on_dev:
            poly_ptr = statement.poly.ptr
        else:
            statement._host = _arr(statement.poly, 1 << statement.n)
            poly_ptr = statement._host.ctypes.data
        h = _vp()
        _check(lib().whir_commit(ctx.handle, C.byref(self.config.params._c()), statement.n, poly_ptr, int(on_dev),
                                 _ptr(pts), len(statement.points), _ptr(evals) if evals.size else None,
                                 C.byref(challenger.c), C.byref(h)))
        return Witness(h, evals)


class Prover:
    """Prover::prove (src/whir/prover/mod.rs:97-128)."""

    def __init__(self, config: WhirConfig):
        self.config = config

    def prove(self, ctx: Context, challenger: DuplexChallenger, witness: Witness) -> np.ndarray:
        cap = self.config.proof_words_bound()
        buf = np.zeros(cap, dtype=np.uint32)
        words = C.c_size_t()
        _check(lib().whir_prove(ctx.handle, witness.handle, C.byref(challenger.c), buf.ctypes.data, cap,
                                C.byref(words)))
        return buf[: words.value].copy()


_PROVE_SETUP: dict = {}


def _prove_setup(params: ProtocolParameters, n: int):
    """The C parameter struct and the proof-length bound of (params, n),
    computed once per distinct pair (this is per-call host work otherwise)."""
    key = (params.security_level, params.pow_bits, params.folding_factor.first, params.folding_factor.rest,
           int(params.soundness_type), params.starting_log_inv_rate, params.rs_domain_initial_reduction_factor,
           params.leaf_hash, params.ds_digest_elems, n)
    v = _PROVE_SETUP.get(key)
    if v is None:
        v = (params._c(), WhirConfig(n, params).proof_words_bound())
        _PROVE_SETUP[key] = v
    return v


def commit_and_prove(ctx: Context, params: ProtocolParameters, n: int, poly, points=None):
    """Domain separator, commit, prove and a post-proof checkpoint sample, as
    in src/whir/mod.rs:103-141. Returns (proof words, checkpoint, user evals)."""
    cparams, cap = _prove_setup(params, n)
    on_dev = isinstance(poly, DeviceArray)
    host = None if on_dev else _arr(poly, 1 << n)
    pts = None if points is None or len(points) == 0 else _arr(points)
    npts = 0 if pts is None else pts.size // (4 * n)
    evals = np.zeros(4 * max(npts, 1), dtype=np.uint32)
    buf = np.empty(cap, dtype=np.uint32)
    words = C.c_size_t()
    cp = np.zeros(4, dtype=np.uint32)
    _check(lib().whir_commit_and_prove(ctx.handle, C.byref(cparams), n, poly.ptr if on_dev else host.ctypes.data,
                                       int(on_dev), _ptr(pts), npts, evals.ctypes.data, buf.ctypes.data, cap,
                                       C.byref(words), cp.ctypes.data))
    return buf[: words.value].copy(), cp, evals[: 4 * npts]


# ---------------------------------------------------------------------------
# Batching and serving (worker pool with HBM-budget admission)
# ---------------------------------------------------------------------------

class ProofRequest:
    """One commit+prove job; keeps its input and output buffers alive."""

    def __init__(self, params: ProtocolParameters, n: int, poly, points=None):
        self.params, self.n = params, n
        self.cfg = WhirConfig(n, params)
        self.on_device = isinstance(poly, DeviceArray)
        self._poly = poly if self.on_device else _arr(poly, 1 << n)
        self.points = None if points is None or len(points) == 0 else _arr(points)
        npts = 0 if self.points is None else self.points.size // (4 * n)
        self.evals = np.zeros(4 * max(npts, 1), dtype=np.uint32)
        self.proof_buf = np.zeros(self.cfg.proof_words_bound(), dtype=np.uint32)
        j = Job()
        j.params = params._c()
        j.n = n
        j.poly = self._poly.ptr if self.on_device else self._poly.ctypes.data
        j.poly_on_device = int(self.on_device)
        j.points = _ptr(self.points)
        j.num_points = npts
        j.evals_out = self.evals.ctypes.data
        j.proof_out = self.proof_buf.ctypes.data
        j.proof_cap = self.proof_buf.size
        self.job = j

    @property
    def proof(self) -> np.ndarray:
        return self.proof_buf[: self.job.proof_words].copy()

    @property
    def checkpoint(self) -> np.ndarray:
        return np.array(list(self.job.checkpoint), dtype=np.uint32)

    @property
    def latency_ms(self) -> float:
        return self.job.t_done_ms - self.job.t_submit_ms


def job_footprint(params: ProtocolParameters, n: int, poly_on_device: bool = False) -> int:
    v = C.c_uint64()
    _check(lib().whir_job_footprint(C.byref(params._c()), n, int(poly_on_device), C.byref(v)))
    return int(v.value)


class Batch:
    """whir_batch: `workers` contexts on one device proving jobs concurrently."""

    def __init__(self, device: int = 0, workers: int = 4, hbm_budget_bytes: int = 120 << 30,
                 p16: Poseidon2Params | None = None, p24: Poseidon2Params | None = None):
        h = _vp()
        _check(lib().whir_batch_create(device, workers, None if p16 is None else C.byref(p16),
                                       None if p24 is None else C.byref(p24), hbm_budget_bytes, C.byref(h)))
        self.handle = h

    def submit(self, req: ProofRequest) -> None:
        _check(lib().whir_batch_submit(self.handle, C.byref(req.job)))

    def memory(self) -> tuple[int, int]:
        """(fixed device bytes of the worker contexts, bytes their pools reserve)."""
        f, r = C.c_uint64(0), C.c_uint64(0)
        _check(lib().whir_batch_memory(self.handle, C.byref(f), C.byref(r)))
        return f.value, r.value

    def set_wait_spin(self, microseconds: int) -> None:
        """Context.set_wait_spin on every worker."""
        _check(lib().whir_batch_set_wait_spin(self.handle, int(microseconds)))

    def set_grind_window(self, mode: int) -> None:
        """Context.set_grind_window on every worker."""
        _check(lib().whir_batch_set_grind_window(self.handle, int(mode)))

    def set_device_transcript(self, enable: bool) -> None:
        """Context.set_device_transcript on every worker (jobs started later)."""
        _check(lib().whir_batch_set_device_transcript(self.handle, int(enable)))

    def wait(self, req: ProofRequest, timeout_ms: int = -1) -> None:
        _check(lib().whir_batch_wait(self.handle, C.byref(req.job), timeout_ms))

    def wait_all(self) -> None:
        _check(lib().whir_batch_wait_all(self.handle))

    def run(self, reqs: list[ProofRequest]) -> None:
        for r in reqs:
            self.submit(r)
        self.wait_all()
        for r in reqs:
            if r.job.status != 0:
                raise WhirError(r.job.status, f"job n={r.n}: {r.job.error.decode()}")

    def close(self) -> None:
        if self.handle:
            lib().whir_batch_destroy(self.handle)
            self.handle = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
