"""Python binding of libflockgpu.so (the B200 Flock prover's C ABI).

The C ABI (include/flock_gpu.h) is the product boundary; this module is a
thin ctypes mirror of it, shaped like the reference worker's use of
`Blake3Setup::new` + `prove_fast` + `to_bytes`
(benchmark-tools/worker/src/main.rs:24-47).  There is no CPU fallback: if
the shared library or a CUDA device is missing, every call raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libflockgpu.so"
DOMAIN = b"flock-bench-v0"
MAX_PROOF_BYTES = 500_000

# every symbol include/flock_gpu.h declares
EXPORTS = (
    "flock_ctx_create", "flock_ctx_destroy", "flock_last_error", "flock_setup_create",
    "flock_setup_destroy", "flock_prove_seed", "flock_prove_blocks", "flock_setup_phase_ms",
    "flock_witness", "flock_ntt_rs_encode", "flock_merkle_tree", "flock_sumcheck_round",
    "flock_pow", "flock_f128_mul", "flock_statement_digest", "flock_bench_ntt",
    "flock_bench_merkle", "flock_bench_sumcheck", "flock_bench_prove", "flock_merkle_root_noalloc",
    "flock_serve_start", "flock_submit", "flock_poll", "flock_sumcheck_round3", "flock_bench_sumcheck3",
    "flock_ntt_autotune", "flock_ntt_rs_encode_plan", "flock_prove_batch", "flock_host_alloc",
    "flock_host_free", "flock_prove_chain", "flock_chain_blocks", "flock_verify", "flock_serve_verify", "flock_verify_bundle",
    "flock_setup_create_blocks", "flock_prove_compressions", "flock_pcs_commit", "flock_prover_data_open",
    "flock_prover_data_destroy", "flock_challenger_create", "flock_challenger_destroy",
    "flock_challenger_observe_label", "flock_challenger_observe_bytes", "flock_challenger_observe_f128",
    "flock_challenger_observe_f128_slice", "flock_challenger_sample_f128", "flock_challenger_sample_f128_vec",
    "flock_challenger_grind_pow", "flock_challenger_verify_pow", "flock_challenger_state_digest",
    "flock_ntt_plan_desc", "flock_bench_ntt_plan", "flock_bench_f128_product", "flock_launch_count",
    "flock_serve_prewarm", "flock_sha256_setup_create", "flock_sha256_prove", "flock_sha256_verify_bundle",
    "flock_sha256_compress", "flock_sha256_statement_digest", "flock_sha256_witness", "flock_sha256_merkle_prove",
    "flock_sha256_merkle_verify", "flock_sha256_merkle_inputs", "flock_setup_set_transcript",
    "flock_ctx_set_transcript", "flock_challenger_create_hash", "flock_merkle_tree_hash",
    "flock_keccak_setup_create", "flock_keccak_prove", "flock_keccak_verify_bundle", "flock_keccak_f",
    "flock_keccak_bench_inputs", "flock_keccak_statement_digest", "flock_keccak_witness", "flock_keccak_comb",
    "flock_zerocheck_round1_deg4", "flock_bench_round1_deg4", "flock_keccak3_setup_create",
    "flock_keccak3_verify_bundle", "flock_keccak3_statement_digest", "flock_keccak3_witness", "flock_keccak3_comb",
    "flock_sha256_prove_chain", "flock_sha256_chain_blocks", "flock_keccak_prove_chain", "flock_keccak_chain_states",
)
# the hash behind Merkle trees / the transcript (HashKind discriminants)
HASH = {"sha256": 0, "blake3": 1}
FLOCK_ERR_CAPACITY = 3
FLOCK_ERR_TIMEOUT = 5
FLOCK_ERR_VERIFY = 6


class FlockJob(ctypes.Structure):
    _fields_ = [("log2_n", ctypes.c_uint32), ("seed", ctypes.c_uint64), ("blocks", ctypes.c_void_p),
                ("domain", ctypes.c_char_p), ("dlen", ctypes.c_size_t)]


class FlockResult(ctypes.Structure):
    _fields_ = [("out", ctypes.c_void_p), ("cap", ctypes.c_size_t), ("out_len", ctypes.c_size_t),
                ("status", ctypes.c_int), ("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double)]
PHASES = ("witness", "rs_encode", "merkle_commit", "zerocheck_round1", "zerocheck_rounds", "lincheck",
          "ring_switch_combine", "ligerito_l0_folds", "ligerito_levels")

_lib = None


class FlockError(RuntimeError):
    pass


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FlockError(f"{LIB_PATH} is not built (run `make -C {HERE}`); there is no CPU fallback")
        lib = ctypes.CDLL(str(LIB_PATH))
        vp, u32, u64, sz, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_int
        lib.flock_last_error.restype = ctypes.c_char_p
        lib.flock_last_error.argtypes = [vp]
        lib.flock_ctx_create.argtypes = [i32, u64, ctypes.POINTER(vp)]
        lib.flock_ctx_destroy.argtypes = [vp]
        lib.flock_setup_create.argtypes = [vp, u32, i32, i32, ctypes.POINTER(vp)]
        lib.flock_setup_destroy.argtypes = [vp]
        lib.flock_launch_count.restype = u64
        lib.flock_launch_count.argtypes = []
        lib.flock_bench_f128_product.argtypes = [vp, i32, i32, ctypes.POINTER(ctypes.c_double)]
        lib.flock_ntt_plan_desc.argtypes = [u32, u32, u32, u32, ctypes.c_char_p, sz]
        lib.flock_bench_ntt_plan.argtypes = [vp, u32, u32, u32, u32, i32, ctypes.POINTER(ctypes.c_double)]
        lib.flock_pcs_commit.argtypes = [vp, vp, u32, vp, ctypes.POINTER(vp)]
        lib.flock_prover_data_open.argtypes = [vp, vp, sz, vp, vp, sz, ctypes.POINTER(sz)]
        lib.flock_prover_data_destroy.argtypes = [vp]
        lib.flock_challenger_create.argtypes = [ctypes.c_char_p, sz, ctypes.POINTER(vp)]
        lib.flock_challenger_destroy.argtypes = [vp]
        lib.flock_challenger_observe_label.argtypes = [vp, ctypes.c_char_p, sz]
        lib.flock_challenger_observe_bytes.argtypes = [vp, ctypes.c_char_p, sz]
        lib.flock_challenger_observe_f128.argtypes = [vp, vp]
        lib.flock_challenger_observe_f128_slice.argtypes = [vp, vp, sz]
        lib.flock_challenger_sample_f128.argtypes = [vp, vp]
        lib.flock_challenger_sample_f128_vec.argtypes = [vp, sz, vp]
        lib.flock_challenger_grind_pow.argtypes = [vp, vp, u32, ctypes.POINTER(u64)]
        lib.flock_challenger_verify_pow.argtypes = [vp, u64, u32]
        lib.flock_challenger_state_digest.argtypes = [vp, vp]
        lib.flock_setup_create_blocks.argtypes = [vp, sz, i32, i32, ctypes.POINTER(vp)]
        lib.flock_prove_compressions.argtypes = [vp, vp, sz, ctypes.c_char_p, sz, vp, sz, ctypes.POINTER(sz)]
        lib.flock_prove_seed.argtypes = [vp, u64, ctypes.c_char_p, sz, vp, sz, ctypes.POINTER(sz)]
        lib.flock_prove_blocks.argtypes = [vp, vp, sz, ctypes.c_char_p, sz, vp, sz, ctypes.POINTER(sz)]
        lib.flock_setup_phase_ms.argtypes = [vp, vp, i32]
        lib.flock_witness.argtypes = [vp, u32, u64, vp, vp, vp]
        lib.flock_ntt_rs_encode.argtypes = [vp, vp, u32, u32, u32, vp]
        lib.flock_ntt_rs_encode_plan.argtypes = [vp, vp, u32, u32, u32, u32, vp]
        lib.flock_ntt_autotune.argtypes = [vp, u32, u32, u32, ctypes.POINTER(ctypes.c_double), ctypes.c_char_p, sz]
        lib.flock_merkle_tree.argtypes = [vp, vp, sz, sz, vp]
        lib.flock_sumcheck_round.argtypes = [vp, vp, vp, sz, vp]
        lib.flock_sumcheck_round3.argtypes = [vp, vp, vp, vp, sz, vp, vp, vp, vp]
        lib.flock_bench_sumcheck3.argtypes = [vp, sz, i32, ctypes.POINTER(ctypes.c_double)]
        lib.flock_pow.argtypes = [vp, vp, u32, ctypes.POINTER(u64)]
        lib.flock_f128_mul.argtypes = [vp, vp, vp, sz, vp]
        lib.flock_statement_digest.argtypes = [u32, vp]
        lib.flock_bench_ntt.argtypes = [vp, u32, u32, u32, i32, ctypes.POINTER(ctypes.c_double)]
        lib.flock_bench_merkle.argtypes = [vp, sz, sz, i32, ctypes.POINTER(ctypes.c_double)]
        lib.flock_bench_sumcheck.argtypes = [vp, sz, i32, ctypes.POINTER(ctypes.c_double)]
        lib.flock_bench_prove.argtypes = [vp, u64, i32, ctypes.POINTER(ctypes.c_double), vp,
                                          ctypes.POINTER(u64)]
        lib.flock_merkle_root_noalloc.argtypes = [vp, sz, sz, vp, vp]
        lib.flock_serve_start.argtypes = [vp, i32]
        lib.flock_serve_prewarm.argtypes = [vp, u32, i32, ctypes.POINTER(i32)]
        lib.flock_zerocheck_round1_deg4.argtypes = [vp, vp, vp, vp, vp, vp, u32, vp, vp, vp]
        lib.flock_bench_round1_deg4.argtypes = [vp, u32, u64, i32, ctypes.POINTER(ctypes.c_double), vp, vp]
        for w in ("", "3"):
            getattr(lib, f"flock_keccak{w}_setup_create").argtypes = [vp, sz, i32, i32, ctypes.POINTER(vp)]
            getattr(lib, f"flock_keccak{w}_verify_bundle").argtypes = [vp, ctypes.c_char_p, sz, ctypes.c_char_p, sz]
            getattr(lib, f"flock_keccak{w}_statement_digest").argtypes = [u32, vp]
            getattr(lib, f"flock_keccak{w}_witness").argtypes = [vp, vp, sz, u32, vp, vp, vp]
            getattr(lib, f"flock_keccak{w}_comb").argtypes = [vp, vp, vp, vp, vp]
        lib.flock_keccak_prove.argtypes = [vp, vp, sz, ctypes.c_char_p, sz, vp, sz, ctypes.POINTER(sz)]
        lib.flock_keccak_verify_bundle.argtypes = [vp, ctypes.c_char_p, sz, ctypes.c_char_p, sz]
        lib.flock_keccak_f.argtypes = [vp]
        lib.flock_keccak_f.restype = None
        lib.flock_keccak_bench_inputs.argtypes = [sz, u64, vp]
        lib.flock_keccak_statement_digest.argtypes = [u32, vp]
        lib.flock_keccak_witness.argtypes = [vp, vp, sz, u32, vp, vp, vp]
        lib.flock_keccak_comb.argtypes = [vp, vp, vp, vp, vp]
        lib.flock_sha256_prove_chain.argtypes = [vp, vp, sz, ctypes.c_char_p, sz, vp, sz, ctypes.POINTER(sz)]
        lib.flock_sha256_chain_blocks.argtypes = [u64, vp, sz, vp]
        lib.flock_keccak_prove_chain.argtypes = [vp, vp, sz, ctypes.c_char_p, sz, vp, sz, ctypes.POINTER(sz)]
        lib.flock_keccak_chain_states.argtypes = [vp, sz, vp]
        lib.flock_sha256_setup_create.argtypes = [vp, sz, i32, i32, ctypes.POINTER(vp)]
        lib.flock_sha256_prove.argtypes = [vp, vp, sz, ctypes.c_char_p, sz, vp, sz, ctypes.POINTER(sz)]
        lib.flock_sha256_verify_bundle.argtypes = [vp, ctypes.c_char_p, sz, ctypes.c_char_p, sz]
        lib.flock_sha256_compress.argtypes = [vp, vp, vp]
        lib.flock_sha256_compress.restype = None
        lib.flock_sha256_statement_digest.argtypes = [u32, vp]
        lib.flock_sha256_witness.argtypes = [vp, vp, sz, u32, vp, vp, vp]
        lib.flock_sha256_merkle_prove.argtypes = [vp, vp, sz, vp, u32, ctypes.c_char_p, sz, vp, sz,
                                                  ctypes.POINTER(sz)]
        lib.flock_sha256_merkle_verify.argtypes = [vp, ctypes.c_char_p, sz, ctypes.c_char_p, sz, u32, vp, sz, vp, vp]
        lib.flock_sha256_merkle_inputs.argtypes = [u32, u32, u64, vp, vp, vp, vp]
        lib.flock_setup_set_transcript.argtypes = [vp, i32]
        lib.flock_ctx_set_transcript.argtypes = [vp, i32]
        lib.flock_challenger_create_hash.argtypes = [ctypes.c_char_p, sz, i32, ctypes.POINTER(vp)]
        lib.flock_merkle_tree_hash.argtypes = [vp, vp, sz, sz, i32, vp]
        lib.flock_submit.argtypes = [vp, ctypes.POINTER(FlockJob), ctypes.POINTER(u64)]
        lib.flock_poll.argtypes = [vp, u64, ctypes.POINTER(FlockResult), i32]
        lib.flock_host_alloc.argtypes = [sz, ctypes.POINTER(vp)]
        lib.flock_host_free.argtypes = [vp]
        lib.flock_prove_batch.argtypes = [vp, ctypes.POINTER(FlockJob), sz, ctypes.POINTER(FlockResult), i32]
        lib.flock_prove_chain.argtypes = [vp, vp, sz, ctypes.c_char_p, sz, vp, sz, ctypes.POINTER(sz)]
        lib.flock_chain_blocks.argtypes = [u64, vp, sz, vp]
        lib.flock_verify.argtypes = [vp, ctypes.c_char_p, sz, ctypes.c_char_p, sz]
        lib.flock_serve_verify.argtypes = [vp, i32]
        lib.flock_verify_bundle.argtypes = [vp, ctypes.c_char_p, sz, ctypes.c_char_p, sz]
        _lib = lib
    return _lib


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def to_records(blocks: np.ndarray, block_len: int = 64, flags: int = 11) -> np.ndarray:
    """(n, 25) benchmark compressions (cv, m, counter_lo) -> (n, 28)
    flock_compression records with the given block_len and flags."""
    blocks = np.ascontiguousarray(blocks, np.uint32).reshape(-1, 25)
    rec = np.zeros((blocks.shape[0], 28), np.uint32)
    rec[:, :25] = blocks
    rec[:, 26] = block_len
    rec[:, 27] = flags
    return rec


def ntt_plan_descs(log_msg_pos: int, lanes: int, log_inv_rate: int) -> list:
    """Descriptions of every candidate pass plan of an RS-encode shape."""
    lib = load()
    out, buf = [], ctypes.create_string_buffer(512)
    while lib.flock_ntt_plan_desc(log_msg_pos, lanes, log_inv_rate, len(out), buf, len(buf)) == 0:
        out.append(buf.value.decode())
    return out


def generate_compressions(log2: int, seed: int) -> np.ndarray:
    """The benchmark inputs on the host, (2^log2, 25) u32: cv[8], m[16],
    counter (benchmark-tools/common/src/lib.rs:25-37 generate_compressions).
    SplitMix64 with state init = seed ^ rotl(log2, 29); draw j of compression
    i uses state init + (25 i + j + 1) * gamma (seed_pipe.rs:114-146)."""
    g = np.uint64(0x9E3779B97F4A7C15)
    init = np.uint64((seed ^ (((log2 << 29) | (log2 >> 35)) & (2**64 - 1))) & (2**64 - 1))
    idx = np.arange(25 << log2, dtype=np.uint64) + np.uint64(1)
    with np.errstate(over="ignore"):
        z = init + idx * g
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z.astype(np.uint32).reshape(-1, 25)


CHAIN_DOMAIN = b"flock_chain-cli"


def sha256_bench_inputs(n: int, seed: int) -> np.ndarray:
    """The sha2_proof bench inputs on the host, (n, 24) u32: h[8], m[16]
    (crates/flock-prover/benches/sha2_proof.rs:56-71): one SplitMix64 stream
    from `seed`, draw j of compression i at state seed + (24 i + j + 1) gamma."""
    g = np.uint64(0x9E3779B97F4A7C15)
    idx = np.arange(24 * n, dtype=np.uint64) + np.uint64(1)
    with np.errstate(over="ignore"):
        z = np.uint64(seed & (2**64 - 1)) + idx * g
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z.astype(np.uint32).reshape(-1, 24)


def sha256_bench_seed(n: int, run: int = 0) -> int:
    """The seed sha2_proof.rs:112 gives run `run` of n compressions."""
    return 0xC0FFEE_5A55 ^ n ^ run


MERKLE_DOMAIN = b"flock-merkle-bench-v0"


def sha256_merkle_inputs(n_log: int, path_log: int = 0, seed: int = None):
    """Honest SHA-256 Merkle paths (benches/sha2_merkle_proof.rs:49-76, the
    path repeated for each of 2^path_log paths): (compressions (2^n_log, 24)
    u32, b_bits (2^n_log,) u8, leaves (2^path_log, 8) u32, root (8,) u32).
    The bench's seed is 0xD15EA5E ^ n."""
    n = 1 << n_log
    seed = 0xD15EA5E ^ n if seed is None else seed
    comps = np.zeros((n, 24), np.uint32)
    b = np.zeros(n, np.uint8)
    leaves = np.zeros((1 << path_log, 8), np.uint32)
    root = np.zeros(8, np.uint32)
    rc = load().flock_sha256_merkle_inputs(n_log, path_log, seed, _ptr(comps), _ptr(b), _ptr(leaves), _ptr(root))
    if rc != 0:
        raise FlockError(f"sha256_merkle_inputs: {rc}")
    return comps, b, leaves, root


def sha256_chain_blocks(seed: int, steps: int, initial_h=None) -> np.ndarray:
    """The flock_chain CLI's honest SHA-256 chain, (steps, 24) u32 records
    (h_in, m) (crates/flock-prover/src/bin/flock_chain.rs:279-316)."""
    out = np.zeros((steps, 24), np.uint32)
    h = None if initial_h is None else np.ascontiguousarray(initial_h, np.uint32)
    rc = load().flock_sha256_chain_blocks(seed, None if h is None else _ptr(h), steps, _ptr(out))
    if rc:
        raise FlockError(f"sha256_chain_blocks: {rc}")
    return out


def sha256_compress(h, m) -> np.ndarray:
    """sha256_compress (sha2.rs:1502-1546): h_in + rounds(h_in, m), 8 u32."""
    h = np.ascontiguousarray(h, np.uint32)
    m = np.ascontiguousarray(m, np.uint32)
    out = np.zeros(8, np.uint32)
    load().flock_sha256_compress(_ptr(h), _ptr(m), _ptr(out))
    return out


def sha256_statement_digest(m: int) -> bytes:
    out = np.zeros(32, np.uint8)
    rc = load().flock_sha256_statement_digest(m, _ptr(out))
    if rc != 0:
        raise FlockError(f"sha256_statement_digest: {rc}")
    return out.tobytes()


def keccak_f(lanes) -> np.ndarray:
    """keccak_f (keccak.rs:423-428, FIPS 202 Keccak-f[1600]) of 25 u64 lanes
    (bit z of lane x + 5y is state bit x + 5y + 25z)."""
    s = np.array(lanes, np.uint64).reshape(25).copy()
    load().flock_keccak_f(_ptr(s))
    return s


def keccak_bench_inputs(n: int, seed: int) -> np.ndarray:
    """The keccak3_proof bench states on the host, (n, 25) u64 lanes
    (benches/keccak3_proof.rs:66-93): one SplitMix64 stream from `seed`, 25
    draws per state, state bit i = bit i mod 64 of draw i / 64."""
    out = np.zeros((n, 25), np.uint64)
    rc = load().flock_keccak_bench_inputs(n, seed, _ptr(out))
    if rc != 0:
        raise FlockError(f"keccak_bench_inputs: {rc}")
    return out


def keccak_chain_states(steps: int, initial=None) -> np.ndarray:
    """The flock_chain CLI's Keccak chain (bin/flock_chain.rs:319-346):
    (steps, 25) u64 successive keccak_f states from `initial` (zero state)."""
    out = np.zeros((steps, 25), np.uint64)
    init = None if initial is None else np.ascontiguousarray(initial, np.uint64)
    rc = load().flock_keccak_chain_states(None if init is None else _ptr(init), steps, _ptr(out))
    if rc:
        raise FlockError(f"keccak_chain_states: {rc}")
    return out


def keccak_bench_seed(n: int, run: int = 0) -> int:
    """The seed benches/keccak3_proof.rs:121-124 gives run `run` of n states."""
    return 0xC0FFEE_BEEF ^ n ^ run


def _kw(width: int) -> str:
    """entry-point suffix: "" for the single encoder (keccak.rs), "3" for the
    3-wide one (keccak3.rs)"""
    if width not in (1, 3):
        raise ValueError("width is 1 (keccak.rs) or 3 (keccak3.rs)")
    return "" if width == 1 else "3"


def keccak_statement_digest(m: int, width: int = 1) -> bytes:
    out = np.zeros(32, np.uint8)
    rc = getattr(load(), f"flock_keccak{_kw(width)}_statement_digest")(m, _ptr(out))
    if rc != 0:
        raise FlockError(f"keccak_statement_digest: {rc}")
    return out.tobytes()


def chain_blocks(seed: int, steps: int, initial_cv=None) -> np.ndarray:
    """The flock_chain CLI's honest BLAKE3 chain, (steps, 28) u32 records
    cv[8], m[16], counter lo/hi, block_len, flags
    (crates/flock-prover/src/bin/flock_chain.rs:178-193, 236-260)."""
    out = np.zeros((steps, 28), np.uint32)
    cv = None if initial_cv is None else np.ascontiguousarray(initial_cv, np.uint32)
    rc = load().flock_chain_blocks(seed, None if cv is None else _ptr(cv), steps, _ptr(out))
    if rc:
        raise FlockError(f"chain_blocks failed ({rc})")
    return out


class PinnedArray:
    """A numpy array over page-locked host memory (flock_host_alloc); the
    memory is freed when this object is."""

    def __init__(self, shape, dtype):
        n = int(np.prod(shape)) * np.dtype(dtype).itemsize
        p = ctypes.c_void_p()
        if load().flock_host_alloc(n, ctypes.byref(p)):
            raise FlockError("flock_host_alloc failed")
        self._p = p
        buf = (ctypes.c_uint8 * n).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=dtype).reshape(shape)

    def __del__(self):
        if getattr(self, "_p", None):
            self.array = None
            load().flock_host_free(self._p)
            self._p = None


def statement_digest(m: int) -> bytes:
    out = np.zeros(32, np.uint8)
    if load().flock_statement_digest(m, _ptr(out)):
        raise FlockError("statement digest failed")
    return out.tobytes()


class Context:
    """One CUDA device (reference: the process-wide rayon pool + allocator)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 150 << 30):
        self.lib = load()
        h = ctypes.c_void_p()
        rc = self.lib.flock_ctx_create(device, hbm_budget_bytes, ctypes.byref(h))
        if rc:
            raise FlockError(f"flock_ctx_create failed ({rc}): no usable CUDA device {device}")
        self.h = h

    def _check(self, rc: int, what: str) -> None:
        if rc:
            raise FlockError(f"{what} failed ({rc}): {self.lib.flock_last_error(self.h).decode()}")

    def close(self) -> None:
        if self.h:
            self.lib.flock_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- serving (continuous batching of proof jobs) ----
    def serve_start(self, slots: int = 4) -> None:
        self._check(self.lib.flock_serve_start(self.h, slots), "serve_start")

    def serve_prewarm(self, log2: int, count: int = 1) -> int:
        """Cache `count` idle setups of 2^log2 in free HBM budget (never
        evicting one); returns how many are cached."""
        n = ctypes.c_int()
        self._check(self.lib.flock_serve_prewarm(self.h, log2, count, ctypes.byref(n)), "serve_prewarm")
        return n.value

    def verify(self, bundle: bytes, domain: bytes = DOMAIN) -> str:
        """'' when the FLOCK v4 bundle verifies (any supported size, no prover
        setup needed), otherwise the name of the failed check."""
        rc = self.lib.flock_verify_bundle(self.h, bundle, len(bundle), domain, len(domain))
        if rc == 0:
            return ""
        if rc == FLOCK_ERR_VERIFY:
            return self.lib.flock_last_error(self.h).decode()
        self._check(rc, "verify_bundle")
        return "error"

    def sha256_verify(self, bundle: bytes, domain: bytes = DOMAIN) -> str:
        """Sha256HybridSetup::verify for any supported size: '' when the
        bundle verifies as a SHA-256 statement, otherwise the failed check."""
        rc = self.lib.flock_sha256_verify_bundle(self.h, bundle, len(bundle), domain, len(domain))
        if rc == 0:
            return ""
        if rc == FLOCK_ERR_VERIFY:
            return self.lib.flock_last_error(self.h).decode()
        self._check(rc, "sha256_verify_bundle")
        return "error"

    def sha256_merkle_verify(self, bundle: bytes, path_log: int, b_bits, leaves, root,
                             domain: bytes = MERKLE_DOMAIN) -> str:
        """verify_merkle_paths_ligerito: '' when the proof verifies against
        the public leaves ((2^path_log, 8) u32), root (8 u32) and bits."""
        b = np.ascontiguousarray(b_bits, np.uint8)
        lv = np.ascontiguousarray(leaves, np.uint32).reshape(-1, 8)
        rt = np.ascontiguousarray(root, np.uint32)
        rc = self.lib.flock_sha256_merkle_verify(self.h, bundle, len(bundle), domain, len(domain), path_log, _ptr(b),
                                                 b.size, _ptr(lv), _ptr(rt))
        if rc == 0:
            return ""
        if rc == FLOCK_ERR_VERIFY:
            return self.lib.flock_last_error(self.h).decode()
        self._check(rc, "sha256_merkle_verify")
        return "error"

    def sha256_witness(self, comps: np.ndarray, n_log: int):
        """(z, a, b) packed row witness of (n, 24) u32 SHA-256 compressions
        over 2^n_log blocks, each (2^n_log, 512) u64."""
        comps = np.ascontiguousarray(comps, np.uint32).reshape(-1, 24)
        z, a, b = (np.zeros((1 << n_log, 512), np.uint64) for _ in range(3))
        self._check(self.lib.flock_sha256_witness(self.h, _ptr(comps), comps.shape[0], n_log, _ptr(z), _ptr(a),
                                                  _ptr(b)), "sha256_witness")
        return z, a, b

    def keccak_verify(self, bundle: bytes, domain: bytes = DOMAIN, width: int = 1) -> str:
        """KeccakSetup::verify (keccak.rs, or keccak3.rs for width 3) for any
        supported size: '' when the bundle verifies, otherwise the failed check."""
        rc = getattr(self.lib, f"flock_keccak{_kw(width)}_verify_bundle")(self.h, bundle, len(bundle), domain,
                                                                         len(domain))
        if rc == 0:
            return ""
        if rc == FLOCK_ERR_VERIFY:
            return self.lib.flock_last_error(self.h).decode()
        self._check(rc, "keccak_verify_bundle")
        return "error"

    def keccak_witness(self, states: np.ndarray, n_log: int, width: int = 1):
        """(z, a, b) packed row witness of (n, 25) u64 Keccak states over
        2^n_log blocks, each (2^n_log, 1024 * (1 or 2)) u64."""
        states = np.ascontiguousarray(states, np.uint64).reshape(-1, 25)
        words = 1024 if width == 1 else 2048
        z, a, b = (np.zeros((1 << n_log, words), np.uint64) for _ in range(3))
        self._check(getattr(self.lib, f"flock_keccak{_kw(width)}_witness")(
            self.h, _ptr(states), states.shape[0], n_log, _ptr(z), _ptr(a), _ptr(b)), "keccak_witness")
        return z, a, b

    def keccak_comb(self, e: np.ndarray, alpha, beta, width: int = 1) -> np.ndarray:
        """The Keccak lincheck's alpha A^T e + B^T e + beta [const] on the GPU
        (e: (2^k_log, 2) u64 lo/hi; alpha, beta: (lo, hi))."""
        k = 1 << (16 if width == 1 else 17)
        e = np.ascontiguousarray(e, np.uint64).reshape(k, 2)
        al, be = np.array(alpha, np.uint64), np.array(beta, np.uint64)
        out = np.zeros((k, 2), np.uint64)
        self._check(getattr(self.lib, f"flock_keccak{_kw(width)}_comb")(self.h, _ptr(e), _ptr(al), _ptr(be),
                                                                        _ptr(out)), "keccak_comb")
        return out

    def round1_deg4(self, a, b, c, d, z, m: int, r):
        """round1_deg4_naive (univariate_skip_deg4.rs:77-165) on the GPU:
        packed rows (2^(m-6) u64 per vector), r ((m, 2) u64) -> (p_abcd, p_z),
        each (192, 2) u64."""
        vs = [np.ascontiguousarray(v, np.uint64) for v in (a, b, c, d, z)]
        rr = np.ascontiguousarray(r, np.uint64).reshape(m, 2)
        pa, pz = np.zeros((192, 2), np.uint64), np.zeros((192, 2), np.uint64)
        self._check(self.lib.flock_zerocheck_round1_deg4(self.h, *[_ptr(v) for v in vs], m, _ptr(rr), _ptr(pa),
                                                         _ptr(pz)), "zerocheck_round1_deg4")
        return pa, pz

    def bench_round1_deg4(self, m: int, seed: int = 1, iters: int = 10):
        """(mean ms, p_abcd, p_z) of the seeded degree-4 round-1 benchmark."""
        ms = ctypes.c_double()
        pa, pz = np.zeros((192, 2), np.uint64), np.zeros((192, 2), np.uint64)
        self._check(self.lib.flock_bench_round1_deg4(self.h, m, seed, iters, ctypes.byref(ms), _ptr(pa), _ptr(pz)),
                    "bench_round1_deg4")
        return ms.value, pa, pz

    def serve_verify(self, on: bool = True) -> None:
        """Self-check every served / batched proof with the verifier."""
        self._check(self.lib.flock_serve_verify(self.h, 1 if on else 0), "serve_verify")

    def submit(self, log2: int, seed: int = 0, blocks=None, domain: bytes = None) -> int:
        """Queue one proof; returns its ticket.  blocks: (2^log2, 25) u32 or None."""
        domain = DOMAIN if domain is None else domain
        job = FlockJob(log2, seed, None, domain, len(domain))
        if blocks is not None:
            blocks = np.ascontiguousarray(blocks, np.uint32).reshape(-1, 25)
            job.blocks = blocks.ctypes.data  # copied by the library before submit returns
        t = ctypes.c_uint64()
        self._check(self.lib.flock_submit(self.h, ctypes.byref(job), ctypes.byref(t)), "submit")
        return t.value

    def poll(self, ticket: int, timeout_ms: int = -1):
        """None while the job runs (after timeout_ms), else a dict with the proof
        bytes, its status and the queue / run / end-to-end latencies in ms."""
        buf = np.zeros(MAX_PROOF_BYTES * 2, np.uint8)
        res = FlockResult(buf.ctypes.data, buf.size, 0, 0, 0.0, 0.0, 0.0)
        rc = self.lib.flock_poll(self.h, ticket, ctypes.byref(res), timeout_ms)
        if rc == FLOCK_ERR_TIMEOUT:
            return None
        self._check(rc, "poll")
        if res.status:
            raise FlockError(f"job {ticket} failed ({res.status}): {self.lib.flock_last_error(self.h).decode()}")
        return {"bytes": buf[: res.out_len].tobytes(), "queue_ms": res.queue_ms, "run_ms": res.run_ms,
                "latency_ms": res.latency_ms}

    def prove_batch(self, jobs, threads: int = 8):
        """Prove [(log2, seed or (2^log2, 25) u32 blocks), ...] as one batch;
        returns a list of dicts like poll()'s."""
        n = len(jobs)
        keep = []
        cj = (FlockJob * max(n, 1))()
        bufs = [np.zeros(MAX_PROOF_BYTES * 2, np.uint8) for _ in range(n)]
        cr = (FlockResult * max(n, 1))()
        for i, (log2, inp) in enumerate(jobs):
            cj[i] = FlockJob(log2, 0, None, DOMAIN, len(DOMAIN))
            if isinstance(inp, np.ndarray):
                blk = np.ascontiguousarray(inp, np.uint32).reshape(-1, 25)
                keep.append(blk)
                cj[i].blocks = blk.ctypes.data
            else:
                cj[i].seed = inp
            cr[i] = FlockResult(bufs[i].ctypes.data, bufs[i].size, 0, 0, 0.0, 0.0, 0.0)
        self._check(self.lib.flock_prove_batch(self.h, cj, n, cr, threads), "prove_batch")
        out = []
        for i in range(n):
            if cr[i].status:
                raise FlockError(f"batch job {i} failed ({cr[i].status}): "
                                 f"{self.lib.flock_last_error(self.h).decode()}")
            out.append({"bytes": bufs[i][: cr[i].out_len].tobytes(), "queue_ms": cr[i].queue_ms,
                        "run_ms": cr[i].run_ms, "latency_ms": cr[i].latency_ms})
        return out

    # ---- kernel-level entry points (host arrays in, host arrays out) ----
    def witness(self, log2: int, seed: int):
        words = (1 << max(log2, 3)) * 128
        z, a, b = (np.zeros(2 * words, np.uint64) for _ in range(3))
        self._check(self.lib.flock_witness(self.h, log2, seed, _ptr(z), _ptr(a), _ptr(b)), "witness")
        return z, a, b

    def ntt_rs_encode(self, msg: np.ndarray, log_msg_pos: int, lanes: int, log_inv_rate: int) -> np.ndarray:
        msg = np.ascontiguousarray(msg, np.uint64)
        assert msg.size == 2 * (lanes << log_msg_pos)
        out = np.zeros(msg.size << log_inv_rate, np.uint64)
        self._check(self.lib.flock_ntt_rs_encode(self.h, _ptr(msg), log_msg_pos, lanes, log_inv_rate, _ptr(out)),
                    "ntt_rs_encode")
        return out

    def ntt_rs_encode_plan(self, msg: np.ndarray, log_msg_pos: int, lanes: int, log_inv_rate: int, plan: int):
        """The encode with candidate pass plan `plan`; None past the last plan."""
        msg = np.ascontiguousarray(msg, np.uint64)
        out = np.zeros(msg.size << log_inv_rate, np.uint64)
        rc = self.lib.flock_ntt_rs_encode_plan(self.h, _ptr(msg), log_msg_pos, lanes, log_inv_rate, plan, _ptr(out))
        if rc == 1:
            return None
        self._check(rc, "ntt_rs_encode_plan")
        return out

    def ntt_autotune(self, log_msg_pos: int, lanes: int, log_inv_rate: int):
        """(best plan ms or -1 if already tuned, plan description)."""
        ms = ctypes.c_double()
        d = ctypes.create_string_buffer(256)
        self._check(self.lib.flock_ntt_autotune(self.h, log_msg_pos, lanes, log_inv_rate, ctypes.byref(ms), d, 256),
                    "ntt_autotune")
        return ms.value, d.value.decode()

    def merkle_tree(self, data: np.ndarray, n_leaves: int, leaf_size: int, hash: str = "blake3") -> np.ndarray:
        data = np.ascontiguousarray(data, np.uint8)
        out = np.zeros((2 * n_leaves - 1) * 32, np.uint8)
        self._check(self.lib.flock_merkle_tree_hash(self.h, _ptr(data), n_leaves, leaf_size, HASH[hash], _ptr(out)),
                    "merkle_tree")
        return out

    def set_transcript(self, hash: str) -> None:
        """The transcript hash the verify-bundle entry points assume."""
        self._check(self.lib.flock_ctx_set_transcript(self.h, HASH[hash]), "ctx_set_transcript")

    def sumcheck_round(self, f: np.ndarray, b: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(f, np.uint64)
        b = np.ascontiguousarray(b, np.uint64)
        out = np.zeros(4, np.uint64)
        self._check(self.lib.flock_sumcheck_round(self.h, _ptr(f), _ptr(b), f.size // 2, _ptr(out)), "sumcheck_round")
        return out

    def sumcheck_round3(self, e: np.ndarray, a: np.ndarray, b: np.ndarray, rho=None):
        """Degree-3 round: (G(1), G(inf)) as 4 u64, after an optional fold of
        a, b at rho ((lo, hi)); returns (msg, a_folded, b_folded)."""
        e, a, b = (np.ascontiguousarray(x, np.uint64) for x in (e, a, b))
        n = a.size // 2
        out = np.zeros(4, np.uint64)
        ao, bo = np.zeros(n, np.uint64), np.zeros(n, np.uint64)
        r = None if rho is None else np.array(rho, np.uint64)
        self._check(self.lib.flock_sumcheck_round3(self.h, _ptr(e), _ptr(a), _ptr(b), n,
                                                   None if r is None else _ptr(r), _ptr(ao), _ptr(bo), _ptr(out)),
                    "sumcheck_round3")
        return (out, None, None) if rho is None else (out, ao, bo)

    def pow(self, digest: bytes, bits: int) -> int:
        d = np.frombuffer(digest, np.uint8).copy()
        n = ctypes.c_uint64()
        self._check(self.lib.flock_pow(self.h, _ptr(d), bits, ctypes.byref(n)), "pow")
        return n.value

    def f128_mul(self, a: np.ndarray, b: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(a, np.uint64)
        b = np.ascontiguousarray(b, np.uint64)
        out = np.zeros_like(a)
        self._check(self.lib.flock_f128_mul(self.h, _ptr(a), _ptr(b), a.size // 2, _ptr(out)), "f128_mul")
        return out

    def bench_ntt(self, log_msg_pos: int, lanes: int, rate: int, iters: int = 5) -> float:
        ms = ctypes.c_double()
        self._check(self.lib.flock_bench_ntt(self.h, log_msg_pos, lanes, rate, iters, ctypes.byref(ms)), "bench_ntt")
        return ms.value

    def bench_ntt_plan(self, log_msg_pos: int, lanes: int, rate: int, plan: int, iters: int = 5) -> float:
        ms = ctypes.c_double()
        self._check(self.lib.flock_bench_ntt_plan(self.h, log_msg_pos, lanes, rate, plan, iters, ctypes.byref(ms)),
                    "bench_ntt_plan")
        return ms.value

    def bench_f128_product(self, variant: int, iters: int = 400) -> float:
        """GF(2^128) products/s by a warp-uniform constant: 0 integer, 1 table, 2 mixed."""
        r = ctypes.c_double()
        self._check(self.lib.flock_bench_f128_product(self.h, variant, iters, ctypes.byref(r)), "bench_f128_product")
        return r.value

    def bench_merkle(self, n_leaves: int, leaf_size: int, iters: int = 5) -> float:
        ms = ctypes.c_double()
        self._check(self.lib.flock_bench_merkle(self.h, n_leaves, leaf_size, iters, ctypes.byref(ms)), "bench_merkle")
        return ms.value

    def bench_sumcheck(self, n: int, iters: int = 5) -> float:
        ms = ctypes.c_double()
        self._check(self.lib.flock_bench_sumcheck(self.h, n, iters, ctypes.byref(ms)), "bench_sumcheck")
        return ms.value


    def bench_sumcheck3(self, n: int, iters: int = 5) -> float:
        ms = ctypes.c_double()
        self._check(self.lib.flock_bench_sumcheck3(self.h, n, iters, ctypes.byref(ms)), "bench_sumcheck3")
        return ms.value


class Challenger:
    """FsChallenger::with_hash(domain, hash) (crates/flock-core/src/
    challenger.rs:170-600) behind the C ABI; values are (lo, hi) pairs of
    u64.  hash: "blake3" (the benchmark's) or "sha256" (FsChallenger::new)."""

    def __init__(self, domain: bytes = DOMAIN, hash: str = "blake3"):
        self.lib = load()
        h = ctypes.c_void_p()
        if self.lib.flock_challenger_create_hash(domain, len(domain), HASH[hash], ctypes.byref(h)):
            raise FlockError("challenger_create failed")
        self.h = h

    def close(self) -> None:
        if self.h:
            self.lib.flock_challenger_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def observe_label(self, label: bytes) -> None:
        self.lib.flock_challenger_observe_label(self.h, label, len(label))

    def observe_bytes(self, data: bytes) -> None:
        self.lib.flock_challenger_observe_bytes(self.h, data, len(data))

    def observe_f128(self, v) -> None:
        a = np.array(v, np.uint64)
        self.lib.flock_challenger_observe_f128(self.h, _ptr(a))

    def observe_f128_slice(self, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, np.uint64).reshape(-1)
        self.lib.flock_challenger_observe_f128_slice(self.h, _ptr(a), a.size // 2)

    def sample_f128(self):
        out = np.zeros(2, np.uint64)
        self.lib.flock_challenger_sample_f128(self.h, _ptr(out))
        return int(out[0]), int(out[1])

    def sample_f128_vec(self, n: int) -> np.ndarray:
        out = np.zeros(2 * max(n, 1), np.uint64)
        self.lib.flock_challenger_sample_f128_vec(self.h, n, _ptr(out))
        return out[: 2 * n]

    def grind_pow(self, ctx: "Context", bits: int) -> int:
        """Smallest valid nonce, absorbed; ctx may be None for at most 6 bits (host search)."""
        n = ctypes.c_uint64()
        rc = self.lib.flock_challenger_grind_pow(self.h, ctx.h if ctx else None, bits, ctypes.byref(n))
        if rc:
            if ctx:
                ctx._check(rc, "challenger_grind_pow")
            raise FlockError(f"challenger_grind_pow failed ({rc})")
        return n.value

    def verify_pow(self, nonce: int, bits: int) -> bool:
        return self.lib.flock_challenger_verify_pow(self.h, nonce, bits) == 0

    def state_digest(self) -> bytes:
        out = np.zeros(32, np.uint8)
        self.lib.flock_challenger_state_digest(self.h, _ptr(out))
        return out.tobytes()


class ProverData:
    """pcs::commit's retained state (codeword + Merkle tree) on the device."""

    def __init__(self, ctx: "Context", z_packed: np.ndarray, m: int):
        self.ctx = ctx
        z = np.ascontiguousarray(z_packed, np.uint64)
        assert z.size == 2 << (m - 7), "z_packed holds 2^(m-7) F128 values"
        root = np.zeros(32, np.uint8)
        h = ctypes.c_void_p()
        ctx._check(ctx.lib.flock_pcs_commit(ctx.h, _ptr(z), m, _ptr(root), ctypes.byref(h)), "pcs_commit")
        self.h, self.m, self.root = h, m, root.tobytes()

    def open(self, positions):
        """(rows (n, 64, 2) u64, multi-proof sibling hashes (k, 32) u8)."""
        pos = np.ascontiguousarray(positions, np.uint64)
        rows = np.zeros((max(pos.size, 1), 64, 2), np.uint64)
        cap = 64 * max(pos.size, 1) + 64
        proof = np.zeros((cap, 32), np.uint8)
        k = ctypes.c_size_t()
        self.ctx._check(self.ctx.lib.flock_prover_data_open(self.h, _ptr(pos), pos.size, _ptr(rows), _ptr(proof), cap,
                                                            ctypes.byref(k)), "prover_data_open")
        return rows[: pos.size], proof[: k.value]

    def close(self) -> None:
        if self.h:
            self.ctx.lib.flock_prover_data_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Sha256Prover:
    """`Sha256HybridSetup::new(n)` (crates/flock-prover/src/r1cs_hashes/
    sha2.rs:1252-1330): SHA-256 compressions, one per 2^15-bit block,
    2^max(3, ceil(log2 n)) slots, BLAKE3 Merkle hashing, fast profile."""

    def __init__(self, ctx: Context, n: int, merkle_hash: str = "blake3", transcript: str = "blake3"):
        h = ctypes.c_void_p()
        ctx._check(ctx.lib.flock_sha256_setup_create(ctx.h, n, HASH[merkle_hash], 0, ctypes.byref(h)),
                   "sha256_setup_create")
        self.ctx, self.n, self.h = ctx, n, h
        ctx._check(ctx.lib.flock_setup_set_transcript(h, HASH[transcript]), "setup_set_transcript")
        self.n_log = max(3, (n - 1).bit_length())
        self._buf = np.zeros(MAX_PROOF_BYTES * 2, np.uint8)

    def close(self) -> None:
        if self.h:
            self.ctx.lib.flock_setup_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def prove(self, comps: np.ndarray, domain: bytes = DOMAIN) -> bytes:
        """prove_fast over (n, 24) u32 compressions (h_in[8], m[16])."""
        comps = np.ascontiguousarray(comps, np.uint32).reshape(-1, 24)
        n = ctypes.c_size_t()
        rc = self.ctx.lib.flock_sha256_prove(self.h, _ptr(comps), comps.shape[0], domain, len(domain),
                                             _ptr(self._buf), self._buf.size, ctypes.byref(n))
        self.ctx._check(rc, "sha256_prove")
        return self._buf[: n.value].tobytes()

    def prove_chain(self, comps: np.ndarray, domain: bytes = CHAIN_DOMAIN) -> bytes:
        """prove_chain over (n, 24) u32 compressions that fill the setup
        (ChainProofBundleLigerito bytes, hash kind Sha2)."""
        comps = np.ascontiguousarray(comps, np.uint32).reshape(-1, 24)
        n = ctypes.c_size_t()
        rc = self.ctx.lib.flock_sha256_prove_chain(self.h, _ptr(comps), comps.shape[0], domain, len(domain),
                                                   _ptr(self._buf), self._buf.size, ctypes.byref(n))
        self.ctx._check(rc, "sha256_prove_chain")
        return self._buf[: n.value].tobytes()

    def prove_merkle(self, comps: np.ndarray, b_bits, path_log: int = 0, domain: bytes = MERKLE_DOMAIN) -> bytes:
        """prove_merkle_paths_ligerito over (n, 24) u32 compressions that fill
        the setup (n a power of two) and n selector bits; bincode of
        (Commitment, MerklePathProofLigerito)."""
        comps = np.ascontiguousarray(comps, np.uint32).reshape(-1, 24)
        b = np.ascontiguousarray(b_bits, np.uint8)
        n = ctypes.c_size_t()
        rc = self.ctx.lib.flock_sha256_merkle_prove(self.h, _ptr(comps), comps.shape[0], _ptr(b), path_log, domain,
                                                    len(domain), _ptr(self._buf), self._buf.size, ctypes.byref(n))
        self.ctx._check(rc, "sha256_merkle_prove")
        return self._buf[: n.value].tobytes()

    def prove_seed(self, seed: int, domain: bytes = DOMAIN) -> bytes:
        """prove_fast over sha256_bench_inputs(n, seed), generated on the GPU."""
        n = ctypes.c_size_t()
        rc = self.ctx.lib.flock_prove_seed(self.h, seed, domain, len(domain), _ptr(self._buf), self._buf.size,
                                           ctypes.byref(n))
        self.ctx._check(rc, "prove_seed")
        return self._buf[: n.value].tobytes()

    def verify(self, bundle: bytes, domain: bytes = DOMAIN) -> str:
        rc = self.ctx.lib.flock_verify(self.h, bundle, len(bundle), domain, len(domain))
        if rc == 0:
            return ""
        if rc == FLOCK_ERR_VERIFY:
            return self.ctx.lib.flock_last_error(self.ctx.h).decode()
        self.ctx._check(rc, "verify")
        return "error"

    def phase_ms(self) -> dict:
        out = np.zeros(len(PHASES), np.float64)
        k = self.ctx.lib.flock_setup_phase_ms(self.h, _ptr(out), len(PHASES))
        return dict(zip(PHASES[:k], out[:k].tolist()))


class KeccakProver:
    """`KeccakSetup::new(n)` (crates/flock-prover/src/r1cs_hashes/keccak.rs:
    870-912): Keccak-f[1600] permutations, one per 2^16-bit block,
    2^max(3, ceil(log2 n)) slots, fast profile; BLAKE3 Merkle hashing unless
    merkle_hash says otherwise.  width = 3: the 3-wide `keccak3::KeccakSetup`
    (keccak3.rs:491-540), three permutations per 2^17-bit block."""

    def __init__(self, ctx: Context, n: int, merkle_hash: str = "blake3", transcript: str = "blake3",
                 width: int = 1):
        h = ctypes.c_void_p()
        ctx._check(getattr(ctx.lib, f"flock_keccak{_kw(width)}_setup_create")(ctx.h, n, HASH[merkle_hash], 0,
                                                                               ctypes.byref(h)),
                   "keccak_setup_create")
        self.ctx, self.n, self.h, self.width = ctx, n, h, width
        ctx._check(ctx.lib.flock_setup_set_transcript(h, HASH[transcript]), "setup_set_transcript")
        self.n_log = max(3, (-(-n // width) - 1).bit_length())
        self._buf = np.zeros(MAX_PROOF_BYTES * 2, np.uint8)

    def close(self) -> None:
        if self.h:
            self.ctx.lib.flock_setup_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def prove(self, states: np.ndarray, domain: bytes = DOMAIN) -> bytes:
        """prove_fast over (n, 25) u64 states."""
        states = np.ascontiguousarray(states, np.uint64).reshape(-1, 25)
        n = ctypes.c_size_t()
        rc = self.ctx.lib.flock_keccak_prove(self.h, _ptr(states), states.shape[0], domain, len(domain),
                                             _ptr(self._buf), self._buf.size, ctypes.byref(n))
        self.ctx._check(rc, "keccak_prove")
        return self._buf[: n.value].tobytes()

    def prove_chain(self, states: np.ndarray, domain: bytes = CHAIN_DOMAIN) -> bytes:
        """prove_chain over (n, 25) u64 states that fill the setup
        (ChainProofBundleLigerito bytes, hash kind Keccak)."""
        states = np.ascontiguousarray(states, np.uint64).reshape(-1, 25)
        n = ctypes.c_size_t()
        rc = self.ctx.lib.flock_keccak_prove_chain(self.h, _ptr(states), states.shape[0], domain, len(domain),
                                                   _ptr(self._buf), self._buf.size, ctypes.byref(n))
        self.ctx._check(rc, "keccak_prove_chain")
        return self._buf[: n.value].tobytes()

    def prove_seed(self, seed: int, domain: bytes = DOMAIN) -> bytes:
        """prove_fast over keccak_bench_inputs(n, seed), generated on the GPU."""
        n = ctypes.c_size_t()
        rc = self.ctx.lib.flock_prove_seed(self.h, seed, domain, len(domain), _ptr(self._buf), self._buf.size,
                                           ctypes.byref(n))
        self.ctx._check(rc, "prove_seed")
        return self._buf[: n.value].tobytes()

    def verify(self, bundle: bytes, domain: bytes = DOMAIN) -> str:
        rc = self.ctx.lib.flock_verify(self.h, bundle, len(bundle), domain, len(domain))
        if rc == 0:
            return ""
        if rc == FLOCK_ERR_VERIFY:
            return self.ctx.lib.flock_last_error(self.ctx.h).decode()
        self.ctx._check(rc, "verify")
        return "error"

    def phase_ms(self) -> dict:
        out = np.zeros(len(PHASES), np.float64)
        k = self.ctx.lib.flock_setup_phase_ms(self.h, _ptr(out), len(PHASES))
        return dict(zip(PHASES[:k], out[:k].tolist()))


class Prover:
    """`Blake3Setup` for 2^log2 compressions with BLAKE3 Merkle hashing
    (crates/flock-prover/src/r1cs_hashes/blake3.rs:4656-5170), or, with
    n_blocks, `Blake3Setup::new(n_blocks)` for any count (2^max(3, ceil(log2
    n)) slots, blake3.rs:1854-1858)."""

    def __init__(self, ctx: Context, log2: int = None, n_blocks: int = None, merkle_hash: str = "blake3",
                 transcript: str = "blake3"):
        h = ctypes.c_void_p()
        mh = HASH[merkle_hash]
        if n_blocks is not None:
            ctx._check(ctx.lib.flock_setup_create_blocks(ctx.h, n_blocks, mh, 0, ctypes.byref(h)), "setup_create_blocks")
            log2 = max(3, (n_blocks - 1).bit_length())
        else:
            ctx._check(ctx.lib.flock_setup_create(ctx.h, log2, mh, 0, ctypes.byref(h)), "setup_create")
            n_blocks = 1 << log2
        self.ctx, self.log2, self.n_blocks = ctx, log2, n_blocks
        self.h = h
        ctx._check(ctx.lib.flock_setup_set_transcript(h, HASH[transcript]), "setup_set_transcript")
        self._buf = np.zeros(MAX_PROOF_BYTES * 2, np.uint8)

    def close(self) -> None:
        if self.h:
            self.ctx.lib.flock_setup_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def prove_seed(self, seed: int, domain: bytes = DOMAIN) -> bytes:
        n = ctypes.c_size_t()
        rc = self.ctx.lib.flock_prove_seed(self.h, seed, domain, len(domain), _ptr(self._buf), self._buf.size,
                                           ctypes.byref(n))
        self.ctx._check(rc, "prove_seed")
        return self._buf[: n.value].tobytes()

    def prove_blocks(self, blocks: np.ndarray, domain: bytes = DOMAIN) -> bytes:
        blocks = np.ascontiguousarray(blocks, np.uint32).reshape(-1, 25)
        n = ctypes.c_size_t()
        rc = self.ctx.lib.flock_prove_blocks(self.h, _ptr(blocks), blocks.shape[0], domain, len(domain),
                                             _ptr(self._buf), self._buf.size, ctypes.byref(n))
        self.ctx._check(rc, "prove_blocks")
        return self._buf[: n.value].tobytes()

    def prove_compressions(self, records: np.ndarray, domain: bytes = DOMAIN) -> bytes:
        """prove_fast over (n_blocks, 28) u32 flock_compression records (cv[8],
        m[16], counter u64 little endian, block_len, flags); the statement's
        slots from n_blocks on hold the all-zero compression."""
        records = np.ascontiguousarray(records, np.uint32).reshape(-1, 28)
        n = ctypes.c_size_t()
        rc = self.ctx.lib.flock_prove_compressions(self.h, _ptr(records), records.shape[0], domain, len(domain),
                                                   _ptr(self._buf), self._buf.size, ctypes.byref(n))
        self.ctx._check(rc, "prove_compressions")
        return self._buf[: n.value].tobytes()

    def prove_chain(self, records: np.ndarray, domain: bytes = CHAIN_DOMAIN) -> bytes:
        """A hash-chain proof (Blake3Setup::prove_chain, blake3.rs:5195) over
        (2^log2, 28) u32 compression records; FLOCK v4 chain bundle bytes."""
        records = np.ascontiguousarray(records, np.uint32).reshape(-1, 28)
        n = ctypes.c_size_t()
        rc = self.ctx.lib.flock_prove_chain(self.h, _ptr(records), records.shape[0], domain, len(domain),
                                            _ptr(self._buf), self._buf.size, ctypes.byref(n))
        self.ctx._check(rc, "prove_chain")
        return self._buf[: n.value].tobytes()

    def verify(self, bundle: bytes, domain: bytes = DOMAIN) -> str:
        """'' when the FLOCK v4 bundle (compression or chain) verifies on this
        setup's statement, otherwise the name of the failed check."""
        rc = self.ctx.lib.flock_verify(self.h, bundle, len(bundle), domain, len(domain))
        if rc == 0:
            return ""
        if rc == FLOCK_ERR_VERIFY:
            return self.ctx.lib.flock_last_error(self.ctx.h).decode()
        self.ctx._check(rc, "verify")
        return "error"

    def bench(self, seed0: int, steps: int):
        """(total device ms of `steps` proofs, mean per-phase ms, kernel launches)."""
        total = ctypes.c_double()
        ph = np.zeros(len(PHASES), np.float64)
        n = ctypes.c_uint64()
        self.ctx._check(self.ctx.lib.flock_bench_prove(self.h, seed0, steps, ctypes.byref(total), _ptr(ph),
                                                       ctypes.byref(n)), "bench_prove")
        return total.value, dict(zip(PHASES, ph.tolist())), n.value

    def phase_ms(self) -> dict:
        out = np.zeros(len(PHASES), np.float64)
        k = self.ctx.lib.flock_setup_phase_ms(self.h, _ptr(out), len(PHASES))
        return dict(zip(PHASES[:k], out[:k].tolist()))
