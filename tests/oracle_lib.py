"""ctypes access to the oracle (oracle/_build/libflockref.so) for the tests.

The oracle is test infrastructure: a CPU restatement of the reference prover
whose proofs the reference's trusted verifier accepts.  Only the tests,
__graft_entry__.smoke() and bench.py's CPU-baseline / reference arm load it.
"""
import ctypes
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parents[1] / "oracle/_build/libflockref.so"


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


class Oracle:
    def __init__(self):
        L = ctypes.CDLL(str(LIB))
        vp, u32, u64, sz, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_int
        L.flockref_prove.argtypes = [u32, u64, vp, sz, ctypes.POINTER(sz)]
        L.flockref_f128_mul.argtypes = [vp, vp, vp]
        L.flockref_f128_mul_n.argtypes = [vp, vp, sz, vp]
        L.flockref_f128_inv.argtypes = [vp, vp]
        L.flockref_phi8_table.argtypes = [vp]
        L.flockref_gf8_mul.argtypes = [ctypes.c_uint8, ctypes.c_uint8]
        L.flockref_gf8_mul.restype = ctypes.c_uint8
        L.flockref_blake3_hash.argtypes = [ctypes.c_char_p, sz, vp]
        L.flockref_blake3_xof.argtypes = [ctypes.c_char_p, sz, vp, sz]
        L.flockref_blake3_leaf_cv.argtypes = [ctypes.c_char_p, sz, vp]
        L.flockref_blake3_parent_cv.argtypes = [ctypes.c_char_p, ctypes.c_char_p, vp]
        L.flockref_generate_compressions.argtypes = [u32, u64, vp]
        L.flockref_witness.argtypes = [u32, u64, vp, vp, vp]
        L.flockref_apply_matrices.argtypes = [vp, i32, vp, vp]
        L.flockref_statement_digest.argtypes = [u32, vp]
        L.flockref_matrix_nnz.argtypes = [i32]
        L.flockref_matrix_nnz.restype = u64
        L.flockref_rs_encode.argtypes = [vp, sz, sz, i32, vp]
        L.flockref_ntt_twiddles.argtypes = [i32, vp]
        L.flockref_merkle_tree.argtypes = [vp, sz, sz, vp]
        L.flockref_merkle_multi_proof.argtypes = [vp, sz, vp, sz, vp, sz]
        L.flockref_merkle_multi_proof.restype = sz
        L.flockref_build_eq.argtypes = [vp, i32, vp]
        L.flockref_lagrange.argtypes = [vp, i32, vp]
        L.flockref_ch_new.argtypes = [ctypes.c_char_p]
        L.flockref_ch_new.restype = vp
        L.flockref_ch_free.argtypes = [vp]
        L.flockref_ch_label.argtypes = [vp, ctypes.c_char_p]
        L.flockref_ch_observe.argtypes = [vp, vp]
        L.flockref_ch_observe_slice.argtypes = [vp, vp, sz]
        L.flockref_ch_bytes.argtypes = [vp, ctypes.c_char_p, sz]
        L.flockref_ch_sample.argtypes = [vp, vp]
        L.flockref_ch_sample_vec.argtypes = [vp, sz, vp]
        L.flockref_ch_grind.argtypes = [vp, u32]
        L.flockref_ch_grind.restype = u64
        L.flockref_ch_digest.argtypes = [vp, vp]
        L.flockref_pow_ok.argtypes = [vp, u64, u32]
        L.flockref_chain_blocks.argtypes = [u64, vp, sz, vp]
        L.flockref_sha256_compress.argtypes = [vp, vp, vp]
        L.flockref_sha256_bench_inputs.argtypes = [sz, u64, vp]
        L.flockref_sha256_min_n_blocks_log.argtypes = [sz]
        L.flockref_sha256_digest.argtypes = [u32, vp]
        L.flockref_sha256_matrix_nnz.argtypes = [i32]
        L.flockref_sha256_matrix_nnz.restype = u64
        L.flockref_sha256_matrix_csr.argtypes = [i32, vp, vp]
        L.flockref_sha256_witness.argtypes = [vp, sz, u32, vp, vp, vp]
        L.flockref_prove_sha256.argtypes = [vp, sz, ctypes.c_char_p, sz, vp, sz, ctypes.POINTER(sz)]
        L.flockref_prove_sha256_zero.argtypes = [u32, ctypes.c_char_p, sz, vp, sz, ctypes.POINTER(sz)]
        L.flockref_sha256_merkle_inputs.argtypes = [u32, u32, u64, vp, vp, vp, vp]
        L.flockref_set_hash_kinds.argtypes = [i32, i32]
        L.flockref_sha256.argtypes = [ctypes.c_char_p, sz, vp]
        L.flockref_ch_new_hash.argtypes = [ctypes.c_char_p, i32]
        L.flockref_ch_new_hash.restype = vp
        L.flockref_merkle_tree_hash.argtypes = [vp, sz, sz, i32, vp]
        L.flockref_prove_sha256_merkle.argtypes = [vp, vp, vp, vp, u32, u32, ctypes.c_char_p, sz, vp, sz,
                                                   ctypes.POINTER(sz), ctypes.POINTER(ctypes.c_int)]
        L.flockref_prove_chain_blocks.argtypes = [vp, u32, ctypes.c_char_p, sz, vp, vp, sz, ctypes.POINTER(sz),
                                                  ctypes.POINTER(ctypes.c_int)]
        L.flockref_prove_records.argtypes = [vp, sz, ctypes.c_char_p, sz, vp, sz, ctypes.POINTER(sz)]
        L.flockref_keccak_f.argtypes = [vp]
        L.flockref_keccak_bench_inputs.argtypes = [sz, u64, vp]
        L.flockref_keccak_digest.argtypes = [i32, u32, vp]
        L.flockref_keccak_witness.argtypes = [i32, vp, sz, u32, vp, vp, vp]
        L.flockref_keccak_comb.argtypes = [i32, vp, vp, vp]
        L.flockref_prove_keccak.argtypes = [i32, vp, sz, ctypes.c_char_p, sz, vp, sz, ctypes.POINTER(sz)]
        L.flockref_last_open_identity_ok.argtypes = []
        L.flockref_sha256_chain_blocks.argtypes = [u64, vp, sz, vp]
        L.flockref_prove_keccak_chain.argtypes = [vp, u32, ctypes.c_char_p, sz, vp, vp, sz, ctypes.POINTER(sz),
                                                  ctypes.POINTER(ctypes.c_int)]
        L.flockref_prove_sha256_chain.argtypes = [vp, u32, ctypes.c_char_p, sz, vp, vp, sz, ctypes.POINTER(sz),
                                                  ctypes.POINTER(ctypes.c_int)]
        L.flockref_round1_deg4.argtypes = [vp, vp, vp, vp, vp, u32, vp, vp, vp]
        L.flockref_time_prove.argtypes = [u32, u64, ctypes.POINTER(sz)]
        L.flockref_time_prove.restype = ctypes.c_double
        self.L = L

    # ---- hash kinds (0 SHA-256, 1 BLAKE3) of the next proofs on this thread
    def set_hash_kinds(self, merkle: str = "blake3", transcript: str = "blake3") -> None:
        k = {"sha256": 0, "blake3": 1}
        self.L.flockref_set_hash_kinds(k[merkle], k[transcript])

    def sha256(self, data: bytes) -> bytes:
        out = np.zeros(32, np.uint8)
        self.L.flockref_sha256(data, len(data), _p(out))
        return out.tobytes()

    def merkle_tree_hash(self, data: np.ndarray, n_leaves: int, leaf_size: int, hash: str) -> np.ndarray:
        data = np.ascontiguousarray(data, np.uint8)
        out = np.zeros((2 * n_leaves - 1) * 32, np.uint8)
        self.L.flockref_merkle_tree_hash(_p(data), n_leaves, leaf_size, {"sha256": 0, "blake3": 1}[hash], _p(out))
        return out

    # ---- Keccak-f[1600] permutations (r1cs_hashes/keccak.rs); a state is 25 u64 lanes
    def keccak_f(self, lanes) -> np.ndarray:
        s = np.array(lanes, np.uint64).copy()
        self.L.flockref_keccak_f(_p(s))
        return s

    def keccak_bench_inputs(self, n: int, seed: int) -> np.ndarray:
        out = np.zeros((n, 25), np.uint64)
        self.L.flockref_keccak_bench_inputs(n, seed, _p(out))
        return out

    # width: 1 = the single encoder (keccak.rs, 2^16-bit blocks), 3 = the
    # 3-wide one (keccak3.rs, 2^17-bit blocks of three permutations)
    def keccak_digest(self, n_log: int, width: int = 1) -> bytes:
        out = np.zeros(32, np.uint8)
        self.L.flockref_keccak_digest(width, n_log, _p(out))
        return out.tobytes()

    def keccak_witness(self, states: np.ndarray, n_log: int, width: int = 1):
        states = np.ascontiguousarray(states, np.uint64).reshape(-1, 25)
        words = 1024 if width == 1 else 2048
        z, a, b = (np.zeros((1 << n_log, words), np.uint64) for _ in range(3))
        self.L.flockref_keccak_witness(width, _p(states), states.shape[0], n_log, _p(z), _p(a), _p(b))
        return z, a, b

    def keccak_comb(self, alpha, e: np.ndarray, width: int = 1) -> np.ndarray:
        """alpha A^T e + B^T e over a block's rows (e: 2^k_log x (lo, hi))."""
        k = 1 << (16 if width == 1 else 17)
        al = np.array(alpha, np.uint64)
        e = np.ascontiguousarray(e, np.uint64).reshape(k, 2)
        out = np.zeros((k, 2), np.uint64)
        self.L.flockref_keccak_comb(width, _p(al), _p(e), _p(out))
        return out

    def prove_keccak(self, states: np.ndarray, domain: bytes = b"flock-bench-v0", width: int = 1) -> bytes:
        states = np.ascontiguousarray(states, np.uint64).reshape(-1, 25)
        buf = np.zeros(2_000_000, np.uint8)
        n = ctypes.c_size_t()
        rc = self.L.flockref_prove_keccak(width, _p(states), states.shape[0], domain, len(domain), _p(buf),
                                         buf.size, ctypes.byref(n))
        assert rc == 0, rc
        return buf[: n.value].tobytes()

    def last_open_identity_ok(self) -> bool:
        """The batched open's claim identity of this thread's last Keccak,
        chain or Merkle-path proof."""
        return bool(self.L.flockref_last_open_identity_ok())

    # ---- degree-4 zerocheck round 1 (zerocheck/univariate_skip_deg4.rs)
    def round1_deg4(self, a, b, c, d, z, m: int, r: np.ndarray):
        """round1_deg4_naive over packed rows (2^(m-6) u64 each) and r
        ((m, 2) u64): (p_abcd, p_z), each (192, 2) u64."""
        vs = [np.ascontiguousarray(v, np.uint64) for v in (a, b, c, d, z)]
        rr = np.ascontiguousarray(r, np.uint64).reshape(m, 2)
        pa, pz = np.zeros((192, 2), np.uint64), np.zeros((192, 2), np.uint64)
        self.L.flockref_round1_deg4(*[_p(v) for v in vs], m, _p(rr), _p(pa), _p(pz))
        return pa, pz

    # ---- SHA-256 compressions (r1cs_hashes/sha2.rs)
    def sha256_compress(self, h, m) -> np.ndarray:
        h, m = np.ascontiguousarray(h, np.uint32), np.ascontiguousarray(m, np.uint32)
        out = np.zeros(8, np.uint32)
        self.L.flockref_sha256_compress(_p(h), _p(m), _p(out))
        return out

    def sha256_bench_inputs(self, n: int, seed: int) -> np.ndarray:
        out = np.zeros((n, 24), np.uint32)
        self.L.flockref_sha256_bench_inputs(n, seed, _p(out))
        return out

    def sha256_digest(self, n_log: int) -> bytes:
        out = np.zeros(32, np.uint8)
        self.L.flockref_sha256_digest(n_log, _p(out))
        return out.tobytes()

    def sha256_matrix(self, which: int):
        nnz = self.L.flockref_sha256_matrix_nnz(which)
        ptr = np.zeros((1 << 15) + 1, np.uint32)
        col = np.zeros(nnz, np.uint16)
        self.L.flockref_sha256_matrix_csr(which, _p(ptr), _p(col))
        return ptr, col

    def sha256_witness(self, comps: np.ndarray, n_log: int):
        comps = np.ascontiguousarray(comps, np.uint32).reshape(-1, 24)
        z, a, b = (np.zeros((1 << n_log, 512), np.uint64) for _ in range(3))
        self.L.flockref_sha256_witness(_p(comps), comps.shape[0], n_log, _p(z), _p(a), _p(b))
        return z, a, b

    def prove_sha256(self, comps: np.ndarray, domain: bytes = b"flock-bench-v0") -> bytes:
        comps = np.ascontiguousarray(comps, np.uint32).reshape(-1, 24)
        buf = np.zeros(2_000_000, np.uint8)
        n = ctypes.c_size_t()
        rc = self.L.flockref_prove_sha256(_p(comps), comps.shape[0], domain, len(domain), _p(buf), buf.size,
                                          ctypes.byref(n))
        assert rc == 0, rc
        return buf[: n.value].tobytes()

    def sha256_merkle_inputs(self, n_log: int, path_log: int, seed: int):
        n = 1 << n_log
        comps = np.zeros((n, 24), np.uint32)
        b = np.zeros(n, np.uint8)
        leaves = np.zeros((1 << path_log, 8), np.uint32)
        root = np.zeros(8, np.uint32)
        self.L.flockref_sha256_merkle_inputs(n_log, path_log, seed, _p(comps), _p(b), _p(leaves), _p(root))
        return comps, b, leaves, root

    def prove_sha256_merkle(self, comps, b, leaves, root, path_log: int,
                            domain: bytes = b"flock-merkle-bench-v0") -> tuple:
        """(bytes, check): check = the shift argument verified from the public
        leaves and root, and the batched open's claim identity."""
        comps = np.ascontiguousarray(comps, np.uint32).reshape(-1, 24)
        b = np.ascontiguousarray(b, np.uint8)
        leaves = np.ascontiguousarray(leaves, np.uint32)
        root = np.ascontiguousarray(root, np.uint32)
        n_log = comps.shape[0].bit_length() - 1
        buf = np.zeros(2_000_000, np.uint8)
        n = ctypes.c_size_t()
        chk = ctypes.c_int()
        rc = self.L.flockref_prove_sha256_merkle(_p(comps), _p(b), _p(leaves), _p(root), n_log, path_log, domain,
                                                 len(domain), _p(buf), buf.size, ctypes.byref(n), ctypes.byref(chk))
        assert rc == 0, rc
        return buf[: n.value].tobytes(), bool(chk.value)

    def prove_sha256_zero(self, n_log: int, domain: bytes = b"flock-bench-v0") -> bytes:
        buf = np.zeros(2_000_000, np.uint8)
        n = ctypes.c_size_t()
        rc = self.L.flockref_prove_sha256_zero(n_log, domain, len(domain), _p(buf), buf.size, ctypes.byref(n))
        assert rc == 0, rc
        return buf[: n.value].tobytes()

    def prove(self, log2: int, seed: int) -> bytes:
        buf = np.zeros(1 << 20, np.uint8)
        n = ctypes.c_size_t()
        rc = self.L.flockref_prove(log2, seed, _p(buf), buf.size, ctypes.byref(n))
        assert rc == 0, rc
        return buf[: n.value].tobytes()

    def prove_records(self, records: np.ndarray, domain: bytes = b"flock-bench-v0") -> bytes:
        """prove_fast over (n, 28) u32 compression records, any n >= 1: the
        statement's slots from n on hold the all-zero compression."""
        records = np.ascontiguousarray(records, np.uint32).reshape(-1, 28)
        buf = np.zeros(1 << 21, np.uint8)
        n = ctypes.c_size_t()
        rc = self.L.flockref_prove_records(_p(records), records.shape[0], domain, len(domain), _p(buf), buf.size,
                                           ctypes.byref(n))
        assert rc == 0, rc
        return buf[: n.value].tobytes()

    def chain_blocks(self, seed: int, steps: int, initial_cv=None) -> np.ndarray:
        """(steps, 28) u32 records of the flock_chain CLI's honest chain."""
        out = np.zeros((steps, 28), np.uint32)
        cv = None if initial_cv is None else _p(np.ascontiguousarray(initial_cv, np.uint32))
        self.L.flockref_chain_blocks(seed, cv, steps, _p(out))
        return out

    def prove_chain(self, records: np.ndarray, domain: bytes, cv_last=None) -> tuple:
        """(chain bundle bytes, check): check is True when the shift argument
        verifies from the bundle's public endpoints and the batched open's
        claim identity holds."""
        records = np.ascontiguousarray(records, np.uint32)
        log2 = records.shape[0].bit_length() - 1
        buf = np.zeros(1 << 21, np.uint8)
        n = ctypes.c_size_t()
        chk = ctypes.c_int(-1)
        cvl = None if cv_last is None else _p(np.ascontiguousarray(cv_last, np.uint32))
        rc = self.L.flockref_prove_chain_blocks(_p(records), log2, domain, len(domain), cvl, _p(buf), buf.size,
                                                ctypes.byref(n), ctypes.byref(chk))
        assert rc == 0, rc
        return buf[: n.value].tobytes(), chk.value == 1

    def sha256_chain_blocks(self, seed: int, steps: int, initial=None) -> np.ndarray:
        """(steps, 24) u32 records (h_in, m) of the CLI's honest SHA-256 chain."""
        out = np.zeros((steps, 24), np.uint32)
        h = None if initial is None else _p(np.ascontiguousarray(initial, np.uint32))
        self.L.flockref_sha256_chain_blocks(seed, h, steps, _p(out))
        return out

    def prove_sha256_chain(self, records: np.ndarray, domain: bytes, cv_last=None) -> tuple:
        """(SHA-256 chain bundle bytes, check), as prove_chain."""
        records = np.ascontiguousarray(records, np.uint32)
        log2 = records.shape[0].bit_length() - 1
        buf = np.zeros(1 << 21, np.uint8)
        n = ctypes.c_size_t()
        chk = ctypes.c_int(-1)
        cvl = None if cv_last is None else _p(np.ascontiguousarray(cv_last, np.uint32))
        rc = self.L.flockref_prove_sha256_chain(_p(records), log2, domain, len(domain), cvl, _p(buf), buf.size,
                                                ctypes.byref(n), ctypes.byref(chk))
        assert rc == 0, rc
        return buf[: n.value].tobytes(), chk.value == 1

    def keccak_chain_states(self, steps: int, initial=None) -> np.ndarray:
        """(steps, 25) u64: successive keccak_f states from `initial` (zero by default)."""
        cur = np.zeros(25, np.uint64) if initial is None else np.array(initial, np.uint64)
        out = np.zeros((steps, 25), np.uint64)
        for i in range(steps):
            out[i] = cur
            cur = self.keccak_f(cur)
        return out

    def prove_keccak_chain(self, states: np.ndarray, domain: bytes, last=None) -> tuple:
        """(Keccak chain bundle bytes, check), as prove_chain."""
        states = np.ascontiguousarray(states, np.uint64).reshape(-1, 25)
        log2 = states.shape[0].bit_length() - 1
        buf = np.zeros(1 << 21, np.uint8)
        n = ctypes.c_size_t()
        chk = ctypes.c_int(-1)
        cl = None if last is None else _p(np.ascontiguousarray(last, np.uint64))
        rc = self.L.flockref_prove_keccak_chain(_p(states), log2, domain, len(domain), cl, _p(buf), buf.size,
                                                ctypes.byref(n), ctypes.byref(chk))
        assert rc == 0, rc
        return buf[: n.value].tobytes(), chk.value == 1

    def f128_mul(self, a, b):
        a = np.ascontiguousarray(a, np.uint64)
        b = np.ascontiguousarray(b, np.uint64)
        out = np.zeros_like(a)
        self.L.flockref_f128_mul_n(_p(a), _p(b), a.size // 2, _p(out))
        return out

    def phi8_table(self):
        out = np.zeros(512, np.uint64)
        self.L.flockref_phi8_table(_p(out))
        return out.reshape(256, 2)

    def blake3(self, data: bytes) -> bytes:
        out = ctypes.create_string_buffer(32)
        self.L.flockref_blake3_hash(data, len(data), out)
        return out.raw

    def xof(self, data: bytes, n: int) -> bytes:
        out = ctypes.create_string_buffer(n)
        self.L.flockref_blake3_xof(data, len(data), out, n)
        return out.raw

    def leaf_cv(self, data: bytes) -> bytes:
        out = ctypes.create_string_buffer(32)
        self.L.flockref_blake3_leaf_cv(data, len(data), out)
        return out.raw

    def parent_cv(self, l: bytes, r: bytes) -> bytes:
        out = ctypes.create_string_buffer(32)
        self.L.flockref_blake3_parent_cv(l, r, out)
        return out.raw

    def compressions(self, log2: int, seed: int) -> np.ndarray:
        out = np.zeros(25 << log2, np.uint32)
        self.L.flockref_generate_compressions(log2, seed, _p(out))
        return out.reshape(-1, 25)

    def witness(self, log2: int, seed: int):
        words = (1 << max(log2, 3)) * 128
        z, a, b = (np.zeros(2 * words, np.uint64) for _ in range(3))
        self.L.flockref_witness(log2, seed, _p(z), _p(a), _p(b))
        return z, a, b

    def apply_matrices(self, z: np.ndarray, n_blocks: int):
        a = np.zeros(n_blocks * 256, np.uint64)
        b = np.zeros(n_blocks * 256, np.uint64)
        self.L.flockref_apply_matrices(_p(np.ascontiguousarray(z[: n_blocks * 256])), n_blocks, _p(a), _p(b))
        return a, b

    def statement_digest(self, n_log: int) -> bytes:
        out = np.zeros(32, np.uint8)
        self.L.flockref_statement_digest(n_log, _p(out))
        return out.tobytes()

    def rs_encode(self, msg: np.ndarray, n_pos: int, lanes: int, rate: int) -> np.ndarray:
        msg = np.ascontiguousarray(msg, np.uint64)
        out = np.zeros(msg.size << rate, np.uint64)
        self.L.flockref_rs_encode(_p(msg), n_pos, lanes, rate, _p(out))
        return out

    def merkle_tree(self, data: np.ndarray, n_leaves: int, leaf_size: int) -> np.ndarray:
        data = np.ascontiguousarray(data, np.uint8)
        out = np.zeros((2 * n_leaves - 1) * 32, np.uint8)
        self.L.flockref_merkle_tree(_p(data), n_leaves, leaf_size, _p(out))
        return out

    def build_eq(self, r: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(r, np.uint64)
        n = r.size // 2
        out = np.zeros(2 << n, np.uint64)
        self.L.flockref_build_eq(_p(r), n, _p(out))
        return out

    def lagrange(self, z: np.ndarray, node_base: int) -> np.ndarray:
        z = np.ascontiguousarray(z, np.uint64)
        out = np.zeros(128, np.uint64)
        self.L.flockref_lagrange(_p(z), node_base, _p(out))
        return out

    def grind(self, domain: bytes, label: bytes, bits: int, hash: str = "blake3") -> tuple:
        c = self.L.flockref_ch_new_hash(domain, {"sha256": 0, "blake3": 1}[hash])
        self.L.flockref_ch_label(c, label)
        d = np.zeros(32, np.uint8)
        self.L.flockref_ch_digest(c, _p(d))
        n = self.L.flockref_ch_grind(c, bits)
        self.L.flockref_ch_free(c)
        return d.tobytes(), n

    def challenger_script(self, domain: bytes, hash: str) -> list:
        """The fixed op script of the transcript tests; returns every sample
        and the final state digest."""
        c = self.L.flockref_ch_new_hash(domain, {"sha256": 0, "blake3": 1}[hash])
        out = []
        self.L.flockref_ch_label(c, b"flock-test-label")
        v = np.array([0x0123456789ABCDEF, 0xFEDCBA9876543210], np.uint64)
        self.L.flockref_ch_observe(c, _p(v))
        s = np.arange(10, dtype=np.uint64)
        self.L.flockref_ch_observe_slice(c, _p(s), 5)
        self.L.flockref_ch_bytes(c, b"\x01\x02\x03", 3)
        one = np.zeros(2, np.uint64)
        self.L.flockref_ch_sample(c, _p(one))
        out.append(one.copy())
        vec = np.zeros(14, np.uint64)
        self.L.flockref_ch_sample_vec(c, 7, _p(vec))
        out.append(vec.copy())
        out.append(self.L.flockref_ch_grind(c, 5))
        d = np.zeros(32, np.uint8)
        self.L.flockref_ch_digest(c, _p(d))
        out.append(d.tobytes())
        self.L.flockref_ch_free(c)
        return out

    def time_prove(self, log2: int, seed: int) -> tuple:
        n = ctypes.c_size_t()
        s = self.L.flockref_time_prove(log2, seed, ctypes.byref(n))
        return s, n.value
