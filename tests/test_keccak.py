"""The Keccak-f[1600] statement on the CPU (crates/flock-prover/src/
r1cs_hashes/keccak.rs): the oracle's permutation against the SHA-3 standard
(hashlib's SHA3-256 and SHAKE128 of single-block messages), the product
library's host permutation and bench inputs against the oracle, the oracle's
row witness against the R1CS semantics (a & b = z, state_24 = keccak_f(state_0),
constant wire, zero padding; the reference's witness and roundtrip tests,
keccak.rs:1580-1770), its lincheck walker against the witness through random
parity checks (A z = a and B z = b, read through alpha A^T e + B^T e), the
statement digests, and the oracle's proofs against the committed fixtures."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "keccak_proofs.json"
GOLDEN3 = Path(__file__).resolve().parent / "golden" / "keccak3_proofs.json"


def _absorb(block: bytes) -> np.ndarray:
    """A zero state XOR a full-rate block (little-endian lanes)."""
    s = np.zeros(25, np.uint64)
    w = np.frombuffer(block + b"\0" * (200 - len(block)), "<u8")
    return s ^ w


def _sponge_one_block(keccak_f, msg: bytes, rate: int, pad: int, out_len: int) -> bytes:
    blk = bytearray(msg + bytes([pad]) + b"\0" * (rate - len(msg) - 1))
    blk[rate - 1] ^= 0x80
    return keccak_f(_absorb(bytes(blk))).astype("<u8").tobytes()[:out_len]


@pytest.mark.parametrize("msg", [b"", b"abc", b"flock keccak-f[1600]", bytes(range(100))])
def test_oracle_permutation_is_sha3(oracle, msg):
    assert _sponge_one_block(oracle.keccak_f, msg, 136, 0x06, 32) == hashlib.sha3_256(msg).digest()
    assert _sponge_one_block(oracle.keccak_f, msg, 168, 0x1F, 64) == hashlib.shake_128(msg).digest(64)


def test_zero_state_known_answer(oracle):
    """keccak_f of the zero state (the Keccak team's known answer, lane 0)."""
    assert int(oracle.keccak_f(np.zeros(25, np.uint64))[0]) == 0xF1258F7940E1DDE7


def test_product_host_permutation_matches_oracle(oracle):
    import flockgpu
    rng = np.random.default_rng(11)
    for _ in range(16):
        s = rng.integers(0, 2**63, 25, np.uint64) ^ (rng.integers(0, 2, 25, np.uint64) << np.uint64(63))
        assert np.array_equal(flockgpu.keccak_f(s), oracle.keccak_f(s))
    assert _sponge_one_block(flockgpu.keccak_f, b"abc", 136, 0x06, 32) == hashlib.sha3_256(b"abc").digest()


def test_bench_inputs_match(oracle):
    import flockgpu
    for n, seed in ((8, 1), (100, flockgpu.keccak_bench_seed(100))):
        assert np.array_equal(flockgpu.keccak_bench_inputs(n, seed), oracle.keccak_bench_inputs(n, seed))


def _bits(v):
    return np.unpackbits(np.ascontiguousarray(v).view(np.uint8), axis=-1, bitorder="little")


def test_witness_rows(oracle):
    """a & b == z in every row; state_0 and state_24 (words 0..24 and 32..56)
    are the input and keccak_f of it with b = 1; the constant word 64 is 1;
    t_r fills words 65..664 and everything after is zero; padding blocks hold
    keccak_f of the zero state."""
    n_log, n = 3, 5
    st = oracle.keccak_bench_inputs(n, 21)
    z, a, b = oracle.keccak_witness(st, n_log)
    assert np.array_equal(a & b, z)
    ones = np.full(25, 2**64 - 1, np.uint64)
    for i in range(1 << n_log):
        s0 = st[i] if i < n else np.zeros(25, np.uint64)
        assert np.array_equal(z[i, :25], s0) and np.array_equal(a[i, :25], s0) and np.array_equal(b[i, :25], ones)
        s24 = oracle.keccak_f(s0)
        assert np.array_equal(z[i, 32:57], s24) and np.array_equal(b[i, 32:57], ones)
        assert z[i, 64] == a[i, 64] == b[i, 64] == 1
        assert not z[i, 25:32].any() and not z[i, 57:64].any()
        assert not (z[i, 665:].any() or a[i, 665:].any() or b[i, 665:].any())


def _parity_checks(oracle, z, a, b, seed):
    """<e, a> == <A^T e, z> and <e, b> == <B^T e, z> for 128 random 0/1
    vectors e at once (bit k of each F128 of e is vector k)."""
    rng = np.random.default_rng(seed)
    e = rng.integers(0, 2**63, (1 << 16, 2), np.uint64) ^ (rng.integers(0, 2, (1 << 16, 2), np.uint64)
                                                          << np.uint64(63))
    bt = oracle.keccak_comb((0, 0), e)        # alpha = 0: B^T e
    at = oracle.keccak_comb((1, 0), e) ^ bt    # alpha = 1: (A + B)^T e
    zb, ab, bb = _bits(z).astype(bool), _bits(a).astype(bool), _bits(b).astype(bool)
    ok_a = np.array_equal(np.bitwise_xor.reduce(e[ab], axis=0), np.bitwise_xor.reduce(at[zb], axis=0))
    ok_b = np.array_equal(np.bitwise_xor.reduce(e[bb], axis=0), np.bitwise_xor.reduce(bt[zb], axis=0))
    return ok_a and ok_b


def test_walker_matches_witness(oracle):
    """The lincheck walker (KeccakLincheckCircuit::fold_alpha_batched,
    keccak.rs:681-848) applies the matrices the witness satisfies: 128 random
    parity checks of A z = a and B z = b per block, for bench states, the
    zero state and the all-ones state."""
    states = np.concatenate([oracle.keccak_bench_inputs(2, 4), np.zeros((1, 25), np.uint64),
                             np.full((1, 25), 2**64 - 1, np.uint64)])
    z, a, b = oracle.keccak_witness(states, 3)
    for i in range(4):
        assert _parity_checks(oracle, z[i], a[i], b[i], 100 + i), i


def test_tampered_witness_fails_the_walker(oracle):
    """A flipped bit of z in state_0 or a t_r row breaks A z = a or B z = b
    (the walker reads every column those rows feed); a flipped state_24 bit
    keeps A z = a (its pin row's A side is the recurrence, its z column is
    read only through C = I) and breaks (A z)(B z) = z instead."""
    z, a, b = oracle.keccak_witness(oracle.keccak_bench_inputs(1, 8), 3)
    for bit in (3, 64 * 7 + 9, 4160 + 1600 * 11 + 100, 4160 + 1600 * 23 + 1599):
        zz = z[0].copy()
        zz[bit // 64] ^= np.uint64(1) << np.uint64(bit % 64)
        assert not _parity_checks(oracle, zz, a[0], b[0], 7), bit
    bit = 2048 + 64 * 24 + 63
    zz = z[0].copy()
    zz[bit // 64] ^= np.uint64(1) << np.uint64(bit % 64)
    assert _parity_checks(oracle, zz, a[0], b[0], 7) and not np.array_equal(a[0] & b[0], zz)


def test_product_statement_digest_matches_oracle(oracle):
    import flockgpu
    for m in (22, 24, 29, 34):
        assert flockgpu.keccak_statement_digest(m) == oracle.keccak_digest(m - 16)
    assert flockgpu.keccak_statement_digest(24) != flockgpu.sha256_statement_digest(24)
    assert flockgpu.keccak_statement_digest(24) != oracle.statement_digest(10)


def test_fixture_digests():
    import flockgpu
    g = json.loads(GOLDEN.read_text())
    for m, d in g["digests"].items():
        assert flockgpu.keccak_statement_digest(int(m)) == bytes.fromhex(d), m


def test_oracle_proof_matches_fixture(oracle):
    g = json.loads(GOLDEN.read_text())
    e = next(p for p in g["proofs"] if p["n"] == 64)
    proof = oracle.prove_keccak(oracle.keccak_bench_inputs(e["n"], e["seed"]))
    assert hashlib.sha256(proof).hexdigest() == e["sha256"] and len(proof) == e["size"]


# ---- the 3-wide encoder (keccak3.rs): three permutations per 2^17-bit block

def test_wide_witness_rows(oracle):
    """keccak3.rs:151-300: sub-keccak s of block i holds input 3 i + s
    (missing ones and padding blocks: the zero state) with state_0 in words
    64 s..64 s + 24 and state_24 in 64 s + 32..; the shared constant is word
    192; t fills words 193..1992 and the tail is zero; a & b = z."""
    n_log, n = 3, 8  # the last block holds two inputs and one zero state
    st = oracle.keccak_bench_inputs(n, 33)
    z, a, b = oracle.keccak_witness(st, n_log, width=3)
    assert z.shape == (8, 2048) and np.array_equal(a & b, z)
    ones = np.full(25, 2**64 - 1, np.uint64)
    for i in range(1 << n_log):
        for s in range(3):
            k = 3 * i + s
            s0 = st[k] if k < n else np.zeros(25, np.uint64)
            assert np.array_equal(z[i, 64 * s:64 * s + 25], s0) and np.array_equal(b[i, 64 * s:64 * s + 25], ones)
            assert np.array_equal(z[i, 64 * s + 32:64 * s + 57], oracle.keccak_f(s0))
            assert not z[i, 64 * s + 25:64 * s + 32].any() and not z[i, 64 * s + 57:64 * s + 64].any()
        assert z[i, 192] == a[i, 192] == b[i, 192] == 1
        assert not (z[i, 1993:].any() or a[i, 1993:].any() or b[i, 1993:].any())


def _parity_checks_wide(oracle, z, a, b, seed):
    rng = np.random.default_rng(seed)
    e = rng.integers(0, 2**63, (1 << 17, 2), np.uint64) ^ (rng.integers(0, 2, (1 << 17, 2), np.uint64)
                                                          << np.uint64(63))
    bt = oracle.keccak_comb((0, 0), e, width=3)
    at = oracle.keccak_comb((1, 0), e, width=3) ^ bt
    zb, ab, bb = _bits(z).astype(bool), _bits(a).astype(bool), _bits(b).astype(bool)
    ok_a = np.array_equal(np.bitwise_xor.reduce(e[ab], axis=0), np.bitwise_xor.reduce(at[zb], axis=0))
    ok_b = np.array_equal(np.bitwise_xor.reduce(e[bb], axis=0), np.bitwise_xor.reduce(bt[zb], axis=0))
    return ok_a and ok_b


def test_wide_walker_matches_witness(oracle):
    """keccak3.rs:430-490: three copies of the recurrence into one comb apply
    the matrices the 3-wide witness satisfies; a flipped t bit of the third
    sub-keccak breaks them."""
    z, a, b = oracle.keccak_witness(oracle.keccak_bench_inputs(5, 9), 3, width=3)
    for i in (0, 1, 2):
        assert _parity_checks_wide(oracle, z[i], a[i], b[i], 200 + i), i
    bit = 12352 + 1600 * (2 * 24 + 7) + 333
    zz = z[0].copy()
    zz[bit // 64] ^= np.uint64(1) << np.uint64(bit % 64)
    assert not _parity_checks_wide(oracle, zz, a[0], b[0], 5)


def test_wide_statement_digest_matches_oracle(oracle):
    import flockgpu
    for m in (22, 25, 34):
        assert flockgpu.keccak_statement_digest(m, width=3) == oracle.keccak_digest(m - 17, width=3)
    assert flockgpu.keccak_statement_digest(25, width=3) != flockgpu.keccak_statement_digest(25)


def test_wide_fixtures(oracle):
    import flockgpu
    g = json.loads(GOLDEN3.read_text())
    for m, d in g["digests"].items():
        assert flockgpu.keccak_statement_digest(int(m), width=3) == bytes.fromhex(d), m
    e = next(p for p in g["proofs"] if p["n"] == 49)
    proof = oracle.prove_keccak(oracle.keccak_bench_inputs(e["n"], e["seed"]), width=3)
    assert hashlib.sha256(proof).hexdigest() == e["sha256"] and len(proof) == e["size"]


# ---- Keccak hash chains (keccak.rs:1000-1060 over chain_common.rs)
CHAIN_GOLDEN = Path(__file__).resolve().parent / "golden" / "keccak_chain_proofs.json"


def test_chain_states_match_oracle(oracle):
    import flockgpu
    assert np.array_equal(flockgpu.keccak_chain_states(20), oracle.keccak_chain_states(20))
    s0 = oracle.keccak_bench_inputs(1, 3)[0]
    assert np.array_equal(flockgpu.keccak_chain_states(5, s0), oracle.keccak_chain_states(5, s0))


def test_oracle_chain_checks(oracle):
    """An honest chain verifies from its public endpoints; a broken link or a
    wrong endpoint does not; the bundle names HashKind::Keccak and carries
    1600-bit endpoints."""
    st = oracle.keccak_chain_states(64)
    proof, ok = oracle.prove_keccak_chain(st, b"flock_chain-cli")
    assert ok and proof[7:11] == b"\x02\x00\x00\x00"
    assert proof[-1608:-1600] == (1600).to_bytes(8, "little")
    bad = st.copy()
    bad[33, 7] ^= np.uint64(1 << 40)
    assert not oracle.prove_keccak_chain(bad, b"flock_chain-cli")[1]
    assert not oracle.prove_keccak_chain(st, b"flock_chain-cli", last=st[9])[1]


def test_oracle_chain_matches_fixture(oracle):
    g = json.loads(CHAIN_GOLDEN.read_text())
    e = next(p for p in g["proofs"] if p["n"] == 64)
    proof, ok = oracle.prove_keccak_chain(oracle.keccak_chain_states(64), b"flock_chain-cli")
    assert ok and hashlib.sha256(proof).hexdigest() == e["sha256"] and len(proof) == e["size"]
