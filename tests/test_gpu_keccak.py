"""The Keccak-f[1600] statement on the GPU (crates/flock-prover/src/
r1cs_hashes/keccak.rs, KeccakSetup::prove_fast / verify): the device witness
kernel and the device lincheck walker against the oracle's, proof bytes
against the oracle's at small sizes and against the committed oracle digests
up to 2^14 permutations, verification (the reference's prove_fast_roundtrip,
keccak.rs:1668-1690) and its rejections, and a full-size proof."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "keccak_proofs.json").read_text())


@pytest.mark.parametrize("n,n_log", [(8, 3), (5, 3), (0, 3), (40, 6)])
def test_witness_matches_oracle(gpu_ctx, oracle, n, n_log):
    rng = np.random.default_rng(n + 23)
    states = rng.integers(0, 2**63, (n, 25), dtype=np.uint64) ^ (rng.integers(0, 2, (n, 25), np.uint64)
                                                                 << np.uint64(63))
    want = oracle.keccak_witness(states, n_log)
    got = gpu_ctx.keccak_witness(states, n_log)
    for name, g, w in zip("zab", got, want):
        assert np.array_equal(g, w), name


def _rand_f128(rng, shape):
    return rng.integers(0, 2**63, shape + (2,), np.uint64) ^ (rng.integers(0, 2, shape + (2,), np.uint64)
                                                             << np.uint64(63))


def test_walker_matches_oracle(gpu_ctx, oracle):
    """comb = alpha A^T e + B^T e + beta [const] on the GPU equals the
    oracle's walker plus beta at the constant column (lincheck.rs:5446 adds
    the pin), for random e, alpha, beta and for alpha = 0, 1."""
    rng = np.random.default_rng(31)
    for alpha in [tuple(_rand_f128(rng, ())), (0, 0), (1, 0)]:
        e = _rand_f128(rng, (1 << 16,))
        beta = _rand_f128(rng, ())
        want = oracle.keccak_comb(alpha, e)
        want[4096] ^= beta
        got = gpu_ctx.keccak_comb(e, alpha, beta)
        assert np.array_equal(got, want), alpha


def test_prove_matches_oracle(gpu_ctx, oracle):
    """n = 64 (m = 22) and n = 100 (128 slots, 28 padding blocks)."""
    import flockgpu
    for n in (64, 100):
        states = flockgpu.keccak_bench_inputs(n, flockgpu.keccak_bench_seed(n))
        p = flockgpu.KeccakProver(gpu_ctx, n)
        try:
            got = p.prove(states)
            assert got == oracle.prove_keccak(states), n
            assert p.verify(got) == ""
        finally:
            p.close()


def test_prove_seed_equals_prove_of_host_inputs(gpu_ctx):
    import flockgpu
    n = 300
    seed = flockgpu.keccak_bench_seed(n)
    p = flockgpu.KeccakProver(gpu_ctx, n)
    try:
        assert p.prove_seed(seed) == p.prove(flockgpu.keccak_bench_inputs(n, seed))
    finally:
        p.close()


@pytest.mark.parametrize("entry", GOLDEN["proofs"], ids=lambda e: str(e["n"]))
def test_sizes_match_oracle_fixture(gpu_ctx, entry):
    import flockgpu
    p = flockgpu.KeccakProver(gpu_ctx, entry["n"])
    try:
        got = p.prove_seed(entry["seed"])
        assert hashlib.sha256(got).hexdigest() == entry["sha256"] and len(got) == entry["size"]
        assert gpu_ctx.keccak_verify(got) == ""
    finally:
        p.close()


def test_verify_rejects(gpu_ctx):
    import flockgpu
    n = 128
    p = flockgpu.KeccakProver(gpu_ctx, n)
    try:
        good = p.prove_seed(7)
        assert gpu_ctx.keccak_verify(good) == ""
        # the SHA-256 statement of the same m (2^8 compressions) is another statement
        assert gpu_ctx.sha256_verify(good) != ""
        assert p.verify(good, domain=b"other-domain") != ""
        for off in (200, len(good) // 2, len(good) - 100):
            bad = bytearray(good)
            bad[off] ^= 1
            assert gpu_ctx.keccak_verify(bytes(bad)) != "", off
    finally:
        p.close()


def test_large_proof_verifies(gpu_ctx):
    """2^16 permutations (m = 32, the BLAKE3 benchmark's statement size):
    prove, verify, and a second proof of the same inputs is byte-identical."""
    import flockgpu
    n = 1 << 16
    p = flockgpu.KeccakProver(gpu_ctx, n)
    try:
        a = p.prove_seed(flockgpu.keccak_bench_seed(n))
        assert p.verify(a) == ""
        assert p.prove_seed(flockgpu.keccak_bench_seed(n)) == a
    finally:
        p.close()


def test_other_entry_points_refuse_a_keccak_setup(gpu_ctx):
    import ctypes
    import flockgpu
    p = flockgpu.KeccakProver(gpu_ctx, 64)
    try:
        blocks = np.zeros((64, 25), np.uint32)
        n = ctypes.c_size_t()
        rc = gpu_ctx.lib.flock_prove_blocks(p.h, flockgpu._ptr(blocks), 64, b"d", 1, flockgpu._ptr(p._buf),
                                            p._buf.size, ctypes.byref(n))
        assert rc == 1 and "Keccak" in gpu_ctx.lib.flock_last_error(gpu_ctx.h).decode()
        comps = np.zeros((64, 24), np.uint32)
        rc = gpu_ctx.lib.flock_sha256_prove(p.h, flockgpu._ptr(comps), 64, b"d", 1, flockgpu._ptr(p._buf),
                                            p._buf.size, ctypes.byref(n))
        assert rc == 1
    finally:
        p.close()


# ---- the 3-wide encoder (keccak3.rs): three permutations per 2^17-bit block
GOLDEN3 = json.loads((Path(__file__).resolve().parent / "golden" / "keccak3_proofs.json").read_text())


@pytest.mark.parametrize("n,n_log", [(24, 3), (8, 3), (0, 3), (100, 6)])
def test_wide_witness_matches_oracle(gpu_ctx, oracle, n, n_log):
    rng = np.random.default_rng(n + 41)
    states = rng.integers(0, 2**63, (n, 25), dtype=np.uint64) ^ (rng.integers(0, 2, (n, 25), np.uint64)
                                                                 << np.uint64(63))
    want = oracle.keccak_witness(states, n_log, width=3)
    got = gpu_ctx.keccak_witness(states, n_log, width=3)
    for name, g, w in zip("zab", got, want):
        assert np.array_equal(g, w), name


def test_wide_walker_matches_oracle(gpu_ctx, oracle):
    rng = np.random.default_rng(43)
    for alpha in [tuple(_rand_f128(rng, ())), (0, 0), (1, 0)]:
        e = _rand_f128(rng, (1 << 17,))
        beta = _rand_f128(rng, ())
        want = oracle.keccak_comb(alpha, e, width=3)
        want[12288] ^= beta
        got = gpu_ctx.keccak_comb(e, alpha, beta, width=3)
        assert np.array_equal(got, want), alpha


def test_wide_prove_matches_oracle(gpu_ctx, oracle):
    """n = 49 (17 blocks: 32 slots, m = 22) and n = 100 (the last block holds
    one permutation and two zero states)."""
    import flockgpu
    for n in (49, 100):
        states = flockgpu.keccak_bench_inputs(n, flockgpu.keccak_bench_seed(n))
        p = flockgpu.KeccakProver(gpu_ctx, n, width=3)
        try:
            got = p.prove(states)
            assert got == oracle.prove_keccak(states, width=3), n
            assert p.verify(got) == ""
            assert p.prove_seed(flockgpu.keccak_bench_seed(n)) == got
        finally:
            p.close()


@pytest.mark.parametrize("entry", GOLDEN3["proofs"], ids=lambda e: str(e["n"]))
def test_wide_sizes_match_oracle_fixture(gpu_ctx, entry):
    import flockgpu
    p = flockgpu.KeccakProver(gpu_ctx, entry["n"], width=3)
    try:
        got = p.prove_seed(entry["seed"])
        assert hashlib.sha256(got).hexdigest() == entry["sha256"] and len(got) == entry["size"]
        assert gpu_ctx.keccak_verify(got, width=3) == ""
        # the single encoder's statement of another m is not this one
        assert gpu_ctx.keccak_verify(got) != ""
    finally:
        p.close()


def test_wide_large_proof_verifies(gpu_ctx):
    """3 * 2^15 permutations (m = 32): prove, verify, and a second proof of
    the same inputs is byte-identical; a flipped byte is rejected."""
    import flockgpu
    n = 3 << 15
    p = flockgpu.KeccakProver(gpu_ctx, n, width=3)
    try:
        a = p.prove_seed(flockgpu.keccak_bench_seed(n))
        assert p.verify(a) == ""
        assert p.prove_seed(flockgpu.keccak_bench_seed(n)) == a
        bad = bytearray(a)
        bad[len(bad) // 3] ^= 4
        assert gpu_ctx.keccak_verify(bytes(bad), width=3) != ""
    finally:
        p.close()


# ---- Keccak hash chains (keccak.rs:1000-1060)
CHAIN_GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "keccak_chain_proofs.json").read_text())


def test_chain_matches_oracle(gpu_ctx, oracle):
    import flockgpu
    for n, start in ((64, None), (128, flockgpu.keccak_bench_inputs(1, 5)[0])):
        states = flockgpu.keccak_chain_states(n, start)
        p = flockgpu.KeccakProver(gpu_ctx, n)
        try:
            got = p.prove_chain(states)
            want, ok = oracle.prove_keccak_chain(states, flockgpu.CHAIN_DOMAIN)
            assert ok and got == want, n
            assert p.verify(got, flockgpu.CHAIN_DOMAIN) == ""
            assert gpu_ctx.keccak_verify(got, flockgpu.CHAIN_DOMAIN) == ""
        finally:
            p.close()


@pytest.mark.parametrize("entry", CHAIN_GOLDEN["proofs"], ids=lambda e: str(e["n"]))
def test_chain_sizes_match_oracle_fixture(gpu_ctx, entry):
    import flockgpu
    p = flockgpu.KeccakProver(gpu_ctx, entry["n"])
    try:
        got = p.prove_chain(flockgpu.keccak_chain_states(entry["n"]))
        assert hashlib.sha256(got).hexdigest() == entry["sha256"] and len(got) == entry["size"]
        assert gpu_ctx.keccak_verify(got, flockgpu.CHAIN_DOMAIN) == ""
    finally:
        p.close()


def test_chain_verify_rejects(gpu_ctx):
    import flockgpu
    n = 64
    states = flockgpu.keccak_chain_states(n)
    p = flockgpu.KeccakProver(gpu_ctx, n)
    try:
        good = p.prove_chain(states)
        assert gpu_ctx.keccak_verify(good, b"another-domain") != ""
        bad = bytearray(good)
        bad[len(bad) // 2] ^= 1
        assert gpu_ctx.keccak_verify(bytes(bad), flockgpu.CHAIN_DOMAIN) != ""
        wrong = bytearray(good)
        wrong[-5] ^= 1  # a bit of the public end state
        assert gpu_ctx.keccak_verify(bytes(wrong), flockgpu.CHAIN_DOMAIN) != ""
        broken = states.copy()
        broken[20, 4] ^= np.uint64(2)
        assert gpu_ctx.keccak_verify(p.prove_chain(broken), flockgpu.CHAIN_DOMAIN) != ""
        # another statement's verifier
        assert gpu_ctx.sha256_verify(good, flockgpu.CHAIN_DOMAIN) != ""
    finally:
        p.close()
    w = flockgpu.KeccakProver(gpu_ctx, 3 * 64, width=3)
    try:
        with pytest.raises(flockgpu.FlockError):
            w.prove_chain(flockgpu.keccak_chain_states(3 * 64))
    finally:
        w.close()
