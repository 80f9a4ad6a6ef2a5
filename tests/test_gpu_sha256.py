"""The SHA-256 compression statement on the GPU (crates/flock-prover/src/
r1cs_hashes/sha2.rs, Sha256HybridSetup::prove_fast / verify): the device
witness kernel against the oracle's witness (z from the boolean witness,
a and b from the matrices), proof bytes against the oracle's at small sizes
and against the committed oracle digests at the bench's sizes, verification,
and the constant-wire pin (sha2.rs:2292 const_pin_all_zero_rejected)."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "sha256_proofs.json").read_text())


@pytest.mark.parametrize("n,n_log", [(8, 3), (5, 3), (0, 3), (40, 6)])
def test_witness_matches_oracle(gpu_ctx, oracle, n, n_log):
    rng = np.random.default_rng(n + 17)
    comps = rng.integers(0, 2**32, (n, 24), dtype=np.uint64).astype(np.uint32)
    want = oracle.sha256_witness(comps, n_log)
    got = gpu_ctx.sha256_witness(comps, n_log)
    for name, g, w in zip("zab", got, want):
        assert np.array_equal(g, w), name


def test_prove_matches_oracle(gpu_ctx, oracle):
    """n = 128 (m = 22) and n = 200 (256 slots, 56 padding blocks)."""
    import flockgpu
    for n in (128, 200):
        comps = flockgpu.sha256_bench_inputs(n, flockgpu.sha256_bench_seed(n))
        p = flockgpu.Sha256Prover(gpu_ctx, n)
        try:
            got = p.prove(comps)
            assert got == oracle.prove_sha256(comps), n
            assert p.verify(got) == ""
        finally:
            p.close()


def test_prove_seed_equals_prove_of_host_inputs(gpu_ctx):
    import flockgpu
    n = 300
    seed = flockgpu.sha256_bench_seed(n)
    p = flockgpu.Sha256Prover(gpu_ctx, n)
    try:
        assert p.prove_seed(seed) == p.prove(flockgpu.sha256_bench_inputs(n, seed))
    finally:
        p.close()


@pytest.mark.parametrize("entry", GOLDEN["proofs"], ids=lambda e: str(e["n"]))
def test_bench_sizes_match_oracle_fixture(gpu_ctx, entry):
    import flockgpu
    p = flockgpu.Sha256Prover(gpu_ctx, entry["n"])
    try:
        got = p.prove_seed(entry["seed"])
        assert hashlib.sha256(got).hexdigest() == entry["sha256"] and len(got) == entry["size"]
        assert gpu_ctx.sha256_verify(got) == ""
    finally:
        p.close()


def test_verify_rejects(gpu_ctx, oracle):
    import flockgpu
    n = 256
    p = flockgpu.Sha256Prover(gpu_ctx, n)
    try:
        good = p.prove_seed(7)
        assert gpu_ctx.sha256_verify(good) == ""
        # the BLAKE3 statement of the same m (2^9 compressions) is another statement
        assert gpu_ctx.verify(good) != ""
        # another transcript domain
        assert p.verify(good, domain=b"other-domain") != ""
        # a flipped byte in the zerocheck / lincheck / opening region
        for off in (200, len(good) // 2, len(good) - 100):
            bad = bytearray(good)
            bad[off] ^= 1
            assert gpu_ctx.sha256_verify(bytes(bad)) != "", off
    finally:
        p.close()
    # the all-zero witness satisfies every row except through the constant
    # wire, which the lincheck pins to 1 in every block
    zero = oracle.prove_sha256_zero(8)
    assert gpu_ctx.sha256_verify(zero) != ""


def test_large_proof_verifies(gpu_ctx):
    """2^19 compressions (m = 34, the largest ladder): prove, verify, and a
    second proof of the same inputs is byte-identical."""
    import flockgpu
    n = 1 << 19
    p = flockgpu.Sha256Prover(gpu_ctx, n)
    try:
        a = p.prove_seed(11)
        assert p.verify(a) == ""
        assert p.prove_seed(11) == a
    finally:
        p.close()


def test_blake3_entry_points_refuse_a_sha256_setup(gpu_ctx):
    import ctypes
    import flockgpu
    p = flockgpu.Sha256Prover(gpu_ctx, 128)
    try:
        blocks = np.zeros((128, 25), np.uint32)
        n = ctypes.c_size_t()
        rc = gpu_ctx.lib.flock_prove_blocks(p.h, flockgpu._ptr(blocks), 128, b"d", 1, flockgpu._ptr(p._buf),
                                            p._buf.size, ctypes.byref(n))
        assert rc == 1 and "SHA-256" in gpu_ctx.lib.flock_last_error(gpu_ctx.h).decode()
    finally:
        p.close()


# ---- SHA-256 hash chains (sha2.rs:1557-1620)
CHAIN_GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "sha256_chain_proofs.json").read_text())


def test_chain_matches_oracle(gpu_ctx, oracle):
    import flockgpu
    for n in (128, 256):
        records = flockgpu.sha256_chain_blocks(n + 1, n)
        p = flockgpu.Sha256Prover(gpu_ctx, n)
        try:
            got = p.prove_chain(records)
            want, ok = oracle.prove_sha256_chain(records, flockgpu.CHAIN_DOMAIN)
            assert ok and got == want, n
            assert p.verify(got, flockgpu.CHAIN_DOMAIN) == ""
            assert gpu_ctx.sha256_verify(got, flockgpu.CHAIN_DOMAIN) == ""
        finally:
            p.close()


@pytest.mark.parametrize("entry", CHAIN_GOLDEN["proofs"], ids=lambda e: str(e["n"]))
def test_chain_sizes_match_oracle_fixture(gpu_ctx, entry):
    import flockgpu
    p = flockgpu.Sha256Prover(gpu_ctx, entry["n"])
    try:
        got = p.prove_chain(flockgpu.sha256_chain_blocks(entry["seed"], entry["n"]))
        assert hashlib.sha256(got).hexdigest() == entry["sha256"] and len(got) == entry["size"]
        assert gpu_ctx.sha256_verify(got, flockgpu.CHAIN_DOMAIN) == ""
    finally:
        p.close()


def test_chain_verify_rejects(gpu_ctx):
    import flockgpu
    n = 128
    records = flockgpu.sha256_chain_blocks(9, n)
    p = flockgpu.Sha256Prover(gpu_ctx, n)
    try:
        good = p.prove_chain(records)
        # another domain, a flipped proof byte, the BLAKE3 statement
        assert gpu_ctx.sha256_verify(good, b"another-domain") != ""
        bad = bytearray(good)
        bad[len(bad) // 2] ^= 1
        assert gpu_ctx.sha256_verify(bytes(bad), flockgpu.CHAIN_DOMAIN) != ""
        assert gpu_ctx.verify(good, flockgpu.CHAIN_DOMAIN) != ""
        # a wrong public endpoint (the last 256 bools of the bundle are cv_last)
        wrong = bytearray(good)
        wrong[-1] ^= 1
        assert gpu_ctx.sha256_verify(bytes(wrong), flockgpu.CHAIN_DOMAIN) != ""
        # a broken chain: the prover runs, the verifier refuses the proof
        broken = records.copy()
        broken[40, 9] ^= 1
        assert gpu_ctx.sha256_verify(p.prove_chain(broken), flockgpu.CHAIN_DOMAIN) != ""
    finally:
        p.close()
