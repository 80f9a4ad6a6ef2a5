"""The BLAKE3 hash-chain statement (Blake3Setup::prove_chain,
crates/flock-prover/src/r1cs_hashes/blake3.rs:5195-5240): 2^n compressions
whose input cv is the previous one's output, proved with the compression
proof's core, a region fold, the shift sumcheck (chain.rs) and one batched
open that adds a packed-direct claim.

The reference's trusted verifier checks only the compression statement, so
the chain is pinned by (i) the oracle's own checks on every proof: the shift
argument verified from the public endpoints on a copy of the transcript
(chain.rs:238-300) and the batched open's claim identity, mirroring the
reference's tests chain_prove_verify_ligerito_roundtrip,
chain_wrong_endpoint_rejects and chain_broken_link_rejects
(blake3.rs:7108-7165); (ii) the compression proof's pins for everything the
two statements share; (iii) bit-identity of the GPU bundle with the oracle,
live at small sizes and through committed digests at 2^14..2^18.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import proofparse

GOLD = Path(__file__).resolve().parent / "golden"
DOMAIN = b"flock_chain-cli"
IV = [0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A, 0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19]


def cv_bits(cv) -> bytes:
    return bytes((int(cv[i // 32]) >> (i % 32)) & 1 for i in range(256))


# ---------------------------------------------------------------- CPU --
def test_oracle_chain_verifies(oracle):
    n = 1 << 8
    recs = oracle.chain_blocks(11, n + 1)  # one more link: its cv is the chain's output
    data, ok = oracle.prove_chain(recs[:n], DOMAIN)
    assert ok
    p = proofparse.parse(data)
    assert p["flavor"] == 3 and p["hash_kind"] == 0 and p["version"] == 4
    assert len(p["shift_rounds"]) == 8 + 1
    assert p["cv0_bits"] == cv_bits(IV)
    assert p["cv_last_bits"] == cv_bits(recs[n, :8])
    assert len(p["s_hat_v"]) == 2
    # the generator's records: counter 0, block_len 64, flags 0, linked cvs
    assert (recs[:, 24:26] == 0).all() and (recs[:, 26] == 64).all() and (recs[:, 27] == 0).all()


def test_oracle_chain_broken_link_rejects(oracle):
    recs = oracle.chain_blocks(12, 1 << 8)
    recs[2, 0] ^= 1  # instance 2's input cv no longer equals instance 1's output
    _, ok = oracle.prove_chain(recs, DOMAIN)
    assert not ok


def test_oracle_chain_wrong_endpoint_rejects(oracle):
    n = 1 << 8
    recs = oracle.chain_blocks(13, n + 1)
    bad = recs[n, :8].copy()
    bad[0] ^= 1
    data, ok = oracle.prove_chain(recs[:n], DOMAIN, cv_last=bad)
    assert not ok
    assert proofparse.parse(data)["cv_last_bits"] == cv_bits(bad)
    _, ok = oracle.prove_chain(recs[:n], DOMAIN, cv_last=recs[n, :8])
    assert ok


def test_oracle_chain_custom_initial_cv(oracle):
    cv = np.arange(1, 9, dtype=np.uint32) * np.uint32(0x01010101)
    recs = oracle.chain_blocks(14, 1 << 8, initial_cv=cv)
    assert (recs[0, :8] == cv).all()
    data, ok = oracle.prove_chain(recs, DOMAIN)
    assert ok and proofparse.parse(data)["cv0_bits"] == cv_bits(cv)


def test_chain_blocks_host_matches_oracle(oracle):
    """The product's host chain builder (flock_chain_blocks) and the oracle's."""
    import flockgpu
    for seed, cv in ((0, None), (99, np.full(8, 0xDEADBEEF, np.uint32))):
        assert np.array_equal(flockgpu.chain_blocks(seed, 300, cv), oracle.chain_blocks(seed, 300, cv))


def test_chain_golden_entries_were_checked():
    rows = json.loads((GOLD / "chain_proofs.json").read_text())
    assert sorted(r["log2"] for r in rows) == [14, 16, 18]
    assert all("shift argument verified" in r["checked_by"] for r in rows)


# ---------------------------------------------------------------- GPU --
@pytest.mark.gpu
@pytest.mark.parametrize("log2,seed", [(8, 1), (9, 2), (10, 3)])
def test_chain_gpu_matches_oracle(gpu_ctx, oracle, log2, seed):
    import flockgpu
    recs = flockgpu.chain_blocks(seed, 1 << log2)
    want, ok = oracle.prove_chain(recs, DOMAIN)
    assert ok
    p = flockgpu.Prover(gpu_ctx, log2)
    try:
        got = p.prove_chain(recs, DOMAIN)
    finally:
        p.close()
    assert got == want, proofparse.first_difference(got, want)


@pytest.mark.gpu
def test_chain_gpu_broken_chain_matches_oracle(gpu_ctx, oracle):
    """A broken chain still gets the honest prover's bytes (which the
    verifier rejects); a custom initial cv and a non-default domain too."""
    import flockgpu
    recs = flockgpu.chain_blocks(21, 1 << 8, np.full(8, 7, np.uint32))
    recs[5, 3] ^= 0x80000000
    want, ok = oracle.prove_chain(recs, b"another-domain")
    assert not ok
    p = flockgpu.Prover(gpu_ctx, 8)
    try:
        assert p.prove_chain(recs, b"another-domain") == want
    finally:
        p.close()


@pytest.mark.gpu
def test_chain_then_compression_on_one_setup(gpu_ctx, oracle):
    """A setup proves chains and compressions in any order: the chain's use of
    the fold buffers leaves nothing behind."""
    import flockgpu
    p = flockgpu.Prover(gpu_ctx, 8)
    try:
        recs = flockgpu.chain_blocks(3, 1 << 8)
        first = p.prove_chain(recs, DOMAIN)
        assert p.prove_seed(5) == oracle.prove(8, 5)
        assert p.prove_chain(recs, DOMAIN) == first
    finally:
        p.close()


@pytest.mark.gpu
@pytest.mark.parametrize("log2", [14, 16, 18])
def test_chain_golden_full_size(gpu_ctx, log2):
    import flockgpu
    rows = [r for r in json.loads((GOLD / "chain_proofs.json").read_text()) if r["log2"] == log2]
    assert rows
    p = flockgpu.Prover(gpu_ctx, log2)
    try:
        for r in rows:
            proof = p.prove_chain(flockgpu.chain_blocks(r["seed"], 1 << log2), r["domain"].encode())
            assert len(proof) == r["size"] and hashlib.sha256(proof).hexdigest() == r["sha256"]
    finally:
        p.close()


@pytest.mark.gpu
def test_chain_rejects_partial_chain(gpu_ctx):
    import flockgpu
    p = flockgpu.Prover(gpu_ctx, 8)
    try:
        with pytest.raises(flockgpu.FlockError):
            p.prove_chain(flockgpu.chain_blocks(1, 200), DOMAIN)
    finally:
        p.close()
