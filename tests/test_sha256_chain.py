"""SHA-256 hash chains (crates/flock-prover/src/r1cs_hashes/sha2.rs:1557-1620,
Sha256HybridSetup::prove_chain / verify_chain over chain_common.rs with the
SHA-256 CHAIN_LAYOUT, :1476-1483) on the CPU: the product's honest-chain
generator against the oracle's and against the compression, and the oracle's
chain prover checked by its own verification of the shift argument from the
public endpoints (the reference's chain tests: an honest chain verifies, a
broken link or a wrong endpoint does not), against the committed fixtures."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "sha256_chain_proofs.json").read_text())
DOMAIN = b"flock_chain-cli"


def test_chain_blocks_match_oracle_and_link(oracle):
    import flockgpu
    for seed, steps in ((1, 16), (7, 300)):
        got = flockgpu.sha256_chain_blocks(seed, steps)
        assert np.array_equal(got, oracle.sha256_chain_blocks(seed, steps))
        for i in range(steps - 1):
            assert np.array_equal(flockgpu.sha256_compress(got[i, :8], got[i, 8:]), got[i + 1, :8])
    iv = np.array([0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a, 0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19],
                  np.uint32)
    assert np.array_equal(flockgpu.sha256_chain_blocks(3, 1)[0, :8], iv)
    h0 = np.arange(8, dtype=np.uint32)
    assert np.array_equal(flockgpu.sha256_chain_blocks(3, 2, h0)[0, :8], h0)


def test_oracle_chain_checks(oracle):
    records = oracle.sha256_chain_blocks(5, 128)
    proof, ok = oracle.prove_sha256_chain(records, DOMAIN)
    assert ok
    broken = records.copy()
    broken[77, 12] ^= 1  # a message word: link 77 -> 78 no longer holds
    assert not oracle.prove_sha256_chain(broken, DOMAIN)[1]
    assert not oracle.prove_sha256_chain(records, DOMAIN, cv_last=records[3, :8])[1]
    # the bundle names its hash: HashKind::Sha2 after the 7-byte header
    assert proof[:7] == b"FLOCK\x04\x03" and proof[7:11] == b"\x01\x00\x00\x00"


def test_oracle_chain_matches_fixture(oracle):
    e = next(p for p in GOLDEN["proofs"] if p["n"] == 128)
    proof, ok = oracle.prove_sha256_chain(oracle.sha256_chain_blocks(e["seed"], e["n"]), DOMAIN)
    assert ok and hashlib.sha256(proof).hexdigest() == e["sha256"] and len(proof) == e["size"]
