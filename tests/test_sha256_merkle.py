"""SHA-256 Merkle paths on the CPU (crates/flock-prover/src/merkle_path.rs,
r1cs_hashes/merkle_path_common.rs, Sha256HybridSetup::prove_merkle_paths_
ligerito): the honest-input generator of the product library against the
oracle's and against SHA-256 itself, and the oracle's prover, whose shift
argument is verified from the public leaves and root (the reference's
honest_roundtrip_accepts / broken_chain_rejects / wrong_leaf_rejects /
wrong_root_rejects tests, merkle_path.rs:640-740) and whose proofs match the
committed fixtures."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "sha256_merkle_proofs.json"


@pytest.mark.parametrize("n_log,path_log", [(7, 0), (8, 2), (9, 9)])
def test_inputs_match_oracle_and_link(oracle, n_log, path_log):
    import flockgpu
    seed = 0xD15EA5E ^ (1 << n_log)
    got = flockgpu.sha256_merkle_inputs(n_log, path_log)
    want = oracle.sha256_merkle_inputs(n_log, path_log, seed)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    comps, b, leaves, root = got
    L = 1 << (n_log - path_log)
    for p in range(1 << path_log):
        cur = leaves[p]
        for i in range(p * L, (p + 1) * L):
            c = comps[i]
            sel = c[16:24] if (b[i] and i % L) else c[8:16]
            assert np.array_equal(sel, cur), i
            cur = oracle.sha256_compress(c[:8], c[8:])
        assert np.array_equal(cur, root)


@pytest.mark.parametrize("path_log", [0, 2])
def test_oracle_honest_paths_verify(oracle, path_log):
    comps, b, leaves, root = oracle.sha256_merkle_inputs(7, path_log, 0xC0FFEE)
    _, ok = oracle.prove_sha256_merkle(comps, b, leaves, root, path_log)
    assert ok


@pytest.mark.parametrize("tamper", ["leaf", "root", "link", "bit"])
def test_oracle_rejects(oracle, tamper):
    comps, b, leaves, root = oracle.sha256_merkle_inputs(7, 0, 0xBAD)
    comps, b, leaves, root = comps.copy(), b.copy(), leaves.copy(), root.copy()
    if tamper == "leaf":
        leaves[0, 0] ^= 1
    elif tamper == "root":
        root[0] ^= 1
    elif tamper == "link":  # the selected half of hash 5 no longer holds hash 4's output
        comps[5, 16 if b[5] else 8] ^= 1
    else:  # a selector bit flipped
        b[9] ^= 1
    _, ok = oracle.prove_sha256_merkle(comps, b, leaves, root, 0)
    assert not ok


def test_oracle_proof_matches_fixture(oracle):
    for e in json.loads(GOLDEN.read_text()):
        if e["n_log"] > 8:
            continue  # the larger ones are checked against the GPU
        comps, b, leaves, root = oracle.sha256_merkle_inputs(e["n_log"], e["path_log"], e["seed"])
        data, ok = oracle.prove_sha256_merkle(comps, b, leaves, root, e["path_log"])
        assert ok and hashlib.sha256(data).hexdigest() == e["sha256"] and len(data) == e["size"]
