"""SHA-256 Merkle paths on the GPU (Sha256HybridSetup::prove_merkle_paths_
ligerito / verify_merkle_paths_ligerito, r1cs_hashes/sha2.rs:1662-1843):
proof bytes against the oracle's at small sizes and against the committed
oracle digests at the Merkle bench's sizes, verification from the public
leaves and root, and rejection of wrong public inputs."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "sha256_merkle_proofs.json").read_text())


@pytest.mark.parametrize("n_log,path_log", [(7, 0), (7, 2), (8, 8)])
def test_merkle_matches_oracle(gpu_ctx, oracle, n_log, path_log):
    import flockgpu
    comps, b, leaves, root = flockgpu.sha256_merkle_inputs(n_log, path_log, seed=31 + n_log)
    want, ok = oracle.prove_sha256_merkle(comps, b, leaves, root, path_log)
    assert ok
    p = flockgpu.Sha256Prover(gpu_ctx, 1 << n_log)
    try:
        got = p.prove_merkle(comps, b, path_log)
    finally:
        p.close()
    assert got == want
    assert gpu_ctx.sha256_merkle_verify(got, path_log, b, leaves, root) == ""


@pytest.mark.parametrize("entry", GOLDEN, ids=lambda e: f'{e["n_log"]}-{e["path_log"]}')
def test_merkle_bench_sizes_match_fixture(gpu_ctx, entry):
    import flockgpu
    comps, b, leaves, root = flockgpu.sha256_merkle_inputs(entry["n_log"], entry["path_log"], entry["seed"])
    p = flockgpu.Sha256Prover(gpu_ctx, 1 << entry["n_log"])
    try:
        got = p.prove_merkle(comps, b, entry["path_log"])
    finally:
        p.close()
    assert hashlib.sha256(got).hexdigest() == entry["sha256"] and len(got) == entry["size"]
    assert gpu_ctx.sha256_merkle_verify(got, entry["path_log"], b, leaves, root) == ""


def test_merkle_verify_rejects(gpu_ctx):
    import flockgpu
    comps, b, leaves, root = flockgpu.sha256_merkle_inputs(8, 1, seed=5)
    p = flockgpu.Sha256Prover(gpu_ctx, 256)
    try:
        good = p.prove_merkle(comps, b, 1)
        # the same inputs proved with a broken link do not verify
        bad_comps = comps.copy()
        bad_comps[7, 16 if b[7] else 8] ^= 1
        broken = p.prove_merkle(bad_comps, b, 1)
    finally:
        p.close()
    assert gpu_ctx.sha256_merkle_verify(good, 1, b, leaves, root) == ""
    assert gpu_ctx.sha256_merkle_verify(broken, 1, b, leaves, root) != ""
    bad_leaves = leaves.copy()
    bad_leaves[1, 3] ^= 1
    assert gpu_ctx.sha256_merkle_verify(good, 1, b, bad_leaves, root) != ""
    bad_root = root.copy()
    bad_root[7] ^= 1
    assert gpu_ctx.sha256_merkle_verify(good, 1, b, leaves, bad_root) != ""
    bad_b = b.copy()
    bad_b[200] ^= 1
    assert gpu_ctx.sha256_merkle_verify(good, 1, bad_b, leaves, root) != ""
    # another number of paths is another statement
    assert gpu_ctx.sha256_merkle_verify(good, 0, b, leaves[:1], root) != ""
    # not a compression bundle
    assert gpu_ctx.sha256_verify(good) != ""


def test_merkle_needs_a_full_power_of_two_setup(gpu_ctx):
    import flockgpu
    comps, b, _, _ = flockgpu.sha256_merkle_inputs(7, 0, seed=1)
    p = flockgpu.Sha256Prover(gpu_ctx, 100)
    try:
        with pytest.raises(flockgpu.FlockError):
            p.prove_merkle(comps[:100], b[:100], 0)
    finally:
        p.close()
