"""The SHA-256 hash option on the GPU: SHA-256 Merkle trees against the
oracle's, the SHA-256 proof of work searched on the device, and whole proofs
with the SHA-256 Merkle hash and / or the SHA-256 transcript (the reference's
defaults, PcsParams::default and FsChallenger::new) against the oracle's and
the committed digests, verified by the product verifier."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "default_hash_proofs.json").read_text())


@pytest.mark.parametrize("n,leaf_size", [(1 << 10, 16), (1 << 8, 48), (1 << 12, 128), (1 << 14, 1024)])
def test_sha256_merkle_tree_matches_oracle(gpu_ctx, oracle, n, leaf_size):
    data = np.random.default_rng(n + leaf_size).integers(0, 256, n * leaf_size, dtype=np.uint8)
    assert np.array_equal(gpu_ctx.merkle_tree(data, n, leaf_size, "sha256"),
                          oracle.merkle_tree_hash(data, n, leaf_size, "sha256"))


@pytest.mark.parametrize("bits", [9, 14])
def test_sha256_pow_on_device(gpu_ctx, oracle, bits):
    import flockgpu
    d, want = oracle.grind(b"flock-pow-test", b"grind", bits, "sha256")
    ch = flockgpu.Challenger(b"flock-pow-test", "sha256")
    ch.observe_label(b"grind")
    assert ch.state_digest() == d
    assert ch.grind_pow(gpu_ctx, bits) == want
    ch.close()


@pytest.mark.parametrize("merkle,transcript", [("sha256", "sha256"), ("sha256", "blake3"), ("blake3", "sha256")])
def test_blake3_statement_with_hash_options_matches_oracle(gpu_ctx, oracle, merkle, transcript):
    import flockgpu
    oracle.set_hash_kinds(merkle, transcript)
    try:
        want = oracle.prove(8, 0x777)
    finally:
        oracle.set_hash_kinds()
    p = flockgpu.Prover(gpu_ctx, 8, merkle_hash=merkle, transcript=transcript)
    try:
        got = p.prove_seed(0x777)
        assert got == want
        assert p.verify(got) == ""
    finally:
        p.close()
    gpu_ctx.set_transcript(transcript)
    try:
        assert gpu_ctx.verify(got) == ""
        gpu_ctx.set_transcript("sha256" if transcript == "blake3" else "blake3")
        assert gpu_ctx.verify(got) != ""
    finally:
        gpu_ctx.set_transcript("blake3")


def test_sha256_statement_with_default_hashes_matches_oracle(gpu_ctx, oracle):
    import flockgpu
    comps = flockgpu.sha256_bench_inputs(128, 9)
    oracle.set_hash_kinds("sha256", "sha256")
    try:
        want = oracle.prove_sha256(comps)
    finally:
        oracle.set_hash_kinds()
    p = flockgpu.Sha256Prover(gpu_ctx, 128, merkle_hash="sha256", transcript="sha256")
    try:
        got = p.prove(comps)
        assert got == want
        assert p.verify(got) == ""
    finally:
        p.close()


@pytest.mark.parametrize("e", GOLDEN, ids=lambda e: f'{e["statement"]}-{e.get("n", e.get("log2"))}-'
                                                    f'{e["merkle_hash"]}-{e["transcript"]}')
def test_default_hash_fixtures(gpu_ctx, e):
    import flockgpu
    if e["statement"] == "sha256":
        p = flockgpu.Sha256Prover(gpu_ctx, e["n"], merkle_hash=e["merkle_hash"], transcript=e["transcript"])
    else:
        p = flockgpu.Prover(gpu_ctx, e["log2"], merkle_hash=e["merkle_hash"], transcript=e["transcript"])
    try:
        got = p.prove_seed(e["seed"])
        assert hashlib.sha256(got).hexdigest() == e["sha256"] and len(got) == e["size"]
        assert p.verify(got) == ""
    finally:
        p.close()
