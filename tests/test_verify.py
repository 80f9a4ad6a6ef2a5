"""The verifier behind flock_verify (Blake3Setup::verify / verify_chain,
crates/flock-core/src/verifier.rs:95-232, r1cs_hashes/chain_common.rs:355-420),
used for self-checking served proofs.

It is pinned by the reference's trusted verifier's judgments on the same
bytes: it accepts every proof that verifier accepted (the golden proofs,
reproduced bit for bit by the GPU prover), and rejects what no verifier may
accept (flipped bits, another transcript domain, another statement size, a
broken chain) -- the reference's tamper tests (verifier_roundtrip.rs, and
blake3.rs:7125-7165 for chains).
"""
import hashlib
import json
import time
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
CHAIN_DOMAIN = b"flock_chain-cli"


@pytest.fixture(scope="module")
def p8(gpu_ctx):
    import flockgpu
    p = flockgpu.Prover(gpu_ctx, 8)
    yield p
    p.close()


def test_accepts_verifier_accepted_goldens(gpu_ctx):
    import flockgpu
    rows = json.loads((GOLD / "verified_proofs.json").read_text())
    for log2 in sorted({r["log2"] for r in rows}):
        p = flockgpu.Prover(gpu_ctx, log2)
        try:
            for r in [r for r in rows if r["log2"] == log2]:
                proof = p.prove_seed(r["seed"])
                assert hashlib.sha256(proof).hexdigest() == r["sha256"]
                assert p.verify(proof) == ""
        finally:
            p.close()


def test_accepts_full_size_golden(gpu_ctx):
    import flockgpu
    r = [r for r in json.loads((GOLD / "verified_proofs_large.json").read_text()) if r["log2"] == 18][0]
    p = flockgpu.Prover(gpu_ctx, 18)
    try:
        proof = p.prove_seed(r["seed"])
        assert hashlib.sha256(proof).hexdigest() == r["sha256"]
        t0 = time.perf_counter()
        assert p.verify(proof) == ""
        print(f"verify 2^18: {1e3 * (time.perf_counter() - t0):.1f} ms")
        assert gpu_ctx.verify(proof) == ""  # and without the setup
    finally:
        p.close()


def test_rejects_bit_flips(p8):
    proof = p8.prove_seed(31)
    assert p8.verify(proof) == ""
    rng = np.random.default_rng(4)
    offs = sorted(set(rng.integers(0, len(proof), 48).tolist()) | {5, 6, 7, 8, 40, 47, len(proof) - 1})
    for off in offs:
        bad = bytearray(proof)
        bad[off] ^= 1 << int(rng.integers(0, 8))
        assert p8.verify(bytes(bad)) != "", off


def test_rejects_truncation_and_trailing_bytes(p8):
    proof = p8.prove_seed(32)
    assert "malformed" in p8.verify(proof[:-1])
    assert "malformed" in p8.verify(proof + b"\0")
    assert "malformed" in p8.verify(b"")


def test_rejects_other_domain_and_size(gpu_ctx, p8):
    import flockgpu
    proof = p8.prove_seed(33)
    assert p8.verify(proof, b"another-domain") != ""
    p9 = flockgpu.Prover(gpu_ctx, 9)
    try:
        assert "size" in p9.verify(proof)
    finally:
        p9.close()


def test_chain_accepts_honest_rejects_broken(p8):
    import flockgpu
    recs = flockgpu.chain_blocks(8, 1 << 8)
    good = p8.prove_chain(recs)
    assert p8.verify(good, CHAIN_DOMAIN) == ""
    # a chain bundle is bound to its domain too
    assert p8.verify(good, b"flock-bench-v0") != ""
    recs[7, 2] ^= 4
    assert p8.verify(p8.prove_chain(recs), CHAIN_DOMAIN) == "verify: chain: shift argument"


def test_chain_rejects_edited_endpoint(p8):
    import flockgpu
    good = p8.prove_chain(flockgpu.chain_blocks(9, 1 << 8))
    bad = bytearray(good)
    bad[-1] ^= 1  # the last bit of cv_last_phys
    assert p8.verify(bytes(bad), CHAIN_DOMAIN) == "verify: chain: shift argument"


def test_chain_full_size_golden_verifies(gpu_ctx):
    import flockgpu
    r = [r for r in json.loads((GOLD / "chain_proofs.json").read_text()) if r["log2"] == 16][0]
    p = flockgpu.Prover(gpu_ctx, 16)
    try:
        proof = p.prove_chain(flockgpu.chain_blocks(r["seed"], 1 << 16), r["domain"].encode())
        assert hashlib.sha256(proof).hexdigest() == r["sha256"]
        assert p.verify(proof, r["domain"].encode()) == ""
    finally:
        p.close()


def test_self_checking_serving(gpu_ctx):
    """Served proofs are checked by the server's verifier threads, batched
    ones by the batch threads; either way the bytes are the plain proofs'."""
    import flockgpu
    jobs = ((8, 1), (9, 2), (8, 3), (10, 6), (8, 7))
    plain = {}
    for l in sorted({l for l, _ in jobs}):
        p = flockgpu.Prover(gpu_ctx, l)
        try:
            for ll, s in jobs:
                if ll == l:
                    plain[(l, s)] = p.prove_seed(s)
        finally:
            p.close()
    ctx = flockgpu.Context(0)
    try:
        ctx.serve_start(2)
        ctx.serve_verify(True)
        tickets = [ctx.submit(l, s) for l, s in jobs]
        for t, job in zip(tickets, jobs):
            r = ctx.poll(t)  # a failed self-check raises
            assert r["bytes"] == plain[job]
        out = ctx.prove_batch([(8, 1), (9, 2)], threads=2)
        assert [o["bytes"] for o in out] == [plain[(8, 1)], plain[(9, 2)]]
        ctx.serve_verify(False)
        assert ctx.poll(ctx.submit(8, 3))["bytes"] == plain[(8, 3)]
    finally:
        ctx.close()


def test_context_verifier_without_setup(gpu_ctx, p8):
    """flock_verify_bundle: the context's own verifier, any size, no setup."""
    import flockgpu
    proof = p8.prove_seed(41)
    chain = p8.prove_chain(flockgpu.chain_blocks(4, 1 << 8))
    assert gpu_ctx.verify(proof) == ""
    assert gpu_ctx.verify(chain, CHAIN_DOMAIN) == ""
    bad = bytearray(proof)
    bad[len(bad) // 2] ^= 1
    assert gpu_ctx.verify(bytes(bad)) != ""
    assert gpu_ctx.verify(proof, b"another-domain") != ""
    assert "malformed" in gpu_ctx.verify(proof[:30])
    p9 = flockgpu.Prover(gpu_ctx, 9)
    try:
        assert gpu_ctx.verify(p9.prove_seed(2)) == ""  # another size on the same verifier
    finally:
        p9.close()


def test_context_verifier_full_size_goldens(gpu_ctx):
    """The setup-free verifier on the largest bundles: the 2^14, 2^16 and
    2^18 proofs the reference's trusted verifier accepted (reproduced bit for
    bit) and the 2^14..2^18 chain goldens, whose opened rows come closest to
    its fixed row buffer."""
    import flockgpu
    proofs = json.loads((GOLD / "verified_proofs_large.json").read_text())
    chains = json.loads((GOLD / "chain_proofs.json").read_text())
    for log2 in sorted({r["log2"] for r in proofs} | {r["log2"] for r in chains}):
        p = flockgpu.Prover(gpu_ctx, log2)
        try:
            for r in [r for r in proofs if r["log2"] == log2]:
                b = p.prove_seed(r["seed"])
                assert hashlib.sha256(b).hexdigest() == r["sha256"]
                assert gpu_ctx.verify(b) == "", log2
            for r in [r for r in chains if r["log2"] == log2]:
                b = p.prove_chain(flockgpu.chain_blocks(r["seed"], 1 << log2))
                assert hashlib.sha256(b).hexdigest() == r["sha256"]
                assert gpu_ctx.verify(b, CHAIN_DOMAIN) == "", log2
        finally:
            p.close()
