"""The SHA-256 hash option of the transcript and of the PCS Merkle trees
(HashKind, crates/flock-core/src/hash.rs:20-30; SHA-256 is the reference's
default): the oracle's SHA-256 against hashlib, the SHA-256 transcript
(FsChallenger::with_hash(.., Sha256), challenger.rs:227-307: squeezes
SHA256(state || ctr LE), PoW SHA256(digest || nonce LE)) rebuilt from its
definition with hashlib, the product's host transcript against the oracle's,
and the SHA-256 Merkle tree (leaf SHA256(bytes), parent SHA256(l || r),
merkle.rs:205-230) against hashlib."""
import hashlib
import struct

import numpy as np
import pytest


@pytest.mark.parametrize("n", [0, 1, 55, 56, 63, 64, 65, 119, 120, 1000, 4096])
def test_oracle_sha256_is_sha256(oracle, n):
    data = bytes((7 * i + 3) & 0xFF for i in range(n))
    assert oracle.sha256(data) == hashlib.sha256(data).digest()


def _le64(v):
    return struct.pack("<Q", v)


def test_sha256_transcript_from_its_definition(oracle):
    """Replay the script's absorbed bytes with hashlib: domain op 1, label op
    2, observe op 3 (kind 1 scalar, 2 slice), bytes op 5, squeeze op 4; a
    squeeze of k bytes is SHA256(state || ctr) for ctr = 0.. and is absorbed."""
    dom = b"flock-hash-test"
    got = oracle.challenger_script(dom, "sha256")
    st = b"\x01" + _le64(len(dom)) + dom
    st += b"\x02" + _le64(16) + b"flock-test-label"
    st += b"\x03\x01" + _le64(0x0123456789ABCDEF) + _le64(0xFEDCBA9876543210)
    st += b"\x03\x02" + _le64(5) + b"".join(_le64(i) for i in range(10))
    st += b"\x05" + _le64(3) + b"\x01\x02\x03"

    def squeeze(state, n):
        out = b""
        ctr = 0
        while len(out) < n:
            out += hashlib.sha256(state + _le64(ctr)).digest()
            ctr += 1
        return out[:n]

    st += b"\x04\x01"
    one = squeeze(st, 16)
    st += one
    assert np.frombuffer(one, np.uint64).tolist() == got[0].tolist()
    st += b"\x04\x02" + _le64(7)
    vec = squeeze(st, 112)
    st += vec
    assert np.frombuffer(vec, np.uint64).tolist() == got[1].tolist()
    # grind_pow(5): the smallest nonce whose SHA256(digest || nonce LE) has 5
    # leading zero bits; the nonce is observed as bytes
    digest = hashlib.sha256(st).digest()
    n = 0
    while hashlib.sha256(digest + _le64(n)).digest()[0] >> 3:
        n += 1
    assert got[2] == n
    st += b"\x05" + _le64(8) + _le64(n)
    assert got[3] == hashlib.sha256(st).digest()


@pytest.mark.parametrize("hash", ["sha256", "blake3"])
def test_product_transcript_matches_oracle(oracle, hash):
    import flockgpu
    dom = b"flock-hash-test"
    want = oracle.challenger_script(dom, hash)
    ch = flockgpu.Challenger(dom, hash)
    ch.observe_label(b"flock-test-label")
    ch.observe_f128((0x0123456789ABCDEF, 0xFEDCBA9876543210))
    ch.observe_f128_slice(np.arange(10, dtype=np.uint64))
    ch.observe_bytes(b"\x01\x02\x03")
    got = [np.array(ch.sample_f128(), np.uint64), np.asarray(ch.sample_f128_vec(7), np.uint64).reshape(-1)]
    got.append(ch.grind_pow(None, 5))
    got.append(ch.state_digest())
    ch.close()
    assert got[0].tolist() == want[0].tolist()
    assert got[1].tolist() == want[1].tolist()
    assert got[2] == want[2] and got[3] == want[3]


@pytest.mark.parametrize("leaf_size", [16, 48, 64, 128, 1024])
def test_oracle_sha256_merkle_tree(oracle, leaf_size):
    n = 16
    data = np.random.default_rng(leaf_size).integers(0, 256, n * leaf_size, dtype=np.uint8)
    tree = oracle.merkle_tree_hash(data, n, leaf_size, "sha256").reshape(-1, 32)
    want = [hashlib.sha256(data[i * leaf_size:(i + 1) * leaf_size].tobytes()).digest() for i in range(n)]
    level, start = want, 0
    nodes = list(want)
    while len(level) > 1:
        level = [hashlib.sha256(level[2 * j] + level[2 * j + 1]).digest() for j in range(len(level) // 2)]
        nodes += level
    assert [bytes(t) for t in tree] == nodes
