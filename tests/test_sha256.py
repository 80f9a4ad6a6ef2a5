"""The SHA-256 compression statement on the CPU (crates/flock-prover/src/
r1cs_hashes/sha2.rs): the oracle's compression against the SHA-256 standard
(hashlib over padded multi-block messages), its R1CS witness against the
matrices (the reference's block_witness_satisfies_matrix_and_matches_reference,
useful_bits_matches_constants and block_r1cs_satisfies_for_one_block tests,
sha2.rs:2125-2386), the product library's host statement (digests of its
matrices) and host compression against the oracle, and the oracle's proofs
against the committed fixtures."""
import hashlib
import json
import struct
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "sha256_proofs.json"
IV = np.array([0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a, 0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19],
              np.uint32)


def _blocks(msg: bytes):
    """FIPS 180-4 padding into 16-word big-endian blocks."""
    padded = msg + b"\x80" + b"\x00" * ((55 - len(msg)) % 64) + struct.pack(">Q", 8 * len(msg))
    return [np.frombuffer(padded[i:i + 64], ">u4").astype(np.uint32) for i in range(0, len(padded), 64)]


def _digest(compress, msg: bytes) -> str:
    h = IV.copy()
    for m in _blocks(msg):
        h = compress(h, m)
    return "".join("%08x" % v for v in h)


@pytest.mark.parametrize("msg", [b"", b"abc", b"abcdbcdecdefdefgefghfghighijhijkijkljklmklmnlmnomnopnopq",
                                 bytes(range(256)) * 3])
def test_oracle_compress_is_sha256(oracle, msg):
    assert _digest(oracle.sha256_compress, msg) == hashlib.sha256(msg).hexdigest()


def test_product_host_compress_matches_oracle(oracle):
    import flockgpu
    rng = np.random.default_rng(5)
    for _ in range(20):
        h, m = rng.integers(0, 2**32, 8, np.uint32), rng.integers(0, 2**32, 16, np.uint32)
        assert np.array_equal(flockgpu.sha256_compress(h, m), oracle.sha256_compress(h, m))
    assert _digest(flockgpu.sha256_compress, b"flock") == hashlib.sha256(b"flock").hexdigest()


def test_bench_inputs_match(oracle):
    import flockgpu
    for n, seed in ((8, 1), (300, flockgpu.sha256_bench_seed(300))):
        assert np.array_equal(flockgpu.sha256_bench_inputs(n, seed), oracle.sha256_bench_inputs(n, seed))


def _bits(z):
    return np.unpackbits(z.view(np.uint8), axis=1, bitorder="little")


def test_witness_satisfies_matrices_and_carries_the_output(oracle):
    """a = A_0 z and b = B_0 z (from the matrices): a & b == z in every row;
    H_out (bits 256..511) is the compression; the constant wire (bit 31400)
    is 1 and bits 31401.. are 0; padding blocks hold the all-zero (h, m)
    compression."""
    n_log, n = 3, 6
    comps = oracle.sha256_bench_inputs(n, 77)
    z, a, b = oracle.sha256_witness(comps, n_log)
    assert np.array_equal(a & b, z)
    zb = _bits(z)
    for i in range(1 << n_log):
        c = comps[i] if i < n else np.zeros(24, np.uint32)
        hout = np.packbits(zb[i, 256:512], bitorder="little").view(np.uint32)
        assert np.array_equal(hout, oracle.sha256_compress(c[:8], c[8:]))
        assert np.array_equal(np.packbits(zb[i, :256], bitorder="little").view(np.uint32), c[:8])
        assert np.array_equal(np.packbits(zb[i, 512:1024], bitorder="little").view(np.uint32), c[8:])
        assert zb[i, 31400] == 1 and not zb[i, 31401:].any()


def test_flipped_witness_bit_breaks_a_row(oracle):
    """Any single flipped carry, AND or materialised bit violates some row
    (the statement pins every useful bit)."""
    comps = oracle.sha256_bench_inputs(8, 3)
    z, a0, b0 = oracle.sha256_witness(comps, 3)
    mats = [oracle.sha256_matrix(w) for w in (0, 1)]
    a, b = _apply(mats, z[:1])
    assert np.array_equal(a, a0[:1]) and np.array_equal(b, b0[:1])
    rng = np.random.default_rng(9)
    for bit in list(rng.integers(1024, 31401, 12)) + [31400, 300, 700]:
        zz = z[:1].copy()
        zz[0, bit // 64] ^= np.uint64(1) << np.uint64(bit % 64)
        a, b = _apply(mats, zz)
        assert not np.array_equal(a & b, zz), bit


def _apply(mats, z):
    """A_0 z, B_0 z of one block from the CSR matrices."""
    zb = _bits(z)[0]
    out = []
    for ptr, col in mats:
        v = np.bitwise_xor.reduceat(zb[col], np.minimum(ptr[:-1], col.size - 1))
        v[np.diff(ptr) == 0] = 0  # reduceat gives an empty row the next row's first term
        out.append(np.packbits(v, bitorder="little").view(np.uint64)[None, :])
    return out


def test_layout_constants(oracle):
    """USEFUL_BITS = 31401, the constant wire last (sha2.rs:108-121): rows
    from 31401 on are empty in A_0 and B_0; row 31400 is z_c * z_c = z_c."""
    for which in (0, 1):
        ptr, col = oracle.sha256_matrix(which)
        assert ptr[31401] == ptr[1 << 15]
        assert list(col[ptr[31400]:ptr[31401]]) == [31400]
        # input rows H_in and M: (v) * (1)
        for r in (0, 255, 512, 1023):
            assert list(col[ptr[r]:ptr[r + 1]]) == ([r] if which == 0 else [31400])


def test_product_statement_digest_matches_oracle(oracle):
    import flockgpu
    for m in (22, 23, 27, 34):
        assert flockgpu.sha256_statement_digest(m) == oracle.sha256_digest(m - 15)
    # a different statement from the BLAKE3 one of the same m
    assert flockgpu.sha256_statement_digest(23) != oracle.statement_digest(9)


def test_fixture_digests():
    g = json.loads(GOLDEN.read_text())
    import flockgpu
    for m, d in g["digests"].items():
        assert flockgpu.sha256_statement_digest(int(m)) == bytes.fromhex(d), m


def test_oracle_proof_matches_fixture(oracle):
    g = json.loads(GOLDEN.read_text())
    e = next(p for p in g["proofs"] if p["n"] == 256)
    proof = oracle.prove_sha256(oracle.sha256_bench_inputs(256, e["seed"]))
    assert hashlib.sha256(proof).hexdigest() == e["sha256"] and len(proof) == e["size"]
