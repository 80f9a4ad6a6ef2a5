"""GPU parity: every kernel entry point and the full prover against the oracle
(bit-exact; the path is pure binary-field / integer arithmetic), plus the
golden proofs the reference's trusted verifier accepted."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def rng_u64(seed, n):
    return np.random.default_rng(seed).integers(0, 2**64, n, dtype=np.uint64)


def test_f128_mul(gpu_ctx, oracle):
    a, b = rng_u64(1, 2 * 512), rng_u64(2, 2 * 512)
    a[:8] = 0
    b[8:16] = np.uint64(2**64 - 1)
    assert np.array_equal(gpu_ctx.f128_mul(a, b), oracle.f128_mul(a, b))


@pytest.mark.parametrize("log2,seed", [(3, 7), (4, 1), (6, 0x00C0FFEEBEEFD15C), (8, 12345)])
def test_witness(gpu_ctx, oracle, log2, seed):
    gz, ga, gb = gpu_ctx.witness(log2, seed)
    oz, oa, ob = oracle.witness(log2, seed)
    assert np.array_equal(gz, oz)
    assert np.array_equal(ga, oa)
    assert np.array_equal(gb, ob)


def test_witness_golden(gpu_ctx):
    for row in json.loads((GOLD / "witness_digests.json").read_text()):
        z, a, b = gpu_ctx.witness(row["log2"], row["seed"])
        assert hashlib.sha256(z.tobytes()).hexdigest() == row["z"]
        assert hashlib.sha256(a.tobytes()).hexdigest() == row["a"]
        assert hashlib.sha256(b.tobytes()).hexdigest() == row["b"]


@pytest.mark.parametrize("lanes,log_pos,rate", [(1, 3, 1), (1, 12, 2), (2, 9, 1), (4, 10, 2), (8, 13, 3),
                                                 (64, 8, 1), (64, 11, 1), (16, 12, 4), (256, 6, 1)])
def test_ntt_rs_encode(gpu_ctx, oracle, lanes, log_pos, rate):
    msg = rng_u64(lanes * 31 + log_pos, 2 * (lanes << log_pos))
    got = gpu_ctx.ntt_rs_encode(msg, log_pos, lanes, rate)
    want = oracle.rs_encode(msg, 1 << log_pos, lanes, rate)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("lanes,log_pos,rate", [(64, 10, 1), (1, 16, 2), (8, 13, 3), (256, 6, 1), (4, 19, 1),
                                                 (64, 13, 1), (128, 9, 2)])
def test_ntt_every_plan(gpu_ctx, oracle, lanes, log_pos, rate):
    """Every pass plan the autotuner may pick gives the oracle's codeword."""
    msg = rng_u64(lanes * 7 + log_pos, 2 * (lanes << log_pos))
    want = oracle.rs_encode(msg, 1 << log_pos, lanes, rate)
    k = 0
    while True:
        got = gpu_ctx.ntt_rs_encode_plan(msg, log_pos, lanes, rate, k)
        if got is None:
            break
        assert np.array_equal(got, want), f"plan {k}"
        k += 1
    assert k >= 2
    ms, desc = gpu_ctx.ntt_autotune(log_pos, lanes, rate)
    assert desc and np.array_equal(gpu_ctx.ntt_rs_encode(msg, log_pos, lanes, rate), want)


@pytest.mark.parametrize("n_leaves,leaf_size", [(1, 64), (2, 32), (16, 48), (1024, 128), (4096, 1024), (2048, 512)])
def test_merkle_tree(gpu_ctx, oracle, n_leaves, leaf_size):
    data = np.random.default_rng(n_leaves + leaf_size).integers(0, 256, n_leaves * leaf_size, dtype=np.uint8)
    assert np.array_equal(gpu_ctx.merkle_tree(data, n_leaves, leaf_size), oracle.merkle_tree(data, n_leaves, leaf_size))


def test_sumcheck_round(gpu_ctx, oracle):
    n = 64
    f, b = rng_u64(5, 2 * n), rng_u64(6, 2 * n)
    F, B = f.reshape(-1, 2), b.reshape(-1, 2)
    u0 = np.bitwise_xor.reduce(oracle.f128_mul(F[0::2].reshape(-1), B[0::2].reshape(-1)).reshape(-1, 2), axis=0)
    u2 = np.bitwise_xor.reduce(
        oracle.f128_mul((F[0::2] ^ F[1::2]).reshape(-1), (B[0::2] ^ B[1::2]).reshape(-1)).reshape(-1, 2), axis=0)
    got = gpu_ctx.sumcheck_round(f, b)
    assert list(got) == [u0[0], u0[1], u2[0], u2[1]]


def _xor_rows(v):
    return np.bitwise_xor.reduce(v.reshape(-1, 2), axis=0)


@pytest.mark.parametrize("log_n", [1, 6, 16])
def test_sumcheck_round_deg2_sizes(gpu_ctx, oracle, log_n):
    n = 1 << log_n
    f, b = rng_u64(50 + log_n, 2 * n), rng_u64(60 + log_n, 2 * n)
    F, B = f.reshape(-1, 2), b.reshape(-1, 2)
    u0 = _xor_rows(oracle.f128_mul(F[0::2].reshape(-1), B[0::2].reshape(-1)))
    u2 = _xor_rows(oracle.f128_mul((F[0::2] ^ F[1::2]).reshape(-1), (B[0::2] ^ B[1::2]).reshape(-1)))
    assert list(gpu_ctx.sumcheck_round(f, b)) == [u0[0], u0[1], u2[0], u2[1]]


def _deg3_expect(oracle, e, a, b):
    A, B = a.reshape(-1, 2), b.reshape(-1, 2)
    a0, a1, b0, b1 = A[0::2].reshape(-1), A[1::2].reshape(-1), B[0::2].reshape(-1), B[1::2].reshape(-1)
    g1 = _xor_rows(oracle.f128_mul(e, oracle.f128_mul(a1, b1)))
    gi = _xor_rows(oracle.f128_mul(e, oracle.f128_mul(a0 ^ a1, b0 ^ b1)))
    return [g1[0], g1[1], gi[0], gi[1]]


def _fold(oracle, x, rho):
    X = x.reshape(-1, 2)
    x0, x1 = X[0::2].reshape(-1), X[1::2].reshape(-1)
    r = np.tile(np.array(rho, np.uint64), x0.size // 2)
    return x0 ^ oracle.f128_mul(r, x0 ^ x1)


@pytest.mark.parametrize("log_n", [1, 5, 16])
def test_sumcheck_round_deg3(gpu_ctx, oracle, log_n):
    """Zerocheck-style round (eq * a * b) over plain F128 vectors."""
    n = 1 << log_n
    a, b, e = rng_u64(70 + log_n, 2 * n), rng_u64(80 + log_n, 2 * n), rng_u64(90 + log_n, n)
    msg, _, _ = gpu_ctx.sumcheck_round3(e, a, b)
    assert list(msg) == _deg3_expect(oracle, e, a, b)


@pytest.mark.parametrize("log_n", [2, 7, 16])
def test_sumcheck_fold_round_deg3(gpu_ctx, oracle, log_n):
    """Fold at rho, then the degree-3 message over the folded pairs."""
    n = 1 << log_n
    a, b, e = rng_u64(100 + log_n, 2 * n), rng_u64(110 + log_n, 2 * n), rng_u64(120 + log_n, n // 2)
    rho = (0x0123456789ABCDEF, 0xFEDCBA9876543210)
    msg, ao, bo = gpu_ctx.sumcheck_round3(e, a, b, rho)
    fa, fb = _fold(oracle, a, rho), _fold(oracle, b, rho)
    assert np.array_equal(ao, fa) and np.array_equal(bo, fb)
    assert list(msg) == _deg3_expect(oracle, e, fa, fb)


@pytest.mark.parametrize("bits", [1, 6, 12])
def test_pow_smallest_nonce(gpu_ctx, oracle, bits):
    digest, nonce = oracle.grind(b"flock-bench-v0", b"gpu-pow-%d" % bits, bits)
    assert gpu_ctx.pow(digest, bits) == nonce


@pytest.fixture(scope="module")
def prover8(gpu_ctx):
    import flockgpu
    p = flockgpu.Prover(gpu_ctx, 8)
    yield p
    p.close()


def test_proof_matches_verifier_accepted_golden(prover8):
    rows = [r for r in json.loads((GOLD / "verified_proofs.json").read_text()) if r["log2"] == 8]
    for r in rows:
        p = prover8.prove_seed(r["seed"])
        assert len(p) == r["size"] and hashlib.sha256(p).hexdigest() == r["sha256"]


def test_proof_matches_oracle_log2_8(prover8, oracle):
    import proofparse
    for seed in (1, 0x00C0FFEEBEEFD15C):
        g, o = prover8.prove_seed(seed), oracle.prove(8, seed)
        assert proofparse.first_difference(g, o) is None
        assert g == o


def test_prove_blocks_equals_prove_seed(prover8, oracle):
    blocks = oracle.compressions(8, 77)
    assert prover8.prove_blocks(blocks) == prover8.prove_seed(77)


def test_prove_blocks_from_pinned_memory(prover8):
    import flockgpu
    pa = flockgpu.PinnedArray((1 << 8, 25), np.uint32)
    pa.array[:] = flockgpu.generate_compressions(8, 78)
    assert prover8.prove_blocks(pa.array) == prover8.prove_seed(78)


@pytest.mark.parametrize("log2", [9, 10, 12])
def test_proof_matches_oracle_larger(gpu_ctx, oracle, log2):
    import flockgpu
    import proofparse
    p = flockgpu.Prover(gpu_ctx, log2)
    try:
        g = p.prove_seed(2024 + log2)
        o = oracle.prove(log2, 2024 + log2)
        assert proofparse.first_difference(g, o) is None
        assert g == o
        assert len(g) <= flockgpu.MAX_PROOF_BYTES
    finally:
        p.close()


def test_golden_larger(gpu_ctx):
    import flockgpu
    rows = [r for r in json.loads((GOLD / "verified_proofs.json").read_text()) if r["log2"] in (9, 10)]
    for log2 in sorted({r["log2"] for r in rows}):
        p = flockgpu.Prover(gpu_ctx, log2)
        try:
            for r in [r for r in rows if r["log2"] == log2]:
                assert hashlib.sha256(p.prove_seed(r["seed"])).hexdigest() == r["sha256"]
        finally:
            p.close()


@pytest.mark.parametrize("log2", [14, 16, 18])
def test_golden_full_size(gpu_ctx, log2):
    """Bit-identity at the benchmark's full size: oracle proofs of 2^14, 2^16
    and 2^18 compressions that the reference's trusted verifier accepted."""
    import flockgpu
    rows = [r for r in json.loads((GOLD / "verified_proofs_large.json").read_text()) if r["log2"] == log2]
    assert rows
    p = flockgpu.Prover(gpu_ctx, log2)
    try:
        for r in rows:
            proof = p.prove_seed(r["seed"])
            assert len(proof) == r["size"] and hashlib.sha256(proof).hexdigest() == r["sha256"]
    finally:
        p.close()


@pytest.mark.parametrize("log2", [12, 19, 20])
def test_golden_gpu_proofs_trusted_harness(gpu_ctx, log2):
    """GPU proofs at sizes the oracle is too slow for (2^19, 2^20) and at
    2^12, made by flock_worker under the reference's trusted harness, which
    drew each seed and verified every proof (make_golden.py --gpu-harness):
    the prover reproduces them bit for bit."""
    import flockgpu
    rows = [r for r in json.loads((GOLD / "gpu_verified_proofs.json").read_text()) if r["log2"] == log2]
    assert rows
    p = flockgpu.Prover(gpu_ctx, log2)
    try:
        for r in rows:
            proof = p.prove_seed(r["seed"])
            assert len(proof) == r["size"] and hashlib.sha256(proof).hexdigest() == r["sha256"]
    finally:
        p.close()


def test_phase_times_reported(prover8):
    prover8.prove_seed(5)
    ph = prover8.phase_ms()
    import flockgpu
    assert list(ph) == list(flockgpu.PHASES) and all(v >= 0 for v in ph.values())


# ---- the kernel microbenchmarks' largest shapes ----
# The oracle's outputs for these seeded inputs are committed as digests
# (tests/golden/kernel_digests.json, make_golden.py --kernels); the inputs are
# regenerated here from the same PCG64 seeds.

def _kernel_digests():
    return json.loads((GOLD / "kernel_digests.json").read_text())


@pytest.mark.parametrize("case", range(3))
def test_ntt_largest_shapes(gpu_ctx, case):
    import make_golden
    row = _kernel_digests()["ntt"][case]
    lm, cols, rate = row["log_msg"], row["columns"], row["log_inv_rate"]
    assert (lm, cols, rate) == make_golden.KERNEL_NTT[case]
    cw = gpu_ctx.ntt_rs_encode(make_golden.ntt_input(lm, cols, rate), lm, cols, rate)
    assert hashlib.sha256(cw.tobytes()).hexdigest() == row["sha256"]


@pytest.mark.parametrize("case", range(3))
def test_merkle_largest_shapes(gpu_ctx, case):
    import make_golden
    row = _kernel_digests()["merkle"][case]
    n, size = row["leaves"], row["leaf_bytes"]
    assert (n, size) == make_golden.KERNEL_MERKLE[case]
    tree = gpu_ctx.merkle_tree(make_golden.merkle_input(n, size), n, size)
    assert hashlib.sha256(tree.tobytes()).hexdigest() == row["sha256"]


def test_sumcheck_round_deg2_2p24(gpu_ctx, oracle):
    """The degree-2 (Ligerito) round message over 2^24 values, against the
    oracle's field products."""
    n = 1 << 24
    f, b = rng_u64(524, 2 * n), rng_u64(525, 2 * n)
    F, B = f.reshape(-1, 2), b.reshape(-1, 2)
    u0 = _xor_rows(oracle.f128_mul(F[0::2].reshape(-1), B[0::2].reshape(-1)))
    u2 = _xor_rows(oracle.f128_mul((F[0::2] ^ F[1::2]).reshape(-1), (B[0::2] ^ B[1::2]).reshape(-1)))
    assert list(gpu_ctx.sumcheck_round(f, b)) == [u0[0], u0[1], u2[0], u2[1]]


@pytest.mark.parametrize("fold", [False, True])
def test_sumcheck_round_deg3_2p24(gpu_ctx, oracle, fold):
    """The degree-3 (zerocheck) round over 2^24 values, with and without the
    fold at rho, against the oracle."""
    n = 1 << 24
    a, b = rng_u64(624 + fold, 2 * n), rng_u64(634 + fold, 2 * n)
    if fold:
        e = rng_u64(644, n // 2)
        rho = (0x0F1E2D3C4B5A6978, 0x8796A5B4C3D2E1F0)
        msg, ao, bo = gpu_ctx.sumcheck_round3(e, a, b, rho)
        fa, fb = _fold(oracle, a, rho), _fold(oracle, b, rho)
        assert np.array_equal(ao, fa) and np.array_equal(bo, fb)
        assert list(msg) == _deg3_expect(oracle, e, fa, fb)
    else:
        e = rng_u64(654, n)
        msg, _, _ = gpu_ctx.sumcheck_round3(e, a, b)
        assert list(msg) == _deg3_expect(oracle, e, a, b)
