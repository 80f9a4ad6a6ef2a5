"""The full prove_fast input contract at the C ABI: Blake3Setup::new(n_blocks)
for any count (2^max(3, ceil(log2 n)) slots, blake3.rs:1854-1858) and
Compression tuples with every field free (u64 counter, block_len, flags;
blake3.rs:1861), the unused slots holding the all-zero compression
(blake3.rs:2527, seed_pipe.rs:210-226)."""
import numpy as np
import pytest


def _records(n: int, seed: int) -> np.ndarray:
    """n random compression records (28 u32), with u64 counters and varied
    block_len / flags (the CLI chain's flags 0, the benchmark's 11, others)."""
    rng = np.random.default_rng(seed)
    rec = rng.integers(0, 2**32, (n, 28), dtype=np.uint64).astype(np.uint32)
    rec[:, 26] = rng.integers(0, 65, n)          # block_len 0..64
    rec[:, 27] = rng.choice([0, 1, 2, 3, 8, 11], n)  # flags
    return rec


def test_oracle_records_equal_benchmark_proof(oracle):
    """The benchmark's compressions as full records (block_len 64, flags 11)
    give the seed proof, which the reference's trusted verifier accepted."""
    import flockgpu
    recs = flockgpu.to_records(oracle.compressions(8, 0x00C0FFEEBEEFD15C))
    assert oracle.prove_records(recs) == oracle.prove(8, 0x00C0FFEEBEEFD15C)


def test_oracle_padding_is_the_zero_compression(oracle):
    """n = 300 compressions prove over 512 slots exactly as the same 300 plus
    212 explicit all-zero compressions."""
    recs = _records(300, 7)
    padded = np.concatenate([recs, np.zeros((212, 28), np.uint32)])
    assert oracle.prove_records(recs) == oracle.prove_records(padded)


@pytest.mark.gpu
@pytest.mark.parametrize("n,seed", [(300, 1), (1000, 2), (129, 3)])
def test_any_count_full_records_match_oracle(gpu_ctx, oracle, n, seed):
    import flockgpu
    import proofparse
    recs = _records(n, seed)
    p = flockgpu.Prover(gpu_ctx, n_blocks=n)
    try:
        assert p.log2 == max(3, (n - 1).bit_length())
        g = p.prove_compressions(recs)
        o = oracle.prove_records(recs)
        assert proofparse.first_difference(g, o) is None
        assert g == o
        assert gpu_ctx.verify(g) == ""
    finally:
        p.close()


@pytest.mark.gpu
def test_full_records_equal_seed_and_blocks_proofs(gpu_ctx):
    import flockgpu
    p = flockgpu.Prover(gpu_ctx, 9)
    try:
        blocks = flockgpu.generate_compressions(9, 99)
        want = p.prove_seed(99)
        assert p.prove_compressions(flockgpu.to_records(blocks)) == want
        assert p.prove_blocks(blocks) == want
    finally:
        p.close()


@pytest.mark.gpu
def test_count_rules(gpu_ctx):
    import flockgpu
    for bad in (0, 1, 128, (1 << 20) + 1):
        with pytest.raises(flockgpu.FlockError):
            flockgpu.Prover(gpu_ctx, n_blocks=bad)
    p = flockgpu.Prover(gpu_ctx, n_blocks=300)
    try:
        with pytest.raises(flockgpu.FlockError):  # prove_fast asserts blocks.len() == n_blocks
            p.prove_compressions(_records(299, 1))
        with pytest.raises(flockgpu.FlockError):
            p.prove_compressions(_records(512, 1))
    finally:
        p.close()
