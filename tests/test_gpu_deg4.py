"""The degree-4 zerocheck round 1 on the GPU (flock_zerocheck_round1_deg4)
against the oracle's round1_deg4_naive (crates/flock-core/src/zerocheck/
univariate_skip_deg4.rs:77-165): random rows and challenges from one row
(m = 6) to 2^14 rows, all-zero and all-ones factors, and the seeded
microbenchmark entry point at the benchmark's smallest size."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GAMMA = np.uint64(0x9E3779B97F4A7C15)


def _rand(rng, shape):
    return rng.integers(0, 2**63, shape, np.uint64) ^ (rng.integers(0, 2, shape, np.uint64) << np.uint64(63))


@pytest.mark.parametrize("m", [6, 7, 9, 12, 16, 20])
def test_random_rows_match_oracle(gpu_ctx, oracle, m):
    rng = np.random.default_rng(100 + m)
    n = 1 << (m - 6)
    vecs = _rand(rng, (5, n))
    r = _rand(rng, (m, 2))
    want = oracle.round1_deg4(*vecs, m, r)
    got = gpu_ctx.round1_deg4(*vecs, m, r)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_constant_rows_match_oracle(gpu_ctx, oracle):
    m = 11
    n = 1 << (m - 6)
    r = _rand(np.random.default_rng(5), (m, 2))
    zero, one = np.zeros(n, np.uint64), np.full(n, 2**64 - 1, np.uint64)
    for vecs in ((zero,) * 5, (one,) * 5, (one, zero, one, one, one), (one, one, one, one, zero)):
        want = oracle.round1_deg4(*vecs, m, r)
        got = gpu_ctx.round1_deg4(*vecs, m, r)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def _splitmix(start: int, count: int) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = np.uint64(start) + (np.arange(count, dtype=np.uint64) + np.uint64(1)) * GAMMA
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def test_bench_entry_point_matches_oracle(gpu_ctx, oracle):
    """benches/round1_deg4.rs's smallest size, m = 16: the benchmark's
    device-generated inputs, regenerated here, give the oracle's message."""
    m, seed = 16, 0xDEC0DE ^ 16
    n = 1 << (m - 6)
    ms, pa, pz = gpu_ctx.bench_round1_deg4(m, seed, iters=3)
    vecs = _splitmix(seed, 5 * n).reshape(5, n)
    r = _splitmix(seed ^ 1, 2 * m).reshape(m, 2)
    want = oracle.round1_deg4(*vecs, m, r)
    assert ms > 0 and np.array_equal(pa, want[0]) and np.array_equal(pz, want[1])
