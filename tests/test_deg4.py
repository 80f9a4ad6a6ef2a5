"""The degree-4 zerocheck round 1 (crates/flock-core/src/zerocheck/
univariate_skip_deg4.rs, round1_deg4_naive) in the oracle, against a second,
independent statement of the same message: each factor's extension to
Lambda4 = {64..255} as the evaluation of its degree-< 64 interpolant over the
nodes S = {0..63} (Lagrange form, GF(2^8) arithmetic in numpy), on sparse
inputs whose sums stay small.  Also the reference's own checks (:214-348):
the message shape, a = b = c = d = 0 gives p_abcd = 0, and with c = d = 1 the
product reduces to a b."""
import numpy as np
import pytest


def _gf8_tables():
    exp = np.zeros(512, np.int64)
    log = np.zeros(256, np.int64)
    x = 1
    for i in range(255):
        exp[i] = x
        log[x] = i
        x2 = x << 1
        if x2 & 0x100:
            x2 ^= 0x11B
        x = x2 ^ x  # multiply by the generator 3
    exp[255:510] = exp[:255]
    return exp, log


EXP, LOG = _gf8_tables()


def _mul(a, b):
    if a == 0 or b == 0:
        return 0
    return int(EXP[LOG[a] + LOG[b]])


def _inv(a):
    return int(EXP[(255 - LOG[a]) % 255])


def _extension():
    """M[l][s]: the Lagrange basis polynomial of node s over S at 64 + l."""
    M = np.zeros((192, 64), np.int64)
    for s in range(64):
        den = 1
        for j in range(64):
            if j != s:
                den = _mul(den, s ^ j)
        inv = _inv(den)
        for l in range(192):
            num = 1
            for j in range(64):
                if j != s:
                    num = _mul(num, (64 + l) ^ j)
            M[l, s] = _mul(num, inv)
    return M


@pytest.fixture(scope="module")
def ext():
    return _extension()


def _row_ext(M, word):
    v = np.zeros(192, np.int64)
    for s in range(64):
        if (int(word) >> s) & 1:
            v ^= M[:, s]
    return v


def _expect(oracle, M, rows, m, r):
    """sum over the given nonzero rows of eq(r[6..], x) phi8(.) by the
    Lagrange statement; rows: {x: (a, b, c, d, z)}."""
    eq = oracle.build_eq(r[6:]).reshape(-1, 2)
    phi = oracle.phi8_table()
    pa = np.zeros((192, 2), np.uint64)
    pz = np.zeros((192, 2), np.uint64)
    for x, words in rows.items():
        ea, eb, ec, ed, ez = (_row_ext(M, w) for w in words)
        for l in range(192):
            prod = _mul(_mul(int(ea[l]), int(eb[l])), _mul(int(ec[l]), int(ed[l])))
            pa[l] ^= oracle.f128_mul(eq[x], phi[prod])
            pz[l] ^= oracle.f128_mul(eq[x], phi[int(ez[l])])
    return pa, pz


def _rand_r(rng, m):
    return rng.integers(0, 2**63, (m, 2), np.uint64) ^ (rng.integers(0, 2, (m, 2), np.uint64) << np.uint64(63))


@pytest.mark.parametrize("m", [6, 8])
def test_oracle_matches_lagrange_statement(oracle, ext, m):
    rng = np.random.default_rng(m)
    n = 1 << (m - 6)
    vecs = np.zeros((5, n), np.uint64)
    rows = {}
    for x in sorted(set(rng.integers(0, n, 2).tolist())):
        words = rng.integers(0, 2**63, 5, np.uint64) ^ (rng.integers(0, 2, 5, np.uint64) << np.uint64(63))
        vecs[:, x] = words
        rows[x] = words
    r = _rand_r(rng, m)
    pa, pz = oracle.round1_deg4(*vecs, m, r)
    ea, ez = _expect(oracle, ext, rows, m, r)
    assert np.array_equal(pa, ea) and np.array_equal(pz, ez)


def test_zero_factors_and_reduction_to_degree_two(oracle):
    """a = b = c = d = 0: p_abcd = 0 (linear_only_path).  c = d = 1: the
    message is that of a, b, 1, 1 in any order of the factors
    (degree4_reduces_to_degree2_when_cd_one)."""
    m = 9
    rng = np.random.default_rng(3)
    n = 1 << (m - 6)
    z = rng.integers(0, 2**63, n, np.uint64)
    zero = np.zeros(n, np.uint64)
    r = _rand_r(rng, m)
    pa, pz = oracle.round1_deg4(zero, zero, zero, zero, z, m, r)
    assert not pa.any() and pz.any()
    a, b = rng.integers(0, 2**63, n, np.uint64), rng.integers(0, 2**63, n, np.uint64)
    one = np.full(n, 2**64 - 1, np.uint64)
    p1, _ = oracle.round1_deg4(a, b, one, one, zero, m, r)
    p2, _ = oracle.round1_deg4(one, a, one, b, zero, m, r)
    assert np.array_equal(p1, p2) and p1.any()
    # all-ones factors extend to the constant 1: p_abcd = sum_x eq_x phi8(1)
    p3, _ = oracle.round1_deg4(one, one, one, one, zero, m, r)
    s = np.bitwise_xor.reduce(oracle.build_eq(r[6:]).reshape(-1, 2), axis=0)
    assert all(np.array_equal(p3[l], s) for l in range(192))
