"""The layer surfaces behind the prove entry point: the transcript
(FsChallenger, challenger.rs:34-100, 170-600) and the PCS commitment
(pcs::commit -> Commitment + ProverData, pcs/commit.rs:143-230), through the
C ABI, against the oracle."""
import ctypes

import numpy as np
import pytest

DOM = b"flock-layer-test-v0"


def _o_sample(L, c):
    out = np.zeros(2, np.uint64)
    L.flockref_ch_sample(c, ctypes.c_void_p(out.ctypes.data))
    return int(out[0]), int(out[1])


def _o_digest(L, c):
    out = np.zeros(32, np.uint8)
    L.flockref_ch_digest(c, ctypes.c_void_p(out.ctypes.data))
    return out.tobytes()


def test_challenger_matches_oracle(oracle):
    """Every observe / sample form, in one script, gives the oracle's
    challenges and state."""
    import flockgpu
    L = oracle.L
    c = L.flockref_ch_new(DOM)
    g = flockgpu.Challenger(DOM)
    try:
        rng = np.random.default_rng(3)
        for step in range(40):
            op = step % 6
            if op == 0:
                lab = b"flock-label-%d" % step
                L.flockref_ch_label(c, lab)
                g.observe_label(lab)
            elif op == 1:
                v = rng.integers(0, 2**64, 2, dtype=np.uint64)
                L.flockref_ch_observe(c, ctypes.c_void_p(v.ctypes.data))
                g.observe_f128((int(v[0]), int(v[1])))
            elif op == 2:
                v = rng.integers(0, 2**64, 2 * (step % 5), dtype=np.uint64)
                L.flockref_ch_observe_slice(c, ctypes.c_void_p(v.ctypes.data), v.size // 2)
                g.observe_f128_slice(v)
            elif op == 3:
                b = rng.integers(0, 256, step, dtype=np.uint8).tobytes()
                L.flockref_ch_bytes(c, b, len(b))
                g.observe_bytes(b)
            elif op == 4:
                assert g.sample_f128() == _o_sample(L, c)
            else:
                n = step % 7
                want = np.zeros(2 * max(n, 1), np.uint64)
                L.flockref_ch_sample_vec(c, n, ctypes.c_void_p(want.ctypes.data))
                assert np.array_equal(g.sample_f128_vec(n), want[: 2 * n])
            assert g.state_digest() == _o_digest(L, c)
    finally:
        L.flockref_ch_free(c)
        g.close()


def test_challenger_verify_pow(oracle):
    """verify_pow accepts the oracle's smallest nonce, rejects the one below
    it, and absorbs the nonce either way."""
    import flockgpu
    L = oracle.L
    c = L.flockref_ch_new(DOM)
    g, h = flockgpu.Challenger(DOM), flockgpu.Challenger(DOM)
    try:
        for x in (L, ):
            x.flockref_ch_label(c, b"pow")
        g.observe_label(b"pow")
        h.observe_label(b"pow")
        nonce = L.flockref_ch_grind(c, 10)
        assert g.verify_pow(nonce, 10)
        assert g.state_digest() == _o_digest(L, c)
        if nonce:
            assert not h.verify_pow(nonce - 1, 10)
        assert h.verify_pow(0, 0) and not flockgpu.Challenger(DOM).verify_pow(1, 0)
    finally:
        L.flockref_ch_free(c)


def test_challenger_grind_on_host(oracle):
    """Grinds of at most 6 bits run on the calling thread (no GPU): the
    smallest nonce, as the oracle's grind_pow finds it."""
    import flockgpu
    L = oracle.L
    for bits in range(0, 7):
        c = L.flockref_ch_new(DOM)
        g = flockgpu.Challenger(DOM)
        try:
            L.flockref_ch_label(c, b"host-grind-%d" % bits)
            g.observe_label(b"host-grind-%d" % bits)
            assert g.grind_pow(None, bits) == L.flockref_ch_grind(c, bits)
            assert g.state_digest() == _o_digest(L, c)
        finally:
            L.flockref_ch_free(c)
    with pytest.raises(flockgpu.FlockError):
        flockgpu.Challenger(DOM).grind_pow(None, 9)  # more bits need the GPU


@pytest.mark.gpu
def test_challenger_grind_on_gpu(gpu_ctx, oracle):
    import flockgpu
    L = oracle.L
    for bits in (1, 9, 14):
        c = L.flockref_ch_new(DOM)
        g = flockgpu.Challenger(DOM)
        try:
            L.flockref_ch_label(c, b"grind")
            g.observe_label(b"grind")
            assert g.grind_pow(gpu_ctx, bits) == L.flockref_ch_grind(c, bits)
            assert g.state_digest() == _o_digest(L, c)
        finally:
            L.flockref_ch_free(c)


@pytest.mark.gpu
@pytest.mark.parametrize("m", [22, 24])
def test_pcs_commit_and_open(gpu_ctx, oracle, m):
    import flockgpu
    z = np.random.default_rng(m).integers(0, 2**64, 2 << (m - 7), dtype=np.uint64)
    pd = flockgpu.ProverData(gpu_ctx, z, m)
    try:
        cw = oracle.rs_encode(z, 1 << (m - 13), 64, 1)
        n_leaves = 1 << (m - 12)
        tree = oracle.merkle_tree(cw.view(np.uint8), n_leaves, 1024)
        assert pd.root == tree[-32:].tobytes()
        pos = np.array(sorted(set(np.random.default_rng(1).integers(0, n_leaves, 150).tolist())), np.uint64)
        rows, proof = pd.open(pos)
        assert np.array_equal(rows.reshape(pos.size, 128), cw.reshape(n_leaves, 128)[pos.astype(np.int64)])
        want = np.zeros((64 * pos.size, 32), np.uint8)
        k = oracle.L.flockref_merkle_multi_proof(ctypes.c_void_p(tree.ctypes.data), n_leaves,
                                                 ctypes.c_void_p(pos.ctypes.data), pos.size,
                                                 ctypes.c_void_p(want.ctypes.data), want.shape[0])
        assert proof.shape[0] == k and np.array_equal(proof, want[:k])
        with pytest.raises(flockgpu.FlockError):
            pd.open(pos[::-1].copy())  # unsorted
    finally:
        pd.close()


@pytest.mark.gpu
def test_pcs_commit_root_is_the_proof_root(gpu_ctx, oracle):
    """Committing the packed witness z of a proof's inputs gives the root the
    proof carries (after the 7-byte FLOCK header)."""
    import flockgpu
    z, _, _ = oracle.witness(9, 31)
    pd = flockgpu.ProverData(gpu_ctx, z, 14 + 9)
    p = flockgpu.Prover(gpu_ctx, 9)
    try:
        assert p.prove_seed(31)[7:39] == pd.root
    finally:
        p.close()
        pd.close()
