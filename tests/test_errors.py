"""Error paths of the C ABI: bad arguments return FLOCK_ERR_ARG (1), a buffer
that is too small returns FLOCK_ERR_CAPACITY (3) with the needed length, an
unfinished job returns FLOCK_ERR_TIMEOUT (5); nothing unwinds across the ABI
and the context stays usable afterwards.  The reference panics on the same
inputs (blake3.rs:4706 n_blocks == 0, :4846 blocks.len() == n_blocks)."""
import ctypes

import numpy as np
import pytest

ERR_ARG, ERR_CAPACITY, ERR_TIMEOUT = 1, 3, 5


def _lib():
    import flockgpu
    return flockgpu.load()


def test_null_handles_rejected_without_a_device():
    lib = _lib()
    vp = ctypes.c_void_p()
    assert lib.flock_setup_create(None, 10, 1, 0, ctypes.byref(vp)) == ERR_ARG
    assert lib.flock_prove_seed(None, 1, b"x", 1, None, 0, None) == ERR_ARG
    assert lib.flock_merkle_tree(None, None, 1, 64, None) == ERR_ARG
    assert lib.flock_ntt_rs_encode(None, None, 4, 1, 1, None) == ERR_ARG
    assert lib.flock_submit(None, None, None) == ERR_ARG
    assert lib.flock_statement_digest(5, None) == ERR_ARG
    assert lib.flock_host_alloc(0, ctypes.byref(vp)) == ERR_ARG
    # hash chains, the verifier and self-checking serving
    assert lib.flock_prove_chain(None, None, 256, b"x", 1, None, 0, None) == ERR_ARG
    assert lib.flock_chain_blocks(1, None, 4, None) == ERR_ARG
    assert lib.flock_verify(None, b"FLOCK", 5, b"x", 1) == ERR_ARG
    assert lib.flock_serve_verify(None, 1) == ERR_ARG
    assert lib.flock_verify_bundle(None, b"FLOCK", 5, b"x", 1) == ERR_ARG


@pytest.mark.gpu
def test_setup_arguments(gpu_ctx):
    lib = gpu_ctx.lib
    h = ctypes.c_void_p()
    for log2, hash_, prof in ((7, 1, 0), (21, 1, 0), (10, 2, 0), (10, 1, 1)):
        assert lib.flock_setup_create(gpu_ctx.h, log2, hash_, prof, ctypes.byref(h)) == ERR_ARG
        assert b"unsupported setup" in lib.flock_last_error(gpu_ctx.h)


@pytest.mark.gpu
def test_prove_arguments_and_capacity(gpu_ctx):
    import flockgpu
    p = flockgpu.Prover(gpu_ctx, 8)
    try:
        lib = gpu_ctx.lib
        blocks = flockgpu.generate_compressions(8, 3)
        out = np.zeros(1 << 20, np.uint8)
        n = ctypes.c_size_t()
        rc = lib.flock_prove_blocks(p.h, blocks.ctypes.data, 255, b"d", 1, out.ctypes.data, out.size, ctypes.byref(n))
        assert rc == ERR_ARG
        small = np.zeros(100, np.uint8)
        rc = lib.flock_prove_seed(p.h, 3, b"flock-bench-v0", 14, small.ctypes.data, small.size, ctypes.byref(n))
        assert rc == ERR_CAPACITY and n.value > 100
        # the setup and context still work
        assert p.prove_seed(3) == p.prove_blocks(blocks)
    finally:
        p.close()


@pytest.mark.gpu
def test_kernel_entry_arguments(gpu_ctx):
    lib = gpu_ctx.lib
    buf = np.zeros(1 << 16, np.uint64)
    b = buf.ctypes.data
    assert lib.flock_merkle_tree(gpu_ctx.h, b, 3, 64, b) == ERR_ARG      # not a power of two
    assert lib.flock_merkle_tree(gpu_ctx.h, b, 0, 64, b) == ERR_ARG      # empty
    assert lib.flock_merkle_tree(gpu_ctx.h, b, 4, 0, b) == ERR_ARG       # empty leaves
    assert lib.flock_merkle_tree(gpu_ctx.h, b, 4, 20, b) == ERR_ARG      # not a multiple of 16 B
    assert lib.flock_merkle_tree(gpu_ctx.h, b, 4, 1040, b) == ERR_ARG    # more than one chunk
    assert lib.flock_ntt_rs_encode(gpu_ctx.h, b, 4, 3, 1, b) == ERR_ARG  # lanes not a power of two
    assert lib.flock_ntt_rs_encode(gpu_ctx.h, b, 4, 1, 0, b) == ERR_ARG  # rate 1
    assert lib.flock_sumcheck_round(gpu_ctx.h, b, b, 3, b) == ERR_ARG
    assert lib.flock_sumcheck_round3(gpu_ctx.h, b, b, b, 1, None, None, None, b) == ERR_ARG
    assert lib.flock_pow(gpu_ctx.h, b, 41, ctypes.byref(ctypes.c_uint64())) == ERR_ARG
    # still usable
    assert gpu_ctx.f128_mul(np.array([2, 0], np.uint64), np.array([3, 0], np.uint64)).tolist() == [6, 0]


@pytest.mark.gpu
def test_serving_arguments_and_timeout():
    import flockgpu
    ctx = flockgpu.Context(0)
    try:
        lib = ctx.lib
        job = flockgpu.FlockJob(25, 1, None, b"d", 1)
        t = ctypes.c_uint64()
        assert lib.flock_submit(ctx.h, ctypes.byref(job), ctypes.byref(t)) == ERR_ARG
        res = flockgpu.FlockResult(None, 0, 0, 0, 0.0, 0.0, 0.0)
        assert lib.flock_poll(ctx.h, 12345, ctypes.byref(res), 0) == ERR_ARG  # serving not started
        assert lib.flock_serve_verify(ctx.h, 1) == ERR_ARG  # nothing to self-check yet
        ctx.serve_start(1)
        assert lib.flock_serve_verify(ctx.h, 0) == 0
        assert lib.flock_poll(ctx.h, 12345, ctypes.byref(res), 0) == ERR_TIMEOUT  # no such job yet
        assert lib.flock_serve_start(ctx.h, 2) == ERR_ARG  # already started
        jobs = (flockgpu.FlockJob * 1)(flockgpu.FlockJob(8, 1, None, b"d", 1))
        results = (flockgpu.FlockResult * 1)()
        assert lib.flock_prove_batch(ctx.h, jobs, 1, results, 0) == ERR_ARG   # no threads
        assert lib.flock_serve_start(ctx.h, 0) == ERR_ARG
    finally:
        ctx.close()


@pytest.mark.gpu
def test_largest_size_deterministic():
    """2^20 compressions, the largest supported size: two proofs of one seed
    are identical, prove_blocks gives the same bytes, and the proof fits the
    harness's 500,000-byte limit."""
    import flockgpu
    ctx = flockgpu.Context(0)
    try:
        p = flockgpu.Prover(ctx, 20)
        a, b = p.prove_seed(2020), p.prove_seed(2020)
        assert a == b and len(a) <= flockgpu.MAX_PROOF_BYTES
        assert p.prove_blocks(flockgpu.generate_compressions(20, 2020)) == a
        p.close()
    finally:
        ctx.close()


def test_statement_entry_points_reject_null_without_a_device():
    """The SHA-256, Keccak, 3-wide Keccak and degree-4 entry points check
    their handles and sizes before touching a device."""
    lib = _lib()
    vp = ctypes.c_void_p()
    out = np.zeros(32, np.uint8)
    for create in (lib.flock_sha256_setup_create, lib.flock_keccak_setup_create, lib.flock_keccak3_setup_create):
        assert create(None, 256, 1, 0, ctypes.byref(vp)) == ERR_ARG
    assert lib.flock_keccak_prove(None, None, 64, b"x", 1, None, 0, None) == ERR_ARG
    assert lib.flock_keccak_prove_chain(None, None, 64, b"x", 1, None, 0, None) == ERR_ARG
    assert lib.flock_sha256_prove_chain(None, None, 128, b"x", 1, None, 0, None) == ERR_ARG
    assert lib.flock_keccak_verify_bundle(None, b"FLOCK", 5, b"x", 1) == ERR_ARG
    assert lib.flock_keccak3_verify_bundle(None, b"FLOCK", 5, b"x", 1) == ERR_ARG
    assert lib.flock_keccak_chain_states(None, 4, None) == ERR_ARG
    assert lib.flock_sha256_chain_blocks(1, None, 4, None) == ERR_ARG
    assert lib.flock_keccak_bench_inputs(4, 1, None) == ERR_ARG
    # digests: sizes outside the statements' range
    assert lib.flock_keccak_statement_digest(5, out.ctypes.data) == ERR_ARG
    assert lib.flock_keccak3_statement_digest(41, out.ctypes.data) == ERR_ARG
    assert lib.flock_keccak_statement_digest(22, None) == ERR_ARG
    assert lib.flock_zerocheck_round1_deg4(None, None, None, None, None, None, 8, None, None, None) == ERR_ARG
    assert lib.flock_bench_round1_deg4(None, 8, 1, 1, None, None, None) == ERR_ARG


@pytest.mark.gpu
def test_statement_setup_sizes(gpu_ctx):
    """Keccak setups need m = k_log + n_log in 22..34: 33..2^18 permutations
    (one per block), 49..3 * 2^17 (three per block); the degree-4 round 1
    takes m in 6..30."""
    import flockgpu
    lib, h = gpu_ctx.lib, ctypes.c_void_p()
    for n in (0, 32, (1 << 18) + 1):
        assert lib.flock_keccak_setup_create(gpu_ctx.h, n, 1, 0, ctypes.byref(h)) == ERR_ARG, n
    for n in (0, 48, (3 << 17) + 1):
        assert lib.flock_keccak3_setup_create(gpu_ctx.h, n, 1, 0, ctypes.byref(h)) == ERR_ARG, n
    assert lib.flock_keccak_setup_create(gpu_ctx.h, 64, 2, 0, ctypes.byref(h)) == ERR_ARG  # unknown Merkle hash
    v = np.zeros(8, np.uint64)
    r = np.zeros((40, 2), np.uint64)
    pa, pz = np.zeros((192, 2), np.uint64), np.zeros((192, 2), np.uint64)
    for m in (5, 31):
        rc = lib.flock_zerocheck_round1_deg4(gpu_ctx.h, *[v.ctypes.data] * 5, m, r.ctypes.data, pa.ctypes.data,
                                             pz.ctypes.data)
        assert rc == ERR_ARG, m
    # a chain must fill its setup: 100 states in a 128-slot setup
    p = flockgpu.KeccakProver(gpu_ctx, 100)
    try:
        with pytest.raises(flockgpu.FlockError):
            p.prove_chain(flockgpu.keccak_chain_states(100))
        # the setup still proves
        assert p.verify(p.prove_seed(3)) == ""
    finally:
        p.close()
