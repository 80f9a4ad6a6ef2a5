"""The allocation-free Merkle root entry point, called through the C ABI with
device pointers, against the allocating flock_merkle_tree on the same leaves.

Two calls in a row with different sizes check that the shared fixed device
array carries nothing from one call into the next.  This file is collected
last so that it also runs after every other test in the same process."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FLOCK_ERR_ARG = 1
FLOCK_ERR_CAPACITY = 3


def _root_noalloc(lib, torch, data: np.ndarray, n_leaves: int, leaf_size: int) -> np.ndarray:
    dev = torch.from_numpy(data).to("cuda")
    root = torch.zeros(32, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    rc = lib.flock_merkle_root_noalloc(ctypes.c_void_p(dev.data_ptr()), n_leaves, leaf_size,
                                       ctypes.c_void_p(root.data_ptr()), None)
    assert rc == 0
    torch.cuda.synchronize()
    return root.cpu().numpy()


def test_merkle_root_noalloc_matches_merkle_tree():
    import torch
    import flockgpu
    device = int(os.environ.get("FLOCK_DEVICE", "0"))
    torch.cuda.set_device(device)
    lib = flockgpu.load()
    ctx = flockgpu.Context(device)
    try:
        rng = np.random.default_rng(0x5EED)
        # largest accepted size first, then a smaller tree with wider leaves:
        # the second call's nodes overlap what the first call left behind
        for n_leaves, leaf_size in ((1 << 15, 64), (1 << 10, 1024), (1, 16)):
            data = rng.integers(0, 256, n_leaves * leaf_size, dtype=np.uint8)
            want = ctx.merkle_tree(data, n_leaves, leaf_size)[-32:]
            got = _root_noalloc(lib, torch, data, n_leaves, leaf_size)
            assert np.array_equal(got, want), (n_leaves, leaf_size)

        # sizes beyond the fixed array and malformed leaves are refused before any work
        big = torch.zeros(16, dtype=torch.uint8, device="cuda")
        root = torch.zeros(32, dtype=torch.uint8, device="cuda")
        p, r = ctypes.c_void_p(big.data_ptr()), ctypes.c_void_p(root.data_ptr())
        assert lib.flock_merkle_root_noalloc(p, 1 << 16, 16, r, None) == FLOCK_ERR_CAPACITY
        assert lib.flock_merkle_root_noalloc(p, 3, 16, r, None) == FLOCK_ERR_ARG
        assert lib.flock_merkle_root_noalloc(p, 1, 24, r, None) == FLOCK_ERR_ARG
    finally:
        ctx.close()
