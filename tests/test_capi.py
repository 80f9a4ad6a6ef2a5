"""CPU-side checks of the C ABI library: it loads, exports every symbol the
header declares, and its host-only statement digest matches the oracle's
(BlockR1cs::statement_digest, crates/flock-core/src/r1cs.rs:334-352)."""
import re
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


def header_symbols():
    text = (REPO / "include/flock_gpu.h").read_text()
    return sorted(set(re.findall(r"\b(flock_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    import flockgpu
    lib = flockgpu.load()
    syms = header_symbols()
    assert len(syms) >= 18
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(flockgpu.EXPORTS)


def test_statement_digest_matches_oracle(oracle):
    import flockgpu
    for n_log in (8, 10):
        assert flockgpu.statement_digest(14 + n_log) == oracle.statement_digest(n_log)


def test_no_cpu_fallback_without_gpu():
    import torch
    import flockgpu
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(flockgpu.FlockError):
        flockgpu.Context(0)


def test_ntt_plans_cover_every_pass_kind():
    """The candidate plans of a 64-lane shape include the warp-per-pair table
    passes (and their mix with integer products) beside the thread-per-pair
    passes, so the parity test of every plan covers all three kernels."""
    import flockgpu
    descs = flockgpu.ntt_plan_descs(13, 64, 1)
    assert any("/tab+imad" in d for d in descs)
    assert any("/tab" in d and "/tab+imad" not in d for d in descs)
    assert any("/tab" not in d for d in descs)
    assert not any("/tab" in d for d in flockgpu.ntt_plan_descs(16, 1, 2))  # one lane: no warp tiles
