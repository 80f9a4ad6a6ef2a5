"""The process boundary: flock_worker speaks the reference benchmark-worker
protocol (benchmark-tools/worker/src/main.rs:14-49): argv LOG2 READY_PATH
PROOF_PATH, READY after the untimed setup, the decimal seed on stdin, the
proof published by writing PROOF_PATH.tmp and renaming it."""
import subprocess
import time
from pathlib import Path

import pytest

WORKER = Path(__file__).resolve().parents[1] / "flock-challenge-multi_b200" / "flock_worker"


def test_worker_rejects_bad_arguments():
    assert WORKER.exists(), "flock_worker is not built"
    assert subprocess.run([str(WORKER)], capture_output=True).returncode == 2
    assert subprocess.run([str(WORKER), "7", "r", "p"], capture_output=True).returncode == 2
    assert subprocess.run([str(WORKER), "9", "r", "p", "d", "x"], capture_output=True).returncode == 2


@pytest.mark.gpu
def test_worker_protocol_matches_prover(tmp_path):
    import flockgpu
    log2, seed = 9, 424242
    ready, proof, rec = tmp_path / "ready", tmp_path / "proof.bin", tmp_path / "rec"
    rec.mkdir()
    # the optional fourth argument records (seed, proof) for harness runs
    p = subprocess.Popen([str(WORKER), str(log2), str(ready), str(proof), str(rec)], stdin=subprocess.PIPE)
    try:
        t0 = time.time()
        while not ready.exists():
            assert p.poll() is None, "worker exited before READY"
            assert time.time() - t0 < 300
            time.sleep(0.05)
        p.stdin.write(f"{seed}\n".encode())
        p.stdin.close()
        assert p.wait(timeout=300) == 0
    finally:
        if p.poll() is None:
            p.kill()
    assert not (tmp_path / "proof.bin.tmp").exists()
    assert (rec / f"proof_{log2}_{seed}.bin").read_bytes() == proof.read_bytes()
    ctx = flockgpu.Context(0)
    try:
        pr = flockgpu.Prover(ctx, log2)
        try:
            assert proof.read_bytes() == pr.prove_seed(seed)
        finally:
            pr.close()
    finally:
        ctx.close()
