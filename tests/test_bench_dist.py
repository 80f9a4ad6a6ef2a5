"""The N > 1 plumbing of bench.py on CPU: two ranks over gloo run the same
init / barrier / max-over-ranks aggregation the GPU ranks run over NCCL
(replicas only: no data-path collective)."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]

RANK_SCRIPT = r"""
import json, os, sys
sys.path.insert(0, sys.argv[1])
import bench
world, rank, local = bench.dist_setup()
bench.barrier(world)
local_ms = 100.0 + 50.0 * rank          # rank 1 is the slower replica
value, max_ms = bench.aggregate(local_ms, world, 10, 4)
seeds = bench.rank_seed_base(rank)
print(json.dumps({"rank": rank, "world": world, "value": value, "max_ms": max_ms, "seed_base": seeds}), flush=True)
import torch.distributed as dist
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_gloo_aggregation(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(RANK_SCRIPT)
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), FLOCK_DIST_BACKEND="gloo")
        procs.append(subprocess.Popen([sys.executable, str(script), str(REPO)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["world"] == 2
        assert o["max_ms"] == 150.0                      # max over ranks, on every rank
        assert abs(o["value"] - (1 << 10) * 4 * 2 / 0.150) < 1e-6
    assert outs[0]["seed_base"] != outs[1]["seed_base"]  # replicas prove different inputs
