"""bench.py's multi-GPU launch on CPU: `--gpus 2` outside torchrun re-launches
itself as two ranks (torch.distributed.run), and each rank takes its own
batch of cities (weak scaling). `--plan --backend gloo` runs the launch and
the sharding without GPU work and prints every rank's share."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_gpus_two_launches_two_ranks_with_disjoint_batches():
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "MASTER_ADDR",
                                                             "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--backend", "gloo",
                        "--plan", "--batch", "3"], capture_output=True, text=True, timeout=240, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    plan = json.loads(lines[0])["plan"]
    assert plan["world"] == 2 and plan["communicator_size"] == 2
    shares = {p["rank"]: p["seeds"] for p in plan["shares"]}
    assert shares == {0: [500000, 500001, 500002], 1: [500003, 500004, 500005]}


def test_world_size_must_match_gpus():
    env = dict(os.environ, WORLD_SIZE="2", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "4", "--plan"],
                       capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode != 0 and "WORLD_SIZE 2" in (r.stderr + r.stdout)


def test_launch_command_and_seed_assignment():
    sys.path.insert(0, os.path.join(ROOT, "qes-public_b200"))
    from qesb import shard

    cmd = shard.launch_command("py", "b.py", 4, 1234, ["--gpus", "4"])
    assert cmd[:3] == ["py", "-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "127.0.0.1" in cmd and cmd[-3:] == ["b.py", "--gpus", "4"]
    assert shard.rank_seeds(10, 2, 3) == [16, 17]
    with pytest.raises(ValueError):
        shard.rank_seeds(10, 0, 1)
