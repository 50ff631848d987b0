"""The bench's multi-rank plumbing on CPU: two gloo ranks join, agree on the
max-over-ranks time, run distinct snapshots, and the reference arm runs on
rank 0 only."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import bench
import torch.distributed as dist
rank, world, local = bench.dist_setup(2, backend="gloo")
t = bench.max_over_ranks(1.5 * (rank + 1), world)
bench.barrier(world)
print(json.dumps({"rank": rank, "world": world, "local": local, "max": t, "seed": bench.replica_seed(rank),
                  "backend": dist.get_backend()}))
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_max_over_ranks_and_seeds():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(r), WORLD_SIZE="2",
                   LOCAL_RANK=str(r), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    outs.sort(key=lambda d: d["rank"])
    assert [d["rank"] for d in outs] == [0, 1]
    assert all(d["world"] == 2 and d["backend"] == "gloo" for d in outs)
    assert all(d["max"] == 3.0 for d in outs)          # every rank reports the slowest rank's time
    assert outs[0]["seed"] != outs[1]["seed"]          # each rank runs its own snapshot


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    bench.run_reference(bench.parse())                  # returns at once, prints nothing
    assert capsys.readouterr().out == ""


def test_config_names_replicas():
    sys.path.insert(0, ROOT)
    import bench
    args = type("Args", (), {"nx": 512, "log2n": 27, "box": 500.0})()
    c = bench.config_dict(args, 4)
    assert c["parallelism"].startswith("replicas x4")
    assert "512^3" in c["workload"]
