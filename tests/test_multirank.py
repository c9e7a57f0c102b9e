"""The multi-GPU plumbing on gloo, world size 2, on the CPU: each replica
draws its own workload, the measurement takes the slowest rank, and the
serving statistics cover every rank's requests (pequod_b200.multirank, as
bench.py uses it under torchrun)."""
import json
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from pequod_b200 import multirank
    from pequod_b200.workloads import serving_requests

    r, w, lr = multirank.env_ranks()
    assert (r, w, lr) == (rank, world, rank)
    dist = multirank.init(w, backend="gloo", timeout_s=60.0)
    slow = multirank.max_over_ranks(dist, [1.0 + rank, 10.0 - rank])
    reqs = serving_requests(rate=200.0, window=0.05, seed=multirank.rank_seed(3, rank))
    done = [(0.1 * (k + 1) + rank, 1000.0 * (k + 1), 1.0 + k + rank) for k in range(3 + rank)]
    gathered = multirank.gather_lists(dist, done)
    summary = multirank.serving_summary(gathered)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"slow": slow, "reqs": reqs, "gathered": gathered, "summary": summary}, f)
    multirank.close(dist)


def test_two_ranks_on_gloo(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r in res:
        assert r["slow"] == [2.0, 10.0]
    # replicas draw different workloads
    assert res[0]["reqs"] != res[1]["reqs"]
    # both ranks see every request, in rank order, and the same statistics
    expect = [[0.1 * (k + 1) + rank, 1000.0 * (k + 1), 1.0 + k + rank] for rank in range(world)
              for k in range(3 + rank)]
    for r in res:
        assert np.allclose(np.array(r["gathered"]), np.array(expect))
        assert r["summary"] == res[0]["summary"]
    lat = np.array([e[0] for e in expect])
    s = res[0]["summary"]
    assert s["runs"] == 7
    assert abs(s["p50_s"] - np.percentile(lat, 50)) < 1e-12
    assert abs(s["p99_s"] - np.percentile(lat, 99)) < 1e-12
    assert abs(s["throughput"] - sum(e[1] for e in expect) / max(e[2] for e in expect)) < 1e-9


def test_single_rank_needs_no_process_group():
    from pequod_b200 import multirank

    assert multirank.init(1) is None
    assert multirank.max_over_ranks(None, [3.0, 4.0]) == [3.0, 4.0]
    assert multirank.gather_lists(None, [1, 2]) == [1, 2]
    multirank.close(None)


def test_reference_arm_under_torchrun(tmp_path):
    """bench.py --impl reference launched as the driver launches it for N = 2:
    rank 0 alone runs the CPU reference and prints one JSON line; rank 1
    exits 0 without work."""
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(root, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "1", "--size", "129"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
