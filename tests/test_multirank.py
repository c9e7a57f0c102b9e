"""The multi-GPU plumbing on gloo, world size 2, on the CPU: one ensemble
workload (a batch of Helmholtz problems, a serving request stream) is
partitioned across the ranks as whole members balanced by their work,
single-run replicas draw their own workload, the measurement takes the
slowest rank, and the serving statistics cover every rank's requests
(pequod_b200.multirank, as bench.py uses it under torchrun)."""
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
    # One shared serving stream and one shared batch, each rank its share.
    stream = serving_requests(rate=200.0, window=0.25, seed=3)
    my_reqs = multirank.shard(stream, [ii * ii * L * n for _, ii, L, n, _ in stream], rank, w)
    batch = [(ii, jj, L) for ii in (65, 129, 257, 513, 1025) for jj in (65, 257, 1025) for L in (1, 3, 5)]
    my_batch = multirank.shard(batch, [i * j * l for i, j, l in batch], rank, w)
    all_reqs = multirank.gather_lists(dist, my_reqs)
    all_batch = multirank.gather_lists(dist, my_batch)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"slow": slow, "reqs": reqs, "gathered": gathered, "summary": summary, "stream": stream,
                   "my_reqs": my_reqs, "batch": batch, "my_batch": my_batch, "all_reqs": all_reqs,
                   "all_batch": all_batch}, f)
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
    # The shared workloads: every member on exactly one rank, and the union
    # of the ranks' shares is the single-rank workload; loads balanced to
    # within the heaviest member.
    for key, mine, allk, wt in (("stream", "my_reqs", "all_reqs", lambda q: q[1] * q[1] * q[2] * q[3]),
                                ("batch", "my_batch", "all_batch", lambda q: q[0] * q[1] * q[2])):
        whole = [tuple(x) for x in res[0][key]]
        assert [tuple(x) for x in res[1][key]] == whole
        shares = [[tuple(x) for x in r[mine]] for r in res]
        assert not set(shares[0]) & set(shares[1])
        assert sorted(shares[0] + shares[1]) == sorted(whole)
        assert sorted(tuple(x) for x in res[0][allk]) == sorted(whole)
        loads = [sum(wt(q) for q in sh) for sh in shares]
        assert max(loads) <= sum(loads) / world + max(wt(q) for q in whole)
        assert min(loads) > 0
    lat = np.array([e[0] for e in expect])
    s = res[0]["summary"]
    assert s["runs"] == 7
    assert abs(s["p50_s"] - np.percentile(lat, 50)) < 1e-12
    assert abs(s["p99_s"] - np.percentile(lat, 99)) < 1e-12
    assert abs(s["throughput"] - sum(e[1] for e in expect) / max(e[2] for e in expect)) < 1e-9


def test_partition_is_balanced_and_deterministic():
    from pequod_b200 import multirank

    rng = np.random.default_rng(7)
    w = list(rng.integers(1, 1000, 200))
    for world in (1, 2, 3, 8):
        parts = multirank.partition(w, world)
        assert parts == multirank.partition(w, world)
        assert sorted(k for p in parts for k in p) == list(range(len(w)))
        loads = [sum(w[k] for k in p) for p in parts]
        assert max(loads) <= sum(w) / world + max(w)
        if world == 8:  # many light items: close to even
            assert max(loads) / (sum(w) / world) < 1.05
    assert multirank.partition([5.0], 4) == [[0], [], [], []]


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
