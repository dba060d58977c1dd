"""bench.py's multi-rank plumbing on the CPU: two gloo ranks rendezvous the
way torchrun starts them, agree on the max and the sum over ranks (the
device timings and the replicas' work), and the reference arm runs on rank 0
alone while the other rank returns at once without work."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, out_dir):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(ws),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    w, r, local = bench._dist()
    assert (w, r, local) == (ws, rank, rank)
    bench._barrier(w)
    mx = bench._max_over_ranks(w, float(rank + 1))
    sm = bench._sum_over_ranks(w, float(rank + 1))
    res = {"max": mx, "sum": sm}
    if rank != 0:
        class A:
            steps, warmup, gpus = 1, 3, ws
        res["reference_rc"] = bench.run_reference(A, w, rank)
    bench._barrier(w)
    import torch.distributed as dist
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump(res, f)


@pytest.mark.timeout(180)
def test_gpus_flag_starts_the_ranks():
    """`python bench.py --gpus 2` without torchrun starts two ranks itself
    (torch.distributed.run); the line rank 0 prints counts both."""
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dry-run"],
                       capture_output=True, text=True, timeout=170, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["n_gpus"] == 2
    assert lines[0]["ranks_reporting"] == 2
    assert lines[0]["rank_id_sum"] == 1


def test_gpus_flag_must_match_the_ranks():
    """Under a launcher that started fewer ranks than --gpus asks for, the
    run refuses instead of reporting the wrong GPU count."""
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dry-run"],
                       capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 2


@pytest.mark.timeout(120)
def test_two_gloo_ranks(tmp_path):
    ws = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, ws, port, str(tmp_path))) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(100)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    r0 = json.load(open(tmp_path / "r0.json"))
    r1 = json.load(open(tmp_path / "r1.json"))
    assert r0["max"] == r1["max"] == 2.0
    assert r0["sum"] == r1["sum"] == 3.0
    assert r1["reference_rc"] == 0
