"""bench.py's contract on CPU: the reference arm prints one JSON line with the required keys,
the replica timing takes the maximum over ranks, and the batched sweep's cases are dealt to
ranks without overlap or loss (world size 2, gloo)."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_json_line():
    env = dict(os.environ, OMP_NUM_THREADS="2")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "c1",
                          "--steps", "2", "--warmup", "1"], capture_output=True, text=True, env=env, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "cell-iters/s"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1


def _worker(rank, port, q):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2)
    q.put((rank, bench.max_over_ranks(10.0 + 5.0 * rank, 2)))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    import socket

    with socket.socket() as sck:
        sck.bind(("127.0.0.1", 0))
        return sck.getsockname()[1]


def _run_ranks(target, world=2):
    import torch.multiprocessing as mp

    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=target, args=(r, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    return dict(q.get(timeout=10) for _ in range(world))


def test_replica_time_is_the_max_over_two_gloo_ranks():
    got = _run_ranks(_worker)
    assert got == {0: 15.0, 1: 15.0}
    assert pytest.approx(15.0) == got[0]


def _deal_worker(rank, port, q):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2)
    meshes, _, _ = bench.make_batch_workload(256)
    cells = [m.n_cells for m in meshes]
    mine = bench.deal_cases(cells, 2)[rank]
    shares = [None, None]
    dist.all_gather_object(shares, mine)  # each rank learns the other's share through the group
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, (shares, cells)))


def test_batch_cases_dealt_to_two_gloo_ranks_are_disjoint_complete_and_balanced():
    """The batched sweep's 256 cases dealt to two ranks (greedy, largest first): each rank's
    share, gathered over the process group, is the same on both ranks; the shares are disjoint,
    cover every case, and their cell totals differ by at most the largest case."""
    got = _run_ranks(_deal_worker)
    (s0, cells), (s1, _) = got[0], got[1]
    assert s0 == s1
    a, b = set(s0[0]), set(s0[1])
    assert not (a & b) and a | b == set(range(256)) and len(s0[0]) + len(s0[1]) == 256
    la, lb = sum(cells[i] for i in a), sum(cells[i] for i in b)
    assert abs(la - lb) <= max(cells)
    assert min(len(a), len(b)) > 64  # both ranks get a real share of the sweep
