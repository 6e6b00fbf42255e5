"""The N>1 path of bench.py (replicas, no data-path collective), run as
two gloo ranks on the CPU: the ranks meet at a barrier, every rank learns
the slowest rank's time, and the whole-job throughput is the rows of all
ranks over that time. Also: a rank other than 0 of the reference arm exits
without work."""
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    from gpudbmetalcodegen_b200 import replicas
    assert replicas.dist_info() == (world, rank, rank)
    pg = replicas.init("gloo", timeout_s=60)
    replicas.barrier(pg)
    # rank r "measured" a step of 1 + r ms and a wall time of 10 - r ms
    step_ms, wall_ms = replicas.max_over_ranks(pg, [1.0 + rank, 10.0 - rank], "cpu")
    rows_per_rank = 1000
    value = rows_per_rank * world / (step_ms / 1e3)
    replicas.barrier(pg)
    replicas.shutdown(pg)
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(f"{step_ms} {wall_ms} {value}\n")


def test_two_gloo_ranks_agree_on_the_slowest_time(tmp_path):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = [open(tmp_path / f"rank{r}.txt").read().split() for r in range(2)]
    for step, wall, value in got:
        assert float(step) == 2.0 and float(wall) == 10.0
        assert float(value) == pytest.approx(2000 / 2e-3)


def test_one_rank_needs_no_process_group(monkeypatch):
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    from gpudbmetalcodegen_b200 import replicas
    assert replicas.init("gloo") is None
    assert replicas.max_over_ranks(None, [3, 4]) == [3.0, 4.0]
    replicas.barrier(None)
    replicas.shutdown(None)


def test_reference_arm_rank_one_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference"], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
