"""The multi-GPU path is replicas only: every rank runs its own copy of the
workload (its own replica seeds), and the aggregate is set by the slowest
rank's time.  Checked here with two gloo ranks on the CPU."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist()
    slow = d.max(1.0 + rank)  # per-rank time: the slowest rank's wins
    d.barrier()
    seeds = [bench.c3_seed(k, d.rank) for k in range(4)]
    q.put((d.rank, d.world, slow, seeds))
    d.close()


def test_two_gloo_ranks_replicas_only():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1] and all(g[1] == 2 for g in got)
    assert all(g[2] == 2.0 for g in got)  # max over ranks
    assert not set(got[0][3]) & set(got[1][3])  # each rank its own replicas


def test_plain_launch_with_several_gpus_starts_one_rank_per_gpu():
    sys.path.insert(0, ROOT)
    import bench

    cmd = bench.launch_command(["--gpus", "4", "--steps", "3"], 4, 29533)
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "--master-addr" in cmd and "127.0.0.1" in cmd
    assert cmd[-4:] == ["--gpus", "4", "--steps", "3"] and cmd[-5].endswith("bench.py")


def test_rank_count_must_match_gpus():
    """Two ranks started for --gpus 3: every rank stops before any work, and
    the launcher reports the failure (gloo on the CPU)."""
    import subprocess

    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2", "--master-addr",
           "127.0.0.1", f"--master-port={_free_port()}", os.path.join(ROOT, "bench.py"), "--gpus", "3"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    assert p.returncode != 0
    assert "--gpus 3 but 2 ranks" in p.stdout + p.stderr
