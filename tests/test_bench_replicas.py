"""The multi-GPU arm of bench.py runs independent replicas (a triangular
solve has no data-path collective); the only cross-rank step is the max of
the ranks' timed totals.  Checked here with world_size 2 over gloo on CPU:
the max-over-ranks throughput, and that the ranks' host analyses of the
same workload give identical plans.  The reference arm runs on rank 0 alone
and prints the contract's line."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)

    def allmax(v):
        t = torch.tensor([v], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # rank r timed 10 solves in (100 + 50 r) ms
    value, ms_per_step = bench.replica_throughput(100.0 + 50.0 * rank, 10, world, allmax)
    q.put((rank, value, ms_per_step))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_throughput_uses_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, ms_per_step in out:
        assert ms_per_step == pytest.approx(15.0)          # slowest rank: 150 ms / 10 solves
        assert value == pytest.approx(2 * 10 * 1000.0 / 150.0)


def _rank_plan(rank, world, port, q):
    # the host side of one replica: the rank's analysis of the bench's small
    # band workload (host-only, no device), digested and gathered over gloo
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    for p in (ROOT, os.path.join(ROOT, "recblock-sptrsv_b200")):
        sys.path.insert(0, p)
    import hashlib

    import bench
    import rbs
    dist.init_process_group("gloo", rank=rank, world_size=world)
    s = bench.make_system("c0", bench.FORWARD)
    plan = rbs.analyse(s["cp"], s["ri"], s["cv"], substitution=bench.FORWARD, lv=-1,
                       opts=rbs.options(host_only=1))
    h = hashlib.sha256()
    for key in ("kernel", "perm", "levelPtr", "recblock_Ptr", "recblock_Index", "recblock_Val", "ca_tab", "lc_tab",
                "block_rows"):
        h.update(key.encode())
        h.update(plan.export(key).tobytes())
    mine = torch.tensor(list(h.digest()), dtype=torch.int64)
    got = [torch.zeros_like(mine) for _ in range(world)]
    dist.all_gather(got, mine)
    q.put((rank, [bytes(t.tolist()).hex() for t in got], int(plan.info().nlevel)))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_build_identical_plans():
    # every rank of `bench.py --gpus N` analyses the same workload for its own
    # GPU; the host analysis is deterministic, so all ranks hold the same
    # plan (same blocks, kernels, layouts) and time the same work
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30000 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_plan, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, digests, nlevel in out:
        assert len(set(digests)) == 1, (rank, digests)
        assert nlevel > 1
    assert out[0][1] == out[1][1]


def test_reference_arm_runs_on_rank0_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    args = type("A", (), {"steps": 1, "warmup": 0, "gpus": 2})()
    bench.run_reference(args)  # returns without work or output on rank 1
    assert capsys.readouterr().out == ""


def test_reference_arm_line_on_rank0():
    # the reference arm's JSON line (host CPU only): the metric of our arm,
    # the CPU configuration it chose, an e2e with no host-device bytes, and
    # the oracle's accuracy on the c1a workload
    import json
    import subprocess
    env = dict(os.environ, RANK="0")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1"], capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    sys.path.insert(0, ROOT)
    import bench
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == "solves/s"
    assert line["value"] > 0 and line["steps"] == 2 and line["warmup"] == 1 and line["higher_is_better"]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == line["value"] and 1 <= cb["cores"] <= bench.cpu_candidates()[-1]
    assert line["e2e"] == {"value": line["value"], "unit": "solves/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["rel_err_vs_x_true"] <= 1e-12


def test_reference_arm_loads_no_library_under_test():
    # the CPU arm builds its inputs with the oracle's generator and solves
    # with the oracle: the only shared object of this repository it maps is
    # oracle/liboracle.so, never recblock-sptrsv_b200/librbs.so
    import subprocess
    code = ("import runpy, sys\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0']\n"
            "runpy.run_path('bench.py', run_name='__main__')\n"
            "maps = open('/proc/self/maps').read().split()\n"
            "print('MAPPED', sorted({w for w in maps if w.endswith('.so') and w.startswith(%r)}))\n" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT,
                         env=dict(os.environ, RANK="0"))
    assert out.returncode == 0, out.stderr[-2000:]
    mapped = eval(out.stdout.strip().splitlines()[-1].split(" ", 1)[1])
    assert mapped == [os.path.join(ROOT, "oracle", "liboracle.so")], mapped
