"""The N > 1 host logic of bench.py on two gloo ranks (CPU): every rank
draws its own seeded workload (weak scaling, no data exchange), the device
time is the max over ranks, the whole-job rate counts every rank's RVEs over
the slowest rank's time, and the reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as tmp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        n, radius, *_ = bench.workload_params(64, bench.rank_seed(rank))
        again, *_ = bench.workload_params(64, bench.rank_seed(rank))
        mine_ms = 100.0 + 50.0 * rank  # stand-in for this rank's device time
        total = bench.max_over_ranks(dist, mine_ms, "cpu")
        sizes = [None] * world
        dist.all_gather_object(sizes, n.tolist())
        q.put((rank, total, sizes, bool(np.array_equal(n, again)),
               bench.whole_job_rate(world, 64, 3, total)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_max_time_and_distinct_workloads():
    world, port = 2, free_port()
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    for rank, total, sizes, det, rate in out:
        assert total == 150.0                      # max over ranks, seen by every rank
        assert det                                 # a rank's workload is reproducible
        assert sizes[0] != sizes[1]                # ranks solve different RVEs
        assert set(sizes[0]) <= {8, 12, 16, 20}
        assert abs(rate - 2 * 64 * 3 / 0.150) < 1e-9


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_line_matches_our_config():
    env = dict(os.environ, RANK="0", WORLD_SIZE="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC
    assert line["unit"] == bench.UNIT and line["higher_is_better"] is True
    assert line["config"]["workload"].startswith("batched tangent: 4096 RVEs per GPU")
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"


def test_reference_arm_samples_the_gpu_arms_rves():
    """The CPU arm and the CPU baseline time RVEs of the GPU arm's own
    workload (same seed, same parameters), not a separate draw."""
    import madmax_b200 as mb
    items = bench.workload_items(64, bench.rank_seed(0))
    descs = bench.workload_descs(mb, 64, bench.rank_seed(0))
    for it, d in zip(items, descs):
        assert it[0] == d.n[0] and it[1] == d.radius
        assert d.E[1] == bench.E_MATRIX * it[2] and (d.nu[0], d.nu[1]) == (it[3], it[4])
    sample = bench.per_size_sample(items, 2)
    assert len(sample) == 8 and sorted({w[0] for w in sample}) == [8, 12, 16, 20]
    assert all(w in items for w in sample)
