"""Multi-process path of bench.py on CPU: ranks are independent replicas (the
substep has no data-path collective) and the reported time is the max over
ranks.  Two gloo ranks run the oracle on their own seeded scenes."""
import json
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica(rank, world, port, outdir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    from oracle import zoracle
    from tests.scenes import build_scene
    from ziran2019_b200 import mpm
    sim = mpm.MpmSimulation(1.0 / 64, gravity=(0, -9.8, 0), precision="fp64", lib=zoracle.lib())
    build_scene(sim, kind="fcr", n=4, seed=rank)
    own = []
    for _ in range(2):
        assert sim.advanceOneTimeStep(1e-3) == 0
        own.append(float(sim.last_stats["ms_total"]))
    worst = bench.barrier_max(sum(own), world)
    x = sim.getParticles()["X"]
    json.dump({"own": sum(own), "max": worst, "x": x.tolist()}, open(os.path.join(outdir, f"r{rank}.json"), "w"))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas_report_the_slowest_rank(tmp_path, oracle):
    world = 2
    mp.start_processes(_replica, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    worst = max(r["own"] for r in res)
    assert all(r["max"] == pytest.approx(worst) for r in res)
    # independent replicas: rank 0 reproduces a single-process run of seed 0
    from tests.scenes import build_scene
    from ziran2019_b200 import mpm
    sim = mpm.MpmSimulation(1.0 / 64, gravity=(0, -9.8, 0), precision="fp64", lib=oracle)
    build_scene(sim, kind="fcr", n=4, seed=0)
    for _ in range(2):
        sim.advanceOneTimeStep(1e-3)
    np.testing.assert_array_equal(np.asarray(res[0]["x"]), sim.getParticles()["X"])
    assert not np.array_equal(np.asarray(res[0]["x"]), np.asarray(res[1]["x"]))
