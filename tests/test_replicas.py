"""The multi-GPU path on CPU: world-size-2 process groups over gloo, as `bench.py --gpus N` runs
them over NCCL. Each rank is an independent replica (its own seed and scene; here the march of
its scene runs on the CPU oracle, so no GPU is needed); the job's throughput is the sum of the
ranks' work over the slowest rank's time. A rank that leaves between steps makes the next
collective (the barrier before the reduction) fail on the other rank with the process group's
error instead of hanging."""
import datetime
import os
import socket

import pytest

WORLD = 2


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, port, mode, q):
    import numpy as np
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=10))
    from turbonerf_b200 import scenes
    from turbonerf_b200.replicas import barrier, job_throughput, replica_seed
    try:
        seed = replica_seed(0x7B0, rank)
        if mode == "leave" and rank == 1:
            q.put((rank, "left"))
            return  # this rank leaves between steps, before the reduction
        import oracle
        sc = scenes.march_scene_single(seed=seed, n_rays=64)
        march = dict(bbox=sc.bbox, cone=sc.cone_angle, dt_min=sc.dt_min, dt_max=sc.dt_max, max_steps=sc.max_steps)
        n_steps, _, _ = oracle.march_count(sc.rays.as_dict(), sc.grid.as_dict(), march)
        samples = int(np.sum(n_steps))
        local_ms = 10.0 * (rank + 1)
        try:
            barrier()
            value, ms, units = job_throughput(local_ms, samples)
            q.put((rank, "ok", seed, samples, value, ms, units))
        except Exception as e:  # noqa: BLE001 - the failure is the result under test
            q.put((rank, "error", type(e).__name__))
    finally:
        if mode != "leave":
            dist.destroy_process_group()


def _run(mode):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, mode, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(WORLD)]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not exit")
    return sorted(out, key=lambda r: r[0])


def test_replicas_sum_work_over_the_slowest_rank():
    r0, r1 = _run("ok")
    assert r0[1] == r1[1] == "ok"
    _, _, seed0, s0, v0, ms0, u0 = r0
    _, _, seed1, s1, v1, ms1, u1 = r1
    assert seed0 == 0x7B0 and seed1 != seed0  # independent replicas
    assert s0 > 0 and s1 > 0 and s0 != s1  # their own scenes
    assert ms0 == ms1 == 20.0  # the slowest rank's time
    assert u0 == u1 == s0 + s1  # all ranks' work
    assert v0 == v1 == pytest.approx((s0 + s1) / 0.020)


def test_a_rank_that_leaves_fails_the_reduction_instead_of_hanging():
    r0, r1 = _run("leave")
    assert r1[1] == "left"
    assert r0[1] == "error"
