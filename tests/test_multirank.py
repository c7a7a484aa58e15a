"""The N > 1 bench path (replicas, max over ranks) with two gloo ranks on
the CPU: every rank steps its own case through the CPU oracle, the slowest
rank sets the time, the aggregate counts every rank's cells."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import sys
    import time
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    import oracle as O
    from mortontrie_amr_b200.case import uniform_box_case
    case = uniform_box_case(n=(8, 8, 8))
    oc = O.OracleCase(case)
    bench.barrier(world)
    t0 = time.perf_counter()
    oc.step(2 + 2 * rank)  # rank 1 does more work: it must set the time
    secs = time.perf_counter() - t0
    agg = bench.aggregate_mlups(512, 2, secs, world)
    slowest = bench.max_over_ranks(secs, world)
    out[rank] = (secs, slowest, agg)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_max_over_ranks():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    secs = [out[r][0] for r in range(world)]
    for r in range(world):
        assert out[r][1] == max(secs)
        assert abs(out[r][2] - world * 512 * 2 / max(secs) / 1e6) < 1e-9
