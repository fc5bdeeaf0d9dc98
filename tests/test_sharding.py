"""Multi-process plumbing of the benchmark on CPU (gloo, world size 2): each
rank takes its own contiguous range of Monte-Carlo instances (weak scaling, no
collective on the data path) and the timings are reduced with MAX, the solve
counts with SUM; the ranks' solutions of their ranges, gathered, equal the
single-process batch's.""" 
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


def _worker(rank, world, port, per_rank, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist = bench.Dist(world)
    try:
        nl, inst = bench.workload(per_rank, dist.rank * per_rank)
        t = dist.max(1.0 + rank)          # per-rank device time
        s = dist.sum(10.0 * (rank + 1))   # per-rank solves
        # each rank solves its own range (the CPU restatement stands in for the
        # GPU on a gloo rank): DC of its instances
        from oracle import pyoracle
        pyoracle.build("port")
        v, st = pyoracle.Oracle("port").run_batch(nl, inst, 0, inst.n, n_threads=1,
                                                  linear_solver=pyoracle.LS_SPARSE, polish_max=8)
        conv = dist.sum(float(sum(x["converged"] for x in st)))
        dist.barrier()
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), kp=inst.mos_kp, vto=inst.mos_vto,
                 t=t, s=s, v=v, conv=conv)
    finally:
        dist.close()


@pytest.mark.timeout(300)
def test_two_ranks_shard_instances_and_reduce(tmp_path):
    world, per_rank = 2, 3
    mp.spawn(_worker, args=(world, _free_port(), per_rank, str(tmp_path)), nprocs=world,
             join=True)
    r = [np.load(tmp_path / f"r{k}.npz") for k in range(world)]
    for z in r:
        assert float(z["t"]) == 2.0 and float(z["s"]) == 30.0
    sys.path.insert(0, ROOT)
    from karam_b200 import circuits
    full = circuits.mc_instances(circuits.config2(), world * per_rank)
    got_kp = np.concatenate([z["kp"] for z in r])
    got_vto = np.concatenate([z["vto"] for z in r])
    # the ranks' ranges are disjoint and together equal the single-process batch
    assert np.array_equal(got_kp, full.mos_kp) and np.array_equal(got_vto, full.mos_vto)
    # and so do their solutions
    from oracle import pyoracle
    v_all, st_all = pyoracle.Oracle("port").run_batch(circuits.config2(), full, 0, full.n, n_threads=1,
                                                      linear_solver=pyoracle.LS_SPARSE, polish_max=8)
    assert np.array_equal(np.concatenate([z["v"] for z in r]), v_all)
    assert float(r[0]["conv"]) == sum(x["converged"] for x in st_all)
