"""CPU, world size 2 over gloo: the multi-rank host path of bench.py.  Each
rank runs its own independent system (seed + rank, replicas, no collective on
the data path); the job value is the sum of the ranks' interacting pairs over
the slowest rank's step time (max over ranks).  The per-rank work here is the
CPU oracle, standing in for the GPU step."""
import json
import os
import socket
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


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    for p in (ROOT, os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import torch.distributed as dist

    import bench
    import ljoracle as O

    ws, r = bench.init_dist("gloo")
    assert (ws, r) == (world, rank)
    seed = 1234 + rank
    x, y, z = O.generate_uniform(seed, 20_000)
    g = O.grid_from_box((0, 0, 0), (1, 1, 1), 0.05)
    pairs = O.config_forces(g, O.bin_particles(g, x, y, z), 0.05, want32=False).pairs
    step_ms = 10.0 + 5.0 * rank          # a slower rank 1
    dist.barrier()
    total = bench.allreduce_sum(float(pairs), ws)
    tmax = bench.allreduce_max(step_ms, ws)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"pairs": pairs, "total": total, "tmax": tmax, "value": total / (tmax * 1e-3)}, f)
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_two_ranks_gloo(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert res[0]["pairs"] != res[1]["pairs"]                 # independent systems (seed + rank)
    for r in res:
        assert r["total"] == res[0]["pairs"] + res[1]["pairs"]
        assert r["tmax"] == 15.0                               # the slowest rank sets the time
        assert r["value"] == pytest.approx(r["total"] / 0.015)
