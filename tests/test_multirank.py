"""Multi-process layout (gloo, world size 2, CPU): ranks agree on the deterministic LPT
assignment of independent systems, cover every system exactly once, and the end-of-run
diagnostics gather returns every rank's record."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, costs, out):
    import datetime

    from blitzar_b200 import sharding

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    bins = sharding.lpt_partition(costs, world)
    mine = bins[rank]
    rec = {"rank": rank, "systems": mine, "particles": int(np.sum(np.asarray(costs)[mine])),
           "seconds": 1.0 + 0.1 * rank}
    recs = sharding.gather_diagnostics(rec)
    out[rank] = recs
    dist.barrier()
    dist.destroy_process_group()


def test_lpt_partition_two_ranks():
    rng = np.random.default_rng(5)
    costs = np.exp(rng.uniform(np.log(1024), np.log(65536), 64)).astype(int)
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, costs.tolist(), out), nprocs=world, join=True)
    a, b = out[0], out[1]
    assert a == b  # both ranks hold every rank's record
    systems = sorted(s for r in a for s in r["systems"])
    assert systems == list(range(len(costs)))
    loads = [r["particles"] for r in a]
    assert max(loads) - min(loads) <= costs.max()
    from blitzar_b200 import sharding

    v = sharding.particle_steps_per_second([r["particles"] for r in a], 10, [r["seconds"] for r in a])
    assert abs(v - costs.sum() * 10 / 1.1) < 1e-6 * v


def test_lpt_is_deterministic_and_balanced():
    from blitzar_b200 import sharding

    costs = [7, 7, 6, 5, 4, 3, 2, 1]
    bins = sharding.lpt_partition(costs, 3)
    assert bins == sharding.lpt_partition(costs, 3)
    loads = sharding.partition_loads(costs, bins)
    assert max(loads) <= 13 and sum(loads) == sum(costs)
