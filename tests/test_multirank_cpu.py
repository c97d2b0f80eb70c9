"""Multi-rank path of bench.py on CPU (gloo, world size 2).

One run per rank, no data-path collective: the whole-job value is the work of
all ranks over the slowest rank's time.  The ranks here advance independent
oracle runs with different seeds, so the test also shows that runs sharded
over ranks are independent (each rank's result equals the same run done
alone)."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from oracle import oracle as O
        from tests.helpers import small_plasma

        p = O.derive(small_plasma(n=6, ppc=2, seed=100 + rank))
        s = O.OracleState(p)
        s.calc_distance()
        s.initialize()
        work = 0
        for it in range(1, 3):
            s.step(it)
            work += s.num_local
        ms = 10.0 * (rank + 1)  # stand-in device times: rank 1 is the slowest
        ms_max, total = bench.combine_ranks(ms, float(work), dist, "cpu")
        out[rank] = (ms_max, total, float(work), float(s.energy()[0]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_combine_and_stay_independent():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    works = [res[r][2] for r in range(world)]
    for r in range(world):
        ms_max, total, _, _ = res[r]
        assert ms_max == 20.0
        assert total == sum(works)
    # each rank's run equals the same run computed alone
    from oracle import oracle as O
    from tests.helpers import small_plasma

    for r in range(world):
        p = O.derive(small_plasma(n=6, ppc=2, seed=100 + r))
        s = O.OracleState(p)
        s.calc_distance()
        s.initialize()
        for it in range(1, 3):
            s.step(it)
        assert np.isclose(s.energy()[0], res[r][3], rtol=0, atol=0)
