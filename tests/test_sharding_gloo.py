"""The multi-rank path on CPU: two gloo ranks each evolve their block of trajectories
(the oracle stands in for the device kernel), all-reduce their sums and take the maximum
of their timings, as bench.py does over NCCL.  The sharded sums must equal one process
running all trajectories, and the blocks of random streams must be disjoint and cover the
single-process ensemble."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from cppqed_b200 import sharding

ARGS = ["--picture", "Sch", "--deltaC", "-1", "--eta", "2", "--kappa", "1", "--cutoff", "12", "--no_quadratures"]
N_PER_RANK = 3
WORLD = 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _block_sums(rank, n):
    """Sum over this rank's trajectories of the final state (real and imaginary parts) and
    the list of streams used."""
    import cppqed_b200 as cqg
    from tests.oracle_lib import Oracle

    model = cqg.Model("PumpedLossyMode_C++QED", ARGS)
    pars = model.run_pars().mcwf
    orc = Oracle()
    s0 = sharding.first_stream(pars.prng_stream, n, rank)
    acc = np.zeros(2 * model.dim)
    streams = []
    for i in range(n):
        psi = orc.trajectory(model, pars, s0 + i, 0.2, 2)["psi"]
        acc += np.concatenate([psi.real, psi.imag])
        streams.append(s0 + i)
    return acc, streams


def _rank_main(rank, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    try:
        acc, streams = _block_sums(rank, N_PER_RANK)
        total = sharding.allreduce_sum(acc, WORLD)
        slowest = sharding.max_over_ranks([10.0 * (rank + 1)], WORLD)
        out.put((rank, total.tolist(), streams, float(slowest[0])))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_sum_to_the_single_process_ensemble():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    results = [q.get(timeout=300) for _ in range(WORLD)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    single, single_streams = _block_sums(0, WORLD * N_PER_RANK)
    for rank, total, streams, slowest in results:
        assert np.allclose(total, single, rtol=1e-13, atol=1e-14)
        assert slowest == 10.0 * WORLD
    all_streams = results[0][2] + results[1][2]
    assert sorted(all_streams) == single_streams and len(set(all_streams)) == len(all_streams)
