"""Multi-process CPU tests (gloo, world size 2) of the multi-GPU host logic:
scene placement by footprint is identical on every rank and covers every scene
once; the timing reductions take the max and the sum over ranks; and a rank
that dies before a collective makes the survivor's collective fail within the
process group's short timeout instead of hanging."""

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


def _worker(rank, world, port, sizes, mode, out):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    from tessera_b200.replicas import Reducer, my_items, place_by_footprint

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    try:
        if mode == "normal":
            mine = my_items(sizes, world, rank)
            gathered = [None] * world
            dist.all_gather_object(gathered, (rank, mine, place_by_footprint(sizes, world)))
            red = Reducer(world, "cpu")
            out[rank] = dict(gathered=gathered, mx=red.max(10.0 + rank), sm=red.sum(1.5 * (rank + 1)))
            red.barrier()
        else:  # rank 1 leaves between steps; rank 0's next collective must fail, not hang
            red = Reducer(world, "cpu")
            red.sum(1.0)
            if rank == 1:
                out[rank] = dict(left=True)
                os._exit(0)
            try:
                red.sum(2.0)
                out[rank] = dict(error=None)
            except Exception as e:  # gloo reports the lost peer or the timeout
                out[rank] = dict(error=type(e).__name__)
    finally:
        if mode == "normal":
            dist.destroy_process_group()


def _run(mode, sizes):
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, mode, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=60)
        assert not p.is_alive(), "a rank hung"
    return dict(out)


def test_placement_and_reductions_over_two_gloo_ranks():
    rng = np.random.default_rng(0)
    sizes = [float(x) for x in np.exp(rng.uniform(np.log(4096), np.log(262144), size=37))]
    out = _run("normal", sizes)
    assert set(out) == {0, 1}
    g0, g1 = out[0]["gathered"], out[1]["gathered"]
    assert g0 == g1
    owner0, owner1 = g0[0][2], g0[1][2]
    assert owner0 == owner1  # every rank computes the same placement
    mine = {r: items for r, items, _ in g0}
    assert sorted(mine[0] + mine[1]) == list(range(len(sizes)))  # each scene exactly once
    loads = [sum(sizes[i] for i in mine[r]) for r in (0, 1)]
    assert abs(loads[0] - loads[1]) <= max(sizes)  # LPT balance bound
    assert out[0]["mx"] == out[1]["mx"] == 11.0
    assert out[0]["sm"] == out[1]["sm"] == 1.5 + 3.0


def test_a_rank_that_leaves_makes_the_next_collective_fail_not_hang():
    out = _run("leave", [1.0, 2.0])
    assert out[1] == dict(left=True)
    assert out[0]["error"] is not None


def test_placement_single_rank_and_validation():
    from tessera_b200.replicas import Reducer, place_by_footprint

    assert place_by_footprint([3, 1, 2], 1) == [0, 0, 0]
    assert place_by_footprint([5, 4, 3, 3], 2) == [0, 1, 1, 0]
    assert Reducer(1).max(3.5) == 3.5 and Reducer(1).sum(2.0) == 2.0
    with pytest.raises(ValueError):
        place_by_footprint([1.0], 0)
