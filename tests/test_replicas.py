"""Replica runs (psb_project_b200/replicas.py) on two CPU processes over gloo:
distinct lattice seeds per rank, the max-over-ranks reduction the bench's
timing uses, and a bounded rendezvous when a peer never joins."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

from psb_project_b200 import replicas  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    r = replicas.init("gloo", timeout_s=30)
    try:
        ms = 10.0 + 5.0 * rank          # a per-rank "time"
        out[rank] = (r.seed(2), r.max_over_ranks(ms), r.world)
        r.barrier()
    finally:
        r.close()


def test_two_ranks_seeds_and_max():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    seeds = {out[r][0] for r in range(world)}
    assert seeds == {2, 2 + replicas.SEED_STRIDE}
    assert all(out[r][1] == 15.0 and out[r][2] == world for r in range(world))


def _lonely(port, q):
    os.environ.update({"RANK": "0", "WORLD_SIZE": "2", "LOCAL_RANK": "0", "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    try:
        replicas.init("gloo", timeout_s=3)
        q.put("joined")
    except Exception as ex:       # the missing peer ends the rendezvous with an error
        q.put(type(ex).__name__)


def test_missing_peer_fails_within_the_timeout():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_lonely, args=(_free_port(), q))
    p.start()
    p.join(60)
    if p.is_alive():
        p.kill()
        pytest.fail("rendezvous did not time out")
    assert q.get(timeout=5) != "joined"


def test_single_process_needs_no_group():
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    r = replicas.init("gloo")
    assert r.world == 1 and r.dist is None and r.max_over_ranks(3.5) == 3.5 and r.seed(7) == 7


def test_assign_scenes_balanced_and_complete():
    import psb_project_b200 as P
    sizes = [s.n for s in P.batch_scenes()]
    for world in (1, 2, 4, 8):
        parts = replicas.assign_scenes(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in parts]
        # LPT: no rank exceeds the mean by more than the largest scene
        assert max(loads) - sum(loads) / world <= max(sizes)
        assert max(loads) <= 1.1 * sum(loads) / world or world == 1 or max(loads) - min(loads) <= max(sizes)
    assert replicas.assign_scenes([5, 3, 3, 1], 2) == [[0, 3], [1, 2]]


def _assign_worker(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import psb_project_b200 as P
    r = replicas.init("gloo", timeout_s=30)
    try:
        sizes = [s.n for s in P.batch_scenes()]
        mine = replicas.assign_scenes(sizes, r.world)[r.rank]
        load = sum(sizes[i] for i in mine)
        out[rank] = (tuple(mine), r.max_over_ranks(load))
        r.barrier()
    finally:
        r.close()


def test_two_ranks_split_the_batch():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_assign_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    a, b = set(out[0][0]), set(out[1][0])
    assert not (a & b) and len(a | b) == 64
    assert out[0][1] == out[1][1]
