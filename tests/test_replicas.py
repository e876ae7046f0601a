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
