"""Box distribution over ranks (no GPU): LPT balance and a world-size-2 gloo
run of the per-rank logic bench.py uses (own shard, max-over-ranks time)."""
import os
import socket

import pytest

from x3div_b200 import b48_boxes, box_points, shard_boxes


def test_b48_is_seeded_and_from_the_five_shapes():
    a, b = b48_boxes(), b48_boxes()
    assert a == b and len(a) == 48
    assert set(a) <= {(96, 96, 96), (128, 256, 64), (200, 100, 150), (256, 256, 256), (64, 512, 64)}
    assert b48_boxes(seed=7) != a


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_lpt_shards_cover_all_boxes_once_and_balance(world):
    boxes = b48_boxes()
    owned = shard_boxes(boxes, world)
    flat = sorted(i for o in owned for i in o)
    assert flat == list(range(len(boxes)))
    loads = [sum(box_points(boxes[i]) for i in o) for o in owned]
    # LPT: the spread is at most the largest box
    assert max(loads) - min(loads) <= max(box_points(b) for b in boxes)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    boxes = b48_boxes()
    mine = shard_boxes(boxes, world)[rank]
    pts = torch.tensor([float(sum(box_points(boxes[i]) for i in mine))], dtype=torch.float64)
    t = torch.tensor([0.5 + rank], dtype=torch.float64)  # a stand-in elapsed time per rank
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(pts, op=dist.ReduceOp.SUM)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    dist.destroy_process_group()
    q.put((rank, float(t.item()), float(pts.item()), gathered))


def test_two_gloo_ranks_own_disjoint_shards():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    total = sum(box_points(b) for b in b48_boxes())
    for rank, tmax, pts, gathered in res:
        assert tmax == 1.5             # max over ranks
        assert pts == float(total)     # every point owned by exactly one rank
        assert sorted(gathered[0] + gathered[1]) == list(range(48))
        assert not set(gathered[0]) & set(gathered[1])
