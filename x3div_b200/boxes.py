"""Box sets and their distribution over ranks.

The batching workload is 48 independent periodic boxes whose shapes are drawn,
with a seed, from {96^3, 128x256x64, 200x100x150, 256^3, 64x512x64}.  Boxes
share no data, so on N GPUs each rank sweeps its own subset: the longest-
processing-time rule (largest box first, onto the least-loaded rank) balances
the points per rank, and no collective is needed on the data path.
"""
from __future__ import annotations

import numpy as np

B48_SHAPES = [(96, 96, 96), (128, 256, 64), (200, 100, 150), (256, 256, 256), (64, 512, 64)]


def b48_boxes(seed: int = 48, count: int = 48):
    """The seeded 48-box set: a list of (nx, ny, nz)."""
    rng = np.random.default_rng(seed)
    idx = rng.integers(0, len(B48_SHAPES), size=count)
    return [B48_SHAPES[i] for i in idx]


def box_points(box) -> int:
    return int(box[0]) * int(box[1]) * int(box[2])


def shard_boxes(boxes, world: int):
    """LPT assignment: returns, per rank, the list of box indices it owns."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(boxes)), key=lambda i: (-box_points(boxes[i]), i))
    load = [0] * world
    owned = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owned[r].append(i)
        load[r] += box_points(boxes[i])
    return [sorted(o) for o in owned]
