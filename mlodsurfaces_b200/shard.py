"""Placement of whole clouds on the GPUs of one node.

The projection shards without any data exchange: a cloud's queries need only
that cloud's tree.  With several resident clouds (the batched and served
forms) each GPU therefore holds whole clouds, and the placement balances the
projection work under each GPU's memory budget.  Every rank computes the same
placement from the same inputs, so no collective is needed to agree on it.
"""
from __future__ import annotations

from typing import Sequence

# Device bytes per point of a resident tree (node records, sorted point
# arrays, per-point areas; about 290 MB for 2M points) and per query of its
# query, point and normal buffers.
TREE_BYTES_PER_POINT = 150
QUERY_BYTES = 36


def cloud_bytes(n_points: int, n_queries: int) -> int:
    """Device memory a resident cloud and its query buffers take."""
    return int(n_points) * TREE_BYTES_PER_POINT + int(n_queries) * QUERY_BYTES


def assign_clouds(work: Sequence[float], nbytes: Sequence[int], n_ranks: int,
                  capacity: int | None = None) -> list[int]:
    """Rank of every cloud: largest work first, each to the rank with the
    least work so far among those with room for it (ties to the lower rank).

    work[i] is cloud i's projection work (e.g. queries x iterations) and
    nbytes[i] its device footprint; capacity bounds the bytes per rank (None:
    unbounded).  The result is deterministic.  Raises ValueError when a cloud
    fits on no rank.  The largest load is at most the mean load plus the
    largest single cloud's work.
    """
    if n_ranks < 1:
        raise ValueError("n_ranks must be at least 1")
    if len(work) != len(nbytes):
        raise ValueError("work and nbytes need one entry per cloud")
    order = sorted(range(len(work)), key=lambda i: (-float(work[i]), i))
    load = [0.0] * n_ranks
    used = [0] * n_ranks
    rank_of = [-1] * len(work)
    for i in order:
        best = -1
        for r in range(n_ranks):
            if capacity is not None and used[r] + int(nbytes[i]) > capacity:
                continue
            if best < 0 or load[r] < load[best]:
                best = r
        if best < 0:
            raise ValueError(f"cloud {i} ({int(nbytes[i])} bytes) fits on no rank within {capacity} bytes")
        rank_of[i] = best
        load[best] += float(work[i])
        used[best] += int(nbytes[i])
    return rank_of
