"""One process per GPU: how the views are split and the gradients summed.

The renders of different views are independent given the surfels and the
photon map (views, passes and pixels shard freely).  Every rank holds
the same surfels, traces the same counter-keyed photons (so the photon maps
are bit-identical without an exchange) and renders its own views; the only
exchange is the sum of the per-surfel gradient arrays.

- shard_cameras(names, rank, world): the cameras of one scene split round
  robin over the ranks.  With the setting camera_seeds = "camera" a
  camera's image and gradient do not depend on the other cameras of a call,
  so the ranks' gradients, summed, equal one process rendering every camera.
- view_offset(rank, world): rank r's ring of views rotated by r / world of
  the camera spacing; N rings of C views interleave into the ring of N*C
  views that shard_cameras splits the same way.
- reduce_gradients(grads): sums the gradient arrays of all ranks in place
  with ONE all-reduce over a flat buffer (eight arrays per step would be
  eight latency-bound collectives).
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence

import torch
import torch.distributed as dist


def shard_cameras(names: Sequence[str], rank: int, world: int) -> List[str]:
    """The cameras rank `rank` of `world` renders: every world-th camera from
    position `rank` (round robin, so the views of a ring spread evenly)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return list(names)[rank::world]


def view_offset(rank: int, world: int) -> float:
    """Ring rotation of rank `rank`'s views, as a fraction of the spacing."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return rank / world


def reduce_gradients(grads: Dict[str, torch.Tensor], group: Optional[dist.ProcessGroup] = None,
                     flat: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Sums `grads` (name -> tensor, all on one device, float32) over the
    ranks of `group` in place.  `flat` may be a preallocated buffer of the
    total size; returns the buffer used."""
    keys = sorted(grads)
    total = sum(grads[k].numel() for k in keys)
    if flat is None or flat.numel() < total:
        flat = torch.empty(total, dtype=torch.float32, device=grads[keys[0]].device)
    off = 0
    for k in keys:
        n = grads[k].numel()
        flat[off:off + n].copy_(grads[k].reshape(-1))
        off += n
    dist.all_reduce(flat[:total], op=dist.ReduceOp.SUM, group=group)
    off = 0
    for k in keys:
        n = grads[k].numel()
        grads[k].copy_(flat[off:off + n].view_as(grads[k]))
        off += n
    return flat
