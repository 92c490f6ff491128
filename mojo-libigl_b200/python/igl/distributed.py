"""Multi-GPU winding numbers: one process per GPU, queries sharded.

The path shards without a data-path collective: every rank holds the whole
mesh (a 327,680-face soup is 24 MB) and evaluates a contiguous block of the
queries. Only the results move:

* forward: each rank's W block is gathered where it is needed
  (``gather_w``; all_gather of equal-sized padded blocks);
* adjoint: dL/do stays with the rank that owns the query; dL/dV has a
  contribution from every query, so the ranks' per-vertex partials are summed
  with one all_reduce (FP64, SUM) of nv x 3 values;
* closest points / signed distance (``points_sharded``): each rank queries its
  block of points against its own copy of the tree; the per-point results are
  gathered like W.

The per-rank compute is a callable, so the same host logic runs the CUDA
kernels on GPUs (NCCL) and any CPU evaluator under gloo (the tests).
"""

from __future__ import annotations

import torch
import torch.distributed as dist


def shard(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous block [lo, hi) of n items owned by `rank` (sizes differ by <= 1)."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def gather_w(w_local: torch.Tensor, n: int, group=None) -> torch.Tensor:
    """Concatenate every rank's block (ranks in order) into the full W on all ranks.

    Works for any per-item tensor: the first dimension is the item axis.
    """
    world = dist.get_world_size(group)
    width = -(-n // world)
    padded = torch.zeros((width,) + tuple(w_local.shape[1:]), dtype=w_local.dtype,
                         device=w_local.device)
    padded[: w_local.shape[0]] = w_local
    blocks = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(blocks, padded, group=group)
    out = [blocks[r][: shard(n, r, world)[1] - shard(n, r, world)[0]] for r in range(world)]
    return torch.cat(out)


def forward_sharded(forward, V, F, O, group=None):
    """W for all queries: this rank evaluates its block with forward(V, F, O_block)."""
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    lo, hi = shard(O.shape[0], rank, world)
    return gather_w(forward(V, F, O[lo:hi]), O.shape[0], group)


def backward_sharded(backward, V, F, O, gW, group=None):
    """(dL/dV summed over all ranks, dL/dO of this rank's block, (lo, hi)).

    backward(V, F, O_block, gW_block) -> (dV_partial (nv, 3), dO_block).
    """
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    lo, hi = shard(O.shape[0], rank, world)
    dV, dO = backward(V, F, O[lo:hi], gW[lo:hi])
    dV = dV.to(torch.float64).contiguous()
    dist.all_reduce(dV, op=dist.ReduceOp.SUM, group=group)
    return dV, dO, (lo, hi)


def points_sharded(query, P, group=None):
    """Per-point results for all of P: this rank evaluates query(P_block).

    `query` returns a tuple of tensors whose first dimension is the block's
    points, e.g. DeviceAABB.query -> (sqrd, index, closest) or
    DeviceAABB.signed_distance -> (S, index, closest, W); each is gathered.
    """
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    lo, hi = shard(P.shape[0], rank, world)
    return tuple(gather_w(t, P.shape[0], group) for t in query(P[lo:hi]))


def gpu_forward(V, F, O, precision: str = "mixed"):
    """Per-rank CUDA forward (the default compute for forward_sharded)."""
    from . import autograd as wa

    tri, ld, nf = wa.triangle_soa(V, F)
    if precision == "mixed":
        return wa.forward_mixed(tri, ld, nf, O)
    if wa.use_prepared_fp64(nf, O.shape[0]):
        return wa.forward_fp64_prepared(tri, ld, nf, O)
    return wa.forward_fp64(tri, ld, nf, O)


def gpu_backward(V, F, O, gW):
    """Per-rank CUDA adjoint through the boundary edges (default for backward_sharded)."""
    from . import autograd as wa

    return wa.backward_edges(V, F, O, gW)
