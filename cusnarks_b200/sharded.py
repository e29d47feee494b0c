"""One MSM split across the ranks of a process group (one process per GPU).

The terms of sum_i k_i P_i are independent, so rank r of W takes the contiguous terms
[r*N/W, (r+1)*N/W) (``shard_range``), runs the MSM of its shard on its own GPU, and the W
partial results (one affine point each: 64 B in G1, 128 B in G2) are exchanged with one
all-gather and added on every rank (``cs_point_sum_device``).  The sum of the partial sums is
the MSM of all terms, and affine Montgomery coordinates are unique, so the result is
word-for-word the single-GPU result.  The reference spreads an MSM over GPUs the same way:
round-robin batches with a host-side reduction of the partial points
(src/python/groth_prover.py:1563 findECPointsDispatch, :1462 assignECPvalues).

The exchange moves one point per rank after milliseconds of bucket work, so it is a plain
collective (NCCL on CUDA tensors, or staged through host memory for gloo), not a fused
kernel: there is no compute to overlap it with.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced term range [lo, hi) of `rank` (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the group")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _torch_sync(t: torch.Tensor):
    if t.is_cuda:
        torch.cuda.synchronize(t.device)


def _gather_points(local: torch.Tensor, group=None) -> torch.Tensor:
    """All ranks' partial points, rank order, on local's device."""
    world = dist.get_world_size(group)
    if world == 1:
        return local.reshape(1, -1)
    on_cuda = local.is_cuda and dist.get_backend(group) == "nccl"
    src = local if on_cuda else local.cpu()
    parts = [torch.empty_like(src) for _ in range(world)]
    dist.all_gather(parts, src, group=group)
    return torch.stack(parts).to(local.device)


def sharded_msm(ctx, scalars: torch.Tensor, points: torch.Tensor, ec2: bool = False, group=None,
                window: int = 0) -> torch.Tensor:
    """sum over all ranks of sum_i scalars[i] * points[i], on every rank.

    scalars: this rank's shard, (n_local, 8) int32 words (normal form); points: (n_local, 16)
    G1 or (n_local, 32) G2 affine Montgomery, both on ctx's GPU.  Returns the affine result
    (16 or 32 int32 words) on that GPU.  Every rank must call it (it is a collective).
    """
    pw = 32 if ec2 else 16
    if scalars.shape[0] != points.shape[0] or points.shape[-1] != pw:
        raise ValueError("scalars and points do not match")
    scalars = scalars.contiguous()
    points = points.contiguous()
    local = torch.empty(pw, dtype=torch.int32, device=points.device)
    n = scalars.shape[0]
    _torch_sync(points)  # the context's stream reads what torch's stream wrote
    if n:
        ctx.msm_device(scalars.data_ptr(), points.data_ptr(), n, local.data_ptr(), ec2=ec2, window=window)
        ctx.sync()
    else:  # an empty shard contributes the point at infinity
        local.copy_(infinity(ec2, points.device))
    parts = _gather_points(local, group)
    out = torch.empty(pw, dtype=torch.int32, device=points.device)
    _torch_sync(parts)
    ctx.point_sum_device(parts.data_ptr(), parts.shape[0], out.data_ptr(), ec2=ec2, dims=2)
    ctx.sync()
    return out


_ONE_MONT_Q = (1 << 256) % 21888242871839275222246405745257275088696311157297823662689037894645226208583


def infinity(ec2: bool = False, device=None) -> torch.Tensor:
    """The reference's affine infinity: G1 (0, 1_mont), G2 (0, 0, 1_mont, 0) (int32 words)."""
    w = np.zeros(32 if ec2 else 16, dtype=np.uint32)
    off = 16 if ec2 else 8
    w[off:off + 8] = [(_ONE_MONT_Q >> (32 * k)) & 0xFFFFFFFF for k in range(8)]
    t = torch.from_numpy(w.view(np.int32).copy())
    return t.to(device) if device is not None else t
