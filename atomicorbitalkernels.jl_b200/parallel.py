"""Several GPUs, one process per GPU (torch.distributed, NCCL on GPUs).

Every pair of a 2C batch and every point of an orbital evaluation is
independent, so the batch is split contiguously over the ranks:

* forward (batch_overlap, evaluate[_ed]): each rank computes its own slice;
  there is no communication.  Scaling is weak (each rank owns its slice).
* (zeta, D) gradient: the pullback is a sum over the batch, so each rank's
  pullback of its slice is a partial gradient and one all-reduce (SUM) of the
  partials completes it -- 2 * ns*K*NZ (overlap) or 2 * nRad*K*NZ (evaluate)
  values, flattened into one buffer so there is one collective per step.
  The position gradient of evaluate (dX) stays local to its slice.

The reference has no multi-device code; this module is the data-parallel
layer around its single-device API (overlap_2c_grad.jl:296-304,
atomicorbitals.jl:254-267).
"""
import torch
import torch.distributed as dist

from . import orbitals as _orbitals
from . import overlap as _overlap


def shard_bounds(n, rank=None, world=None):
    """[lo, hi) of rank's contiguous share of n items (the first n % world
    ranks take one extra)."""
    if rank is None:
        rank = dist.get_rank() if dist.is_initialized() else 0
    if world is None:
        world = dist.get_world_size() if dist.is_initialized() else 1
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of size {world}")
    base, extra = divmod(int(n), world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard(x, rank=None, world=None, axis=-1):
    """rank's contiguous slice of x along `axis` (the batch axis: last for the
    reference's column-major (3, B) / (N, N, B) arrays)."""
    n = x.shape[axis]
    lo, hi = shard_bounds(n, rank, world)
    idx = [slice(None)] * x.ndim
    idx[axis] = slice(lo, hi)
    return x[tuple(idx)]


def allreduce_sum(tensors, group=None):
    """Sum a list of tensors over the ranks with one collective (flattened into
    one buffer of the first tensor's dtype and device); returns new tensors of
    the input shapes.  Without an initialised process group: the inputs."""
    tensors = list(tensors)
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return tensors
    flat = torch.cat([t.reshape(-1).to(tensors[0].dtype) for t in tensors])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    out, o = [], 0
    for t in tensors:
        out.append(flat[o:o + t.numel()].reshape(t.shape).to(t.dtype))
        o += t.numel()
    return out


def overlap_pullback_ps(dS_local, orb, XA_local, XB_local, ps, st, group=None, pullback=None):
    """(zeta, D) gradient of a sharded 2C batch: the local pullback_ps of this
    rank's slice (dS_local, XA_local, XB_local), summed over the ranks.
    `pullback` replaces the local pullback (same signature and result)."""
    g = (pullback or _overlap.pullback_ps)(dS_local, orb, XA_local, XB_local, ps, st)
    dz, dD = allreduce_sum([g["Rnl"]["zeta"], g["Rnl"]["D"]], group)
    return {"Rnl": {"zeta": dz, "D": dD}, "Ylm": {}}


def evaluate_pullback_ps(dP_local, basis, X_local, ps, st, group=None, pullback=None):
    """(zeta, D) gradient of a sharded orbital evaluation, summed over the
    ranks (the local result's other entries are returned unchanged)."""
    g = (pullback or _orbitals.pullback_ps)(dP_local, basis, X_local, ps, st)
    dz, dD = allreduce_sum([g["Rnl"]["zeta"], g["Rnl"]["D"]], group)
    out = dict(g)
    out["Rnl"] = dict(g["Rnl"], zeta=dz, D=dD)
    return out
