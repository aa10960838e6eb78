"""Multi-GPU sweeps: one process per GPU, each sweeping its own slice of the grid.

The points of a sweep are independent (the reference integrates one point per thread with no
exchange between points, gqis/N_Level_Kernel.cu), so a sweep over G GPUs needs no collective on its
data path: rank r sweeps its own rows of the parameter grid and the results are only assembled
where they are needed. A fit over a sharded map adds one all-reduce of its P + 1 loss and gradient
sums per evaluation (``fit_loss_gradient``). The
timing convention of a multi-GPU measurement is the maximum over ranks of each rank's device time.
These helpers work with any torch.distributed backend (``nccl`` on GPUs, ``gloo`` for the CPU tests).
"""

from __future__ import annotations

import numpy as np


def shard_rows(num_rows, world_size, rank):
    """Contiguous ``[begin, end)`` of ``num_rows`` grid rows owned by ``rank`` (sizes differ by <= 1)."""
    if world_size < 1 or not (0 <= rank < world_size):
        raise ValueError("rank must lie in [0, world_size)")
    base, extra = divmod(int(num_rows), int(world_size))
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def weak_axis(full_axis, world_size, rank):
    """The slice of a sweep axis of ``world_size`` equal tiles that ``rank`` sweeps (weak scaling)."""
    full_axis = np.asarray(full_axis)
    if len(full_axis) % world_size:
        raise ValueError("weak scaling needs the axis length to be a multiple of the world size")
    b, e = shard_rows(len(full_axis), world_size, rank)
    return full_axis[b:e]


def _device_for(dist):
    import torch
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(value):
    """Maximum of a float over the ranks of the default process group (the value itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(values):
    """Sum of a small float64 vector over the ranks of the default process group, with one all-reduce
    (the values themselves without a group)."""
    import torch
    import torch.distributed as dist
    vec = np.asarray(values, dtype=np.float64).reshape(-1)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vec
    t = torch.as_tensor(vec, device=_device_for(dist))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def fit_loss_gradient(mean_map, grad_map, data_map):
    """Least-squares fit of a sharded interferogram: each rank passes its rows of the model map
    <O>_avg(theta) (``mean_map``, (rows, ny)), of its gradient d<O>_avg/dtheta (``grad_map``,
    (rows, ny, P), from ``gqis.adjoint``) and of the measured map (``data_map``). Returns
    (loss, dloss/dtheta) of loss = sum over the whole grid of (<O>_avg - data)^2, the same on every
    rank: the P + 1 per-rank sums meet in one all-reduce. Torch tensors (any device) or arrays."""
    def host(x):
        return x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)
    m, g, y = host(mean_map), host(grad_map), host(data_map)
    r = np.real(m).astype(np.float64) - np.real(y).astype(np.float64)
    if g.shape[:2] != r.shape:
        raise ValueError(f"gradient map {g.shape} does not match the model map {r.shape}")
    local = np.concatenate([[np.sum(r * r)], 2.0 * np.einsum("ij,ijk->k", r, np.real(g).astype(np.float64))])
    total = allreduce_sum(local)
    return float(total[0]), total[1:]


def gather_rows(local_map, num_rows):
    """Assemble the full ``(num_rows, ...)`` map on every rank from each rank's ``shard_rows`` slice
    (an all-gather: only for maps that are needed whole, e.g. to fit them)."""
    import torch
    import torch.distributed as dist
    local = np.asarray(local_map)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return local
    ws, dev = dist.get_world_size(), _device_for(dist)
    rows = [shard_rows(num_rows, ws, r) for r in range(ws)]
    width = max(e - b for b, e in rows)
    real = np.iscomplexobj(local)
    buf = np.zeros((width,) + local.shape[1:], dtype=np.complex128 if real else np.float64)
    buf[:len(local)] = local
    t = torch.as_tensor(np.stack([buf.real, buf.imag]) if real else buf[None], device=dev)
    parts = [torch.empty_like(t) for _ in range(ws)]
    dist.all_gather(parts, t)
    out = []
    for (b, e), part in zip(rows, parts):
        p = part.cpu().numpy()
        p = p[0] + 1j * p[1] if real else p[0]
        out.append(p[:e - b])
    return np.concatenate(out).astype(local.dtype, copy=False)
