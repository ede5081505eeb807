"""Data-parallel training of the warm-start network across processes, one per
GPU (torch.distributed; NCCL on GPUs, gloo works for host-side tests).

Every rank runs its own planet, so every rank holds its own training pairs.
A step: each rank accumulates the gradients of `batch` of its pairs
(`unet_accumulate`), the FP32 gradient buffers are summed over the ranks in
place (one all-reduce of the network's 359,761 floats), and every rank
applies the same Adam step with the sum divided by batch x world
(`unet_apply`). Ranks that start from the same `unet_init` seed and the same
output gain therefore keep identical weights. The gain (the RMS of the
stored targets) is agreed first: each rank's mean square is averaged over
the ranks.

The solver argument needs unet_train (0 steps sets the local gain),
unet_info, unet_set_gain, unet_accumulate, unet_grads and unet_apply, as
FluidSolver provides.
"""
import torch
import torch.distributed as dist


def agree_gain(solver, group=None):
    """Set the same output gain on every rank: sqrt of the rank-mean of G^2."""
    solver.unet_train(0, 1, 0.0, 1)                      # 0 steps: sets the local gain from the pairs
    g = float(solver.unet_info()["gain"])
    t = torch.tensor([g * g], dtype=torch.float64, device=_device(solver))
    world = dist.get_world_size(group)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    G = float((t / world).sqrt().item())
    solver.unet_set_gain(G)
    return G


def train_data_parallel(solver, steps, batch=4, lr=1e-3, seed=1, group=None):
    """`steps` synchronous Adam steps of batch x world samples; returns the
    mean loss per sample over all ranks and steps."""
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    total = torch.zeros(1, dtype=torch.float64, device=_device(solver))
    for it in range(steps):
        # distinct draws on every rank and step
        loss = solver.unet_accumulate(batch, (seed * 1000003 + it * world + rank) & 0xffffffff)
        g = solver.unet_grads()
        dist.all_reduce(g, op=dist.ReduceOp.SUM, group=group)
        solver.unet_apply(lr, batch * world)
        total += loss
    dist.all_reduce(total, op=dist.ReduceOp.SUM, group=group)
    return float(total.item()) / max(1, steps * batch * world)


def _device(solver):
    g = solver.unet_grads()
    return g.device
