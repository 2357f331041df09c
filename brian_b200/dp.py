"""Data-parallel training of the proposal network across ranks.

Each rank holds the whole training set (the simulator's (features,
parameters) pairs) and one copy of the network.  Every optimiser step takes
one global batch of the epoch's row order -- the same order on every rank,
drawn from (seed, epoch) -- and rank r computes the mean-loss gradient of its
contiguous share of it; the flat gradients are summed over the ranks by one
all-reduce (NCCL for GPU tensors, gloo for host tensors) and every rank takes
the same Adam step from the sum times 1/ranks, so the copies stay equal.
With one rank the steps are bg_mlp_train's, bit for bit.

A worker adapts one network copy:

    rows                       training-set size
    epoch_order(seed, epoch)   draws the epoch's row order
    step_gradients(batch, row0) -> (mean loss, gradient)
    as_tensor(gradient)        a torch tensor sharing the gradient's memory
    apply_gradients(gradient, lr, scale)

``ProposalWorker`` wraps the engine's network (bg_mlp_*).  There is no
counterpart in the reference (its fitting starts the optimisers from
uniform draws, modelfitting.py:479-516).
"""
import numpy as np

__all__ = ["ProposalWorker", "train_data_parallel"]


class ProposalWorker(object):
    """A worker over an ``MLPHandle`` whose training set is loaded."""

    def __init__(self, handle):
        self.h = handle
        self.rows = handle.rows

    def epoch_order(self, seed, epoch):
        self.h.epoch_order(seed, epoch)

    def step_gradients(self, batch, row0):
        return self.h.step_gradients(batch, row0)

    def as_tensor(self, grad):
        return grad.torch()

    def apply_gradients(self, grad, lr, scale):
        import torch
        # the all-reduce ran on torch's stream; the update runs on the handle's
        torch.cuda.current_stream(grad.device).synchronize()
        self.h.apply_gradients(grad, lr, scale)


def train_data_parallel(worker, epochs, global_batch, lr, seed, group=None):
    """`epochs` passes over the training set in steps of `global_batch`
    rows split evenly over the ranks of `group` (the default process group,
    or a single rank when torch.distributed is not initialised).  Returns the
    mean loss of each epoch over all ranks' steps."""
    import torch
    import torch.distributed as dist
    multi = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if multi else 1
    rank = dist.get_rank(group) if multi else 0
    if global_batch % world:
        raise ValueError("the global batch must split evenly over %d ranks" % world)
    local = global_batch // world
    steps = worker.rows // global_batch
    if steps < 1:
        raise ValueError("training set smaller than one global batch")
    losses = []
    for ep in range(epochs):
        worker.epoch_order(seed, ep)
        total = 0.0
        for s in range(steps):
            loss, grad = worker.step_gradients(local, s * global_batch + rank * local)
            if world > 1:
                dist.all_reduce(worker.as_tensor(grad), op=dist.ReduceOp.SUM, group=group)
            worker.apply_gradients(grad, lr, 1.0 / world)
            total += loss
        mean = torch.tensor([total / steps], dtype=torch.float64)
        if world > 1:
            if dist.get_backend(group) == "nccl":
                mean = mean.cuda()
            dist.all_reduce(mean, op=dist.ReduceOp.SUM, group=group)
        losses.append(float(mean.cpu()[0]) / world)
    return np.array(losses)
