"""Runs split over the ranks of a torch.distributed job (one GPU per rank)
where the work partitions without a per-step exchange.

The STDP scale-up (Poisson inputs onto independent LIF outputs, all to all)
shards by output columns: every rank draws the same Poisson spikes (they are
a function of seed, step and index), simulates its own outputs with their
columns of W, and the plastic weights, output spikes and traces are gathered
once at the end.  The reference has no multi-GPU simulation of one network
(its distribution is playdoh's across fits, modelfitting.py:446-518); the
fits themselves are split by modelfitting.distributed_modelfitting.
"""
import numpy as np

__all__ = ["shard_range", "stdp_scaleup_sharded"]


def shard_range(n, rank, world):
    """[lo, hi) of rank `rank` among `world` contiguous near-equal shards."""
    return n * rank // world, n * (rank + 1) // world


def _gather(obj, group):
    import torch.distributed as dist
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, obj, group=group)
    return parts


def stdp_scaleup_sharded(steps, seed=2024, nin=10000, nout=4096, process_group=None, **kw):
    """The STDP scale-up for `steps` steps with the outputs split over the
    ranks; every rank returns the full results: W (nin x nout, the
    connection's dtype), output spikes (steps, indices in 0..nout) in
    (step, index) order, the traces A_pre (the same on every rank) and
    A_post, and the final v of the outputs."""
    import torch.distributed as dist
    from . import workloads
    from .clock import reinit_default_clock
    world = dist.get_world_size(process_group)
    rank = dist.get_rank(process_group)
    lo, hi = shard_range(nout, rank, world)
    reinit_default_clock()
    d = workloads.stdp_scaleup(seed=seed, nin=nin, nout=nout, spike_record=hi - lo, out_range=(lo, hi), **kw)
    d["net"].run(steps * d["outputs"].clock.dt)
    a_pre, a_post = d["stdp"]._traces()
    s, i = d["M"]._record()
    local = {"lo": lo, "W": d["C"]._weights().reshape(nin, hi - lo).copy(), "steps": s.copy(),
             "idx": i.astype(np.int64) + lo, "A_pre": a_pre.copy(), "A_post": a_post.copy(),
             "v": np.array(d["outputs"].v)}
    d["net"]._invalidate()
    parts = sorted(_gather(local, process_group), key=lambda p: p["lo"])
    steps_all = np.concatenate([p["steps"] for p in parts])
    idx_all = np.concatenate([p["idx"] for p in parts])
    order = np.lexsort((idx_all, steps_all))
    return {"W": np.concatenate([p["W"] for p in parts], axis=1), "steps": steps_all[order],
            "idx": idx_all[order], "A_pre": parts[0]["A_pre"],
            "A_post": np.concatenate([p["A_post"] for p in parts]), "v": np.concatenate([p["v"] for p in parts]),
            "world_size": world}
