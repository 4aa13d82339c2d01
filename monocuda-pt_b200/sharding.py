"""How a multi-GPU render splits its work.

Pixels and samples are independent, so each rank renders whole samples of the
full image from its own replica of the scene and BVH: rank r takes the sample
indices [r * (steps + warmup), (r + 1) * (steps + warmup)), the first `steps`
of them timed and the rest as warm-up. With the counter-based RNG a sample's
draws depend only on (seed, pixel, sample index), so the ranks' samples are
distinct and the sum of their accumulation buffers (one all-reduce at the end)
equals one process rendering all of those samples. Nothing else is exchanged.
"""


def sample_ranges(rank, world, steps, warmup):
    """(timed, warm-up) sample-index ranges of one rank."""
    if not 0 <= rank < world:
        raise ValueError("rank %d outside world of %d" % (rank, world))
    if steps < 0 or warmup < 0:
        raise ValueError("negative step count")
    base = rank * (steps + warmup)
    return range(base, base + steps), range(base + steps, base + steps + warmup)


def all_timed_samples(world, steps, warmup):
    """Every timed sample index of the job, in rank order."""
    out = []
    for r in range(world):
        out.extend(sample_ranges(r, world, steps, warmup)[0])
    return out


def reduce_accumulation(acc, world):
    """Sums the ranks' accumulation buffers in place (every rank gets the sum)."""
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(acc)
    return acc
