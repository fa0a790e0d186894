"""Instance sharding across GPUs / processes.

The commit path shards by AIR instance: every instance's LDE + tree is self-contained, and the
only thing ranks exchange is the 32-byte roots — as the reference distributes instances over
MPI processes and GPU streams (common/src/distribution_ctx.rs:55-..., is_my_process_instance
:288; roots gathered by mpi_ctx.rs:248).  Assignment is longest-processing-time-first on the
commit cost NExt * nCols (elements written and hashed).
"""
import heapq


def commit_cost(nbits, nbits_ext, ncols):
    return (1 << nbits_ext) * max(1, ncols)


def assign_instances(shapes, world):
    """shapes: list of (nBits, nBitsExt, nCols); returns the owning rank of each instance."""
    order = sorted(range(len(shapes)), key=lambda i: (-commit_cost(*shapes[i]), i))
    heap = [(0, r) for r in range(world)]
    owner = [0] * len(shapes)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + commit_cost(*shapes[i]), r))
    return owner


def my_instances(shapes, world, rank):
    owner = assign_instances(shapes, world)
    return [i for i, r in enumerate(owner) if r == rank]


def gather_roots(local_roots, n_instances, dist=None):
    """local_roots: {instance: [4 ints]} on this rank -> full list on every rank (all_gather_object)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        parts = [local_roots]
    else:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, local_roots)
    out = [None] * n_instances
    for part in parts:
        for i, root in part.items():
            out[i] = root
    return out
