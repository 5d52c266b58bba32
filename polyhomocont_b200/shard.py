"""Path sharding across GPUs (one process per GPU).

Paths of one system are independent (src/solve.f90:190-208), so a solve
splits into contiguous path ranges, one per rank, with no collective on the
data path: each rank tracks its range on its own GPU, the per-path records
are gathered to rank 0 in global path order, and rank 0 runs the
order-dependent host bookkeeping (phc_finish_solve), which makes the result
identical to a single-GPU solve.
"""
import numpy as np


def path_range(npaths, rank, world):
    """Contiguous, balanced 1-based range (k0, count) of rank's paths."""
    base, extra = divmod(int(npaths), int(world))
    count = base + (1 if rank < extra else 0)
    k0 = 1 + rank * base + min(rank, extra)
    return k0, count


def finish_solve(n, paths, x, options=None):
    """Host bookkeeping on gathered records (phc_finish_solve)."""
    from . import result_from_arrays
    return result_from_arrays(n, paths, x, options)


class ShardFailure(RuntimeError):
    """A rank could not track its path range; raised on every rank that
    reaches the gather (rank 0 names the failed ranks)."""


def solve_sharded(sys, rank, world, group=None, options=None, gpu=None, runner=None,
                  npaths=None):
    """solve() over `world` ranks. runner(k0, count) -> (paths, z, x) tracks a
    path range; by default the GPU (phc_solve_paths on this rank's device).
    npaths: solve only the first npaths paths (default: all of them).
    Returns the SolveResult on rank 0 and None elsewhere. With world == 1
    no process group is needed.

    Failure handling: a rank whose tracking raises still takes part in the
    gather, with an error record instead of its paths, so rank 0 learns at
    once which ranks failed and raises ShardFailure, and the failed rank
    re-raises its own error. A rank that dies outright leaves the gather to
    the process group's timeout, which ends it with an error on the others."""
    from . import default_gpu_options, default_options, solve_paths
    o = options if options is not None else default_options()
    npaths = sys.bezout() if npaths is None else int(npaths)
    n = sys.nvars()
    k0, count = path_range(npaths, rank, world)
    err = None
    try:
        if runner is None:
            g = gpu if gpu is not None else default_gpu_options(device=rank)
            paths, z, x, st = solve_paths(sys, o, g, k0=k0, count=count)
            if st != 0:
                raise RuntimeError(f"solve_paths on rank {rank}: status {st}")
        else:
            paths, z, x = runner(k0, count)
        mine = (k0, np.asarray(paths), np.asarray(z), np.asarray(x))
    except Exception as e:  # reported through the gather, re-raised below
        err = e
        mine = (k0, None, None, f"{type(e).__name__}: {e}")
    if world == 1:
        parts = [mine]
    else:
        import torch.distributed as dist
        parts = [None] * world if rank == 0 else None
        dist.gather_object(mine, parts, dst=0, group=group)
    if err is not None:
        raise ShardFailure(f"rank {rank} failed to track paths {k0}..{k0 + count - 1}") from err
    if rank != 0:
        return None
    failed = [(r, p[3]) for r, p in enumerate(parts) if p[1] is None]
    if failed:
        raise ShardFailure("ranks failed: " + "; ".join(f"{r}: {m}" for r, m in failed))
    parts.sort(key=lambda p: p[0])
    paths = np.concatenate([p[1] for p in parts])
    z = np.concatenate([p[2] for p in parts])
    x = np.concatenate([p[3] for p in parts])
    res = finish_solve(n, paths, x, o)
    res.z = z
    return res
