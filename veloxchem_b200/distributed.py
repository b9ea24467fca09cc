"""Multi-rank Fock builds over torch.distributed.

The reference splits the work items of one build round-robin over MPI ranks
(``CFockDriver::compute(screener, rank, nodes, ...)``,
src/t4c_func/FockDriver.cpp:234-290, ``omp::partition_tasks``,
src/general/OpenMPFunc.hpp:89-112) and sums the partial Fock matrices on the
root (``comm.reduce``, src/pymodule/scfdriver.py:1977).  Here the same split
runs one rank per GPU and the sum is one ``all_reduce`` (NCCL over NVLink for
CUDA tensors, gloo for host arrays) of the nao x nao FP64 partial.

Two partitions of the work items are available (``partition``):

* ``'round_robin'``: the reference's deal, item g to rank g mod nodes (the
  partial matrices are the reference's own rank shares);
* ``'balanced'``: longest-processing-time-first over the items' estimated
  costs (primitive quartets x per-primitive flops of the class, plus the
  per-quartet transform and digestion flops), so that every rank gets about
  the same work; the sum over ranks is the same full build.
"""

import numpy as np

PARTITIONS = {'round_robin': 0, 'balanced': 1}


def group_rank_size(group=None):
    """(rank, size) of the calling process in ``group`` (the default group
    when None), or (0, 1) when torch.distributed is not initialised."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def reduce_fock(partial, group=None):
    """Sum of the per-rank partial Fock matrices, returned on every rank.

    ``partial`` is a NumPy array (reduced with the group's backend on a CPU
    tensor) or a torch tensor (reduced in place on its device)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return partial
    if isinstance(partial, np.ndarray):
        # reduce a copy: the caller's partial matrix stays unchanged; NCCL
        # reduces device tensors only, so the copy goes through the rank's GPU
        t = torch.from_numpy(np.array(partial, dtype=np.float64, copy=True))
        if dist.get_backend(group) == 'nccl':
            t = t.to(torch.device('cuda', torch.cuda.current_device()))
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
            return t.cpu().numpy()
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t.numpy()
    dist.all_reduce(partial, op=dist.ReduceOp.SUM, group=group)
    return partial


def distributed_fock(screener, density, label, exchange_factor, omega, ithreshold, group=None,
                     partition='round_robin'):
    """Full Fock matrix on every rank of ``group``: each rank builds its share
    of the work items (its own rank and the group's size, ``partition`` as in
    the module docstring) on its own GPU, then the shares sum."""
    from .fockdriver import FockDriver
    rank, nodes = group_rank_size(group)
    screener.set_partition(partition)
    try:
        drv = FockDriver((rank, nodes))
        local = drv.compute(screener, density, label, exchange_factor, omega, ithreshold)
    finally:
        screener.set_partition('round_robin')
    full = reduce_fock(local.full_matrix().to_numpy(), group)
    out = density.copy()
    out.zero()
    out.set_values(full)
    return out
