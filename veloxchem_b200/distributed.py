"""Multi-rank Fock builds over torch.distributed.

The reference splits the work items of one build round-robin over MPI ranks
(``CFockDriver::compute(screener, rank, nodes, ...)``,
src/t4c_func/FockDriver.cpp:234-290) and sums the partial Fock matrices on the
root (``comm.reduce``, src/pymodule/scfdriver.py:1977).  Here the same split
runs one rank per GPU and the sum is one ``all_reduce`` (NCCL over NVLink for
CUDA tensors, gloo for host arrays) of the nao x nao FP64 partial.
"""

import numpy as np


def reduce_fock(partial, group=None):
    """Sum of the per-rank partial Fock matrices, returned on every rank.

    ``partial`` is a NumPy array (reduced with the group's backend on a CPU
    tensor) or a torch tensor (reduced in place on its device)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return partial
    if isinstance(partial, np.ndarray):
        # reduce a copy: the caller's partial matrix stays unchanged
        t = torch.from_numpy(np.array(partial, dtype=np.float64, copy=True))
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t.numpy()
    dist.all_reduce(partial, op=dist.ReduceOp.SUM, group=group)
    return partial


def distributed_fock(screener, density, label, exchange_factor, omega, ithreshold, group=None):
    """Full Fock matrix on every rank of ``group``: each rank builds its share
    of the work items (rank/nodes split) on its own GPU, then the shares sum."""
    import torch.distributed as dist
    from .fockdriver import FockDriver
    drv = FockDriver(group if dist.is_initialized() else None)
    local = drv.compute(screener, density, label, exchange_factor, omega, ithreshold)
    full = reduce_fock(local.full_matrix().to_numpy(), group)
    out = density.copy()
    out.zero()
    out.set_values(full)
    return out
