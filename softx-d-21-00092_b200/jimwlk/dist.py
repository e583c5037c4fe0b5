"""Event-sharded runs on several GPUs, one process per GPU.

The events of an ensemble are independent, so each rank evolves its own and
measures them (Engine.measure_ensemble or Engine.step_measure_ensemble).  The
ensemble over all ranks' events is then the sum of the ranks' sums and squared
sums: the statistics reduction of gfield::reduce (field.h:1521-1536) carried
across processes.  This is the only collective of a sharded run.
"""
from __future__ import annotations

import numpy as np


def allreduce_ensemble(sum_h: np.ndarray, err_h: np.ndarray, group=None):
    """Sum the ranks' ensemble fields in place (complex N x N host arrays, as
    returned by measure_ensemble) over the torch.distributed process group.

    With the NCCL backend the arrays travel through the current CUDA device,
    with gloo they stay on the host.  A single process returns them unchanged."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return sum_h, err_h
    nccl = dist.get_backend(group) == "nccl"
    dev = torch.device("cuda", torch.cuda.current_device()) if nccl else torch.device("cpu")
    both = np.stack([np.ascontiguousarray(sum_h), np.ascontiguousarray(err_h)])
    t = torch.view_as_real(torch.from_numpy(both)).to(dev)  # float64 pairs: a plain SUM
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    out = torch.view_as_complex(t.cpu().contiguous()).numpy()
    sum_h[...] = out[0]
    err_h[...] = out[1]
    return sum_h, err_h
