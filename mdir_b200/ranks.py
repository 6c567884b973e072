"""What ranks exchange when a workload runs on several GPUs (one process a
GPU, torch.distributed; NCCL on the GPUs, gloo in the CPU tests).

The single box does not shard (replicas: each rank its own box, the job's
time the slowest rank's).  Frames do: the batch shares its frames by
bin-packing on atom counts (`batch.shard`) and gathers the per-frame
energies back into frame order; the force-matching gradient sums the
ranks' parameter gradients in f64 (one all-reduce).  MDIR runs frames one
after another in one process (D251) and has no counterpart."""

import numpy as np
import torch
import torch.distributed as dist


def max_over_ranks(value, device=None):
    """The largest of the ranks' values (a float); the value itself with one rank."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_gradients(*tensors):
    """Sums f64 gradient tensors over the ranks in place, flattened into one
    buffer so that the exchange is one all-reduce; returns them."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return tensors
    flat = torch.cat([t.reshape(-1).to(torch.float64) for t in tensors])
    dist.all_reduce(flat)
    at = 0
    for t in tensors:
        k = t.numel()
        t.copy_(flat[at:at + k].reshape(t.shape).to(t.dtype))
        at += k
    return tensors


def gather_frame_values(frames, mine, values):
    """The per-frame values of all ranks in frame order: `mine` are this
    rank's frame numbers, `values` its (len(mine), ...) array."""
    values = np.asarray(values)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        out = np.zeros((frames,) + values.shape[1:], dtype=values.dtype)
        out[np.asarray(mine, dtype=np.int64)] = values
        return out
    got = [None] * dist.get_world_size()
    dist.all_gather_object(got, (list(mine), values.tolist()))
    out = np.zeros((frames,) + values.shape[1:], dtype=values.dtype)
    seen = np.zeros(frames, dtype=bool)
    for frames_r, vals_r in got:
        idx = np.asarray(frames_r, dtype=np.int64)
        if seen[idx].any():
            raise ValueError("a frame evaluated on two ranks")
        seen[idx] = True
        out[idx] = np.asarray(vals_r, dtype=values.dtype).reshape((len(idx),) + values.shape[1:])
    if not seen.all():
        raise ValueError("frames evaluated on no rank")
    return out
