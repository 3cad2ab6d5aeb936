"""Multi-GPU host logic: the solver path does not shard (one mesh per GPU and
no collective on the data path), so N GPUs run N independent replicas, or a
batch of independent cases split across ranks.  The only collectives are the
timing reduction (max over ranks) and, for split batches, gathering per-case
results on rank 0.  Both work over NCCL (CUDA tensors) and gloo (CPU).
"""
import torch
import torch.distributed as dist


def _device():
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x):
    """The maximum of a host float over all ranks (x itself without a group)."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(ms_local, steps):
    """Whole-job rate of N replicas that each ran `steps` units in ms_local
    device milliseconds: N * steps / max over ranks of the time."""
    ws = dist.get_world_size() if dist.is_initialized() else 1
    ms = max_over_ranks(ms_local)
    return ws * steps / (ms / 1e3), ms


def cases_for_rank(ncases, rank, world_size):
    """Indices of the independent cases rank `rank` solves (round robin)."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("bad rank or world size")
    return list(range(rank, ncases, world_size))


def gather_case_results(local, ncases, rank, world_size):
    """Per-case float results (a dict index -> value on each rank) collected
    into one list on every rank, in case order."""
    if world_size == 1 or not dist.is_initialized():
        return [local[i] for i in range(ncases)]
    t = torch.zeros(ncases, dtype=torch.float64, device=_device())
    for i, v in local.items():
        t[i] = v
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().tolist()
