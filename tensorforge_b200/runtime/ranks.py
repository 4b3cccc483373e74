"""One process per GPU: rank setup and the few collectives a batched run needs.

Elements of a batch are independent, so a multi-GPU run shards elements across ranks with
no data-path collective (weak scaling: every rank owns its own elements and replicated
shared operands). The only cross-rank steps are bookkeeping: agreeing on a decision every
rank must take identically (which variant is timed), barriers around timed regions and
the slowest rank's time. Every rank calls these in the same order.
"""
import datetime
import os


def env_rank():
  """(rank, world size, local rank) from the launcher's environment (1 process: 0, 1, 0)."""
  return (int(os.environ.get('RANK', '0')), int(os.environ.get('WORLD_SIZE', '1')),
          int(os.environ.get('LOCAL_RANK', '0')))


def init(backend='nccl', timeout_s=120):
  """Join the process group (MASTER_ADDR / MASTER_PORT from the environment) with a short
  timeout, so that ranks waiting for a rank that died end with an error instead of
  hanging; returns torch.distributed, or None for a single process."""
  rank, world, local = env_rank()
  if world <= 1:
    return None
  import torch
  import torch.distributed as dist
  if backend == 'nccl':
    torch.cuda.set_device(local)
  dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
  return dist


def _device(dist):
  import torch
  return torch.device('cuda', torch.cuda.current_device()) if dist.get_backend() == 'nccl' else torch.device('cpu')


def max_over_ranks(value, dist):
  """The largest `value` over all ranks (the slowest rank's time for a timed region)."""
  if dist is None:
    return float(value)
  import torch
  t = torch.tensor([float(value)], device=_device(dist), dtype=torch.float64)
  dist.all_reduce(t, op=dist.ReduceOp.MAX)
  return float(t.item())


def all_ranks(flag, dist):
  """True only if `flag` holds on every rank: a decision all ranks then take alike."""
  if dist is None:
    return bool(flag)
  import torch
  t = torch.tensor([1 if flag else 0], device=_device(dist), dtype=torch.int32)
  dist.all_reduce(t, op=dist.ReduceOp.MIN)
  return bool(t.item())


def rank_seed(base, rank):
  """Seed of a rank's synthetic elements: distinct data per rank, reproducible per rank."""
  return base + rank


def aggregate_rate(world, elements_per_rank, ms):
  """Whole-job elements/s of a weak-scaled run timed by the slowest rank."""
  return world * elements_per_rank / (ms / 1e3)
