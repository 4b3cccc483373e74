"""Multi-rank bookkeeping of weak-scaled runs (runtime/ranks.py) with 2 gloo ranks on CPU."""
import os
import socket

import pytest


def _free_port():
  with socket.socket() as s:
    s.bind(('127.0.0.1', 0))
    return s.getsockname()[1]


def _worker(rank, world, port, q):
  os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                    LOCAL_RANK=str(rank))
  from tensorforge_b200.runtime import ranks
  try:
    dist = ranks.init('gloo', timeout_s=30)
    out = {
      'env': ranks.env_rank(),
      'max': ranks.max_over_ranks(1.5 + rank, dist),
      'all_true': ranks.all_ranks(True, dist),
      'one_false': ranks.all_ranks(rank == 0, dist),
      'seed': ranks.rank_seed(1234, rank),
    }
    # the bench's sequence for one timed region: barrier, work, barrier, slowest rank's time
    dist.barrier()
    work = sum(range(10000 * (rank + 1)))  # ranks take different times
    dist.barrier()
    out['timed'] = ranks.max_over_ranks(10.0 * (rank + 1), dist)
    out['rate'] = ranks.aggregate_rate(world, 500000, out['timed'])
    out['work'] = work
    dist.destroy_process_group()
    q.put((rank, out))
  except Exception as e:  # reported to the parent; a rank never hangs the test
    q.put((rank, repr(e)))


def test_two_gloo_ranks_agree():
  import torch.multiprocessing as mp
  ctx = mp.get_context('spawn')
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
  for p in procs:
    p.start()
  results = dict(q.get(timeout=120) for _ in procs)
  for p in procs:
    p.join(timeout=60)
  for r in range(2):
    assert isinstance(results[r], dict), results[r]
    assert results[r]['env'] == (r, 2, r)
    assert results[r]['max'] == 2.5
    assert results[r]['all_true'] is True
    assert results[r]['one_false'] is False
    assert results[r]['timed'] == 20.0
    assert results[r]['rate'] == pytest.approx(2 * 500000 / 0.020)
  assert results[0]['seed'] != results[1]['seed']


def test_single_process_needs_no_group(monkeypatch):
  from tensorforge_b200.runtime import ranks
  for k in ('RANK', 'WORLD_SIZE', 'LOCAL_RANK'):
    monkeypatch.delenv(k, raising=False)
  assert ranks.env_rank() == (0, 1, 0)
  assert ranks.init('gloo') is None
  assert ranks.max_over_ranks(3.0, None) == 3.0
  assert ranks.all_ranks(False, None) is False
  assert ranks.aggregate_rate(1, 1000, 2.0) == pytest.approx(5e5)


def _worker_dies(rank, world, port, q):
  os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                    LOCAL_RANK=str(rank))
  from tensorforge_b200.runtime import ranks
  dist = ranks.init('gloo', timeout_s=5)
  dist.barrier()
  if rank == 1:
    q.put((rank, 'left'))
    q.close()
    q.join_thread()  # the message is out before the process goes
    os._exit(0)  # leaves between steps, with no collective in flight
  try:
    ranks.max_over_ranks(1.0, dist)
    q.put((rank, 'no error'))
  except Exception as e:
    q.put((rank, f'error: {type(e).__name__}'))


def test_a_rank_that_leaves_makes_the_next_collective_fail():
  import torch.multiprocessing as mp
  ctx = mp.get_context('spawn')
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_worker_dies, args=(r, 2, port, q)) for r in range(2)]
  for p in procs:
    p.start()
  results = dict(q.get(timeout=60) for _ in procs)
  for p in procs:
    p.join(timeout=60)
  assert results[1] == 'left'
  assert results[0].startswith('error'), results[0]
