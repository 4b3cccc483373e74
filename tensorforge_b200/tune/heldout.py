"""Held-out checks of the learned cost model against the exhaustive tuner.

`heldout_specs` names chains of the seeded 2,000-chain tuning set that the shipped model
never trained on (the 20 % test split of tune.run); `evaluate` measures every variant of
each chain on the current GPU (the exhaustive tuner's timings) and scores a predictor's
picks:

  regret(pick) = (measured time of pick - measured best) / measured best

for the predictor's top-1, the best measured of its top-k and the planner's own choice
(the method without the learned part).
"""
import time

import numpy as np

from .chains import random_chains
from .run import is_test_chain


def heldout_specs(n=40, total=2000, seed=0):
  """The first `n` test-split chains of random_chains(total, seed)."""
  return [s for s in random_chains(total, seed=seed) if is_test_chain(s.index)][:n]


def small_specs(n, seed, hi=48, max_bytes=16 << 20):
  """A small seeded campaign (sizes up to `hi`, batches capped at `max_bytes` per operand)."""
  return random_chains(n, seed=seed, hi=hi, max_bytes=max_bytes)


_SOURCE_HASH = []


def _package_hash():
  """Hash of the package's Python sources: a cached chain record is valid for one version."""
  import hashlib
  import os
  if not _SOURCE_HASH:
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    h = hashlib.sha1()
    for d, _, files in sorted(os.walk(root)):
      if '_kcache' in d or '__pycache__' in d:
        continue
      for f in sorted(files):
        if f.endswith('.py'):
          with open(os.path.join(d, f), 'rb') as fh:
            h.update(f.encode() + fh.read())
    _SOURCE_HASH.append(h.hexdigest()[:16])
  return _SOURCE_HASH[0]


def _build_cached(spec, flags):
  """build_chain with its record cached beside the library (generating ~20 variants in
  Python costs seconds per chain; the record is keyed by the chain and the package sources)."""
  import hashlib
  import os
  import pickle
  from .autotune import build_chain
  from .variants import space_signature
  from ..runtime.build import CACHE
  key = hashlib.sha1(f'{spec.key()}|{spec.seed}|{space_signature()}|{_package_hash()}|{flags}'.encode()).hexdigest()[:20]
  path = os.path.join(CACHE, f'chain_{key}.pkl')
  if os.path.exists(path):
    with open(path, 'rb') as f:
      cb = pickle.load(f)
    if cb.so_path and os.path.exists(os.path.join(CACHE, os.path.basename(cb.so_path))):
      cb.so_path = os.path.join(CACHE, os.path.basename(cb.so_path))
      return cb
  cb = build_chain(spec, extra_flags=flags)
  os.makedirs(CACHE, exist_ok=True)
  tmp = f'{path}.{os.getpid()}.tmp'
  with open(tmp, 'wb') as f:
    pickle.dump(cb, f)
  os.replace(tmp, path)
  return cb


def build_all(specs, jobs=8):
  """Variant libraries of every chain (host work; nvcc runs in parallel; built without
  line information: they are timed, never profiled)."""
  from concurrent.futures import ThreadPoolExecutor
  from ..runtime.build import NO_LINEINFO
  with ThreadPoolExecutor(max_workers=jobs) as pool:
    return list(pool.map(lambda s: _build_cached(s, (NO_LINEINFO,)), specs))


def measure_all(builds, time_limit=None):
  """[(ChainBuild, results)] for the chains measured within `time_limit` seconds."""
  from .autotune import measure_chain
  t0 = time.time()
  out = []
  for cb in builds:
    if time_limit is not None and time.time() - t0 > time_limit:
      break
    out.append((cb, measure_chain(cb)))
  return out


def score(records, predict, k=5):
  """Per-chain regrets of the predictor's top-1 / top-k and of the planner default."""
  rows = []
  for cb, res in records:
    idx = [j for j, r in enumerate(res) if r['ok']]
    if len(idx) < 2:
      continue
    ms = np.array([res[j]['ms'] for j in idx])
    pred = np.asarray(predict([cb.feats[j] for j in idx]))
    order = list(np.argsort(pred))
    best = ms.min()
    row = {'chain': cb.spec.index, 'variants': len(idx),
           'top1': float(ms[order[0]] / best - 1), f'top{k}': float(ms[order[:k]].min() / best - 1)}
    row['default'] = float(ms[idx.index(cb.default)] / best - 1) if cb.default in idx else None
    rows.append(row)
  return rows


def summary(rows, k=5):
  def stats(key):
    v = np.array([r[key] for r in rows if r[key] is not None])
    if len(v) == 0:
      return None
    return {'mean': float(v.mean()), 'median': float(np.median(v)), 'within_10pct': float((v <= 0.10).mean()),
            'n': int(len(v))}
  return {'chains': len(rows), 'top1': stats('top1'), f'top{k}': stats(f'top{k}'), 'default': stats('default')}
