"""Tuning run: build and time every variant of N random chains, then train and score the
cost model on a held-out split.

    python -m tensorforge_b200.tune.run --chains 2000 --jobs 32 --time-limit 1800 --out DIR

Chain libraries are compiled by a pool of `--jobs` worker processes (spawn start method, so
they never inherit this process's CUDA context) while this process measures finished
libraries on the GPU, in chain order, until `--time-limit` seconds have passed. Per-chain
timings are cached in DIR/cache; a rerun with the same DIR resumes and does not compile the
cached chains again. Chains are split by a multiplicative hash of their index into training
(80 %) and test sets; the cost model is trained on the training chains by the CUDA MLP
kernels and scored on the test chains:

  regret(pick) = (measured time of pick - exhaustive best) / exhaustive best

for the model's top-1, the best measured of its top-5 and the planner default. Writes
DIR/dataset.npz, DIR/model.npz and DIR/summary.json and prints the summary.
"""
import argparse
import concurrent.futures as cf
import json
import math
import multiprocessing as mp
import os
import time

import numpy as np


def _build(spec, kcache, compile=True):
  if kcache:
    os.environ['TFB_KCACHE'] = kcache
  from .autotune import build_chain
  t = time.time()
  cb = build_chain(spec, compile=compile)
  return cb, time.time() - t


def is_test_chain(index):
  """Deterministic 20 % held-out split of chain indices."""
  return (index * 2654435761) % 1000 < 200


def collect(specs, jobs, time_limit, out, kcache=None, keep_libs=False, log=print):
  """Build (pool) and measure (this process) chains; returns the measured records."""
  from .autotune import measure_chain, is_cached, gpu_signature
  t0 = time.time()
  ctx = mp.get_context('spawn')
  records = []
  cache = os.path.join(out, 'cache')
  sig = gpu_signature()
  pool = cf.ProcessPoolExecutor(max_workers=jobs, mp_context=ctx)
  # chains with cached timings are not compiled again (their records are still generated)
  futs = [pool.submit(_build, s, kcache, not is_cached(cache, s, sig)) for s in specs]
  build_s = []
  try:
    for i, f in enumerate(futs):
      left = time_limit - (time.time() - t0)
      if left <= 0:
        break
      try:
        cb, bt = f.result(timeout=left)
      except cf.TimeoutError:
        break
      except Exception as e:  # a chain that does not generate or compile is reported and skipped
        log(f'chain {specs[i].index}: build failed: {str(e).splitlines()[0][:200]}')
        continue
      if cb.so_path is not None:
        build_s.append(bt)
      try:
        res = measure_chain(cb, cache=cache)
      except Exception as e:  # the planner default itself failed to launch
        log(f'chain {specs[i].index}: measurement failed: {str(e).splitlines()[0][:200]}')
        continue
      records.append((cb, res))
      if not keep_libs and kcache and cb.so_path is not None:
        try:
          os.remove(cb.so_path)
        except OSError:
          pass
      if len(records) % 25 == 0:
        log(f'{len(records)} chains measured, {time.time() - t0:.0f} s')
  finally:
    pool.shutdown(wait=False, cancel_futures=True)
  return records, build_s


def dataset(records):
  X, y, chain, var, ok, default = [], [], [], [], [], []
  for cb, res in records:
    for j, (f, r) in enumerate(zip(cb.feats, res)):
      X.append(f)
      y.append(math.log(max(r['ms'], 1e-4)))
      chain.append(cb.spec.index)
      var.append(j)
      ok.append(r['ok'])
      default.append(j == cb.default)
  return (np.array(X, np.float32), np.array(y, np.float32), np.array(chain), np.array(var),
          np.array(ok), np.array(default))


def score(model, records, k=5):
  """Per-test-chain regrets of model top-1, model top-k and the planner default."""
  from .cost_model import top_k, regret
  rows = []
  for cb, res in records:
    if not is_test_chain(cb.spec.index):
      continue
    idx = [j for j, r in enumerate(res) if r['ok']]
    if len(idx) < 2:
      continue
    ms = [res[j]['ms'] for j in idx]
    pred = model.predict([cb.feats[j] for j in idx])
    picks = top_k(pred, k)
    d = idx.index(cb.default) if cb.default in idx else None
    rows.append({'chain': cb.spec.index, 'variants': len(idx),
                 'top1': regret(ms, picks[:1]), f'top{k}': regret(ms, picks),
                 'default': regret(ms, [d]) if d is not None else None})
  return rows


def summarise(rows, k=5):
  def stats(key):
    v = np.array([r[key] for r in rows if r[key] is not None])
    if len(v) == 0:
      return None
    return {'mean': float(v.mean()), 'median': float(np.median(v)), 'p90': float(np.percentile(v, 90)),
            'within_10pct': float((v <= 0.10).mean()), 'n': int(len(v))}
  return {'top1': stats('top1'), f'top{k}': stats(f'top{k}'), 'default': stats('default')}


def main(argv=None):
  ap = argparse.ArgumentParser()
  ap.add_argument('--chains', type=int, default=2000)
  ap.add_argument('--seed', type=int, default=0)
  ap.add_argument('--jobs', type=int, default=max(1, (os.cpu_count() or 2) - 1))
  ap.add_argument('--time-limit', type=float, default=1800)
  ap.add_argument('--out', default='tune_out')
  ap.add_argument('--kcache', default=None, help='kernel build cache for the tuning libraries')
  ap.add_argument('--steps', type=int, default=4000)
  ap.add_argument('--keep-libs', action='store_true')
  a = ap.parse_args(argv)
  from .chains import random_chains
  os.makedirs(a.out, exist_ok=True)
  specs = random_chains(a.chains, seed=a.seed)
  t0 = time.time()
  records, build_s = collect(specs, a.jobs, a.time_limit, a.out, a.kcache, a.keep_libs)
  collect_s = time.time() - t0
  X, y, chain, var, ok, default = dataset(records)
  np.savez(os.path.join(a.out, 'dataset.npz'), X=X, y=y, chain=chain, variant=var, ok=ok, default=default)
  from .cost_model import CostModel
  train = np.array([not is_test_chain(c) for c in chain]) & ok
  model = CostModel(seed=a.seed)
  t1 = time.time()
  hist = model.fit(X[train], y[train], steps=a.steps)
  fit_s = time.time() - t1
  model.save(os.path.join(a.out, 'model.npz'))
  rows = score(model, records)
  test = np.array([is_test_chain(c) for c in chain]) & ok
  pred = model.predict(X[test]) if test.any() else np.zeros(0)
  summary = {
    'chains_requested': a.chains, 'chains_measured': len(records), 'jobs': a.jobs,
    'cpu_count': os.cpu_count(), 'collect_s': collect_s, 'build_s_mean': float(np.mean(build_s)) if build_s else None,
    'variants_measured': int(len(y)), 'variants_failed_check': int((~ok).sum()),
    'train_rows': int(train.sum()), 'test_rows': int(test.sum()), 'fit_s': fit_s,
    'loss_first': hist[0][1] if hist else None, 'loss_last': hist[-1][1] if hist else None,
    'test_rmse_log': float(np.sqrt(np.mean((pred - y[test]) ** 2))) if test.any() else None,
    'regret': summarise(rows), 'test_chains': len(rows),
  }
  with open(os.path.join(a.out, 'summary.json'), 'w') as f:
    json.dump({'summary': summary, 'per_chain': rows, 'loss_history': hist}, f, indent=1)
  print(json.dumps(summary))


if __name__ == '__main__':
  main()
