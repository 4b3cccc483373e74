"""Time the reference's OpenMP-backend kernel on the host cores (separate process).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py). Runs in its own interpreter so that
the system OpenMP runtime is loaded (a process that imported torch carries torch's
older bundled libgomp, which lacks symbols the reference build needs).

    python -m oracle.cpu_bench --tag bench_chain_o6_float --case chain_o6 --seconds 8
    python -m oracle.cpu_bench ... --fixed 4096 --steps 5 --warmup 1
Prints one JSON object.
"""
import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
  ap = argparse.ArgumentParser()
  ap.add_argument('--tag', required=True)
  ap.add_argument('--case', required=True)
  ap.add_argument('--seconds', type=float, default=8.0)
  ap.add_argument('--max-elements', type=int, default=200000)
  ap.add_argument('--fixed', type=int, default=0)
  ap.add_argument('--steps', type=int, default=1)
  ap.add_argument('--warmup', type=int, default=1)
  a = ap.parse_args()
  os.environ['OMP_TARGET_OFFLOAD'] = 'DISABLED'  # the CPU baseline never runs on an offload device
  import numpy as np
  from oracle import cases, harness, ref_omp
  rk = ref_omp.RefKernel(a.tag)
  fp = np.float64 if 'double' in a.tag else np.float32
  descrs = cases.build(a.case, cases.ns_from_module('tensorforge_b200'))

  def setup(n):
    lay, mem = harness.make_memory(descrs, n, seed=2, extra_offsets=False, dtype=fp)
    host = {k: v.astype(fp) for k, v in mem.buffers.items()}
    return lay, host, mem.scalars

  def timed(n, reps):
    lay, host, sc = setup(n)
    out = []
    for _ in range(reps):
      t = time.perf_counter()
      rk.run(lay, host, n, scalars=sc)
      out.append(time.perf_counter() - t)
    return out

  timed(64, 1)
  if a.fixed:
    n = a.fixed
    timed(n, a.warmup)
    times = timed(n, a.steps)
  else:
    cal = 512
    rate = cal / min(timed(cal, 2))
    n = int(min(a.max_elements, max(cal, rate * a.seconds)))
    n = (n + 7) // 8 * 8
    times = timed(n, a.steps)
  cores = len(os.sched_getaffinity(0)) if hasattr(os, 'sched_getaffinity') else os.cpu_count()
  med = sorted(times)[len(times) // 2]
  print(json.dumps({'elements': n, 'times': times, 'elements_per_s': n / (sum(times) / len(times)),
                    'median_s': med, 'elements_per_s_median': n / med,
                    'cores': cores, 'omp_threads': os.environ.get('OMP_NUM_THREADS', 'all')}))


if __name__ == '__main__':
  main()
