"""Record what the reference generator does with the GEMM-suite cases this generator rejects.

Usage (reads the reference source tree through oracle.ref_omp.REFERENCE_ROOT):

    python tests/golden/make_suite_reference.py

For every case of gemm_suites.json that tensorforge_b200 rejects at generation, the
reference generator is run (OpenMP backend, oracle/ref_omp.py). If it generates, its kernel
is built and run on the host in a child process over 2 elements whose buffers carry guard
zones of 8,192 values on both sides; the record says what the kernel wrote:
  * `within_box`: entries changed inside the destination's bounding box,
  * `outside_box`: entries changed in the element's data outside the box,
  * `outside_data`: entries changed in the guard zones (outside every element's data),
  * `box_relative_err`: max error of the box entries against the box-relative GEMM
    C_box = alpha * op(A_box) * op(B_box) (None when the box shapes do not match).
Writes suite_reference_behaviour.json next to this file.
"""
import json
import multiprocessing as mp
import os
import sys
import traceback

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
GUARD = 8192
N = 2


class _Lay:
  def __init__(self, name, slot, starts):
    self.name, self.kind, self.slot, self.starts, self.extra_offset = name, 'strided', slot, starts, 0


def _run_case(case, q):
  try:
    from oracle import cases, ref_omp
    tag = 'suite_' + case['id'].replace('/', '_')
    builder = lambda ns: cases.suite_gemm(ns, case['a'], case['b'], case['c'], case['trans_a'],  # noqa: E731
                                          case['trans_b'], case['alpha'])
    try:
      ref_omp.build(tag, builder, 'double')
    except Exception as e:  # the reference generator (or its output) fails
      q.put({'generates': False, 'error': traceback.format_exception_only(type(e), e)[-1].strip()[:200]})
      return
    rk = ref_omp.RefKernel(tag)
    params = [n for t, n in ref_omp.parse_params(rk.header) if '*' in t and n not in ('flags', 'streamPtr')]
    mats = {}
    for t, name in ref_omp.parse_params(rk.header):
      pass
    # operand order of the reference ABI: C (m0), A (m1), B (m2) for GemmDescr
    order = {'m0': case['c'], 'm1': case['a'], 'm2': case['b']}
    rng = np.random.default_rng(3)
    bufs, lays, full = {}, [], {}
    for name in params:
      m = order[name]
      vol = m['rows'] * m['cols']
      full[name] = rng.uniform(-1, 1, 2 * GUARD + N * vol)
      bufs[name] = full[name][GUARD:]
      lays.append(_Lay(name, vol, np.arange(N) * vol))
    before = {k: v.copy() for k, v in full.items()}
    rk.run(lays, bufs, N, scalars={})
    c, a, b = case['c'], case['a'], case['b']
    out = full['m0']
    changed = out != before['m0']
    vol = c['rows'] * c['cols']
    inside = np.zeros_like(changed)
    r0, c0, r1, c1 = c['bbox']
    for e in range(N):
      base = GUARD + e * vol
      for col in range(c0, c1):
        inside[base + col * c['rows'] + r0: base + col * c['rows'] + r1] = True
    data = np.zeros_like(changed)
    data[GUARD:GUARD + N * vol] = True
    rec = {'generates': True, 'kernel': rk.base_name,
           'within_box': int((changed & inside).sum()), 'outside_box': int((changed & data & ~inside).sum()),
           'outside_data': int((changed & ~data).sum()),
           'inputs_changed': int(sum((full[k] != before[k]).sum() for k in full if k != 'm0'))}

    def box(m, buf, e, trans):
      R0, C0, R1, C1 = m['bbox']
      mat = buf[GUARD + e * m['rows'] * m['cols']:][:m['rows'] * m['cols']].reshape(m['cols'], m['rows']).T
      sub = mat[R0:R1, C0:C1]
      return sub.T if trans else sub
    errs = []
    for e in range(N):
      A, B = box(a, before['m1'], e, case['trans_a']), box(b, before['m2'], e, case['trans_b'])
      C = box(c, out, e, False)
      if A.shape[1] != B.shape[0] or C.shape != (A.shape[0], B.shape[1]):
        errs = None
        break
      errs.append(float(np.abs(C - case['alpha'] * (A @ B)).max()))
    rec['box_relative_err'] = None if errs is None else max(errs)
    q.put(rec)
  except Exception as e:
    q.put({'generates': True, 'error': traceback.format_exception_only(type(e), e)[-1].strip()[:200]})


def main():
  from oracle import cases
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.common.exceptions import GenerationError
  from tensorforge_b200.generators.generator import Generator
  suites = json.load(open(os.path.join(HERE, 'gemm_suites.json')))
  ns = cases.ns_from_module('tensorforge_b200')
  out = {}
  ctx = mp.get_context('spawn')
  for case in suites:
    g = Generator(cases.suite_gemm(ns, case['a'], case['b'], case['c'], case['trans_a'], case['trans_b'],
                                   case['alpha']), Context('sm_100a', 'cuda', FloatingPointType.FLOAT, Options()))
    try:
      g.generate()
      continue
    except GenerationError as e:
      ours = str(e).split(' in ')[0].split(' of ')[0][:60]
    q = ctx.Queue()
    p = ctx.Process(target=_run_case, args=(case, q))
    p.start()
    p.join(600)
    if p.is_alive():
      p.kill()
      rec = {'generates': True, 'error': 'timed out'}
    elif p.exitcode != 0:
      rec = {'generates': True, 'error': f'host process died with exit code {p.exitcode}'}
    else:
      rec = q.get()
    rec['ours'] = ours
    out[case['id']] = rec
    print(case['id'], rec, flush=True)
  with open(os.path.join(HERE, 'suite_reference_behaviour.json'), 'w') as f:
    json.dump(out, f, indent=1, sort_keys=True)


if __name__ == '__main__':
  main()
