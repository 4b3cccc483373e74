"""Expand the reference's GEMM YAML test suites into concrete cases (tests/golden/gemm_suites.json).

Usage: python tests/golden/make_gemm_suites.py [reference root]
(default: oracle.ref_omp.REFERENCE_ROOT, i.e. $TFB_REFERENCE_ROOT or the recipe's checkout)

Reads tests/gemms/testsuites/*.yaml of the reference. A value written as a string that
contains "param" and names a list of the suite is a parameter; a suite's cases are the product of its parameter
lists (as the reference's loader enumerates them), deduplicated, and at most 12 per suite
are kept: evenly spaced over the product, so that first and last are included. `beta` is
recorded but has no effect (GemmDescr drops it in the reference and here), and the
`gemm_type` parameter only selects reference code paths, so it is dropped.
"""
import itertools
import json
import os
import sys

import yaml

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
KEEP = 12


def _params(spec):
  names = sorted({v for v in _walk(spec) if isinstance(v, str) and 'param' in v and v in spec})
  return [n for n in names if 'gemm_type' not in n]


def _walk(x):
  if isinstance(x, dict):
    for v in x.values():
      yield from _walk(v)
  elif isinstance(x, list):
    for v in x:
      yield from _walk(v)
  else:
    yield x


def _subst(x, values):
  if isinstance(x, dict):
    return {k: _subst(v, values) for k, v in x.items()}
  if isinstance(x, list):
    return [_subst(v, values) for v in x]
  if isinstance(x, str) and x in values:
    return values[x]
  return x


def _yes(v):
  return v is True or str(v).lower() in ('yes', 'true', '1')


def expand(spec):
  names = _params(spec)
  combos = list(itertools.product(*[spec[n] for n in names])) if names else [()]
  cases, seen = [], set()
  for combo in combos:
    s = _subst(spec, dict(zip(names, combo)))
    case = {'suite': spec['test_base_name'], 'trans_a': _yes(s['trans_a']), 'trans_b': _yes(s['trans_b']),
            'alpha': float(s['alpha']), 'beta': float(s['beta']), 'num_elements': int(s['num_elements']),
            'a': {k: s['matrix_a'][k] for k in ('rows', 'cols', 'addressing', 'bbox')},
            'b': {k: s['matrix_b'][k] for k in ('rows', 'cols', 'addressing', 'bbox')},
            'c': {k: s['matrix_c'][k] for k in ('rows', 'cols', 'addressing', 'bbox')}}
    key = json.dumps(case, sort_keys=True)
    if key not in seen:
      seen.add(key)
      cases.append(case)
  if len(cases) > KEEP:
    step = (len(cases) - 1) / (KEEP - 1)
    cases = [cases[round(i * step)] for i in range(KEEP)]
  return cases


def main():
  from oracle.ref_omp import REFERENCE_ROOT
  root = sys.argv[1] if len(sys.argv) > 1 else REFERENCE_ROOT
  suite_dir = os.path.join(root, 'tests', 'gemms', 'testsuites')
  out = []
  for fn in sorted(os.listdir(suite_dir)):
    with open(os.path.join(suite_dir, fn)) as f:
      doc = yaml.safe_load(f)
    for spec in doc['test_suites']:
      for i, case in enumerate(expand(spec)):
        case['id'] = f'{fn[:-5]}/{spec["test_base_name"]}/{i}'
        out.append(case)
  with open(os.path.join(HERE, 'gemm_suites.json'), 'w') as f:
    json.dump(out, f, indent=0)
  print(len(out), 'cases')


if __name__ == '__main__':
  main()
