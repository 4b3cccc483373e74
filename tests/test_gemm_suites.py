"""The reference's GEMM YAML suites (expanded into tests/golden/gemm_suites.json): every case
generates, and the FP64 oracle agrees with an independent numpy statement of a GEMM on
bounding boxes (transposes, sub-boxes, leading dimensions, alpha)."""
import json
import os

import numpy as np
import pytest

from oracle import cases, harness, multilinear

HERE = os.path.dirname(os.path.abspath(__file__))
SUITES = json.load(open(os.path.join(HERE, 'golden', 'gemm_suites.json')))


def _build(case, ns_root='tensorforge_b200'):
  ns = cases.ns_from_module(ns_root)
  return cases.suite_gemm(ns, case['a'], case['b'], case['c'], case['trans_a'], case['trans_b'], case['alpha'])


def _ranges(case):
  """Index ranges of m, k, n: intersections of the *operands'* absolute boxes (the reference's
  multilinear semantics, multilinear.py:58-96: the destination's box only places the
  result); a suite written for box-relative GEMMs can have empty ones."""
  def box(m, trans):
    r0, c0, r1, c1 = m['bbox']
    rows, cols = (r0, r1), (c0, c1)
    return (cols, rows) if trans else (rows, cols)
  (am, ak), (bk, bn) = box(case['a'], case['trans_a']), box(case['b'], case['trans_b'])
  inter = lambda *rs: (max(r[0] for r in rs), min(r[1] for r in rs))
  return am, inter(ak, bk), bn


def _reader(buf, start, m, compact):
  """X(r, c) for absolute stored coordinates, addressed as the reference does: the element
  pointer is the box's first entry, the leading dimension the stored row count, or the
  box's for a lead-less, non-transposed operand (read through a compact copy of its box)."""
  r0, c0, r1, _ = m['bbox']
  ld = (r1 - r0) if compact else m['rows']
  return lambda r, c: buf[start + (r - r0) + (c - c0) * ld]


@pytest.mark.parametrize('case', SUITES, ids=[c['id'] for c in SUITES])
def test_suite_case_generates_and_oracle_matches_numpy(case):
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.exceptions import GenerationError
  from tensorforge_b200.generators.generator import Generator
  (m0, m1), (k0, k1), (n0, n1) = _ranges(case)
  g = Generator(_build(case), Context('sm_100a', 'cuda', FloatingPointType.FLOAT, Options()))
  c = case['c']
  fits = (m0 - c['bbox'][0] >= 0 and m1 - c['bbox'][0] <= c['rows'] and
          n0 - c['bbox'][1] >= 0 and n1 - c['bbox'][1] <= c['cols'])
  if m1 <= m0 or k1 <= k0 or n1 <= n0 or not fits:
    # empty ranges, or results that would be stored outside the destination: rejected
    with pytest.raises(GenerationError):
      g.generate()
    return
  g.generate()
  descrs = _build(case)
  n = 3
  lay, mem = harness.make_memory(descrs, n, seed=1, dtype=np.float64)
  before = {l.name: mem.buffers[l.name].copy() for l in lay if l.kind == 'strided'}
  multilinear.evaluate(descrs, mem, n, quirks=False)
  out = [l for l in lay if l.tensor.direction.name != 'SOURCE'][0]
  ins = [l for l in lay if l.kind == 'strided' and l is not out]
  a_l = [l for l in ins if list(l.tensor.shape) == [case['a']['rows'], case['a']['cols']]][0]
  b_l = [l for l in ins if l is not a_l][0]
  for e in range(n):
    A = _reader(before[a_l.name], a_l.starts[e], case['a'], compact=False)
    B = _reader(before[b_l.name], b_l.starts[e], case['b'], compact=not case['trans_b'])
    C = _reader(mem.buffers[out.name], out.starts[e], case['c'], compact=False)
    for i in range(m0, m1):
      for j in range(n0, n1):
        acc = 0.0
        for k in range(k0, k1):
          a = A(k, i) if case['trans_a'] else A(i, k)
          bv = B(j, k) if case['trans_b'] else B(k, j)
          acc += a * bv
        assert abs(C(i, j) - case['alpha'] * acc) <= 1e-12 * (1 + abs(acc))


BEHAVIOUR = json.load(open(os.path.join(HERE, 'golden', 'suite_reference_behaviour.json')))


@pytest.mark.parametrize('case', SUITES, ids=[c['id'] for c in SUITES])
def test_rejected_case_has_a_recorded_reference_behaviour(case):
  """Every suite case this generator rejects is one the reference cannot serve either
  (tests/golden/make_suite_reference.py ran the reference generator on each): it does not
  generate (NameError on transposes), or its kernel writes outside the destination's
  bounding box or outside the element's data (or the host process dies)."""
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.exceptions import GenerationError
  from tensorforge_b200.generators.generator import Generator
  g = Generator(_build(case), Context('sm_100a', 'cuda', FloatingPointType.FLOAT, Options()))
  try:
    g.generate()
    assert case['id'] not in BEHAVIOUR
    return
  except GenerationError:
    pass
  rec = BEHAVIOUR[case['id']]
  if not rec['generates']:
    assert 'Error' in rec['error']
  elif 'error' in rec:
    assert 'died' in rec['error'] or 'timed out' in rec['error']
  else:
    assert rec['outside_box'] > 0 or rec['outside_data'] > 0
