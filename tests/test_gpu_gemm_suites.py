"""GPU: the reference's GEMM YAML suites (tests/golden/gemm_suites.json) against the FP64
oracle: sub-boxes, leading dimensions, transposes and alpha, FP32 with the reference
suite's tolerance (1e-5 of the output's largest magnitude)."""
import json
import os

import numpy as np
import pytest

from oracle import cases, harness, multilinear

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
SUITES = json.load(open(os.path.join(HERE, 'golden', 'gemm_suites.json')))


@pytest.mark.parametrize('case', SUITES, ids=[c['id'] for c in SUITES])
def test_suite_case_matches_oracle(case):
  import torch
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.common.exceptions import GenerationError
  from tensorforge_b200.generators.generator import Generator
  from tensorforge_b200.runtime import compile_generator
  ns = cases.ns_from_module('tensorforge_b200')
  build = lambda: cases.suite_gemm(ns, case['a'], case['b'], case['c'], case['trans_a'], case['trans_b'], case['alpha'])
  g = Generator(build(), Context('sm_100a', 'cuda', FloatingPointType.FLOAT, Options()))
  try:
    g.generate()
  except GenerationError:
    pytest.skip('rejected at generation (empty range or result outside the destination)')
  k = compile_generator(g)
  descrs = build()
  n = max(case['num_elements'], 17)
  lay, mem = harness.make_memory(descrs, n, seed=3)
  dev, kw = {}, {'numElements': n}
  for l in lay:
    if l.kind == 'scalar':
      kw[l.name] = mem.scalars[l.name]
      continue
    dev[l.name] = torch.tensor(mem.buffers[l.name], dtype=torch.float32, device='cuda')
    kw[l.name] = dev[l.name]
    if l.kind == 'strided':
      kw[f'{l.name}_extraOffset'] = l.extra_offset
  k(**kw)
  torch.cuda.synchronize()
  multilinear.evaluate(descrs, mem, n, quirks=False)
  for l in lay:
    if l.kind == 'strided' and l.tensor.direction.name != 'SOURCE':
      got = dev[l.name].double().cpu().numpy()
      ref = mem.buffers[l.name]
      assert np.abs(got - ref).max() <= 1e-5 * max(1e-30, np.abs(ref).max())
