"""GPU: Options(tuner='exhaustive') times every variant at generation time and keeps the
fastest; the kernel it picks matches the oracle."""
import numpy as np
import pytest

from oracle import cases, harness, multilinear

pytestmark = pytest.mark.gpu


def test_exhaustive_tuner_picks_a_correct_variant():
  import torch
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.generators.generator import Generator
  from tensorforge_b200.runtime import compile_generator
  from tensorforge_b200.tune.variants import variant_space
  ns = cases.ns_from_module('tensorforge_b200')
  g = Generator(cases.build('gemm_add', ns), Context('sm_100a', 'cuda', FloatingPointType.FLOAT,
                                                      Options(tuner='exhaustive')))
  g.generate()
  heur = Generator(cases.build('gemm_add', ns), Context('sm_100a', 'cuda', FloatingPointType.FLOAT, Options()))
  heur.generate()
  assert len(variant_space(heur.get_chain(), 4)) >= 2
  k = compile_generator(g)
  descrs = cases.build('gemm_add', ns)
  n = 513
  lay, mem = harness.make_memory(descrs, n, seed=4)
  dev, kw = {}, {'numElements': n}
  for l in lay:
    dev[l.name] = torch.tensor(mem.buffers[l.name], dtype=torch.float32, device='cuda')
    kw[l.name] = dev[l.name]
    if l.kind == 'strided':
      kw[f'{l.name}_extraOffset'] = l.extra_offset
  k(**kw)
  torch.cuda.synchronize()
  multilinear.evaluate(descrs, mem, n)
  for l in lay:
    if l.kind == 'strided' and l.tensor.direction.name != 'SOURCE':
      got = dev[l.name].double().cpu().numpy()
      assert np.abs(got - mem.buffers[l.name]).max() <= 1e-5 * np.abs(mem.buffers[l.name]).max()
