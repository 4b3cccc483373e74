"""GPU: chains that only fit 227 KB of shared memory through region reuse, against the
FP64 oracle (a sample of the 27 seeded tuning chains that were rejected without reuse,
including one whose shared sparse operands share memory and are re-expanded per tile)."""
import numpy as np
import pytest

from oracle import harness, multilinear
from tests.test_generic_liveness import _generate

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('index', [117, 549, 1641, 1932])
def test_reuse_chain_matches_oracle(index):
  import torch
  from tensorforge_b200.runtime import compile_generator
  g = _generate(index)
  k = compile_generator(g)
  descrs = g.descr_list
  n = 7
  lay, mem = harness.make_memory(descrs, n, seed=index)
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
      ref = mem.buffers[l.name]
      assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max(), l.name
