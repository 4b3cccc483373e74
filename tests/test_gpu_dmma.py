"""GPU: FP64 tensor-core (DMMA) chains vs the FP64 oracle.

The DMMA path contracts A_t * (B * R_t) instead of the reference's (A_t * B) * R_t and
sums in another order, so results differ from the oracle by FP64 rounding only: the
tolerance is a relative L2 error of 1e-12 over the whole output.
"""
import numpy as np
import pytest

from oracle import cases, harness, multilinear

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _run(case, n, seed=5, dist='uniform', use_flags=False):
  import torch
  from tensorforge_b200.kernels import make
  from tensorforge_b200.runtime import compile_generator
  g = make(case, 'double', precision='dmma')
  assert g.get_plan().strategy == 'dmma', g.get_plan()
  k = compile_generator(g)
  descrs = cases.build(case, cases.ns_from_module('tensorforge_b200'))
  lay, mem = harness.make_memory(descrs, n, seed=seed, dist=dist, dtype=np.float64)
  flags = harness.make_flags(n, seed) if use_flags else None
  dev, kw = {}, {'numElements': n}
  for l in lay:
    dev[l.name] = torch.tensor(mem.buffers[l.name], dtype=torch.float64, device='cuda')
    kw[l.name] = dev[l.name]
    if l.kind == 'strided':
      kw[f'{l.name}_extraOffset'] = l.extra_offset
  if flags is not None:
    kw['flags'] = torch.tensor(flags, dtype=torch.int32, device='cuda')
  k(**kw)
  torch.cuda.synchronize()
  multilinear.evaluate(descrs, mem, n, flags=flags)
  out = [l for l in lay if l.kind == 'strided' and l.tensor.direction.name != 'SOURCE'][0]
  return dev[out.name].cpu().numpy(), mem.buffers[out.name], out, flags


@pytest.mark.parametrize('n', [1, 9, 333, 4099])
def test_chain_o6_dmma(n):
  got, ref, _, _ = _run('chain_o6', n)
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= TOL, rel


def test_chain_o6_dmma_flags():
  got, ref, out, flags = _run('chain_o6', 517, use_flags=True)
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= TOL, rel
  for e in np.nonzero(flags == 0)[0][:5]:
    s = out.starts[e]
    assert np.array_equal(got[s:s + 504], ref[s:s + 504])


@pytest.mark.parametrize('case', ['chain_o4_q27', 'chain_o3_dense'])
def test_other_shapes_dmma(case):
  got, ref, _, _ = _run(case, 301, dist='loguniform')
  rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
  assert rel <= TOL, rel
