"""GPU parity: generated sm_100a kernels vs the reference's own kernels (golden vectors).

Tolerances follow the reference's test suite convention (relative to the output's max
magnitude): 1e-5 for FP32, 1e-12 for FP64.
"""
import numpy as np
import pytest

from oracle import cases
from tests.golden_io import golden_files, golden_ids, load, device_args

pytestmark = pytest.mark.gpu


def _run_case(meta, z, options=None):
  import torch
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.generators.generator import Generator
  from tensorforge_b200.runtime import compile_generator
  ns = cases.ns_from_module('tensorforge_b200')
  ftype = FloatingPointType.FLOAT if meta['fp'] == 'float' else FloatingPointType.DOUBLE
  g = Generator(cases.build(meta['case'], ns), Context('sm_100a', 'cuda', ftype, options or Options()))
  g.generate()
  k = compile_generator(g)
  bufs, kwargs, keep = device_args(z, meta, torch)
  k(**kwargs)
  torch.cuda.synchronize()
  return {n: b.double().cpu().numpy() for n, b in bufs.items()}


@pytest.mark.parametrize('path', golden_files(), ids=golden_ids())
def test_generic_matches_reference(path):
  from tensorforge_b200.common.context import Options
  z, meta = load(path)
  out = _run_case(meta, z, Options(variant={'strategy': 'generic'}))
  tol = 1e-5 if meta['fp'] == 'float' else 1e-12
  for s in meta['symbols']:
    if s['kind'] in ('scalar', 'shared'):
      continue
    ref = z[f'out_{s["name"]}'].astype(np.float64)
    if meta['case'] == 'gemm_alpha':
      continue  # reference drops alpha; checked against the oracle below
    scale = max(1e-30, float(np.abs(ref).max()))
    assert np.abs(out[s['name']] - ref).max() <= tol * scale, s['name']


@pytest.mark.parametrize('path', golden_files(), ids=golden_ids())
def test_default_plan_matches_reference(path):
  z, meta = load(path)
  if meta['case'] == 'gemm_alpha':
    pytest.skip('reference drops alpha')
  out = _run_case(meta, z)
  tol = 1e-5 if meta['fp'] == 'float' else 1e-12
  for s in meta['symbols']:
    if s['kind'] in ('scalar', 'shared'):
      continue
    ref = z[f'out_{s["name"]}'].astype(np.float64)
    scale = max(1e-30, float(np.abs(ref).max()))
    assert np.abs(out[s['name']] - ref).max() <= tol * scale, s['name']


def test_alpha_is_applied():
  """GemmDescr alpha != 1 scales the product (the reference silently drops it)."""
  import torch
  from oracle import harness, multilinear
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context
  from tensorforge_b200.generators.generator import Generator
  from tensorforge_b200.runtime import compile_generator
  ns = cases.ns_from_module('tensorforge_b200')
  d = cases.build('gemm_alpha', ns)
  n = 37
  lay, mem = harness.make_memory(d, n, seed=9)
  g = Generator(d, Context('sm_100a', 'cuda', FloatingPointType.FLOAT))
  g.generate()
  k = compile_generator(g)
  dev = {l.name: torch.tensor(mem.buffers[l.name], dtype=torch.float32, device='cuda') for l in lay if l.kind != 'scalar'}
  kw = {'numElements': n}
  for l in lay:
    if l.kind == 'scalar':
      kw[l.name] = mem.scalars[l.name]
    else:
      kw[l.name] = dev[l.name]
      if l.kind == 'strided':
        kw[f'{l.name}_extraOffset'] = l.extra_offset
  k(**kw)
  multilinear.evaluate(d, mem, n, quirks=False)
  for l in lay:
    if l.kind == 'strided' and l.tensor.direction.name != 'SOURCE':
      got = dev[l.name].double().cpu().numpy()
      assert np.abs(got - mem.buffers[l.name]).max() <= 1e-5 * np.abs(mem.buffers[l.name]).max()
