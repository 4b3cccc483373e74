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


COLPROG_VARIANTS = [
  {'strategy': 'colprog', 'a_source': 'const'},
  {'strategy': 'colprog', 'a_source': 'smem'},
  {'strategy': 'colprog', 'a_source': 'smem', 'cols': 2},
  {'strategy': 'colprog', 'a_source': 'const', 'prefetch': 0, 'threads': 256},
  {'strategy': 'colprog', 'a_source': 'mixed', 'const_terms': 1, 'upitch': 'odd', 'min_blocks': 3},
  {'strategy': 'colprog', 'a_source': 'smem', 'threads': 256, 'rsplit': 2, 'min_blocks': 2},
  {'strategy': 'colprog', 'a_source': 'smem', 'threads': 256, 'rsplit': 2, 'cols': 2},
]


@pytest.mark.parametrize('variant', COLPROG_VARIANTS, ids=lambda v: ','.join(f'{k}={x}' for k, x in v.items() if k != 'strategy'))
@pytest.mark.parametrize('case', ['chain_o6', 'c0_gemm_ptr'])
def test_column_program_variants_match_reference(case, variant):
  """Every column-program variant the planner or the tuner can pick, on the golden vectors."""
  from tensorforge_b200.common.context import Options
  paths = [p for p in golden_files() if load(p)[1]['case'] == case and load(p)[1]['fp'] == 'float']
  assert paths
  z, meta = load(paths[0])
  out = _run_case(meta, z, Options(variant=variant))
  for s in meta['symbols']:
    if s['kind'] in ('scalar', 'shared'):
      continue
    ref = z[f'out_{s["name"]}'].astype(np.float64)
    scale = max(1e-30, float(np.abs(ref).max()))
    assert np.abs(out[s['name']] - ref).max() <= 1e-5 * scale, s['name']


@pytest.mark.parametrize('n', [1, 9, 10, 28, 1001])
@pytest.mark.parametrize('quantities', [9, 27])
def test_large_basis_column_program(quantities, n):
  """84-basis chains (9.5k unrolled FMAs per column, 256-thread CTAs by default) against the
  FP64 oracle, at sizes around the tile (9 elements for 27 quantities, 28 for 9), with flags."""
  import torch
  from oracle import harness, multilinear
  from tensorforge_b200.kernels import mixed_catalogue
  from tensorforge_b200.runtime import compile_generator
  g = dict(mixed_catalogue())[f'mixed_84x{quantities}']
  assert g.get_plan().strategy == 'colprog' and g.get_plan().params['threads'] == 256
  k = compile_generator(g)
  descrs = g.descr_list
  lay, mem = harness.make_memory(descrs, n, seed=5)
  flags = harness.make_flags(n, 5)
  dev = {l.name: torch.tensor(mem.buffers[l.name], dtype=torch.float32, device='cuda') for l in lay if l.kind != 'scalar'}
  kw = {'numElements': n, 'flags': torch.tensor(flags, dtype=torch.int32, device='cuda')}
  for l in lay:
    kw[l.name] = dev[l.name]
    if l.kind == 'strided':
      kw[f'{l.name}_extraOffset'] = l.extra_offset
  assert all(l.kind in ('strided', 'shared') for l in lay)
  k(**kw)
  torch.cuda.synchronize()
  multilinear.evaluate(descrs, mem, n, flags=flags)
  for l in lay:
    if l.kind == 'strided' and l.tensor.direction.name != 'SOURCE':
      got = dev[l.name].double().cpu().numpy()
      ref = mem.buffers[l.name]
      assert np.linalg.norm(got - ref) <= 1e-6 * np.linalg.norm(ref)
      for e in np.nonzero(flags == 0)[0]:  # masked elements keep their values exactly
        s = l.starts[e]
        assert np.array_equal(got[s:s + 84 * quantities], ref[s:s + 84 * quantities])
