"""GPU: elementwise stages (alone and fused with contractions) against the FP64 oracle.

FP32 kernels are compared with the oracle run in FP64 with its floating-point
temporaries rounded to FP32 on assignment (as the kernel's registers are), so branch
decisions agree; tolerance |got - ref| <= 1e-5 * (1 + |ref|) per entry (CUDA's
single-precision math functions are accurate to a few ulp). FP64: 1e-12 * (1 + |ref|).
"""
import numpy as np
import pytest

from oracle import harness, multilinear
from tensorforge_b200 import workloads as W
from tensorforge_b200.kernels import EW_LAUNCH_SHAPES

pytestmark = pytest.mark.gpu


def run_case(name, n, fp='float', seed=3, flags=None, variant=None):
  import torch
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.generators.generator import Generator
  from tensorforge_b200.runtime import compile_generator
  ns = W.ns_from_module('tensorforge_b200')
  ftype = FloatingPointType.FLOAT if fp == 'float' else FloatingPointType.DOUBLE
  g = Generator(W.build_elementwise(name, ns), Context('sm_100a', 'cuda', ftype, Options(variant=variant)))
  g.generate()
  k = compile_generator(g)
  descrs = W.build_elementwise(name, ns)
  npdt = np.float32 if fp == 'float' else np.float64
  lay, mem = harness.make_memory(descrs, n, seed=seed, dtype=npdt)
  dt = torch.float32 if fp == 'float' else torch.float64
  dev, kw, keep = {}, {'numElements': n}, []
  for l in lay:
    if l.kind == 'scalar':
      kw[l.name] = mem.scalars[l.name]
      continue
    b = torch.tensor(mem.buffers[l.name], dtype=dt, device='cuda')
    dev[l.name] = b
    if l.kind == 'ptr':
      ptrs = torch.tensor(b.data_ptr() + (l.starts - l.extra_offset).astype(np.int64) * b.element_size(),
                          dtype=torch.int64, device='cuda')
      keep.append(ptrs)
      kw[l.name] = ptrs
      kw[f'{l.name}_extraOffset'] = l.extra_offset
    elif l.kind == 'strided':
      kw[l.name] = b
      kw[f'{l.name}_extraOffset'] = l.extra_offset
    else:
      kw[l.name] = b
  if flags is not None:
    kw['flags'] = torch.tensor(flags, dtype=torch.int32, device='cuda')
  k(**kw)
  torch.cuda.synchronize()
  multilinear.evaluate(descrs, mem, n, flags=flags, fp32=(fp == 'float'))
  outs = [l for l in lay if l.kind in ('strided', 'ptr') and l.tensor.direction.name != 'SOURCE']
  assert outs
  return [(dev[l.name].double().cpu().numpy(), mem.buffers[l.name], l) for l in outs], g


def check(results, fp):
  tol = 1e-5 if fp == 'float' else 1e-12
  for got, ref, l in results:
    err = np.abs(got - ref) / (1.0 + np.abs(ref))
    assert err.max() <= tol, (l.name, float(err.max()), int(err.argmax()))


@pytest.mark.parametrize('fp', ['float', 'double'])
@pytest.mark.parametrize('name', list(W.EW_CASES))
def test_case_matches_oracle(name, fp):
  check(run_case(name, W.EW_CASES[name][2], fp)[0], fp)


@pytest.mark.parametrize('n', [1, 2, 999])
def test_element_counts(n):
  check(run_case('ew_control', n)[0], 'float')
  check(run_case('ew_fused_chain', n)[0], 'float')


def test_flags_leave_elements_untouched():
  n = 301
  flags = (np.arange(n) % 3 != 1).astype(np.int32)
  results, _ = run_case('ew_fused_chain', n, flags=flags)
  check(results, 'float')


@pytest.mark.parametrize('variant', EW_LAUNCH_SHAPES, ids=lambda v: f"G{v['threads_per_element']}E{v['elements_per_block']}U{v.get('points_per_lane', 4)}")
def test_launch_shapes(variant):
  """Lane groups narrower and wider than a warp, several elements per CTA."""
  for name in ('ew_update', 'ew_feeds_contraction', 'ew_views', 'ew_control'):
    check(run_case(name, 77, variant=variant)[0], 'float')


@pytest.mark.parametrize('name', ['ew_chain_epilogue', 'ew_chain_epilogue_add'])
def test_epilogue_column_program_and_generic_agree_with_oracle(name):
  """The fused epilogue (column program) and the same descriptors on the generic generator."""
  res, g = run_case(name, 333)
  assert g.get_plan().strategy == 'colprog'
  check(res, 'float')
  res, g = run_case(name, 333, variant={'strategy': 'generic'})
  assert g.get_plan().strategy == 'generic'
  check(res, 'float')


def test_epilogue_flags():
  n = 250
  flags = (np.arange(n) % 4 != 2).astype(np.int32)
  check(run_case('ew_chain_epilogue', n, flags=flags)[0], 'float')
