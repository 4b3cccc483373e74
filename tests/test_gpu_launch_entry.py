"""GPU: the status-returning entry point `tfb_launch_<name>` (same parameters as the
reference's `launcher_<name>`), called directly through ctypes for every generator
strategy on the golden vectors of the reference's own kernels."""
import ctypes

import numpy as np
import pytest

from oracle import cases
from tests.golden_io import golden_files, load, device_args

pytestmark = pytest.mark.gpu

# (golden case, fp, generator options, tolerance relative to the output's max magnitude)
CONFIGS = [
  ('chain_o6', 'float', {'variant': {'strategy': 'generic'}}, 1e-5),
  ('chain_o6', 'float', {}, 1e-5),                                     # column program
  ('chain_o6', 'float', {'precision': 'tf32x3'}, 1e-5),                # tensor cores, form U
  ('chain_o6', 'float', {'precision': 'tf32x3', 'variant': {'form': 'b'}}, 1e-5),
  ('c0_gemm_ptr', 'float', {'precision': 'tf32x3'}, 1e-5),             # form B, pointer arrays
  ('chain_o6', 'double', {'precision': 'dmma'}, 1e-12),
]


def _entry(case, fp, opts):
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.generators.generator import Generator
  from tensorforge_b200.runtime import compile_generator
  from tensorforge_b200.runtime.kernel import _ctype
  ns = cases.ns_from_module('tensorforge_b200')
  ftype = FloatingPointType.FLOAT if fp == 'float' else FloatingPointType.DOUBLE
  g = Generator(cases.build(case, ns), Context('sm_100a', 'cuda', ftype, Options(**opts)))
  g.generate()
  k = compile_generator(g)
  lib = ctypes.CDLL(k.so_path, mode=ctypes.RTLD_LOCAL)
  fn = getattr(lib, f'tfb_launch_{g.get_base_name()}')
  fn.argtypes = [_ctype(t) for t, _ in g.abi_params()]
  fn.restype = ctypes.c_int
  return g, fn


def _args(g, kwargs, n, stream):
  out = []
  for c_type, name in g.abi_params():
    if name == 'numElements':
      out.append(n)
    elif name == 'flags':
      out.append(None)
    elif name == 'streamPtr':
      out.append(stream)
    else:
      v = kwargs.get(name, 0 if name.endswith('_extraOffset') else None)
      out.append(int(v.data_ptr()) if hasattr(v, 'data_ptr') else v)
  return out


@pytest.mark.parametrize('case,fp,opts,tol', CONFIGS,
                         ids=[f'{c}-{f}-{o.get("precision", "plain")}-{o.get("variant", {}).get("strategy", o.get("variant", {}).get("form", "default"))}'
                              for c, f, o, _ in CONFIGS])
def test_status_entry_matches_reference(case, fp, opts, tol):
  import torch
  paths = [p for p in golden_files() if load(p)[1]['case'] == case and load(p)[1]['fp'] == fp]
  assert paths
  z, meta = load(paths[0])
  g, fn = _entry(case, fp, opts)
  bufs, kwargs, keep = device_args(z, meta, torch)
  stream = torch.cuda.Stream()
  outs = [s['name'] for s in meta['symbols'] if s['kind'] not in ('scalar', 'shared')
          and not np.array_equal(z[f'out_{s["name"]}'], z[f'in_{s["name"]}'])]
  assert outs

  # zero elements: success, nothing written
  before = {n: bufs[n].clone() for n in outs}
  assert fn(*_args(g, kwargs, 0, stream.cuda_stream)) == 0
  torch.cuda.synchronize()
  for n in outs:
    assert torch.equal(bufs[n], before[n]), n

  # the golden batch on a side stream
  assert fn(*_args(g, kwargs, int(z['n']), stream.cuda_stream)) == 0
  stream.synchronize()
  for n in outs:
    ref = z[f'out_{n}'].astype(np.float64)
    got = bufs[n].double().cpu().numpy()
    assert np.abs(got - ref).max() <= tol * max(1e-30, float(np.abs(ref).max())), n
