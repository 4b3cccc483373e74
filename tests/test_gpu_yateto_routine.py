"""GPU: the chain generated through the yateto gateway runs from its routine file, called
through the gateway's own call site (pointer arrays with extra offsets, a shared sparse
compute constant), and matches the FP64 oracle at the FP32 tolerance (1e-5 of the output's
largest magnitude)."""
import ctypes

import numpy as np
import pytest

from oracle import harness, multilinear

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('n', [1, 37, 1000])
def test_routine_runs_through_call_site(tmp_path, n):
  import torch
  from tensorforge_b200.runtime.build import build_library
  from tests.yateto_routine import generate_routine
  g, descrs, source = generate_routine(tmp_path)
  lib = ctypes.CDLL(build_library(source))
  lay, mem = harness.make_memory(descrs, n, seed=11)
  args, keep, dev = [], [], {}
  for l in lay:
    b = torch.tensor(mem.buffers[l.name], dtype=torch.float32, device='cuda')
    dev[l.name] = b
    if l.kind == 'ptr':
      ptrs = torch.tensor(b.data_ptr() + (l.starts - l.extra_offset).astype(np.int64) * 4, dtype=torch.int64, device='cuda')
      keep.append(ptrs)
      args += [ctypes.c_void_p(ptrs.data_ptr()), ctypes.c_uint(l.extra_offset)]
    elif l.kind == 'strided':
      args += [ctypes.c_void_p(b.data_ptr()), ctypes.c_uint(l.extra_offset)]
    else:
      args.append(ctypes.c_void_p(b.data_ptr()))
  stream = torch.cuda.current_stream().cuda_stream
  args += [ctypes.c_size_t(n), ctypes.c_void_p(None), ctypes.c_void_p(stream)]
  lib.yateto_execute(*args)
  torch.cuda.synchronize()
  multilinear.evaluate(descrs, mem, n)
  outs = [l for l in lay if l.tensor.direction.name != 'SOURCE']
  assert outs
  for l in outs:
    got = dev[l.name].double().cpu().numpy()
    ref = mem.buffers[l.name]
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()
