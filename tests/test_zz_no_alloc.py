"""GPU: the allocation-free grouped launch matches the regular grouped launch.

Some callers cannot call cudaMalloc: an application whose external memory manager owns
every device allocation and hands out only the operand buffers, or a latency-critical loop
where an allocation could block on a device-wide synchronisation. The regular grouped entry
point needs a device work table and a device counter from its caller;
tfb_grouped_launch_noalloc_<set> needs neither (its group records go to the kernel by value,
its work counter sits in a static device array of the library), so the caller passes only
inputs and outputs. This file is collected last on purpose: a failure here leaves every
other GPU test already run.
"""
import ctypes

import numpy as np
import pytest

from oracle import cases, harness

pytestmark = pytest.mark.gpu

SHAPES = [(10, 9, 37), (20, 27, 19), (35, 9, 101), (56, 9, 64), (84, 27, 23)]


def _kernel():
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context
  from tensorforge_b200.generators.generator import Generator
  from tensorforge_b200.grouped import GroupedKernel
  ns = cases.ns_from_module('tensorforge_b200')
  gens, descrs = [], []
  for b, q, _ in SHAPES:
    g = Generator(cases.mixed_chain(ns, b, q), Context('sm_100a', 'cuda', FloatingPointType.FLOAT))
    g.generate()
    gens.append(g)
    descrs.append(cases.mixed_chain(ns, b, q))
  return GroupedKernel(gens), descrs


def _buffers(descrs, seed):
  import torch
  out = []
  for gi, ((b, q, n), d) in enumerate(zip(SHAPES, descrs)):
    lay, mem = harness.make_memory(d, n, seed=seed + gi)
    dev, kw = {}, {'numElements': n}
    for l in lay:
      dev[l.name] = torch.tensor(mem.buffers[l.name], dtype=torch.float32, device='cuda')
      kw[l.name] = dev[l.name]
      if l.kind in ('strided', 'ptr'):
        kw[f'{l.name}_extraOffset'] = l.extra_offset
    out.append((dev, kw))
  return out


def test_noalloc_matches_regular_entry_point_twice():
  import torch
  from tensorforge_b200.grouped import launch_noalloc
  gk, descrs = _kernel()
  ref = _buffers(descrs, 50)
  gk.prepare([kw for _, kw in ref]).launch()
  torch.cuda.synchronize()
  for call in range(2):
    # fresh outputs each call: the second call must not depend on the first call's scratch
    bufs = _buffers(descrs, 50)
    launch_noalloc(gk, [kw for _, kw in bufs])
    torch.cuda.synchronize()
    for (rdev, _), (bdev, _) in zip(ref, bufs):
      for name in rdev:
        a = rdev[name].double().cpu().numpy()
        b = bdev[name].double().cpu().numpy()
        assert np.abs(a - b).max() <= 1e-5 * max(1.0, np.abs(a).max()), (call, name)


def test_noalloc_fewer_groups_and_an_empty_group():
  """num_groups below the fused set's size and a zero-element group between non-empty ones
  (both go through the kernel's tile-offset scan): the groups launched match the regular
  entry point, the others keep their inputs."""
  import torch
  from tensorforge_b200.grouped import launch_noalloc
  gk, descrs = _kernel()
  used = len(SHAPES) - 1

  def trimmed(bufs):
    kws = [dict(kw) for _, kw in bufs]
    kws[1]['numElements'] = 0
    return kws

  ref = _buffers(descrs, 70)
  kws = trimmed(ref)
  kws[used]['numElements'] = 0  # the regular entry point takes every group: empty the last
  gk.prepare(kws).launch()
  untouched = _buffers(descrs, 70)
  for call in range(2):
    bufs = _buffers(descrs, 70)
    launch_noalloc(gk, trimmed(bufs)[:used])
    torch.cuda.synchronize()
    for gi, ((rdev, _), (bdev, _), (udev, _)) in enumerate(zip(ref, bufs, untouched)):
      for name in rdev:
        a = rdev[name].double().cpu().numpy()
        b = bdev[name].double().cpu().numpy()
        assert np.abs(a - b).max() <= 1e-5 * max(1.0, np.abs(a).max()), (call, gi, name)
        if gi in (1, used):
          assert np.array_equal(b, udev[name].double().cpu().numpy()), (call, gi, name)


def test_noalloc_rejects_null_records():
  import torch
  gk, _ = _kernel()
  gk._load()
  fn = getattr(gk._lib, f'tfb_grouped_launch_noalloc_{gk.name}')
  fn.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p]
  fn.restype = ctypes.c_int
  assert fn(None, 1, torch.cuda.current_stream().cuda_stream) == 1  # cudaErrorInvalidValue


def test_noalloc_rejects_too_many_groups():
  import torch
  from tensorforge_b200.grouped import _GroupArgs
  gk, _ = _kernel()
  gk._load()
  fn = getattr(gk._lib, f'tfb_grouped_launch_noalloc_{gk.name}')
  fn.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p]
  fn.restype = ctypes.c_int
  recs = (_GroupArgs * (len(SHAPES) + 1))()
  rc = fn(ctypes.addressof(recs), len(SHAPES) + 1, torch.cuda.current_stream().cuda_stream)
  assert rc == 1  # cudaErrorInvalidValue
