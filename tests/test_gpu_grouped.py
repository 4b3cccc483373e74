"""GPU: mixed-shape persistent launch (one kernel over a work table, CUDA-graph replay)."""
import numpy as np
import pytest

from oracle import cases, harness, multilinear

pytestmark = pytest.mark.gpu

SHAPES = [(10, 9, 37), (20, 27, 19), (35, 9, 101), (56, 9, 64), (84, 27, 23)]


def _groups():
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context
  from tensorforge_b200.generators.generator import Generator
  ns = cases.ns_from_module('tensorforge_b200')
  gens, descrs = [], []
  for b, q, _ in SHAPES:
    d = cases.mixed_chain(ns, b, q)
    g = Generator(d, Context('sm_100a', 'cuda', FloatingPointType.FLOAT))
    g.generate()
    gens.append(g)
    descrs.append(cases.mixed_chain(ns, b, q))
  return gens, descrs


def _setup(descrs, use_flags=False):
  import torch
  per = []
  for gi, ((b, q, n), d) in enumerate(zip(SHAPES, descrs)):
    lay, mem = harness.make_memory(d, n, seed=10 + gi)
    dev, kw = {}, {'numElements': n}
    for l in lay:
      dev[l.name] = torch.tensor(mem.buffers[l.name], dtype=torch.float32, device='cuda')
      kw[l.name] = dev[l.name]
      if l.kind in ('strided', 'ptr'):
        kw[f'{l.name}_extraOffset'] = l.extra_offset
    flags = harness.make_flags(n, gi) if use_flags else None
    if flags is not None:
      kw['flags'] = torch.tensor(flags, dtype=torch.int32, device='cuda')
    per.append((lay, mem, dev, kw, flags))
  return per


def _check(descrs, per):
  for (b, q, n), d, (lay, mem, dev, kw, flags) in zip(SHAPES, descrs, per):
    multilinear.evaluate(d, mem, n, flags=flags)
    out = [l for l in lay if l.kind == 'strided' and l.tensor.direction.name != 'SOURCE'][0]
    got = dev[out.name].double().cpu().numpy()
    ref = mem.buffers[out.name]
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max(), (b, q)


def test_grouped_matches_oracle():
  import torch
  from tensorforge_b200.grouped import GroupedKernel
  gens, descrs = _groups()
  gk = GroupedKernel(gens)
  per = _setup(descrs)
  launch = gk.prepare([p[3] for p in per])
  launch.launch()
  torch.cuda.synchronize()
  _check(descrs, per)


@pytest.mark.parametrize('threads,prefetch', [(128, True), (256, False)])
def test_grouped_variants_match_oracle(threads, prefetch):
  """128 threads per CTA with the prefetch stage (each tile fetches the next same-group work
  item's inputs during its last K stage; the default at 256 threads), and 256 threads
  without it."""
  import torch
  from tensorforge_b200.grouped import GroupedKernel
  gens, descrs = _groups()
  gk = GroupedKernel(gens, threads=threads, prefetch=prefetch)
  per = _setup(descrs, use_flags=True)
  launch = gk.prepare([p[3] for p in per])
  launch.launch()
  torch.cuda.synchronize()
  _check(descrs, per)


def test_grouped_flags_and_graph_replay():
  import torch
  from tensorforge_b200.grouped import GroupedKernel
  gens, descrs = _groups()
  gk = GroupedKernel(gens)
  per = _setup(descrs, use_flags=True)
  launch = gk.prepare([p[3] for p in per])
  launch.capture()
  # the graph replays the counter reset as well: two replays give the same result
  launch.replay()
  launch.replay()
  torch.cuda.synchronize()
  _check(descrs, per)


def test_grouped_equals_separate_launches():
  import torch
  from tensorforge_b200.grouped import GroupedKernel
  from tensorforge_b200.runtime import compile_generator
  gens, descrs = _groups()
  gk = GroupedKernel(gens)
  per_a = _setup(descrs)
  per_b = _setup(descrs)
  gk.prepare([p[3] for p in per_a]).launch()
  for g, p in zip(gens, per_b):
    compile_generator(g)(**p[3])
  torch.cuda.synchronize()
  for pa, pb in zip(per_a, per_b):
    for name in pa[2]:
      a, bb = pa[2][name].cpu().numpy(), pb[2][name].cpu().numpy()
      assert np.abs(a - bb).max() <= 1e-5 * max(1.0, np.abs(bb).max())


def test_per_group_graph_matches_oracle():
  """The per-group mode: every group through its own launcher on side streams, eagerly and
  replayed from one CUDA graph, with flags."""
  import torch
  from tensorforge_b200.grouped import GroupedKernel
  gens, descrs = _groups()
  gk = GroupedKernel(gens)
  per = _setup(descrs, use_flags=True)
  pg = gk.prepare_per_group([p[3] for p in per], streams=3)
  assert sorted(g for lane in pg.lanes for g in lane) == list(range(len(SHAPES)))
  pg.launch()
  torch.cuda.synchronize()
  _check(descrs, per)
  # replay: the kernels are deterministic and masked elements are never written, so with the
  # outputs zeroed before the capture (its warm-up launch refills them) and again before the
  # replay, the replay must reproduce the captured state bit for bit
  outs = [[l for l in p[0] if l.kind == 'strided' and l.tensor.direction.name != 'SOURCE'][0] for p in per]
  for p, o in zip(per, outs):
    p[2][o.name].zero_()
  pg.capture()
  torch.cuda.synchronize()
  captured = [p[2][o.name].clone() for p, o in zip(per, outs)]
  assert all(bool(c.abs().sum() > 0) for c in captured)
  for p, o in zip(per, outs):
    p[2][o.name].zero_()
  pg.replay()
  torch.cuda.synchronize()
  for p, o, c in zip(per, outs, captured):
    assert torch.equal(p[2][o.name], c), o.name
