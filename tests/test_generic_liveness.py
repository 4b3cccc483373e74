"""Shared-memory liveness and region reuse in the generic generator (CPU).

The 27 random chains (of the 2,000 seeded tuning chains) whose temporaries and expanded
sparse operands do not fit 227 KB when every region has its own memory now generate,
and in every layout two regions that are live in the same stage never share memory.
"""
import pytest

from tensorforge_b200.codegen.generic import (assign_offsets, live_ranges, region_sizes, shared_regions,
                                              _stage_access, _sparse_box, _prod)

# random_chains(2000, seed=0) indices that needed more than 227 KB without region reuse
REUSE_CHAINS = [41, 80, 117, 157, 393, 439, 525, 549, 552, 661, 672, 721, 818, 861, 955, 965, 976, 1035, 1037,
                1209, 1213, 1272, 1339, 1388, 1641, 1774, 1932]


def _generate(index):
  from tensorforge_b200 import workloads
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.generators.generator import Generator
  from tensorforge_b200.tune.chains import random_chains, build_descriptors
  spec = random_chains(2000, seed=0)[index]
  ns = workloads.ns_from_module('tensorforge_b200')
  g = Generator(build_descriptors(spec, ns), Context('sm_100a', 'cuda', FloatingPointType.FLOAT,
                                                     Options(variant={'strategy': 'generic'})))
  g.generate()
  return g


def _check_disjoint(sizes, ranges, offsets):
  names = list(sizes)
  for i, a in enumerate(names):
    for b in names[i + 1:]:
      live_together = not (ranges[a][1] < ranges[b][0] or ranges[b][1] < ranges[a][0])
      mem_overlap = offsets[a] < offsets[b] + sizes[b] and offsets[b] < offsets[a] + sizes[a]
      assert not (live_together and mem_overlap), (a, b)
    assert offsets[a] % 4 == 0


@pytest.mark.parametrize('index', REUSE_CHAINS)
def test_chain_that_needed_reuse_generates_within_227_kb(index):
  g = _generate(index)
  ch = g.get_chain()
  summed = sum(region_sizes(ch).values()) + sum(_prod(_sparse_box(o)) for o in ch.operands
                                                  if o.kind == 'shared' and o.sparse)
  assert summed * 4 > 227 * 1024                 # did not fit without reuse
  assert g.get_plan().smem_bytes <= 227 * 1024   # fits with it
  sizes, ranges = region_sizes(ch), live_ranges(ch)
  offsets, _ = assign_offsets(sizes, ranges)
  _check_disjoint(sizes, ranges, offsets)


def test_shared_regions_reuse_only_across_disjoint_stages():
  g = _generate(1641)   # two shared sparse operands of ~14k values each, used in stages 0 and 1
  ch = g.get_chain()
  offsets, total, resident = shared_regions(ch)
  ops = [o for o in ch.operands if o.kind == 'shared' and o.sparse]
  assert len(resident) < len(ops)
  access = [_stage_access(st) for st in ch.stages]
  sizes = {o.name: (_prod(_sparse_box(o)) + 3) // 4 * 4 for o in ops}
  ranges = {}
  for o in ops:
    used = [i for i, (_, r) in enumerate(access) if id(o) in r]
    ranges[o.name] = (min(used), max(used))
  _check_disjoint(sizes, ranges, offsets)
  assert total < sum(sizes.values())


def test_temporary_chain_reuses_dead_temporaries():
  """A four-stage chain: T1 dies in stage 1, so T3 (written in stage 2) takes its memory."""
  from tensorforge_b200 import workloads
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.generators.generator import Generator
  ns = workloads.ns_from_module('tensorforge_b200')
  A = ns.Addressing
  x = ns.Tensor([16, 16], A.STRIDED)
  descrs, cur = [], x
  for si in range(4):
    other = ns.Tensor([16, 16], A.NONE)
    ops = [ns.SubTensor(other), ns.SubTensor(cur)]
    dest = ns.Tensor([16, 16], A.STRIDED) if si == 3 else ns.generate_tmp_tensor(ops, [[0, -1], [-1, 1]])
    descrs.append(ns.MultilinearDescr(ns.SubTensor(dest), ops, [[0, -1], [-1, 1]], [[0, 1], [0, 1]]))
    cur = dest
  g = Generator(descrs, Context('sm_100a', 'cuda', FloatingPointType.FLOAT, Options(variant={'strategy': 'generic'})))
  g.generate()
  ch = g.get_chain()
  sizes, ranges = region_sizes(ch), live_ranges(ch)
  offsets, total = assign_offsets(sizes, ranges)
  assert len(sizes) == 3 and total == 2 * 256   # three 16x16 temporaries in two slots
  _check_disjoint(sizes, ranges, offsets)
