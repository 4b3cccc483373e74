"""Named kernel configurations built ahead of time (tests, smoke, benchmark).

Each entry is a Generator for a chain from the case catalogue with a given precision /
strategy. `build()` in __graft_entry__ compiles all of them so that the GPU machine
only loads prebuilt libraries.
"""
from .common.basic_types import FloatingPointType
from .common.context import Context, Options
from .generators.generator import Generator

FP = {'float': FloatingPointType.FLOAT, 'double': FloatingPointType.DOUBLE}

# (case, fp, options kwargs) beyond the golden-vector cases
EXTRA = [
  ('chain_o6', 'float', {}),
  ('chain_o6', 'float', {'variant': {'strategy': 'generic'}}),
  ('chain_o6', 'float', {'precision': 'tf32x3'}),
  ('chain_o6', 'float', {'precision': 'bf16x3'}),
  ('chain_o4_q27', 'float', {'precision': 'tf32x3'}),
  ('chain_o6_ptr', 'float', {'precision': 'tf32x3'}),
  ('chain_o6', 'float', {'precision': 'tf32x3', 'variant': {'pipe': 1}}),
  ('chain_o6', 'float', {'precision': 'tf32x3', 'variant': {'form': 'u'}}),
  ('chain_o6', 'float', {'precision': 'tf32x3', 'variant': {'form': 'u', 'pipe': 2}}),
  ('chain_o6', 'float', {'precision': 'tf32x3', 'variant': {'form': 'u', 'ahead': 1}}),
  ('chain_o6', 'float', {'precision': 'tf32x3', 'variant': {'form': 'b'}}),
  ('c0_gemm_ptr', 'float', {'precision': 'tf32x3', 'variant': {'form': 'b'}}),
  ('c0_gemm_strided', 'float', {'precision': 'tf32x3', 'variant': {'form': 'b'}}),
  ('chain_o6', 'float', {'precision': 'tf32x3', 'variant': {'form': 'b', 'acc': 2, 'bbuf': 2}}),
  ('chain_o6', 'float', {'precision': 'tf32x3', 'variant': {'form': 'b', 'bbuf': 2}}),
  ('chain_o6', 'float', {'precision': 'tf32x3', 'variant': {'form': 'b', 'ws': 1}}),
  ('c0_gemm_ptr', 'float', {'precision': 'tf32x3', 'variant': {'form': 'b', 'ws': 1}}),
  ('c0_gemm_strided', 'float', {'precision': 'tf32x3', 'variant': {'form': 'b', 'ws': 1}}),
  ('c0_gemm_ptr', 'float', {'precision': 'tf32x3', 'variant': {'form': 'u'}}),
  ('c0_gemm_strided', 'float', {'precision': 'tf32x3', 'variant': {'form': 'u'}}),
  ('c0_gemm_ptr', 'float', {'precision': 'tf32x3', 'variant': {'form': 'b', 'acc': 2, 'bbuf': 2}}),
  ('c0_gemm_strided', 'float', {'precision': 'tf32x3', 'variant': {'form': 'b', 'acc': 2, 'bbuf': 2}}),
  ('c0_gemm_ptr', 'float', {'precision': 'tf32x3'}),
  ('c0_gemm_strided', 'float', {'precision': 'tf32x3'}),
  ('gemm_add', 'float', {'precision': 'tf32x3'}),
  ('chain_o3_dense', 'float', {'precision': 'tf32x3'}),
  ('sparse_a_shared', 'float', {'precision': 'tf32x3'}),
  ('chain_o6', 'float', {'precision': 'bf16x3', 'variant': {'pipe': 1}}),
  ('chain_o6', 'double', {}),
  ('chain_o6', 'double', {'variant': {'strategy': 'colprog'}}),
  ('chain_o6', 'float', {'variant': {'strategy': 'colprog', 'a_source': 'mixed', 'const_terms': 1, 'upitch': 'odd',
                                     'min_blocks': 3}}),
  ('c0_gemm_ptr', 'float', {'variant': {'strategy': 'colprog', 'a_source': 'mixed', 'const_terms': 1, 'upitch': 'odd',
                                        'min_blocks': 3}}),
  ('chain_o6', 'double', {'precision': 'dmma'}),
  ('chain_o4_q27', 'double', {'precision': 'dmma'}),
  ('chain_o3_dense', 'double', {'precision': 'dmma'}),
  ('c0_gemm_ptr', 'float', {}),
] + [(f'kat_matmul_{v}', 'float', o) for v in ('ab', 'atb', 'abt', 'atbt')
     for o in ({}, {'variant': {'strategy': 'generic', 'threads_per_element': 32, 'elements_per_block': 4}})]


def make(case, fp='float', **opts):
  from . import workloads as cases
  ns = cases.ns_from_module('tensorforge_b200')
  g = Generator(cases.build(case, ns), Context('sm_100a', 'cuda', FP[fp], Options(**opts)))
  g.generate()
  return g


def catalogue():
  import glob
  import json
  import os
  import numpy as np
  root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
  out, seen = [], set()

  def add(case, fp, opts):
    key = (case, fp, json.dumps(opts, sort_keys=True))
    if key in seen:
      return
    seen.add(key)
    try:
      out.append((f'{case}/{fp}/{key[2]}', make(case, fp, **opts)))
    except Exception:  # a variant that does not apply to this chain is skipped
      if not opts:
        raise

  for path in sorted(glob.glob(os.path.join(root, 'tests', 'golden', '*.npz'))):
    meta = json.loads(bytes(np.load(path)['meta']).decode())
    add(meta['case'], meta['fp'], {})
    add(meta['case'], meta['fp'], {'variant': {'strategy': 'generic'}})
  for case, fp, opts in EXTRA:
    add(case, fp, opts)
  return out


EW_LAUNCH_SHAPES = [
  {'strategy': 'generic', 'threads_per_element': 32, 'elements_per_block': 4},
  {'strategy': 'generic', 'threads_per_element': 128, 'elements_per_block': 2},
  {'strategy': 'generic', 'threads_per_element': 8, 'elements_per_block': 16},
  {'strategy': 'generic', 'threads_per_element': 16, 'elements_per_block': 4, 'points_per_lane': 8},
  {'strategy': 'generic', 'threads_per_element': 64, 'elements_per_block': 1, 'points_per_lane': 1},
]


def elementwise_catalogue():
  """(name, Generator) for the elementwise workloads: both precisions, plus the launch
  shapes the tests sweep and the benchmark's variants."""
  from . import workloads
  from .common.basic_types import FloatingPointType
  from .common.context import Context, Options
  from .generators.generator import Generator
  ns = workloads.ns_from_module('tensorforge_b200')
  out = []

  def add(name, fp, variant=None):
    ftype = FloatingPointType.FLOAT if fp == 'float' else FloatingPointType.DOUBLE
    g = Generator(workloads.build_elementwise(name, ns), Context('sm_100a', 'cuda', ftype, Options(variant=variant)))
    g.generate()
    out.append((f'{name}/{fp}/{variant}', g))

  for name in workloads.EW_CASES:
    for fp in ('float', 'double'):
      add(name, fp)
  for v in EW_LAUNCH_SHAPES:
    for name in ('ew_update', 'ew_feeds_contraction', 'ew_views', 'ew_control'):
      add(name, 'float', v)
  for v in EW_BENCH_VARIANTS:
    add('ew_update', 'float', v)
  for name in ('ew_chain_epilogue', 'ew_chain_epilogue_add'):
    add(name, 'float', {'strategy': 'generic'})
  return out


EW_BENCH_VARIANTS = [
  {'strategy': 'generic', 'threads_per_element': g, 'elements_per_block': e, 'points_per_lane': u}
  for g, e, u in ((64, 1, 1), (64, 1, 4), (64, 1, 8), (64, 4, 4), (32, 8, 4), (128, 2, 4), (256, 1, 2),
                  (512, 1, 1))
]


def mixed_catalogue():
  """(name, Generator) for the groups of the mixed-shape workload under their own default
  plans (the benchmark's separate-launch comparison and the large-basis parity tests)."""
  from . import workloads as cases
  ns = cases.ns_from_module('tensorforge_b200')
  out = []
  for b, q, _ in cases.mixed_shape_groups():
    g = Generator(cases.mixed_chain(ns, b, q), Context('sm_100a', 'cuda', FP['float']))
    g.generate()
    out.append((f'mixed_{b}x{q}', g))
  return out


def grouped_catalogue():
  """Grouped (mixed-shape) kernels used by the tests and the benchmark."""
  from . import workloads as cases
  from .grouped import GroupedKernel
  ns = cases.ns_from_module('tensorforge_b200')
  out = []
  sets = {
    'test': [(10, 9), (20, 27), (35, 9), (56, 9), (84, 27)],
    'bench_c3': [(b, q) for b, q, _ in cases.mixed_shape_groups()],
  }
  for tag, shapes in sets.items():
    gens = []
    for b, q in shapes:
      g = Generator(cases.mixed_chain(ns, b, q), Context('sm_100a', 'cuda', FP['float']))
      g.generate()
      gens.append(g)
    out.append((tag, GroupedKernel(gens)))
  return out
