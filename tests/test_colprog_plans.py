"""Column-program plan selection (no GPU): the FMA cap and the 256-thread widening."""
from tensorforge_b200 import workloads as cases
from tensorforge_b200.kernels import make, Generator, Context, FP, Options


def _mixed(b, q, variant=None):
  ns = cases.ns_from_module('tensorforge_b200')
  g = Generator(cases.mixed_chain(ns, b, q), Context('sm_100a', 'cuda', FP['float'], Options(variant=variant or {})))
  g.generate()
  return g.get_plan()


def test_large_basis_chains_run_as_wide_column_programs():
  # 84x84 A at 45 %, three terms: 9.5k unrolled FMAs, above the old cap, below the new one
  for q in (9, 27):
    p = _mixed(84, q)
    assert p.strategy == 'colprog', p
    assert p.params['threads'] == 256 and p.params['prefetch'] == 1, p


def test_explicit_threads_are_kept():
  p = _mixed(84, 27, {'strategy': 'colprog', 'threads': 128})
  assert p.strategy == 'colprog' and p.params['threads'] == 128


def test_two_cta_column_programs_stay_at_128_threads():
  assert make('chain_o6', 'float').get_plan().params['threads'] == 128
  # the FP64 column program would lose its prefetch stage at 256 threads: not widened
  p = make('chain_o6', 'double', variant={'strategy': 'colprog'}).get_plan()
  assert p.params['threads'] == 128 and p.params['prefetch'] == 1


def test_unimplemented_precisions_are_rejected():
  import pytest
  for p in ('fp16x3', 'auto', 'fp8'):
    with pytest.raises(ValueError):
      Options(precision=p)
