"""Tensor-core plan selection and layouts (no GPU): operand forms U and B, the form-B tile
choice under the TMEM and shared-memory limits, and that every variant compiles for sm_100a."""
import pytest

from tensorforge_b200.kernels import make
from tensorforge_b200.codegen.tcsplit_b import layout_b, blocks_of, SMEM_MAX
from tensorforge_b200.plan.chains import match_left_chain


def _shape(case):
  return match_left_chain(make(case, 'float').get_chain())


def test_default_is_form_u():
  p = make('chain_o6', 'float', precision='tf32x3').get_plan()
  assert p.strategy == 'tcsplit' and 'form' not in p.params and p.params['pipe'] == 3


def test_warp_specialised_pipeline_eligibility():
  """pipe 3 (separate epilogue warps, two A slots, two accumulator pairs) needs TF32
  splits, a U pass per term with K a multiple of 4, and TMEM for 2 slots + 2 pairs."""
  assert make('chain_o4_q27', 'float', precision='tf32x3').get_plan().params['pipe'] == 3
  assert make('chain_o6', 'float', precision='bf16x3').get_plan().params['pipe'] == 2
  assert make('chain_o3_dense', 'float', precision='tf32x3').get_plan().params['pipe'] == 2   # K = 10
  assert make('chain_o6', 'float', precision='tf32x3', variant={'pipe': 2}).get_plan().params['pipe'] == 2


@pytest.mark.parametrize('acc,bbuf', [(1, 1), (1, 2), (2, 1), (2, 2)])
def test_form_b_layout_limits(acc, bbuf):
  L = layout_b(_shape('chain_o6'), acc, bbuf)
  assert L is not None
  assert L['tmem'] <= 512 and L['total'] <= SMEM_MAX
  assert L['n_mma'] % 16 == 0 and L['te'] * L['P'] <= L['n_mma'] <= 256
  # the largest tile: one more element would break a limit
  bigger = layout_b(_shape('chain_o6'), acc, bbuf, L['te'] + 1)
  assert bigger is None


def test_form_b_blocks():
  assert blocks_of(1) == [(0, 0, True)]
  assert blocks_of(3) == [(0, 1, False), (2, 2, True)]
  assert blocks_of(5) is None


def test_form_b_declines_other_chains():
  # accumulating output, rows above 64 and terms with different inputs keep form U
  from tensorforge_b200 import workloads
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.generators.generator import Generator
  assert layout_b(_shape('gemm_add')) is None                  # out += A B
  ns = workloads.ns_from_module('tensorforge_b200')
  g = Generator(workloads.volume_chain(ns, basis=84, quantities=9), Context('sm_100a', 'cuda', FloatingPointType.FLOAT, Options()))
  g.generate()
  assert layout_b(match_left_chain(g.get_chain())) is None     # 84 rows do not fit a 64-lane half
  assert layout_b(_shape('chain_o4_q27'))['te'] == 256 // 27 or layout_b(_shape('chain_o4_q27'))['tmem'] <= 512
  s = _shape('chain_o6')
  assert s.M == 56 and layout_b(s)['blocks'] == blocks_of(3)


def test_form_b_variants_compile():
  from tensorforge_b200.runtime.build import build_library
  for v in ({'form': 'b'}, {'form': 'b', 'acc': 2, 'bbuf': 2}):
    for case in ('chain_o6', 'c0_gemm_ptr'):
      g = make(case, 'float', precision='tf32x3', variant=v)
      assert g.get_plan().params['form'] == 'b'
      build_library(g.get_source())
