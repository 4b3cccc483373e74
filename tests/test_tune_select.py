"""Generation-time variant selection (no GPU): Options(tuner='model') ranks the variant space
with the shipped cost model on the host."""
import pytest

from tensorforge_b200.common.basic_types import FloatingPointType as FP
from tensorforge_b200.common.context import Context, Options
from tensorforge_b200.generators.generator import Generator
from tensorforge_b200.tune import select, variants
from tensorforge_b200.tune.autotune import make_generator, build_descriptors, _ns
from tensorforge_b200.tune.chains import random_chains
from oracle import cases


def _gen(descrs, fp=FP.FLOAT, **opts):
  g = Generator(descrs, Context('sm_100a', 'cuda', fp, Options(**opts)))
  g.generate()
  return g


def test_model_tuner_picks_a_variant_of_the_space():
  for spec in random_chains(12, seed=21, hi=40):
    base = make_generator(spec)
    space = variants.variant_space(base.get_chain(), 4)
    want = select.model_choice(base.get_chain(), 4)
    g = Generator(build_descriptors(spec, _ns()), Context('sm_100a', 'cuda', FP.FLOAT, Options(tuner='model')))
    g.generate()
    if want is None:
      assert len(space) < 2
      continue
    assert want in space
    assert g.get_plan().strategy == want['strategy']
    # same launcher ABI whatever the variant
    assert g.abi_params() == base.abi_params()


def test_model_tuner_keeps_heuristic_plans_where_it_does_not_apply():
  ns = cases.ns_from_module('tensorforge_b200')
  heur = _gen(cases.build('chain_o6', ns), FP.DOUBLE)
  tuned = _gen(cases.build('chain_o6', ns), FP.DOUBLE, tuner='model')   # FP64: not modelled
  assert tuned.get_plan().key() == heur.get_plan().key()
  tc = _gen(cases.build('chain_o6', ns), precision='tf32x3', tuner='model')  # tensor cores: one plan
  assert tc.get_plan().strategy == 'tcsplit'


def test_unknown_tuner_is_rejected():
  with pytest.raises(ValueError):
    Options(tuner='fastest')


def test_tensor_core_variants_in_the_exhaustive_space():
  ns = cases.ns_from_module('tensorforge_b200')
  g = _gen(cases.build('chain_o6', ns), precision='tf32x3')
  space = variants.variant_space(g.get_chain(), 4, 'tf32x3')
  kinds = {(v['form'], v.get('pipe'), v.get('bbuf')) for v in space}
  assert ('u', 3, None) in kinds and ('u', 2, None) in kinds and ('b', None, 1) in kinds
  for v in space:   # each realises a distinct tensor-core plan
    assert _gen(cases.build('chain_o6', ns), precision='tf32x3', variant=v).get_plan().strategy == 'tcsplit'


def test_points_per_lane_in_the_exhaustive_space_only():
  ns = cases.ns_from_module('tensorforge_b200')
  g = _gen(cases.build_elementwise('ew_update', ns))
  full = variants.variant_space(g.get_chain(), 4)
  model = variants.variant_space(g.get_chain(), 4, model_only=True)
  assert {v.get('points_per_lane') for v in full} == set(variants.POINTS_PER_LANE)
  assert all('points_per_lane' not in v for v in model) and len(full) == 4 * len(model)
  # the default (4 points) keeps the feature vector the model was trained on
  d = dict(model[0])
  assert variants.variant_features(g.get_chain(), d) == variants.variant_features(g.get_chain(), dict(d, points_per_lane=4))


def test_model_inference_falls_back_to_the_host_without_a_gpu():
  import torch
  if torch.cuda.is_available():
    pytest.skip('a GPU is present: inference runs there (tests/test_gpu_tune_select.py)')
  spec = random_chains(3, seed=5, hi=40)[0]
  g = Generator(build_descriptors(spec, _ns()), Context('sm_100a', 'cuda', FP.FLOAT, Options(tuner='model')))
  g.generate()
  assert select.last_inference in ('host', None)
