"""GPU: what the learned part gains over the method without it.

A small seeded campaign (60 random chains, sizes up to 48) is measured exhaustively on
the GPU; a fresh cost model is trained on the training split by the CUDA MLP kernels and
its picks on the held-out chains are compared with the planner's own choice (the method
without the learned part): the best measured of the model's top 5 must be faster, on
average over the held-out chains, than the planner's pick.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_trained_model_beats_the_planner_on_held_out_chains():
  from tensorforge_b200.tune import heldout
  from tensorforge_b200.tune.cost_model import CostModel
  from tensorforge_b200.tune.run import is_test_chain
  builds = heldout.build_all(heldout.small_specs(60, seed=77))
  records = heldout.measure_all(builds)
  train = [(cb, res) for cb, res in records if not is_test_chain(cb.spec.index)]
  test = [(cb, res) for cb, res in records if is_test_chain(cb.spec.index)]
  X = [f for cb, res in train for f, r in zip(cb.feats, res) if r['ok']]
  y = [np.log(max(r['ms'], 1e-4)) for cb, res in train for r in res if r['ok']]
  model = CostModel(seed=0)
  hist = model.fit(np.array(X), np.array(y), steps=1500)
  assert hist[-1][1] < hist[0][1]            # the CUDA training kernels reduce the loss
  s = heldout.summary(heldout.score(test, model.predict))
  print(s)
  assert s['chains'] >= 8
  assert s['top5']['mean'] < s['default']['mean'], s
