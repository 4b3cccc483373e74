"""Autotuner host logic and the cost-model oracle (no GPU)."""
import math

import numpy as np
import pytest

from oracle import mlp as ref_mlp
from tensorforge_b200.tune.chains import random_chains
from tensorforge_b200.tune import autotune, variants, run
from tensorforge_b200.tune.cost_model import top_k, regret


def test_random_chains_seeded_and_in_range():
  a = random_chains(200, seed=0)
  b = random_chains(200, seed=0)
  assert [s.key() for s in a] == [s.key() for s in b]
  assert [s.key() for s in random_chains(5, seed=1)] != [s.key() for s in a[:5]]
  for s in a:
    assert 1 <= len(s.stages) <= 4
    assert 4 <= s.x_rows <= 128 and 4 <= s.x_cols <= 128
    rows, cols = s.x_rows, s.x_cols
    for st in s.stages:
      assert 0.1 <= st.density <= 1.0
      assert 4 <= st.rows <= 128 and 4 <= st.cols <= 128
      # chaining consistency: the contracted size is the previous stage's M (left) or N (right)
      if st.side == 'left':
        assert st.k == rows and st.cols == cols
      else:
        assert st.k == cols and st.rows == rows
      rows, cols = st.rows, st.cols
    assert 64 <= s.batch <= 1_000_000


def test_random_chain_distribution():
  specs = random_chains(2000, seed=0)
  lengths = np.bincount([len(s.stages) for s in specs], minlength=5)[1:]
  assert all(400 <= c <= 600 for c in lengths)
  logb = np.log10([s.batch for s in specs if s.batch > 10_000])
  assert logb.min() >= 4.0 and logb.max() <= 6.0


def test_variant_library_dedupes_and_contains_default():
  spec = random_chains(1, seed=3, hi=24)[0]
  src, gens, default = autotune.variant_library(spec)
  keys = [g.get_plan().key() for _, g in gens]
  assert len(set(keys)) == len(keys)
  names = [g.get_base_name() for _, g in gens]
  assert len(set(names)) == len(names)
  for n in names:
    assert f'launcher_{n}(' in src
  base = autotune.make_generator(spec)
  assert gens[default][1].get_plan().key() == base.get_plan().key()
  # every variant keeps the chain's launcher ABI
  assert all(g.abi_params() == base.abi_params() for _, g in gens)


def test_features_shape_and_finite():
  for spec in random_chains(20, seed=5, hi=32):
    base = autotune.make_generator(spec)
    for v in variants.variant_space(base.get_chain()):
      f = variants.features(base.get_chain(), v, spec.batch)
      assert len(f) == variants.NFEAT
      assert all(math.isfinite(x) for x in f)


def test_split_is_deterministic_20_percent():
  test = [run.is_test_chain(i) for i in range(2000)]
  assert 0.17 < np.mean(test) < 0.23
  assert test == [run.is_test_chain(i) for i in range(2000)]


def test_regret_and_topk():
  ms = [2.0, 1.0, 4.0, 1.05]
  assert regret(ms, [1]) == 0.0
  assert regret(ms, [0]) == pytest.approx(1.0)
  assert regret(ms, [0, 3]) == pytest.approx(0.05)
  assert top_k(np.array([3.0, 1.0, 2.0, 0.5]), 2) == [3, 1]


def test_mlp_oracle_gradients_match_finite_differences():
  rng = np.random.default_rng(0)
  p = ref_mlp.init(1).astype(np.float64)
  X = rng.normal(size=(16, ref_mlp.IN))
  T = rng.normal(size=16)
  g = ref_mlp.grads(p, X, T)
  idx = rng.choice(ref_mlp.NPARAMS, 60, replace=False)
  h = 1e-6
  for q in idx:
    e = np.zeros_like(p)
    e[q] = h
    fd = (ref_mlp.loss(p + e, X, T) - ref_mlp.loss(p - e, X, T)) / (2 * h)
    assert abs(fd - g[q]) < 1e-7 + 1e-5 * abs(g[q])


def test_cost_model_init_matches_oracle_layout():
  from tensorforge_b200.tune.cost_model import CostModel
  p = CostModel._init_params(None, 0)
  assert p.shape == (ref_mlp.NPARAMS,)
  assert np.array_equal(p, ref_mlp.init(0))
