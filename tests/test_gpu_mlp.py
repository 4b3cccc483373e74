"""CUDA cost-model kernels (csrc/mlp.cu) against the FP64 oracle, and a small tuning run."""
import numpy as np
import pytest

from oracle import mlp as ref_mlp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def model():
  from tensorforge_b200.tune.cost_model import CostModel
  return CostModel(seed=2)


def _batch(B, seed=0):
  import torch
  rng = np.random.default_rng(seed)
  X = rng.normal(size=(B, ref_mlp.IN)).astype(np.float32)
  T = rng.normal(size=B).astype(np.float32)
  return X, T, torch.tensor(X, device='cuda'), torch.tensor(T, device='cuda')


@pytest.mark.parametrize('B', [1, 7, 256, 3001])
def test_forward_matches_oracle(model, B):
  X, _, Xd, _ = _batch(B)
  p = model.params.cpu().numpy()
  y = model.forward(Xd).cpu().numpy()
  y_ref, _, _ = ref_mlp.forward(p, X)
  # FP32 accumulation over 32 + 64 + 64 terms
  assert np.max(np.abs(y - y_ref)) <= 1e-5 * (1 + np.max(np.abs(y_ref)))


@pytest.mark.parametrize('B', [1, 33, 1024])
def test_gradients_and_loss_match_oracle(model, B):
  X, T, Xd, Td = _batch(B, seed=B)
  p = model.params.cpu().numpy()
  loss, g = model.gradients(Xd, Td)
  g = g.cpu().numpy()
  g_ref = ref_mlp.grads(p, X, T)
  assert np.max(np.abs(g - g_ref)) <= 1e-4 * (1 + np.max(np.abs(g_ref)))
  assert float(loss.item()) == pytest.approx(ref_mlp.loss(p, X, T), rel=1e-5)


def test_adam_step_matches_numpy():
  from tensorforge_b200.tune.cost_model import CostModel
  m = CostModel(seed=3)
  X, T, Xd, Td = _batch(64, seed=9)
  p0 = m.params.cpu().numpy().astype(np.float64)
  mm = np.zeros_like(p0)
  vv = np.zeros_like(p0)
  p = p0.copy()
  for step in range(1, 4):
    g = ref_mlp.grads(p, X, T)
    m.gradients(Xd, Td)
    m.adam_step(1e-3)
    mm = 0.9 * mm + 0.1 * g
    vv = 0.999 * vv + 0.001 * g * g
    p = p - 1e-3 * (mm / (1 - 0.9 ** step)) / (np.sqrt(vv / (1 - 0.999 ** step)) + 1e-8)
  assert np.max(np.abs(m.params.cpu().numpy() - p)) <= 2e-5


def test_fit_learns_a_smooth_function():
  from tensorforge_b200.tune.cost_model import CostModel
  rng = np.random.default_rng(4)
  X = rng.uniform(-1, 1, size=(4000, ref_mlp.IN)).astype(np.float32)
  y = (np.sin(X[:, 0] * 2) + X[:, 1] * X[:, 2] + 0.5 * X[:, 3]).astype(np.float32)
  m = CostModel(seed=0)
  hist = m.fit(X[:3000], y[:3000], steps=1500, lr=3e-3, batch=1024)
  assert hist[-1][1] < 0.1 * hist[0][1]
  pred = m.predict(X[3000:])
  # held-out error well below the target's spread (28 of the 32 inputs are noise)
  assert np.sqrt(np.mean((pred - y[3000:]) ** 2)) < 0.5 * np.std(y[3000:])


def test_tuning_run_measures_consistent_variants(tmp_path):
  """Every variant of a few small chains computes the planner default's result."""
  from tensorforge_b200.tune.chains import random_chains
  from tensorforge_b200.tune.autotune import build_chain, measure_chain
  for spec in random_chains(3, seed=11, hi=20):
    cb = build_chain(spec)
    res = measure_chain(cb, cache=str(tmp_path))
    assert len(res) == len(cb.names) >= 2
    assert all(r['ok'] for r in res), [(r['variant'], r['err']) for r in res]
    assert all(r['ms'] > 0 for r in res)
    # the cache answers a second call without relaunching
    assert measure_chain(cb, cache=str(tmp_path)) == res
