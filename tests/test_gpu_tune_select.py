"""GPU: Options(tuner='exhaustive') times every variant at generation time and keeps the
fastest; the kernel it picks matches the oracle."""
import numpy as np
import pytest

from oracle import cases, harness, multilinear

pytestmark = pytest.mark.gpu


def test_exhaustive_tuner_picks_a_correct_variant():
  import torch
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.generators.generator import Generator
  from tensorforge_b200.runtime import compile_generator
  from tensorforge_b200.tune.variants import variant_space
  ns = cases.ns_from_module('tensorforge_b200')
  g = Generator(cases.build('gemm_add', ns), Context('sm_100a', 'cuda', FloatingPointType.FLOAT,
                                                      Options(tuner='exhaustive')))
  g.generate()
  heur = Generator(cases.build('gemm_add', ns), Context('sm_100a', 'cuda', FloatingPointType.FLOAT, Options()))
  heur.generate()
  assert len(variant_space(heur.get_chain(), 4)) >= 2
  k = compile_generator(g)
  descrs = cases.build('gemm_add', ns)
  n = 513
  lay, mem = harness.make_memory(descrs, n, seed=4)
  dev, kw = {}, {'numElements': n}
  for l in lay:
    dev[l.name] = torch.tensor(mem.buffers[l.name], dtype=torch.float32, device='cuda')
    kw[l.name] = dev[l.name]
    if l.kind == 'strided':
      kw[f'{l.name}_extraOffset'] = l.extra_offset
  k(**kw)
  torch.cuda.synchronize()
  multilinear.evaluate(descrs, mem, n)
  for l in lay:
    if l.kind == 'strided' and l.tensor.direction.name != 'SOURCE':
      got = dev[l.name].double().cpu().numpy()
      assert np.abs(got - mem.buffers[l.name]).max() <= 1e-5 * np.abs(mem.buffers[l.name]).max()


def test_model_choice_runs_the_network_on_the_gpu():
  """Options(tuner='model') evaluates the cost model with the CUDA MLP kernels when a GPU
  is present; its predictions match the host evaluation of the same weights."""
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.generators.generator import Generator
  from tensorforge_b200.tune import select
  from tensorforge_b200.tune.cost_model import host_predict
  from tensorforge_b200.tune.variants import variant_space, features
  ns = cases.ns_from_module('tensorforge_b200')
  g = Generator(cases.build('three_matrices', ns), Context('sm_100a', 'cuda', FloatingPointType.FLOAT,
                                                            Options(tuner='model')))
  g.generate()
  assert select.last_inference == 'gpu'
  chain = g.get_chain()
  feats = [features(chain, v, 100000) for v in variant_space(chain, 4)]
  params, mean, std = select._load_model()
  host = host_predict(params, mean, std, feats)
  dev = select.predict(feats)
  assert np.abs(dev - host).max() <= 1e-3 * max(1.0, np.abs(host).max())


def test_exhaustive_tuner_over_tensor_core_variants():
  """Options(tuner='exhaustive', precision='tf32x3') times the tensor-core variants (forms U
  and B, both producer pipelines) and keeps the fastest; its kernel meets 1e-6."""
  import torch
  from tensorforge_b200.common.basic_types import FloatingPointType
  from tensorforge_b200.common.context import Context, Options
  from tensorforge_b200.generators.generator import Generator
  from tensorforge_b200.runtime import compile_generator
  from tensorforge_b200.tune.variants import variant_space
  ns = cases.ns_from_module('tensorforge_b200')
  g = Generator(cases.build('chain_o6', ns), Context('sm_100a', 'cuda', FloatingPointType.FLOAT,
                                                      Options(precision='tf32x3', tuner='exhaustive')))
  g.generate()
  assert g.get_plan().strategy == 'tcsplit'
  assert len(variant_space(g.get_chain(), 4, 'tf32x3')) >= 3
  k = compile_generator(g)
  descrs = cases.build('chain_o6', ns)
  n = 999
  lay, mem = harness.make_memory(descrs, n, seed=6)
  dev, kw = {}, {'numElements': n}
  for l in lay:
    dev[l.name] = torch.tensor(mem.buffers[l.name], dtype=torch.float32, device='cuda')
    kw[l.name] = dev[l.name]
    if l.kind == 'strided':
      kw[f'{l.name}_extraOffset'] = l.extra_offset
  k(**kw)
  torch.cuda.synchronize()
  multilinear.evaluate(descrs, mem, n)
  for l in lay:
    if l.kind == 'strided' and l.tensor.direction.name != 'SOURCE':
      got = dev[l.name].double().cpu().numpy()
      ref = mem.buffers[l.name]
      assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-6
