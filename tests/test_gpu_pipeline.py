"""GPU: the host-batch pipeline (runtime/pipeline.py) equals one launch over the batch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('opts', [{}, {'precision': 'tf32x3'}], ids=['colprog', 'tf32x3'])
@pytest.mark.parametrize('n,slices', [(10007, 4), (5, 8), (4099, 1)])
def test_pipeline_matches_single_launch(opts, n, slices):
  import torch
  from tensorforge_b200.kernels import make
  from tensorforge_b200.runtime import compile_generator
  from tensorforge_b200.runtime.pipeline import HostPipeline
  g = make('chain_o6', 'float', **opts)
  k = compile_generator(g)
  gen = torch.Generator().manual_seed(n)
  host, dev, ref = {}, {}, {}
  for t, _ in g.abi_symbols():
    size = t.spp.count_nz() if t.addressing.name == 'NONE' else n * t.get_real_volume()
    host[t.name] = (torch.rand(size, generator=gen) * 2 - 1).pin_memory()
    dev[t.name] = torch.zeros(size, device='cuda')
    ref[t.name] = host[t.name].cuda()
  out = [t.name for t, _ in g.abi_symbols() if t.direction.name != 'SOURCE'][0]
  k(numElements=n, **ref)
  HostPipeline(k, g, slices=slices, streams=3)(host, dev, n)
  torch.cuda.current_stream().synchronize()
  np.testing.assert_array_equal(host[out].numpy(), ref[out].cpu().numpy())
