"""GPU: the reference's yateto matmul known-answer tests (tests/code-gen/matmul/ssm_86_Eigen/
KernelTest.t.h), C = op(A) op(B) on 32x32 pointer-array operands with the test's inputs,
relative L2 error against the test's loops below its 1.19e-5 bound."""
import numpy as np
import pytest

from tests.test_kat_matmul import KAT, ROLE, kat_inputs, kat_reference, kat_memory

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('variant', [None, {'strategy': 'generic', 'threads_per_element': 32, 'elements_per_block': 4}],
                         ids=['default', 'G32E4'])
@pytest.mark.parametrize('n', [1, 50])
@pytest.mark.parametrize('name', KAT)
def test_kat(name, n, variant):
  import torch
  from tensorforge_b200.kernels import make
  from tensorforge_b200.runtime import compile_generator
  g = make(name, 'float', **({'variant': variant} if variant else {}))
  k = compile_generator(g)
  descrs, lay, mem = kat_memory(name, n)
  kw, keep, dev = {'numElements': n}, [], {}
  for l in lay:
    b = torch.tensor(mem.buffers[l.name], dtype=torch.float32, device='cuda')
    dev[l.name] = b
    ptrs = torch.tensor(b.data_ptr() + (l.starts - l.extra_offset).astype(np.int64) * 4, dtype=torch.int64, device='cuda')
    keep.append(ptrs)
    kw[l.name] = ptrs
    kw[f'{l.name}_extraOffset'] = l.extra_offset
  k(**kw)
  torch.cuda.synchronize()
  A, B, _ = kat_inputs()
  want = kat_reference(name, A, B)
  rc = ROLE[name][2]
  l = {x.name: x for x in lay}[rc]
  got_all = dev[rc].double().cpu().numpy()
  for e in range(n):
    got = got_all[l.starts[e]:l.starts[e] + 1024]
    assert np.sqrt(np.sum((got - want) ** 2) / np.sum(want ** 2)) < 1.19e-5
