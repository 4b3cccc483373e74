"""The CPU oracle reproduces the reference's own generated kernels (golden vectors)."""
import numpy as np
import pytest

from oracle import cases, multilinear
from tests.golden_io import golden_files, golden_ids, load, oracle_memory


@pytest.mark.parametrize('path', golden_files(), ids=golden_ids())
def test_oracle_matches_reference_kernels(path):
  z, meta = load(path)
  descrs = cases.build(meta['case'], cases.ns_from_module('tensorforge_b200'))
  mem = oracle_memory(z, meta)
  multilinear.evaluate(descrs, mem, int(z['n']), quirks=True)
  tol = 1e-5 if meta['fp'] == 'float' else 1e-12
  for s in meta['symbols']:
    if s['kind'] in ('scalar', 'shared'):
      continue
    ref = z[f'out_{s["name"]}'].astype(np.float64)
    got = mem.buffers[s['name']]
    scale = max(1e-30, float(np.abs(ref).max()))
    assert np.abs(got - ref).max() <= tol * scale, s['name']


def test_reference_failures_recorded():
  import os
  from tests.golden_io import GOLDEN
  txt = open(os.path.join(GOLDEN, 'reference_failures.txt')).read()
  assert 'trans_a' in txt and 'LeadLoop' in txt


def test_alpha_quirk_and_intended_semantics():
  """The reference drops GemmDescr's alpha (its value table is keyed by index tuples);
  the oracle reproduces that with quirks=True and computes alpha*A*B with quirks=False."""
  from oracle import harness
  d = cases.build('gemm_alpha', cases.ns_from_module('tensorforge_b200'))
  lay, mem = harness.make_memory(d, 4, seed=3, dtype=np.float64)
  import copy
  m2 = copy.deepcopy(mem)
  multilinear.evaluate(d, mem, 4, quirks=True)
  multilinear.evaluate(d, m2, 4, quirks=False)
  out = [l for l in lay if l.kind != 'shared'][0]
  a = mem.buffers[out.name][out.starts[0]:out.starts[0] + 48]
  b = m2.buffers[out.name][out.starts[0]:out.starts[0] + 48]
  assert np.all(a == 0.0) and np.abs(b).max() > 0
