"""The reference's yateto matmul known-answer tests (tests/code-gen/matmul/ssm_86_Eigen/
KernelTest.t.h:20-86 and the three cases after it): 32x32 C = op(A) op(B) with inputs
A[i] = i % 512 + 1, B[i] = (i + 1) % 512 + 1 (flat column-major), relative L2 error below
1.19e-5. Here (no GPU): the launcher prototypes against the fixture's (subroutine.h:3-6,
parameter kinds and order), and the oracle against the test's own loops."""
import numpy as np
import pytest

from oracle import cases, harness, multilinear

KAT = ['kat_matmul_ab', 'kat_matmul_atb', 'kat_matmul_abt', 'kat_matmul_atbt']
# subroutine.h:3-6: parameter types in order (names aside)
PROTO = {
  'kat_matmul_ab': ['float**', 'unsigned', 'const float**', 'unsigned', 'const float**', 'unsigned'],
  'kat_matmul_atb': ['const float**', 'unsigned', 'const float**', 'unsigned', 'float**', 'unsigned'],
  'kat_matmul_abt': ['const float**', 'unsigned', 'float**', 'unsigned', 'const float**', 'unsigned'],
  'kat_matmul_atbt': ['const float**', 'unsigned', 'float**', 'unsigned', 'const float**', 'unsigned'],
}
ROLE = {  # which ABI symbol (m-order) is A, B, C
  'kat_matmul_ab': ('m1', 'm2', 'm0'),
  'kat_matmul_atb': ('m0', 'm1', 'm2'),
  'kat_matmul_abt': ('m0', 'm2', 'm1'),
  'kat_matmul_atbt': ('m0', 'm2', 'm1'),
}


def kat_inputs():
  i = np.arange(1024)
  return (i % 512 + 1).astype(np.float64), ((i + 1) % 512 + 1).astype(np.float64), ((i + 2) % 512 + 1).astype(np.float64)


def kat_reference(name, A, B):
  """The KernelTest loops: _tmp0[i + 32 j] += a(i, k) * b(k, j) with a, b read as written there."""
  a = A.reshape(32, 32, order='F')
  b = B.reshape(32, 32, order='F')
  ta = a.T if name in ('kat_matmul_atb', 'kat_matmul_atbt') else a
  tb = b.T if name in ('kat_matmul_abt', 'kat_matmul_atbt') else b
  return (ta @ tb).reshape(-1, order='F')


def kat_memory(name, n):
  descrs = cases.build(name, cases.ns_from_module('tensorforge_b200'))
  lay, mem = harness.make_memory(descrs, n, seed=0, extra_offsets=False)
  A, B, C = kat_inputs()
  ra, rb, rc = ROLE[name]
  by = {l.name: l for l in lay}
  for sym, vals in ((ra, A), (rb, B), (rc, C)):
    l = by[sym]
    for e in range(n):
      mem.buffers[sym][l.starts[e]:l.starts[e] + 1024] = vals
  return descrs, lay, mem


@pytest.mark.parametrize('name', KAT)
def test_launcher_prototype_matches_fixture(name):
  from tensorforge_b200.kernels import make
  g = make(name, 'float')
  types = [c for c, _ in g.abi_params()][:-3]
  assert types == PROTO[name]
  assert [c for c, _ in g.abi_params()][-3:] == ['size_t', 'unsigned*', 'void*']


@pytest.mark.parametrize('name', KAT)
def test_oracle_matches_kernel_test_loops(name):
  descrs, lay, mem = kat_memory(name, 2)
  multilinear.evaluate(descrs, mem, 2)
  A, B, _ = kat_inputs()
  want = kat_reference(name, A, B)
  rc = ROLE[name][2]
  l = {x.name: x for x in lay}[rc]
  for e in range(2):
    got = mem.buffers[rc][l.starts[e]:l.starts[e] + 1024]
    assert np.sqrt(np.sum((got - want) ** 2) / np.sum(want ** 2)) < 1.19e-5
