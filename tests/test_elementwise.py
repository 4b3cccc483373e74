"""Elementwise statements (no GPU): the optree builders, generation and its checks, the
yateto `add_scalar` entry, and the oracle against per-element numpy written out by hand."""
import math

import numpy as np
import pytest

from oracle import harness, multilinear
from tensorforge_b200 import workloads as W
from tensorforge_b200.common.basic_types import Addressing, FloatingPointType as FP
from tensorforge_b200.common.context import Context, Options
from tensorforge_b200.common.exceptions import GenerationError
from tensorforge_b200.common.matrix.boundingbox import BoundingBox
from tensorforge_b200.common.matrix.spp import ListSPP
from tensorforge_b200.common.matrix.tensor import Tensor, SubTensor
from tensorforge_b200.common.operation import Operation
from tensorforge_b200.generators import optree as ot
from tensorforge_b200.generators.descriptions import ElementwiseDescr, MultilinearDescr
from tensorforge_b200.generators.generator import Generator

NS = W.ns_from_module('tensorforge_b200')


def _gen(descrs, fp=FP.FLOAT):
  g = Generator(descrs, Context('sm_100a', 'cuda', fp, Options()))
  g.generate()
  return g


def _run_oracle(name, n=None, seed=1, flags=None):
  descrs = W.build_elementwise(name, NS)
  n = n or W.EW_CASES[name][2]
  lay, mem = harness.make_memory(descrs, n, seed=seed)
  before = {k: v.copy() for k, v in mem.buffers.items()}
  multilinear.evaluate(descrs, mem, n, flags=flags)
  return {l.name: l for l in lay}, before, mem


def _block(lay, buf, e):
  """Element e's values of a dense batched symbol, shaped column-major."""
  shape = lay.tensor.shape
  vol = int(np.prod(shape))
  s = lay.starts[e]
  return buf[s:s + vol].reshape(shape, order='F')


# ------------------------------------------------------------------ oracle by hand
def test_oracle_update_by_hand():
  lay, before, mem = _run_oracle('ew_update')
  s = mem.scalars['m1']
  for e in range(W.EW_CASES['ew_update'][2]):
    q = _block(lay['m0'], before['m0'], e)
    t = q * s
    want = np.where(t > 0, t * np.exp(-t * t), 0.5 * t)
    assert np.allclose(_block(lay['m2'], mem.buffers['m2'], e), want, rtol=0, atol=1e-15)


HAND = {
  'exp': np.exp, 'log': lambda x: np.log(np.abs(x) + 0.5), 'expm1': np.expm1, 'logp1': lambda x: np.log1p(np.abs(x)),
  'sqrt': lambda x: np.sqrt(np.abs(x)), 'cbrt': np.cbrt, 'rsqrt': lambda x: 1 / np.sqrt(np.abs(x) + 0.25),
  'rcbrt': lambda x: 1 / np.cbrt(x + 2), 'pow': lambda x: (np.abs(x) + 0.5) ** 1.3, 'sin': lambda x: np.sin(3 * x),
  'cos': lambda x: np.cos(3 * x), 'tan': np.tan, 'asin': lambda x: np.arcsin(0.9 * x),
  'acos': lambda x: np.arccos(0.9 * x), 'atan': lambda x: np.arctan(4 * x), 'sinh': lambda x: np.sinh(2 * x),
  'cosh': lambda x: np.cosh(2 * x), 'tanh': lambda x: np.tanh(2 * x), 'asinh': lambda x: np.arcsinh(3 * x),
  'acosh': lambda x: np.arccosh(np.abs(x) + 1.5), 'atanh': lambda x: np.arctanh(0.9 * x),
  'erf': lambda x: np.vectorize(math.erf)(2 * x), 'gamma': lambda x: np.vectorize(math.gamma)(x + 2),
  'abs': np.abs, 'neg': lambda x: -x, 'rcp': lambda x: 1 / (x + 2), 'ceil': lambda x: np.ceil(4 * x),
  'floor': lambda x: np.floor(4 * x), 'round': lambda x: np.trunc(4 * x + np.copysign(0.5, x)),
  'trunc': lambda x: np.trunc(4 * x), 'sign': np.sign, 'mod': lambda x: np.fmod(8 * x, 3),
  'min': lambda x: np.minimum(x, 0.25), 'max': lambda x: np.maximum(x, -0.25), 'square': lambda x: x * x,
  'div': lambda x: x / (x * x + 1),
}


def test_oracle_functions_by_hand():
  assert set(HAND) == {n for n, _ in W.EW_FUNCTIONS}
  lay, before, mem = _run_oracle('ew_functions')
  for e in range(W.EW_CASES['ew_functions'][2]):
    q = _block(lay['m0'], before['m0'], e)
    out = _block(lay['m1'], mem.buffers['m1'], e)
    for f, (name, _) in enumerate(W.EW_FUNCTIONS):
      assert np.allclose(out[:, :, f], HAND[name](q), rtol=1e-14, atol=1e-14), name


def test_sinh_is_not_sin():
  # the reference's Operation enum makes SINH an alias of SIN; here each is its own
  assert Operation.SINH is not Operation.SIN and ot.sinh(1.0).optype == Operation.SINH


def test_oracle_control_by_hand():
  lay, before, mem = _run_oracle('ew_control')
  for e in range(W.EW_CASES['ew_control'][2]):
    q = _block(lay['m0'], before['m0'], e)
    p = _block(lay['m1'], before['m1'], e)
    got = _block(lay['m2'], mem.buffers['m2'], e)
    for idx in np.ndindex(q.shape):
      qv, pv = q[idx], p[idx]
      x = qv * qv + 1.0
      y, i = x, 0
      while i < 6:
        y = 0.5 * (y + x / y)
        i += 1
      o = y
      if qv > 0 and not (pv < -0.5):
        o = o + pv
      if qv < 0 or pv > 0.5:
        o = o - float(math.fmod(int(4 * pv), 3)) * 0.125
      o = o + (2.0 if ((qv > 0) != (pv > 0)) else float(i & 3))
      assert got[idx] == pytest.approx(o, rel=1e-15, abs=1e-15)


def test_oracle_fused_chain_by_hand():
  lay, before, mem = _run_oracle('ew_fused_chain')
  K = before['m0'].reshape(lay['m0'].tensor.shape, order='F')
  s = mem.scalars['m3']
  for e in range(W.EW_CASES['ew_fused_chain'][2]):
    q = _block(lay['m1'], before['m1'], e)
    o0 = _block(lay['m2'], before['m2'], e)
    want = o0 + np.maximum(K @ q, 0) * s
    assert np.allclose(_block(lay['m2'], mem.buffers['m2'], e), want, rtol=1e-13, atol=1e-13)


def test_oracle_feeds_contraction_by_hand():
  lay, before, mem = _run_oracle('ew_feeds_contraction')
  K = before['m2'].reshape(lay['m2'].tensor.shape, order='F')
  for e in range(W.EW_CASES['ew_feeds_contraction'][2]):
    q = _block(lay['m0'], before['m0'], e)
    want = (K @ np.tanh(q)) ** 2
    assert np.allclose(_block(lay['m1'], mem.buffers['m1'], e), want, rtol=1e-13, atol=1e-13)


def test_oracle_views_by_hand():
  lay, before, mem = _run_oracle('ew_views')
  B = before['m1'].reshape(6, 5, order='F')
  for e in range(W.EW_CASES['ew_views'][2]):
    q = _block(lay['m0'], before['m0'], e)
    want = _block(lay['m2'], before['m2'], e).copy()
    for n0 in range(6):
      for n1 in range(5):
        want[2 + n0, 1 + n1] = q[3 + n1, 4 + n0] * 2 + B[n0, n1]
    assert np.allclose(_block(lay['m2'], mem.buffers['m2'], e), want, rtol=0, atol=1e-15)


def test_oracle_sparse_read_by_hand():
  lay, before, mem = _run_oracle('ew_sparse_read')
  S = lay['m0'].tensor
  for e in range(W.EW_CASES['ew_sparse_read'][2]):
    dense = np.zeros(S.shape)
    s0 = lay['m0'].starts[e]
    for pos, (i, j) in enumerate(S.spp.list):
      dense[i, j] = before['m0'][s0 + pos]
    assert np.allclose(_block(lay['m1'], mem.buffers['m1'], e), 2 * dense + 1, rtol=0, atol=1e-15)


def test_oracle_flags_skip_elements():
  flags = np.array([1, 0] * 18 + [1], dtype=np.int32)
  lay, before, mem = _run_oracle('ew_update', flags=flags)
  for e in np.nonzero(flags == 0)[0]:
    assert np.array_equal(_block(lay['m2'], mem.buffers['m2'], e), _block(lay['m2'], before['m2'], e))


# ------------------------------------------------------------------ builders
def test_builder_shortcuts():
  x = ot.tensor(Tensor([4], Addressing.STRIDED))
  assert ot.mul(x, 1) is x and ot.mul(1.0, x) is x
  assert ot.mul(x, -1).optype == Operation.NEG
  assert (x ** 0.5).optype == Operation.SQRT and (x ** -0.5).optype == Operation.RSQRT
  assert (x ** (1 / 3)).optype == Operation.CBRT and (x ** -1).optype == Operation.RCP
  assert (x ** 2).optype == Operation.MUL and (x ** 1) is x
  assert (1 / x).optype == Operation.RCP and (x / 1) is x and (x / -1).optype == Operation.NEG
  assert ot.pow(math.e, x).optype == Operation.EXP
  assert ot.immc(True).fptype == FP.BOOL and ot.immc(3).fptype == FP.INT and ot.immc(2.5).fptype == FP.FLOAT
  assert (x < 1).optype == Operation.LT and (x == 1).optype == Operation.EQ
  with pytest.raises(TypeError):
    bool(x < 1)


def test_descr_directions_and_abi_order():
  d = W.build_elementwise('ew_update', NS)
  g = _gen(d)
  params = g.abi_params()
  assert params[0] == ('const float*', 'm0') and params[2] == ('float', 'm1') and params[3] == ('float*', 'm2')
  assert params[-3:] == [('size_t', 'numElements'), ('unsigned*', 'flags'), ('void*', 'streamPtr')]
  # read and written -> SOURCESINK, not const
  g2 = _gen(W.build_elementwise('ew_fused_chain', NS))
  assert ('float**', 'm2') in g2.abi_params()


def test_kernel_names_are_stable():
  names = {}
  for case in W.EW_CASES:
    a = _gen(W.build_elementwise(case, NS)).get_base_name()
    b = _gen(W.build_elementwise(case, NS)).get_base_name()
    assert a == b, case
    names[a] = case
  assert len(names) == len(W.EW_CASES)


def _two(shape=(6, 4)):
  return Tensor(list(shape), Addressing.STRIDED), Tensor(list(shape), Addressing.STRIDED)


@pytest.mark.parametrize('make', [
  # a shared tensor is read only
  lambda: [ot.assign(ot.tensor(Tensor([6, 4], Addressing.NONE)), ot.tensor(_two()[0]))],
  # a sparse tensor is not written
  lambda: [ot.assign(ot.tensor(Tensor([6, 4], Addressing.STRIDED, spp=ListSPP([(0, 0), (2, 1)], [6, 4]))),
                     ot.tensor(_two()[0]))],
  # written without every index: points would collide
  lambda: (lambda Q, O: [ot.assign(ot.tensor(O, indices=[-1]), ot.tensor(Q))])(
    Tensor([6, 4], Addressing.STRIDED), Tensor([6], Addressing.STRIDED)),
  # written and read through another index order
  lambda: (lambda Q: [ot.assign(ot.tensor(Q), ot.tensor(Q, indices=[-2, -1]) + 1.0)])(Tensor([5, 5], Addressing.STRIDED)),
  # gap in the indices
  lambda: (lambda Q, O: [ot.assign(ot.tensor(O, indices=[-1, -3]), ot.tensor(Q, indices=[-1, -3]))])(*_two()),
  # index count does not match the rank
  lambda: (lambda Q, O: [ot.assign(ot.tensor(O), ot.tensor(Q, indices=[-1]))])(*_two()),
  # bitwise operator on floating-point values
  lambda: (lambda Q, O: [ot.assign(ot.tensor(O), ot.tensor(Q) & ot.tensor(Q))])(*_two()),
  # a scalar argument is passed by value and cannot be assigned
  lambda: (lambda Q: [ot.assign(ot.scalar(Tensor([], Addressing.SCALAR)), ot.tensor(Q))])(_two()[0]),
  # a temporary read before anything wrote it
  lambda: (lambda Q, O: [ot.assign(ot.tensor(O), ot.tensor(Tensor([6, 4], Addressing.STRIDED, is_tmp=True)))])(*_two()),
])
def test_rejected_statements(make):
  with pytest.raises(GenerationError):
    _gen([ElementwiseDescr(make())])


def test_view_reaching_outside_is_rejected():
  Q = Tensor([6, 4], Addressing.STRIDED, bbox=BoundingBox([2, 0], [6, 4]))
  O = Tensor([6, 4], Addressing.STRIDED)
  # the view starts at row 2 of a tensor whose box starts at 2: rows 2..5 map to address
  # rows 0..3, inside; a view box from row 0 would map below the tensor
  _gen([ElementwiseDescr([ot.assign(ot.tensor(SubTensor(O, BoundingBox([0, 0], [4, 4]))),
                                    ot.tensor(SubTensor(Q, BoundingBox([2, 0], [6, 4]))))])])
  with pytest.raises(GenerationError):
    _gen([ElementwiseDescr([ot.assign(ot.tensor(O), ot.tensor(SubTensor(Q, BoundingBox([0, 0], [6, 4]))))])])


def test_unbound_variable_is_rejected():
  class Node:  # a yateto-like tensor node that no frontend bound
    name = 'x'
    memoryLayout = None
  with pytest.raises(GenerationError):
    ElementwiseDescr([ot.assign(ot.tensor(Node()), 1.0)])


def test_double_precision_literals_and_math():
  g = _gen(W.build_elementwise('ew_update', NS), FP.DOUBLE)
  k = g.get_kernel()
  assert 'exp(' in k and 'expf(' not in k and 'const double' in k


def test_emitted_sources_compile():
  """nvcc cross-compiles the emitted kernels for sm_100a (no GPU needed)."""
  from tensorforge_b200.runtime.build import build_library
  for case in ('ew_control', 'ew_functions', 'ew_fused_chain'):
    for fp in (FP.FLOAT, FP.DOUBLE):
      build_library(_gen(W.build_elementwise(case, NS), fp).get_source())


# ------------------------------------------------------------------ yateto gateway
class _Rng:
  def __init__(self, start, stop):
    self.start, self.stop = start, stop


class DenseMemoryLayout:  # the gateway tells dense layouts by this class name
  def __init__(self, shape):
    self._bbox = [_Rng(0, s) for s in shape]

  def bbox(self):
    return self._bbox

  def alignedStride(self):
    return False


class _EqSpp:
  def __init__(self, shape):
    self.shape = shape

  def nnzbounds(self):
    return [(0, s - 1) for s in self.shape]


class _YTensor:
  def __init__(self, name, shape, tmp=False):
    self.name = name
    self.memoryLayout = DenseMemoryLayout(shape)
    self.eqspp = _EqSpp(shape)
    self.is_compute_constant = False
    self.is_temporary = tmp
    self.values = None
    self.datatype = None
    self.addressing = None


class _YScalar:
  def __init__(self, name):
    self._name = name
    self.datatype = None

  def name(self):
    return self._name


class _Arch:
  name = 'sm_100'
  backend = 'cuda'
  typename = 'float'


def test_yateto_add_scalar():
  from tensorforge_b200.frontend.yateto import GpuKernelGeneratorV1

  class Cpp(list):
    def __call__(self, s):
      self.append(s)

  class Cache(dict):
    def addRoutine(self, name, writer):
      self[name] = writer

  Q, O, T = _YTensor('Q', [8, 3]), _YTensor('O', [8, 3]), _YTensor('tmp0', [8, 3], tmp=True)
  s = _YScalar('dt')
  gen = GpuKernelGeneratorV1(_Arch())
  stmts = [ot.assign(ot.tensor(T), ot.tensor(Q) * ot.scalar(s)),
           ot.assign(ot.tensor(O), ot.tensor(O) + ot.max(ot.tensor(T), 0.0))]
  assert gen.add_scalar([Q, s, T, O], stmts, [[-1, -2], [], [-1, -2], [-1, -2]]) == 0
  cpp, cache = Cpp(), Cache()
  g = gen.generate(cpp, cache)
  assert len(cache) == 1 and g.get_base_name() in cache
  assert [t.alias for t, _ in g.abi_symbols()] == ['Q', 'dt', 'O']
  assert [c for c, _ in g.abi_params()][:5] == ['const float**', 'unsigned', 'float', 'float**', 'unsigned']
  assert 'const_cast<const float**>(Q)' in cpp[0] and 'extraOffset_O' in cpp[0]


# ------------------------------------------------------------------ epilogues on the column program
@pytest.mark.parametrize('name', ['ew_chain_epilogue', 'ew_chain_epilogue_add'])
def test_oracle_chain_epilogue_by_hand(name):
  fn, kw, n = W.EW_CASES[name]
  full = fn(NS, **kw)
  chain = W.volume_chain(NS, basis=kw.get('basis', 56), quantities=kw.get('quantities', 9), seed=kw.get('seed', 0))
  if kw.get('accumulate'):
    chain[1].add = True
  lay_f, mem_f = harness.make_memory(full, n, seed=5)
  lay_c, mem_c = harness.make_memory(chain, n, seed=5)
  for name_ in mem_c.buffers:  # the chain's operands are drawn first, identically
    assert np.array_equal(mem_c.buffers[name_], mem_f.buffers[name_])
  before = {k: v.copy() for k, v in mem_f.buffers.items()}
  multilinear.evaluate(full, mem_f, n)
  multilinear.evaluate(chain, mem_c, n)
  lay = {l.name: l for l in lay_f}
  out = [l.name for l in lay_c if l.tensor is chain[1].dest.tensor][0]
  s = mem_f.scalars['m9']
  for e in range(n):
    c = _block(lay[out], mem_c.buffers[out], e)
    want = np.where(c > 0, c, 0.1 * c) + _block(lay['m8'], before['m8'], e) * s
    assert np.allclose(_block(lay[out], mem_f.buffers[out], e), want, rtol=1e-13, atol=1e-13)


def test_epilogue_plans():
  for fp in (FP.FLOAT, FP.DOUBLE):
    g = _gen(W.build_elementwise('ew_chain_epilogue', NS), fp)
    assert g.get_plan().strategy == 'colprog', g.get_plan()
    assert '// elementwise epilogue' in g.get_kernel()
  # tensor-core precision requested: the epilogue keeps the chain on the column program
  g = Generator(W.build_elementwise('ew_chain_epilogue', NS),
                Context('sm_100a', 'cuda', FP.FLOAT, Options(precision='tf32x3')))
  g.generate()
  assert g.get_plan().strategy == 'colprog'
  # an elementwise stage that writes another tensor is not an epilogue: generic generator
  d = W.volume_chain(NS, basis=20, quantities=9)
  out = d[-1].dest.tensor
  other = Tensor([20, 9], Addressing.STRIDED)
  d.append(ElementwiseDescr([ot.assign(ot.tensor(other), ot.tensor(out) * 2.0)]))
  assert _gen(d).get_plan().strategy == 'generic'
  # one between the contractions: generic as well
  d = W.volume_chain(NS, basis=20, quantities=9, terms=2)
  out = d[-1].dest.tensor
  d.insert(2, ElementwiseDescr([ot.assign(ot.tensor(out), ot.tensor(out) * 2.0)]))
  assert _gen(d).get_plan().strategy == 'generic'
