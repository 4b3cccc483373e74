"""yateto gateway with mock yateto objects (yateto itself is not installed here)."""
import os

import pytest

from tensorforge_b200 import interop
from tensorforge_b200.common.basic_types import Addressing


class Rng:
  def __init__(self, start, stop):
    self.start, self.stop = start, stop


class DenseMemoryLayout:
  def __init__(self, shape):
    self._bbox = [Rng(0, s) for s in shape]

  def bbox(self):
    return self._bbox

  def alignedStride(self):
    return False


class CSCMemoryLayout(DenseMemoryLayout):
  def __init__(self, shape, entries):
    super().__init__(shape)
    self._entries = entries

  def entries(self, rows, cols):
    return [e for e in self._entries if e[0] in rows and e[1] in cols]


class EqSpp:
  def __init__(self, shape):
    self.shape = shape

  def nnzbounds(self):
    return [(0, s - 1) for s in self.shape]


class YTensor:
  def __init__(self, name, shape, const=False, tmp=False, layout=None):
    self.name = name
    self.memoryLayout = layout or DenseMemoryLayout(shape)
    self.eqspp = EqSpp(shape)
    self.is_compute_constant = const
    self.is_temporary = tmp
    self.values = None
    self.datatype = None
    self.addressing = None
    self.indices = 'ij'[:len(shape)]


class Arch:
  name = 'sm_100'
  backend = 'cuda'
  typename = 'float'


class Cpp:
  def __init__(self):
    self.lines, self.included = [], []

  def __call__(self, s):
    self.lines.append(s)

  def includes(self, hs):
    self.included += hs


class Cache:
  def __init__(self):
    self.routines = {}

  def addRoutine(self, name, writer):
    self.routines[name] = writer


def test_routine_generator_is_frontend():
  fe = interop.get_routine_generator(None)
  assert fe.__name__ == 'YatetoFrontend'
  assert interop.use_fusedgemm_cost() is True
  assert interop.get_version().strip()


def test_legacy_chain_generates_call_site_and_routine(tmp_path):
  FE = interop.get_routine_generator(None)
  fe = FE(Arch())
  K = YTensor('kDivM', (56, 56), const=True,
              layout=CSCMemoryLayout((56, 56), [(i, j) for j in range(56) for i in range(56) if (i * 7 + j) % 3]))
  Q = YTensor('Q', (56, 9))
  S = YTensor('star', (9, 9))
  T = YTensor('_tmp0', (56, 9), tmp=True)
  out = YTensor('Qout', (56, 9))
  fe.add_linear_operation(T, [K, Q], [[0, -1], [-1, 1]], [[0, 1], [0, 1]], False)
  fe.add_linear_operation(out, [T, S], [[0, -1], [-1, 1]], [[0, 1], [0, 1]], False)
  cpp, cache = Cpp(), Cache()
  g = fe.generate(cpp, cache)
  call = cpp.lines[0]
  assert call.startswith(f'launcher_{g.get_base_name()}(')
  assert 'const_cast<const float*>(kDivM)' in call
  assert 'extraOffset_Q' in call and 'numElements, flags, streamPtr' in call
  writer = cache.routines[g.get_base_name()]
  path = tmp_path / 'subroutine.cu'
  header = writer('r', str(path))
  assert header.startswith('void launcher_')
  text = path.read_text()
  assert f'launcher_{g.get_base_name()}' in text and '__global__' in text
  c = Cpp()
  writer.header(c)
  assert 'tensorforge_aux.h' in c.included
  # compute constant -> shared, others -> pointer arrays
  kinds = {t.alias: t.addressing for t, _ in g.abi_symbols()}
  assert kinds['kDivM'] == Addressing.NONE and kinds['Q'] == Addressing.PTR_BASED


def test_dictionary_api():
  FE = interop.get_routine_generator(None)
  fe = FE(Arch())
  fe.add_tensor({'name': 'A', 'datatype': 'f32', 'storage': {'shape': [8, 8], 'type': 'full'}, 'addressing': '&',
                 'values': None, 'flags': {'temporary': False, 'constant': True}})
  fe.add_tensor({'name': 'B', 'datatype': 'f32', 'storage': {'shape': [8, 4], 'type': 'full'}, 'addressing': 'n*N+o&',
                 'values': None, 'flags': {'temporary': False, 'constant': False}})
  fe.add_tensor({'name': 'C', 'datatype': 'f32', 'storage': {'shape': [8, 4], 'type': 'spp',
                 'entries': [(i, j) for j in range(4) for i in range(8)]}, 'addressing': 'n&+o&',
                 'values': None, 'flags': {'temporary': False, 'constant': False}})
  fe.add_operation({'type': 'multilinear', 'result': {'name': 'C', 'spp': None},
                    'args': [{'name': 'A', 'spp': None}, {'name': 'B', 'spp': None}],
                    'target': [[0, -1], [-1, 1]], 'permute': [[0, 1], [0, 1]],
                    'linear': {'alpha': None, 'add': True}, 'condition': []})
  cpp, cache = Cpp(), Cache()
  g = fe.generate(cpp, cache)
  assert len(cache.routines) == 1
  assert 'extraOffset_B' in cpp.lines[0]
