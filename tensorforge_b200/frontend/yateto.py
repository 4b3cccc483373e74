"""yateto gateway: turns yateto's operation stream into one generated kernel per routine.

Same classes and call protocol as tensorforge/frontend/yateto.py:19-398:
`YatetoFrontend(arch)` with `add_linear_operation(dest, ops, target, permute, add)`
(the legacy object API), `add_tensor(dict)` / `add_operation(dict)` (the dictionary API)
and `generate(cpp, routineCache)`, which emits the launcher call into yateto's kernel
source (`cpp`) and registers a `TensorForgeWriter` that appends kernel + launcher to the
routine file and returns the launcher prototype for the header.

Addressing strings follow the reference (frontend/yateto.py:224-233): '&' shared,
'n*N+o&' strided, 'n&+o&' pointer array, '' scalar. In the legacy API, compute
constants are shared, temporaries strided and everything else pointer-based
(frontend/yateto.py:270-277). Call sites pass sources through `const_cast` and the
`extraOffset_<name>` members of yateto's kernel structs (frontend/yateto.py:325-345).
"""
from ..common.basic_types import Addressing, FloatingPointType, DataFlowDirection
from ..common.context import Context
from ..common.aux import generate_tmp_tensor
from ..common.exceptions import GenerationError
from ..common.matrix.tensor import Tensor, SubTensor
from ..common.matrix.spp import FullSPP, ListSPP
from ..common.matrix.boundingbox import BoundingBox
from ..generators.descriptions import MultilinearDescr, ElementwiseDescr
from ..generators.generator import Generator
from ..interface import YatetoInterface

ADDRESSING = {'&': Addressing.NONE, 'n*N+o&': Addressing.STRIDED, 'n&+o&': Addressing.PTR_BASED, '': Addressing.SCALAR}


class TensorForgeWriter:
  """Routine-cache entry: appends one kernel + launcher to yateto's routine file."""

  def __init__(self, generator, headers):
    self._headers = list(dict.fromkeys(list(headers) + list(generator.get_helper_headers())))
    self._generator = generator
    self._basename = generator.get_base_name()

  def target(self):
    return 'gpu'

  def __eq__(self, other):
    return isinstance(other, TensorForgeWriter) and self._basename == other._basename

  def __hash__(self):
    return hash(self._basename)

  def header(self, cpp):
    cpp.includes(self._headers)

  def __call__(self, routineName, fileName):
    with open(fileName, 'a', encoding='utf-8') as f:
      f.write(self._generator.get_kernel())
      f.write('\n')
      f.write(self._generator.get_launcher())
      f.write('\n')
    return self._generator.get_header()


class GpuKernelGeneratorV1:
  def __init__(self, arch):
    self._arch = arch
    self._cache = {}
    self._tmp = {}
    self._descr_list = []

  # ------------------------------------------------------------------ legacy object API
  def add_operation(self, dest, ops, target, permute, add):
    self._cache_operands(dest, ops, target, permute)
    self._descr_list.append(MultilinearDescr(self._sub(dest), [self._sub(op) for op in ops],
                                             target, permute, add=add))
    return 0

  def _is_scalar(self, op):
    return not hasattr(op, 'memoryLayout') and not isinstance(op, (float, int))

  def _sub(self, op):
    if isinstance(op, (float, int)):
      return SubTensor(Tensor([], Addressing.SCALAR, data=[op]))
    if self._is_scalar(op):
      return SubTensor(self._cache[op.name()])
    tensor = self._cache[op.name]
    bounds = op.eqspp.nnzbounds() if not callable(op.eqspp) else op.eqspp().nnzbounds()
    box = BoundingBox([lo for lo, _ in bounds], [hi + 1 for _, hi in bounds])
    # restrict the view to the tensor's own box (yateto's nonzero bounds may be looser)
    lower = [max(a, b) for a, b in zip(box.lower(), tensor.bbox.lower())]
    upper = [min(a, b) for a, b in zip(box.upper(), tensor.bbox.upper())]
    return SubTensor(tensor, BoundingBox(lower, upper))

  def _storage(self, layout):
    return layout.storage() if type(layout).__name__ == 'MemoryLayoutView' else layout

  def _addressing(self, term):
    if getattr(term, 'addressing', None) is not None:
      a = term.addressing
      return ADDRESSING[a] if isinstance(a, str) else a
    if term.is_compute_constant:
      return Addressing.NONE
    if term.is_temporary:
      return Addressing.STRIDED
    return Addressing.PTR_BASED

  def _make(self, op):
    if isinstance(op, (float, int)):
      return
    if self._is_scalar(op):
      name = op.name()
      if name not in self._cache:
        self._cache[name] = Tensor([], Addressing.SCALAR, alias=name, datatype=getattr(op, 'datatype', None))
      return
    if op.is_temporary:
      if op.name not in self._tmp:
        raise GenerationError(f'temporary {op.name} is used before it is produced')
      self._cache[op.name] = self._tmp[op.name]
      return
    tml = self._storage(op.memoryLayout)
    rng = tml.bbox()
    shape = [r.stop for r in rng]
    pattern = None
    if type(tml).__name__ != 'DenseMemoryLayout':
      pattern = tml.entries(range(rng[0].start, rng[0].stop), range(rng[1].start, rng[1].stop))
    t = YatetoInterface.gen_matrix(shape, rng, addressing=self._addressing(op), name=op.name,
                                   is_tmp=False, permute=None, pattern=pattern,
                                   values=getattr(op, 'values', None), datatype=getattr(op, 'datatype', None))
    if op.name not in self._cache or not t.is_same(self._cache[op.name]):
      self._cache[op.name] = t

  def _cache_operands(self, dest, ops, target, permute):
    for op in ops:
      self._make(op)
    if dest.is_temporary:
      if dest.name not in self._tmp:
        t = generate_tmp_tensor([self._sub(op) for op in ops], target, alias=dest.name)
        self._tmp[dest.name] = t
      self._cache[dest.name] = self._tmp[dest.name]
    else:
      self._make(dest)

  def _name(self, op):
    return op.name() if self._is_scalar(op) else op.name

  def add_scalar(self, ops, statements, indices):
    """Elementwise statements over yateto tensors (frontend/yateto.py:127-149).

    `statements` are optree statements whose tensor variables were made from the yateto
    nodes in `ops`; `indices[i]` is the index list of ops[i] (-1 for n0, -2 for n1, ...).
    Scalars take no indices. A temporary that the statements write before anything
    produced it becomes a new strided temporary with the layout's shape.
    """
    index_of = {}
    for op, idx in zip(ops, indices):
      if isinstance(op, (float, int)):
        continue
      if getattr(op, 'is_temporary', False) and op.name not in self._tmp:
        tml = self._storage(op.memoryLayout)
        rng = tml.bbox()
        t = Tensor([r.stop for r in rng], Addressing.STRIDED,
                   BoundingBox([r.start for r in rng], [r.stop for r in rng]), op.name, True)
        self._tmp[op.name] = t
      self._make(op)
      index_of[self._name(op)] = [] if self._is_scalar(op) else list(idx)

    def assigner(pre):
      if self._is_scalar(pre):
        self._make(pre)
        index_of.setdefault(pre.name(), [])
      name = self._name(pre)
      if name not in index_of:
        raise GenerationError(f'{name} is used by the statements but not listed in ops')
      return self._sub(pre), index_of[name]

    for st in statements:
      st.assignTensor(assigner)
    self._descr_list.append(ElementwiseDescr(statements))
    return 0

  # ------------------------------------------------------------------ dictionary API
  def add_tensor(self, d):
    name = d['name']
    datatype = FloatingPointType.ytt2enum(d['datatype']) if 'datatype' in d else None
    storage = d['storage']
    shape = list(storage['shape'])
    kind = storage['type']
    bbox, spp = None, None
    if kind == 'bbox':
      lower = list(storage['start'])
      bbox = BoundingBox(lower, [s + z for s, z in zip(lower, storage['sizes'])])
    elif kind == 'spp':
      spp = ListSPP(storage['entries'], shape)
    addressing = ADDRESSING[d.get('addressing', '&')]
    flags = d.get('flags', {})
    self._cache[name] = Tensor(shape, addressing, bbox, name, bool(flags.get('temporary', False)), spp,
                               d.get('values'), datatype)

  def add_operation_new(self, d):
    if d['type'] != 'multilinear':
      raise GenerationError(f'operation type {d["type"]!r} is not supported by the sm_100a generator')
    ref = lambda x: SubTensor(self._cache[x['name']])  # noqa: E731
    result = ref(d['result'])
    args = [ref(a) for a in d['args']]
    add = bool(d.get('linear', {}).get('add', False))
    self._descr_list.append(MultilinearDescr(result, args, d['target'], d['permute'], add=add))
    return 0

  # ------------------------------------------------------------------ generation
  def _fptype(self):
    if hasattr(self._arch, 'typename'):
      return FloatingPointType.str2enum(self._arch.typename)
    return FloatingPointType.FLOAT

  def _call_site(self, generator):
    mat, off = {}, {}
    for name, t in self._cache.items():
      if t.direction == DataFlowDirection.SOURCE and t.addressing != Addressing.SCALAR:
        dt = self._fptype() if t.datatype is None else t.datatype
        mat[name] = f'const_cast<const {dt}{t.addressing.to_pointer()}>({name})'
      else:
        mat[name] = name
      off[name] = '0' if (t.is_tmp or t.addressing == Addressing.NONE) else f'extraOffset_{name}'
    return generator.generate_call_site(mat, off, 'numElements', 'flags', 'streamPtr')

  def generate(self, cpp, routine_cache, options=None):
    context = Context(arch=self._arch.name, backend=self._arch.backend, fp_type=self._fptype(), options=options)
    g = Generator(self._descr_list, context)
    g.register()
    cpp(self._call_site(g))
    g.generate()
    # everything the emitted kernels and launchers use (PRELUDE of tensorforge_b200.codegen)
    headers = ['cuda_runtime.h', 'cstdint', 'cstddef', 'atomic', 'mutex', 'cstdio'] + context.get_vm().get_headers()
    routine_cache.addRoutine(g.get_base_name(), TensorForgeWriter(g, headers))
    return g


class YatetoFrontend:
  def __init__(self, arch):
    self.generator = GpuKernelGeneratorV1(arch)

  def generate(self, cpp, cache):
    return self.generator.generate(cpp, cache)

  def add_linear_operation(self, dest, ops, target, permute, add):
    return self.generator.add_operation(dest, ops, target, permute, add)

  def add_operation(self, description):
    return self.generator.add_operation_new(description)

  def add_tensor(self, tensor):
    return self.generator.add_tensor(tensor)
